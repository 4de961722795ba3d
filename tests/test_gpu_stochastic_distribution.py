"""Stochastic quenches compared in distribution with the reference's own noisy kernel.

The reference's periodic bulk kernel (KZM_bulk_ldg.cu, built from its sources into oracle/_ref
and run on the GPU in FP64) draws its Langevin noise from a splitmix64 stream; this library
draws it from Philox4x32-7. Single trajectories therefore differ, but their statistics over
seeds must agree. A 32^3 periodic box is quenched to 300 K from the same 12 isotropic initial
fields (|Q| ~ 1e-3) with noise kT/dx^3 at 300 K; at four times the means over seeds of the
average order S, the free energy and the defect line density must agree within 4 combined
standard errors (plus 1 % of the mean for quantities whose spread is tiny).
"""
import math

import numpy as np
import pytest

from gpu_helpers import fp32
from oracle.oracle import OrcBulkParams, RefKZM
from lcdrsimulator_b200 import KZMSolver
from lcdrsimulator_b200.physics import bulk_ABC

pytestmark = pytest.mark.gpu

N, D, KAPPA, GAMMA, DT = 32, 1e-8, 6e-12, 0.1, 2e-9
CHECKS = [100, 300, 600, 1000]
SEEDS = list(range(12))
KEYS = ("avg_S", "total", "defect_line_density")


def test_noisy_quench_statistics_match_reference_kernel(oracle):
    ref = RefKZM()
    bp = OrcBulkParams(N, N, N, D, D, D, KAPPA, GAMMA, DT, 0.0, 0.1, 0.25)
    A, B, C = bulk_ABC(0.044e6, 1.413e6, 1.153e6, 300.0, 307.0)
    sigma = math.sqrt(2.0 * (1.0 / GAMMA) * (1.380649e-23 * 300.0 / D ** 3) * DT)
    mine = {k: np.zeros((len(SEEDS), len(CHECKS))) for k in KEYS}
    theirs = {k: np.zeros((len(SEEDS), len(CHECKS))) for k in KEYS}
    s = KZMSolver(N, N, N, D, D, D, KAPPA, GAMMA)
    for a, seed in enumerate(SEEDS):
        q0 = fp32(oracle.bulk_init(bp, 1000 + seed, 1e-3))
        s.upload(q0)
        q = q0.copy()
        done = 0
        for b, t in enumerate(CHECKS):
            s.step(t - done, A, B, C, DT, noise_sigma=sigma, seed=77 + seed, step_index=done)
            q = ref.run(bp, q, t - done, A, B, C, noise_sigma=sigma, seed=77 + seed, iter0=done)
            done = t
            o_m = s.observe(A, B, C)
            o_r = ref.observe(bp, q, A, B, C)
            for k in KEYS:
                mine[k][a, b] = o_m[k]
                theirs[k][a, b] = o_r[k]
    s.close()
    n = len(SEEDS)
    for k in KEYS:
        for b, t in enumerate(CHECKS):
            m1, m2 = mine[k][:, b].mean(), theirs[k][:, b].mean()
            se = math.sqrt(mine[k][:, b].var(ddof=1) / n + theirs[k][:, b].var(ddof=1) / n)
            assert np.isfinite([m1, m2, se]).all()
            assert abs(m1 - m2) <= 4.0 * se + 0.01 * abs(m2), (k, t, m1, m2, se)
    # the quench does order the box
    assert theirs["avg_S"][:, -1].mean() > 0.2
