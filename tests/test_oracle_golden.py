"""Pins the FP64 oracle's whole-step semantics to the reference's own FP64 CUDA code (CPU only).

The fixtures under tests/golden/ were produced by tests/golden/make_golden.py, which runs the
reference's QSR.cu and KZM_bulk_ldg.cu kernels (compiled from the reference sources) on a GPU.
"""
import ast
import glob
import hashlib
import os

import numpy as np
import pytest

from oracle.oracle import make_params, OrcBulkParams

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
QSR_FILES = sorted(glob.glob(os.path.join(GOLDEN, "qsr_*.npz")))


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype=np.float64).tobytes()).hexdigest()


@pytest.mark.skipif(not QSR_FILES, reason="golden fixtures not generated yet")
@pytest.mark.parametrize("path", QSR_FILES, ids=[os.path.basename(p) for p in QSR_FILES])
def test_oracle_matches_reference_cuda_fixture(oracle, path):
    z = np.load(path, allow_pickle=False)
    Nx, Ny, Nz = (int(v) for v in z["grid"])
    p = ast.literal_eval(str(z["params"]))
    op = make_params(Nx=Nx, Ny=Ny, Nz=Nz, T_star=307.0, **p)
    g, fl = oracle.geometry(op)
    if float(z["delta_eff"]) != 0.0:  # recorded by the generator
        assert g.delta_eff == pytest.approx(float(z["delta_eff"]), rel=1e-14)
    q0 = oracle.init(op, g, 0, 42, 0.5)
    assert _sha(q0) == str(z["init_sha"]), "initial field differs from the one the fixture was made from"
    T, S, dt, steps = float(z["T"]), float(z["S_shell"]), float(z["dt"]), int(z["steps"])
    if int(z["imex"]):
        q1 = oracle.step_imex(op, g, fl, q0, T, S, 4 * dt, op.L1, 25, n=steps)
    else:
        q1 = oracle.step_explicit(op, g, fl, q0, T, S, dt, n=steps)
    ref = z["q_final"]
    assert np.abs(q1 - ref).max() <= 1e-12 * np.abs(ref).max()
    o = oracle.observe(op, g, fl, ref, T, S)
    for k in ("bulk", "elastic", "anchoring", "radiality", "avg_S", "max_S", "defect_density"):
        assert o[k] == pytest.approx(float(z["obs_" + k]), rel=1e-12, abs=1e-300), k
    # checker = |sum_even - sum_odd| / sum (QSR.cu:2839-2873): a cancelling difference, so its
    # rounding error is a few ulps of the sums (absolute), not of the small ratio
    assert o["checker_rel"] == pytest.approx(float(z["obs_checker_rel"]), rel=0, abs=1e-13), "checker_rel"
    # the reference sums the xi proxy with FP64 atomics (QSR.cu:1042-1106): order-dependent rounding
    assert o["xi_grad_proxy"] == pytest.approx(float(z["obs_xi_grad_proxy"]), rel=1e-12), "xi_grad_proxy"
    for k in ("defect_count", "defect_plaquettes", "xi_edges"):
        assert o[k] == int(z["obs_" + k]), k


@pytest.mark.skipif(not os.path.exists(os.path.join(GOLDEN, "kzm_periodic.npz")), reason="no KZM fixture")
def test_oracle_matches_reference_kzm_fixture(oracle):
    z = np.load(os.path.join(GOLDEN, "kzm_periodic.npz"))
    bp = OrcBulkParams(16, 8, 24, 1e-8, 1.1e-8, 0.9e-8, 6e-12, 0.1, 1e-10, 0.0, 0.1, 0.25)
    q0 = oracle.bulk_init(bp, 12345, 0.2)
    assert _sha(q0) == str(z["init_sha"])
    A, B, C = float(z["A"]), float(z["B"]), float(z["C"])
    q1 = oracle.bulk_step(bp, q0, A, B, C, n=int(z["steps"]))
    assert np.abs(q1 - z["q_final"]).max() <= 1e-12 * np.abs(z["q_final"]).max()
    o = oracle.bulk_observe(bp, z["q_final"], A, B, C)
    for k in ("bulk", "elastic", "total", "avg_S", "max_S", "defect_line_density", "xi_grad_proxy"):
        assert o[k] == pytest.approx(float(z["obs_" + k]), rel=1e-12), k
    assert o["defect_plaquettes_used"] == int(z["obs_defect_plaquettes_used"])
    assert o["nonzero_defect_plaquettes"] == int(z["obs_nonzero_defect_plaquettes"])
