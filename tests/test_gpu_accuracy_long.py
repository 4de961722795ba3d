"""Long-run accuracy of the FP32 device path against the FP64 oracle on identical noise-free
inputs: the anisotropic weak-anchoring physics of the 256^3 workload (L1/L2/L3 = 6/3/1e-12 N,
W = 1e-5 J/m^2, boundary_S = 0.6, T = 302 K, random directors S0 = 0.5) on a 64^3 grid with a
droplet of R = 28 cells, 5000 explicit steps at dt_max, observed every 1000 steps.

Run twice: plain FP32 storage and compensated storage (each value kept as two FP32 words). The
plain run's error grows like a random walk of per-step FP32 rounding of the stored field; the
compensated run must meet field max error <= 1e-5 and RMS <= 1e-6 (relative to max |Q|) and free
energy <= 1e-7 (relative to |F|). With LDG_ACCURACY_OUT set, the measured errors are also written
there as JSON.
"""
import json
import os

import numpy as np
import pytest

from gpu_helpers import make_pair, fp32, rel_err, rms_rel
from lcdrsimulator_b200.physics import DtRequest, estimate_stable_dt_window

pytestmark = pytest.mark.gpu

CASE = dict(Nx=64, Ny=64, Nz=64, L1=6e-12, L2=3e-12, L3=1e-12, W=1e-5, droplet_radius_cells=28.0, kappa=0.0)
T, S_SHELL, STEPS, EVERY = 302.0, 0.6, 5000, 1000


BARS = {0: (3e-5, 3e-6, 1e-7), 1: (1e-5, 1e-6, 1e-7)}


@pytest.mark.parametrize("compensated", [0, 1])
def test_long_run_fp32_matches_fp64(oracle, compensated):
    op, solver, d = make_pair(compensated=compensated, **CASE)
    g, fl = oracle.geometry(op)
    r = DtRequest(dx=d["dx"], dy=d["dy"], dz=d["dz"], gamma=d["gamma"], a=d["a"], b=d["b"], c=d["c"],
                  T_star=d["T_star"], modechoice=d["bulk_modechoice"], kappa=d["kappa"], L1=d["L1"], L2=d["L2"],
                  L3=d["L3"], S0=0.5, T_a=T, T_b=T)
    dt = estimate_stable_dt_window(r)["dt_max"]
    q = fp32(oracle.init(op, g, 0, 42, 0.5))
    solver.upload(q)
    rows = []
    for t in range(EVERY, STEPS + 1, EVERY):
        solver.step(EVERY, T, S_SHELL, dt)
        q = oracle.step_explicit(op, g, fl, q, T, S_SHELL, dt, n=EVERY)
        got = solver.download()
        F_gpu = solver.observe(T, S_SHELL)["total"]
        F_ref = oracle.observe(op, g, fl, q, T, S_SHELL)["total"]
        rows.append(dict(step=t, field_max=rel_err(got, q), field_rms=rms_rel(got, q),
                         energy=abs(F_gpu - F_ref) / abs(F_ref)))
    solver.close()
    out = os.environ.get("LDG_ACCURACY_OUT")
    if out:
        with open(f"{out}.{compensated}", "w") as f:
            json.dump(dict(case=CASE, compensated=compensated, T=T, S_shell=S_SHELL, dt=dt, rows=rows), f)
    bmax, brms, benergy = BARS[compensated]
    for row in rows:
        assert row["field_max"] <= bmax, row
        assert row["field_rms"] <= brms, row
        assert row["energy"] <= benergy, row
