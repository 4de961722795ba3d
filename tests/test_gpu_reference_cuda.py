"""The B200 path against the reference's own FP64 CUDA kernels run on the same GPU.

The reference kernels (QSR.cu compiled from the reference sources into oracle/_ref/) are
the checker here; they show that the oracle restates the reference and that the FP32 fused
path tracks the reference's FP64 multi-kernel chain.
"""
import numpy as np
import pytest

from gpu_helpers import make_pair, fp32, rel_err
from lcdrsimulator_b200.physics import bulk_ABC, S_eq

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refcuda():
    from oracle.oracle import RefCUDA
    try:
        return RefCUDA()
    except FileNotFoundError:
        pytest.skip("reference CUDA build (oracle/_ref/qsr_cuda_ref.so) not available")


CASES = {
    "l1_strong_40": (dict(Nx=40, Ny=40, Nz=40, L1=6e-12), 300.0, None),
    "l123_weak_32": (dict(Nx=32, Ny=24, Nz=40, L1=6e-12, L2=3e-12, L3=1e-12, W=1e-5), 302.0, 0.6),
}


@pytest.mark.parametrize("name", list(CASES))
def test_oracle_equals_reference_cuda(oracle, refcuda, name):
    kw, T, S = CASES[name]
    op, solver, d = make_pair(**kw)
    solver.close()
    g, fl = oracle.geometry(op)
    S_shell = S if S is not None else S_eq(*bulk_ABC(d["a"], d["b"], d["c"], T, d["T_star"]))
    q0 = oracle.init(op, g, 0, 42, 0.5)
    refcuda.create(op)
    refcuda.upload(q0)
    for _ in range(20):
        refcuda.step(T, S_shell, 1.5e-10)
    rq = refcuda.download()
    ro = refcuda.observe(T, S_shell, d["Nz"] // 2)
    refcuda.destroy()
    oq = oracle.step_explicit(op, g, fl, q0, T, S_shell, 1.5e-10, n=20)
    assert rel_err(oq, rq) <= 1e-12
    oo = oracle.observe(op, g, fl, rq, T, S_shell)
    for k in ("bulk", "elastic", "anchoring", "radiality", "avg_S", "max_S"):
        assert oo[k] == pytest.approx(ro[k], rel=1e-12, abs=1e-300), k


@pytest.mark.parametrize("name", list(CASES))
def test_fused_fp32_tracks_reference_cuda(oracle, refcuda, name):
    kw, T, S = CASES[name]
    op, solver, d = make_pair(**kw)
    g, fl = oracle.geometry(op)
    S_shell = S if S is not None else S_eq(*bulk_ABC(d["a"], d["b"], d["c"], T, d["T_star"]))
    q0 = fp32(oracle.init(op, g, 0, 42, 0.5))
    refcuda.create(op)
    refcuda.upload(q0)
    for _ in range(200):
        refcuda.step(T, S_shell, 1.5e-10)
    rq = refcuda.download()
    ro = refcuda.observe(T, S_shell, d["Nz"] // 2)
    refcuda.destroy()
    solver.upload(q0)
    solver.step(200, T, S_shell, 1.5e-10)
    assert rel_err(solver.download(), rq) <= 1e-5
    so = solver.observe(T, S_shell)
    assert so["total"] == pytest.approx(ro["bulk"] + ro["elastic"] + ro["anchoring"], rel=1e-5)
    solver.close()


# Step time of the fused FP32 path against the reference's FP64 kernel chain on the same GPU.
# The default benchmark workload (256^3, droplet R = 120 cells, L1/L2/L3 = 6/3/1e-12 N,
# W = 1e-5 J/m^2, boundary_S = 0.6, T = 302 K) and the plain strong-anchoring relaxation of a
# 64^3 grid (R = 28 cells, L1 only, T = 300 K), both from the reference's seeded random directors.
TIMING = {
    "anisotropic_weak_256": (dict(Nx=256, Ny=256, Nz=256, kappa=0.0, L1=6e-12, L2=3e-12, L3=1e-12, W=1e-5,
                                  droplet_radius_cells=120.0), 302.0, 0.6, 50, 5),
    "plain_relaxation_64": (dict(Nx=64, Ny=64, Nz=64, kappa=0.0, L1=6e-12, droplet_radius_cells=28.0), 300.0, None,
                            400, 100),
}


@pytest.mark.parametrize("name", list(TIMING))
def test_step_time_against_reference_cuda_chain(refcuda, name):
    import json
    import os
    import torch
    kw, T, S, n_ours, n_ref = TIMING[name]
    op, solver, d = make_pair(**kw)
    S_shell = S if S is not None else S_eq(*bulk_ABC(d["a"], d["b"], d["c"], T, d["T_star"]))
    dt = 1.5e-10
    q0 = solver.initial_field(0, 42, 0.5)
    solver.upload(q0)
    solver.autotune(T, S_shell, dt, trial_steps=5)
    stream = torch.cuda.ExternalStream(solver.stream())
    args = solver.step_args(T, S_shell, dt)
    for s in range(3):
        args.step_index = s
        solver.step_raw(1, args)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for s in range(n_ours):
        args.step_index = 3 + s
        solver.step_raw(1, args)
    e1.record(stream)
    e1.synchronize()
    ours = e0.elapsed_time(e1) / n_ours
    assert np.isfinite(solver.download()).all()
    solver.close()
    refcuda.create(op)
    refcuda.upload(q0)
    refcuda.time_steps(T, S_shell, dt, 2)  # warm-up
    ref = refcuda.time_steps(T, S_shell, dt, n_ref) / n_ref
    refcuda.destroy()
    cells = d["Nx"] * d["Ny"] * d["Nz"]
    rec = dict(workload=name, cells=cells, ours_ms_per_step=ours, reference_cuda_ms_per_step=ref,
               ours_cell_updates_per_s=cells / (ours * 1e-3), reference_cell_updates_per_s=cells / (ref * 1e-3),
               speedup=ref / ours)
    out = os.environ.get("LDG_REF_TIMING_OUT")
    if out:
        with open(f"{out}.{name}", "w") as f:
            json.dump(rec, f)
    # one fused FP32 launch per step against the reference's seven FP64 kernels per step
    assert ours * 3.0 < ref, rec


def test_periodic_step_time_against_reference_kernel():
    """The periodic quench step (256^3 box, kappa = 6e-12 N, T = 300 K, Langevin noise kT/dx^3)
    against the reference's FP64 update kernel (KZM_bulk_ldg.cu) on the same GPU and input."""
    import json
    import math
    import os
    import torch
    from oracle.oracle import OrcBulkParams, RefKZM
    from lcdrsimulator_b200 import KZMSolver
    try:
        ref = RefKZM()
    except FileNotFoundError:
        pytest.skip("reference CUDA build (oracle/_ref/kzm_cuda_ref.so) not available")
    N, D, KAPPA, GAMMA, DT = 256, 1e-8, 6e-12, 0.1, 1.6e-9
    A, B, Cc = bulk_ABC(0.044e6, 1.413e6, 1.153e6, 300.0, 307.0)
    sigma = math.sqrt(2.0 * (1.0 / GAMMA) * (1.380649e-23 * 300.0 / D ** 3) * DT)
    q0 = np.random.default_rng(5).normal(0.0, 1e-3, N * N * N * 5)
    s = KZMSolver(N, N, N, D, D, D, KAPPA, GAMMA)
    s.upload(q0)
    stream = torch.cuda.ExternalStream(s.stream())
    s.step(3, A, B, Cc, DT, noise_sigma=sigma, seed=9, step_index=0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = 50
    e0.record(stream)
    s.step(n, A, B, Cc, DT, noise_sigma=sigma, seed=9, step_index=3)
    e1.record(stream)
    e1.synchronize()
    ours = e0.elapsed_time(e1) / n
    assert np.isfinite(s.download()).all()
    s.close()
    bp = OrcBulkParams(N, N, N, D, D, D, KAPPA, GAMMA, DT, 0.0, 0.1, 0.25)
    theirs = ref.time_steps(bp, q0, 3, 20, A, B, Cc, noise_sigma=sigma, seed=9) / 20
    sites = N ** 3
    rec = dict(workload="periodic_quench_256", cells=sites, ours_ms_per_step=ours, reference_cuda_ms_per_step=theirs,
               ours_cell_updates_per_s=sites / (ours * 1e-3), reference_cell_updates_per_s=sites / (theirs * 1e-3),
               speedup=theirs / ours)
    out = os.environ.get("LDG_REF_TIMING_OUT")
    if out:
        with open(f"{out}.periodic_quench_256", "w") as f:
            json.dump(rec, f)
    assert ours * 2.0 < theirs, rec
