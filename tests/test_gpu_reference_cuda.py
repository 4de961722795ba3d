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
