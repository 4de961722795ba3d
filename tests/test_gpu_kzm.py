"""GPU parity of the periodic bulk (KZM_bulk_ldg) CUDA path against the FP64 oracle."""
import math

import numpy as np
import pytest

from gpu_helpers import fp32, rel_err
from oracle.oracle import OrcBulkParams
from lcdrsimulator_b200 import KZMSolver
from lcdrsimulator_b200.physics import bulk_ABC

pytestmark = pytest.mark.gpu


def _pair(Nx, Ny, Nz, dx=1e-8, dy=1e-8, dz=1e-8, kappa=6e-12, gamma=0.1, dt=1e-10, cap=0.0):
    bp = OrcBulkParams(Nx, Ny, Nz, dx, dy, dz, kappa, gamma, dt, cap, 0.1, 0.25)
    s = KZMSolver(Nx, Ny, Nz, dx, dy, dz, kappa, gamma, q_norm_cap=cap)
    return bp, s


@pytest.mark.parametrize("shape", [(24, 20, 16), (7, 5, 6), (2, 3, 4), (33, 17, 9)])
def test_periodic_steps_match_oracle(oracle, shape):
    bp, s = _pair(*shape, dy=1.1e-8)
    q0 = fp32(oracle.bulk_init(bp, 12345, 0.05))
    A, B, C = bulk_ABC(0.044e6, 1.413e6, 1.153e6, 300.0, 307.0)
    s.upload(q0)
    s.step(10, A, B, C, bp.dt)
    want = oracle.bulk_step(bp, q0, A, B, C, n=10)
    assert rel_err(s.download(), want) <= 2e-6


def test_periodic_cap_matches_oracle(oracle):
    bp, s = _pair(16, 16, 16, cap=0.3)
    q0 = fp32(oracle.bulk_init(bp, 1, 0.4))
    A, B, C = bulk_ABC(0.044e6, 1.413e6, 1.153e6, 295.0, 307.0)
    s.upload(q0)
    s.step(5, A, B, C, bp.dt)
    want = oracle.bulk_step(bp, q0, A, B, C, n=5)
    assert rel_err(s.download(), want) <= 2e-6


def test_periodic_observables_match_oracle(oracle):
    bp, s = _pair(24, 20, 16)
    A, B, C = bulk_ABC(0.044e6, 1.413e6, 1.153e6, 295.0, 307.0)
    q = oracle.bulk_init(bp, 99, 0.3)
    q = fp32(oracle.bulk_step(bp, q, A, B, C, n=50))
    s.upload(q)
    got = s.observe(A, B, C)
    want = oracle.bulk_observe(bp, q, A, B, C)
    for k in ("bulk", "elastic", "total", "avg_S", "max_S", "defect_line_density", "xi_grad_proxy",
              "defect_density_per_plaquette"):
        assert got[k] == pytest.approx(want[k], rel=1e-10), k
    for k in ("defect_plaquettes_used", "nonzero_defect_plaquettes"):
        assert got[k] == want[k], k
    assert want["nonzero_defect_plaquettes"] > 0


def test_periodic_noise_statistics(oracle):
    # zero field at A = 0: one step is pure noise with the requested sigma
    bp, s = _pair(32, 32, 32)
    s.upload(np.zeros(5 * 32 ** 3))
    sigma = math.sqrt(2.0 * (1.0 / 0.1) * 1e3 * 1e-12)
    s.step(1, 0.0, 1e6, 1e6, 1e-12, noise_sigma=sigma, seed=777, step_index=3)
    z = s.download() / sigma
    assert abs(z.mean()) < 0.01 and abs(z.std() - 1.0) < 0.01
    # different steps draw different numbers, same step reproduces
    s.upload(np.zeros(5 * 32 ** 3))
    s.step(1, 0.0, 1e6, 1e6, 1e-12, noise_sigma=sigma, seed=777, step_index=3)
    assert np.array_equal(s.download() / sigma, z)


@pytest.mark.parametrize("kernel", ["default", "async"])
@pytest.mark.parametrize("shape", [(64, 40, 70), (33, 17, 9), (2, 3, 4), (32, 8, 32), (40, 13, 5)])
def test_tiled_periodic_kernel_matches_direct(oracle, shape, kernel, monkeypatch):
    # the z-marching tiled kernels (two sites per thread by default, one site per thread with
    # LDG_KZM_KERNEL=async) and the one-thread-per-site kernel agree, with noise
    if kernel != "default":
        monkeypatch.setenv("LDG_KZM_KERNEL", kernel)
    A, B, C = bulk_ABC(0.044e6, 1.413e6, 1.153e6, 300.0, 307.0)
    bp, s = _pair(*shape, dy=1.1e-8)
    q0 = fp32(oracle.bulk_init(bp, 5, 0.05))
    s.upload(q0)
    s.step(6, A, B, C, bp.dt, noise_sigma=1e-4, seed=99, step_index=10)
    tiled = s.download()
    s.close()
    monkeypatch.setenv("LDG_KZM_KERNEL", "direct")
    bp, s2 = _pair(*shape, dy=1.1e-8)
    s2.upload(q0)
    s2.step(6, A, B, C, bp.dt, noise_sigma=1e-4, seed=99, step_index=10)
    direct = s2.download()
    s2.close()
    assert rel_err(tiled, direct) <= 1e-6
