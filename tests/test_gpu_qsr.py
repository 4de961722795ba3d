"""GPU parity of the confined-droplet CUDA path against the FP64 oracle, through the C ABI.

Tolerances (FP32 device fields vs FP64 oracle, relative to max |Q|):
  * a few explicit steps from an identical FP32-representable field: <= 2e-6
  * 2000 explicit steps (32^3, L1, strong anchoring): field <= 1e-5, free energy <= 1e-6
  * FP64 reductions on an identical FP32-representable field: energies <= 1e-10 relative,
    integer counts exact.
"""
import math

import numpy as np
import pytest

from gpu_helpers import make_pair, fp32, rel_err, rms_rel
from lcdrsimulator_b200.physics import bulk_ABC, S_eq, estimate_stable_dt_window, DtRequest

pytestmark = pytest.mark.gpu

STEP_CASES = {
    "L1_strong": dict(Nx=32, Ny=32, Nz=32, L1=6e-12),
    "kappa_strong": dict(Nx=24, Ny=24, Nz=24, L1=0.0, kappa=6.5e-12),
    "L1L2L3_weak": dict(Nx=24, Ny=20, Nz=28, L1=6e-12, L2=3e-12, L3=1e-12, W=1e-5),
    "ravnik_L3_weak": dict(Nx=20, Ny=20, Nz=20, bulk_modechoice=2, L1=6e-12, L3=2e-12, W=1e-5),
    "aniso_spacing_L2": dict(Nx=20, Ny=24, Nz=18, dy=1.2e-8, dz=0.9e-8, L1=6e-12, L2=2e-12, W=2e-5),
    "odd_grid_all_terms": dict(Nx=13, Ny=11, Nz=9, L1=6e-12, L2=3e-12, L3=1e-12, W=1e-5),
    "radius_override_weak": dict(Nx=32, Ny=32, Nz=32, droplet_radius_cells=10.0, L1=6e-12, W=1e-5),
    "minimum_grid_3": dict(Nx=3, Ny=3, Nz=3, L1=6e-12, L2=3e-12, L3=1e-12, W=1e-5),
    "negative_W": dict(Nx=16, Ny=16, Nz=16, L1=6e-12, W=-1e-6),
    # grids with tiles whose halo lies inside the grid (k0 = 32, j0 = 8): the face-free interior
    # path of the tiled kernel, with the droplet surface crossing those tiles
    "interior_tiles_L1L2L3_weak": dict(Nx=12, Ny=20, Nz=72, L1=6e-12, L2=3e-12, L3=1e-12, W=1e-5,
                                  droplet_radius_cells=9.0),
    "interior_tiles_L2_strong": dict(Nx=12, Ny=20, Nz=72, L1=6e-12, L2=3e-12, W=0.0, droplet_radius_cells=9.0),
    "interior_tiles_kappa_weak": dict(Nx=14, Ny=24, Nz=80, L1=0.0, kappa=6.5e-12, W=2e-5, droplet_radius_cells=30.0),
}


def _dt(d, T):
    r = DtRequest(dx=d["dx"], dy=d["dy"], dz=d["dz"], gamma=d["gamma"], a=d["a"], b=d["b"], c=d["c"],
                  T_star=d["T_star"], modechoice=d["bulk_modechoice"], kappa=d["kappa"], L1=d["L1"], L2=d["L2"],
                  L3=d["L3"], S0=0.5, T_a=T, T_b=T)
    return estimate_stable_dt_window(r)["dt_max"]


@pytest.mark.parametrize("name", list(STEP_CASES))
def test_explicit_steps_match_oracle(oracle, name):
    op, solver, d = make_pair(**STEP_CASES[name])
    g, fl = oracle.geometry(op)
    geo = solver.geometry()
    assert geo["shell_cells"] == g.shell_count
    assert geo["delta_eff"] == pytest.approx(g.delta_eff, rel=1e-14)
    T, S_shell = 302.0, 0.6
    q0 = fp32(oracle.init(op, g, 0, 42, 0.5))
    dt = _dt(d, T)
    solver.upload(q0)
    solver.step(5, T, S_shell, dt)
    got = solver.download()
    want = oracle.step_explicit(op, g, fl, q0, T, S_shell, dt, n=5)
    assert rel_err(got, want) <= 2e-6, (name, rel_err(got, want))
    solver.close()


def test_q_norm_cap_matches_oracle(oracle):
    op, solver, d = make_pair(Nx=16, Ny=16, Nz=16, L1=6e-12)
    g, fl = oracle.geometry(op)
    q0 = fp32(oracle.init(op, g, 0, 5, 1.1))
    cap = 1.0 * math.sqrt(2.0 / 3.0)
    dt = _dt(d, 300.0)
    solver.upload(q0)
    solver.step(3, 300.0, 0.9, dt, q_norm_cap=cap)
    want = oracle.step_explicit(op, g, fl, q0, 300.0, 0.9, dt, q_norm_cap=cap, n=3)
    assert rel_err(solver.download(), want) <= 2e-6


IMEX_CASES = dict(STEP_CASES, chunked_planes_strong=dict(Nx=70, Ny=12, Nz=20, L1=6e-12, droplet_radius_cells=9.0))


@pytest.mark.parametrize("name,iters", [("L1_strong", 25), ("L1L2L3_weak", 25), ("odd_grid_all_terms", 25),
                                        ("L1_strong", 2), ("interior_tiles_L2_strong", 7),
                                        ("chunked_planes_strong", 25), ("chunked_planes_strong", 4)])
def test_imex_steps_match_oracle(oracle, name, iters):
    # grids with several 32-plane chunks, interior tiles, odd sweep counts
    op, solver, d = make_pair(**IMEX_CASES[name])
    g, fl = oracle.geometry(op)
    q0 = fp32(oracle.init(op, g, 0, 7, 0.5))
    T, S_shell, L_stab = 301.0, 0.6, d["L1"]
    dt = 4 * _dt(d, T)
    solver.upload(q0)
    solver.step(3, T, S_shell, dt, semi_implicit=True, L_stab=L_stab, jacobi_iters=iters)
    want = oracle.step_imex(op, g, fl, q0, T, S_shell, dt, L_stab, iters, n=3)
    assert rel_err(solver.download(), want) <= 2e-6


@pytest.mark.parametrize("name", ["L1_strong", "L1L2L3_weak", "radius_override_weak", "odd_grid_all_terms"])
def test_observables_match_oracle_on_identical_field(oracle, name):
    op, solver, d = make_pair(**STEP_CASES[name])
    g, fl = oracle.geometry(op)
    q = oracle.init(op, g, 0, 9, 0.6)
    q = fp32(oracle.step_explicit(op, g, fl, q, 300.0, 0.6, _dt(d, 300.0), n=20))
    solver.upload(q)
    got = solver.observe(300.0, 0.6)
    want = oracle.observe(op, g, fl, q, 300.0, 0.6)
    for k in ("bulk", "elastic", "anchoring", "total", "radiality", "avg_S", "max_S"):
        assert got[k] == pytest.approx(want[k], rel=1e-10, abs=1e-300), k
    for k in ("radiality_count", "core_count", "defect_count", "defect_plaquettes", "xi_edges"):
        assert got[k] == want[k], k
    for k in ("defect_density", "xi_grad_proxy", "checker_rel"):
        if math.isnan(want[k]):
            assert math.isnan(got[k]), k
        else:
            assert got[k] == pytest.approx(want[k], rel=1e-9), k
    assert got["nonfinite_cells"] == 0


def test_nematic_matches_oracle(oracle):
    op, solver, d = make_pair(Nx=16, Ny=12, Nz=20, L1=6e-12)
    g, fl = oracle.geometry(op)
    q = fp32(oracle.init(op, g, 0, 3, 0.5))
    solver.upload(q)
    got = solver.nematic()
    want = oracle.nematic(q)
    assert np.abs(got - want).max() < 1e-12


def test_long_run_fp32_error_budget(oracle):
    # 2000 explicit steps, L1 + strong anchoring, equilibrium shell order.
    op, solver, d = make_pair(Nx=32, Ny=32, Nz=32, L1=6e-12, T_star=307.0)
    g, fl = oracle.geometry(op)
    T = 300.0
    S_shell = S_eq(*bulk_ABC(d["a"], d["b"], d["c"], T, d["T_star"]))
    q0 = fp32(oracle.init(op, g, 0, 42, 0.5))
    dt = _dt(d, T)
    solver.upload(q0)
    solver.step(2000, T, S_shell, dt)
    got = solver.download()
    want = oracle.step_explicit(op, g, fl, q0, T, S_shell, dt, n=2000)
    assert rel_err(got, want) <= 1e-5
    assert rms_rel(got, want) <= 1e-6
    eg = solver.observe(T, S_shell)["total"]
    ew = oracle.observe(op, g, fl, want, T, S_shell)["total"]
    assert eg == pytest.approx(ew, rel=1e-6)


@pytest.mark.parametrize("grid", [dict(Nx=8, Ny=8, Nz=8), dict(Nx=12, Ny=20, Nz=72, droplet_radius_cells=9.0)])
def test_noise_stream_matches_philox_box_muller(oracle, grid):
    # With Q = 0, A = 0 (T = T*) and no gradients the update is the noise alone, so the device
    # noise can be read back and compared with Philox4x32-7 + Box-Muller evaluated here. The
    # device radius uses the hardware base-2 logarithm (absolute error <= 2^-22 near u = 1), so a
    # normal may be off by 2e-4 in absolute terms where |z| is tiny, 1e-5 relative elsewhere.
    # The second grid has tiles on the face-free interior path.
    op, solver, d = make_pair(L1=6e-12, W=1e-5, **grid)
    g, fl = oracle.geometry(op)
    solver.upload(np.zeros(5 * grid["Nx"] * grid["Ny"] * grid["Nz"]))
    sigma, seed, step = 1e-3, 0x1234ABCD5678EF01, 17
    solver.step(1, d["T_star"], 0.0, 1e-12, noise_sigma=sigma, seed=seed, step_index=step)
    got = solver.download().reshape(-1, 5)
    move = (fl & 2) != 0  # evolving cells (ORC_EVOLVE with W > 0)
    k0, k1 = seed & 0xFFFFFFFF, seed >> 32
    idx = np.flatnonzero(move)
    m21 = (1 << 21) - 1
    for cell in idx[:: max(1, len(idx) // 40)]:
        w = oracle.philox([int(cell), 0, step & 0xFFFFFFFF, step >> 32], [k0, k1], rounds=7)
        f = [w[0] & m21, w[1] & m21, w[2] & m21, w[3] & m21, ((w[0] >> 21) << 10) | (w[1] >> 22),
             ((w[2] >> 21) << 10) | (w[3] >> 22)]
        u = [(x + 1.0) / 2097152.0 for x in f]
        r = [math.sqrt(-2.0 * math.log(u[0])), math.sqrt(-2.0 * math.log(u[2])), math.sqrt(-2.0 * math.log(u[4]))]
        z = [r[0] * math.cos(2 * math.pi * u[1]), r[0] * math.sin(2 * math.pi * u[1]),
             r[1] * math.cos(2 * math.pi * u[3]), r[1] * math.sin(2 * math.pi * u[3]),
             r[2] * math.cos(2 * math.pi * u[5])]
        assert np.allclose(got[cell], sigma * np.array(z), rtol=2e-5, atol=2e-4 * sigma)
    assert np.all(got[~move] == 0.0)
    # distribution: zero mean, unit variance over all evolving cells and components
    zs = got[move].ravel() / sigma
    assert abs(zs.mean()) < 0.1 and abs(zs.var() - 1.0) < 0.15


def test_step_rejects_bad_arguments(oracle):
    from lcdrsimulator_b200 import LdgError
    op, solver, d = make_pair(Nx=8, Ny=8, Nz=8)
    with pytest.raises(LdgError, match="no field"):
        solver.step(1, 300.0, 0.5, 1e-10)
    solver.upload(np.zeros(5 * 512))
    with pytest.raises(LdgError, match="dt"):
        solver.step(1, 300.0, 0.5, -1.0)
    with pytest.raises(LdgError, match="expected"):
        solver.upload(np.zeros(10))


@pytest.mark.parametrize("name", ["L1L2L3_weak", "odd_grid_all_terms", "radius_override_weak", "L1_strong"])
def test_tiled_matches_direct_kernel(oracle, name, monkeypatch):
    # The TMA-tiled kernel (default) and the direct kernel evaluate the same arithmetic.
    op, solver, d = make_pair(**STEP_CASES[name])
    g, fl = oracle.geometry(op)
    q0 = fp32(oracle.init(op, g, 0, 21, 0.5))
    dt = _dt(d, 302.0)
    solver.upload(q0)
    solver.step(7, 302.0, 0.6, dt)
    tiled = solver.download()
    solver.close()
    monkeypatch.setenv("LDG_QSR_KERNEL", "direct")
    op2, solver2, _ = make_pair(**STEP_CASES[name])
    solver2.upload(q0)
    solver2.step(7, 302.0, 0.6, dt)
    direct = solver2.download()
    solver2.close()
    assert rel_err(tiled, direct) <= 1e-6
    want = oracle.step_explicit(op, g, fl, q0, 302.0, 0.6, dt, n=7)
    assert rel_err(tiled, want) <= 2e-6


def test_tiled_plan_counts(oracle):
    op, solver, d = make_pair(Nx=64, Ny=64, Nz=64, droplet_radius_cells=20.0, L1=6e-12, W=1e-5)
    geo = solver.geometry()
    g, fl = oracle.geometry(op)
    assert geo["written_cells"] == int(((fl & 2) != 0).sum())  # W > 0: moving cells only
    assert geo["written_cells"] <= geo["active_cells"] < geo["box_cells"]


def test_compensated_storage_round_trip_and_steps(oracle):
    # upload / download keep ~48 bits; a few steps stay at the FP32 parity bar
    op, solver, d = make_pair(Nx=20, Ny=24, Nz=36, L1=6e-12, L2=3e-12, W=1e-5, compensated=1)
    g, fl = oracle.geometry(op)
    q0 = np.asarray(oracle.init(op, g, 0, 3, 0.5))
    solver.upload(q0)
    assert np.abs(solver.download() - q0).max() <= 1e-13 * np.abs(q0).max()
    T, S_shell = 302.0, 0.6
    dt = _dt(d, T)
    solver.step(5, T, S_shell, dt)
    want = oracle.step_explicit(op, g, fl, q0, T, S_shell, dt, n=5)
    assert rel_err(solver.download(), want) <= 2e-6
    # an IMEX step drops the low words: the field continues from its high words
    solver.step(1, T, S_shell, dt, semi_implicit=True, L_stab=d["L1"], jacobi_iters=3)
    q1 = solver.download()
    solver.upload(q1)
    assert np.array_equal(np.asarray(q1, np.float32).astype(np.float64), q1)


def test_autotune_restores_field_and_keeps_results(oracle):
    op, solver, d = make_pair(**STEP_CASES["interior_tiles_L1L2L3_weak"])
    g, fl = oracle.geometry(op)
    q0 = fp32(oracle.init(op, g, 0, 11, 0.5))
    T, S_shell = 302.0, 0.6
    dt = _dt(d, T)
    solver.upload(q0)
    n0 = solver.launch_count()
    chunk = solver.autotune(T, S_shell, dt, trial_steps=3)
    assert chunk in (8, 12, 16, 24, 32, 48, 64)
    assert solver.launch_count() == n0
    assert np.array_equal(solver.download(), q0)
    solver.step(4, T, S_shell, dt)
    want = oracle.step_explicit(op, g, fl, q0, T, S_shell, dt, n=4)
    assert rel_err(solver.download(), want) <= 2e-6
