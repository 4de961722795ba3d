"""GPU parity of the droplet ensemble (one persistent launch per step over many droplets).

Each instance of an ensemble must follow the same trajectory as a standalone solver stepped
one step at a time with the reference's quench protocol (QSR.cu:2679-2687): temperature per
step, equilibrium or custom shell order, Philox noise keyed by the instance seed. Both run the
same per-tile routine, so the comparison tolerance (relative to max |Q|) is 2e-6, the FP32
bar; one instance is also checked against the FP64 oracle.
"""
import numpy as np
import pytest

from gpu_helpers import fp32, rel_err
from oracle.oracle import make_params
from lcdrsimulator_b200 import EnsembleSolver, QSRSolver, LdgError, QsrObserveArgs
from lcdrsimulator_b200.physics import bulk_ABC, S_eq

pytestmark = pytest.mark.gpu

MATERIAL = dict(dx=1e-8, dy=1e-8, dz=1e-8, a=0.044e6, b=1.413e6, c=1.153e6, T_star=307.0, bulk_modechoice=1,
                gamma=0.1)

CASES = {
    # weak anchoring, all elastic terms, linear ramp, custom shell order
    "weak_L1L2L3_ramp_custom": dict(
        params=dict(kappa=0.0, L1=6e-12, L2=3e-12, L3=1e-12, W=1e-5, dt=1.5e-10, q_norm_cap=0.0,
                    boundary_custom=1, boundary_S=0.6, protocol=2),
        instances=[dict(N=20, T_high=312.0, T_low=300.0, pre_equil_iters=5, ramp_iters=20, seed=11),
                   dict(N=24, T_high=310.0, T_low=302.0, pre_equil_iters=0, ramp_iters=30, seed=12),
                   dict(N=28, droplet_radius_cells=10.0, T_high=309.0, T_low=301.0, pre_equil_iters=12,
                        ramp_iters=7, seed=13),
                   # large enough for tiles on the face-free interior path
                   dict(N=72, droplet_radius_cells=30.0, T_high=311.0, T_low=299.0, pre_equil_iters=3,
                        ramp_iters=25, seed=14)]),
    # strong anchoring, L1 only, step quench, equilibrium shell order S_eq(T)
    "strong_L1_step_equilibrium": dict(
        params=dict(kappa=0.0, L1=6e-12, L2=0.0, L3=0.0, W=0.0, dt=1.5e-10, q_norm_cap=0.0,
                    boundary_custom=0, boundary_S=0.0, protocol=1),
        instances=[dict(N=16, T_high=312.0, T_low=300.0, pre_equil_iters=10, ramp_iters=0, seed=3),
                   dict(N=22, T_high=311.0, T_low=296.0, pre_equil_iters=20, ramp_iters=0, seed=4)]),
}


def temperature(inst, protocol, it):
    if it < inst["pre_equil_iters"]:
        return inst["T_high"]
    if protocol == 1:
        return inst["T_low"]
    t = it - inst["pre_equil_iters"]
    if t <= 0:
        return inst["T_high"]
    if t >= inst["ramp_iters"]:
        return inst["T_low"]
    return inst["T_high"] + (inst["T_low"] - inst["T_high"]) * (t / inst["ramp_iters"])


def shell_order(p, T):
    if p["boundary_custom"]:
        return p["boundary_S"]
    return max(S_eq(*bulk_ABC(p["a"], p["b"], p["c"], T, p["T_star"], p["bulk_modechoice"])), 0.0)


def standalone(p, inst):
    return QSRSolver(Nx=inst["N"], Ny=inst["N"], Nz=inst["N"], dx=p["dx"], dy=p["dy"], dz=p["dz"], a=p["a"],
                     b=p["b"], c=p["c"], T_star=p["T_star"], bulk_modechoice=p["bulk_modechoice"], kappa=p["kappa"],
                     L1=p["L1"], L2=p["L2"], L3=p["L3"], W=p["W"], gamma=p["gamma"],
                     droplet_radius_cells=inst.get("droplet_radius_cells", 0.0))


def run_standalone(p, inst, q0, n_steps):
    s = standalone(p, inst)
    s.upload(q0)
    for it in range(n_steps):
        T = temperature(inst, p["protocol"], it)
        s.step(1, T, shell_order(p, T), p["dt"], q_norm_cap=p["q_norm_cap"],
               noise_sigma=inst.get("noise_sigma", 0.0), seed=inst["seed"], step_index=it)
    out = s.download()
    s.close()
    return out


def build(case, **override):
    c = CASES[case]
    p = dict(MATERIAL)
    p.update(c["params"])
    p.update(override)
    instances = [dict(EnsembleSolver.INSTANCE_DEFAULTS, **i) for i in c["instances"]]
    return p, instances


@pytest.mark.parametrize("case", list(CASES))
def test_ensemble_matches_standalone_steps(case):
    p, instances = build(case)
    n_steps = 45   # one captured graph of 32 launches plus 13 direct launches
    ens = EnsembleSolver(instances, **p)
    ens.initial_fields(init_mode=0, S0=0.5)
    q0 = [ens.download(n) for n in range(len(instances))]
    ens.step(n_steps)
    assert ens.step_index == n_steps
    for n, inst in enumerate(instances):
        got = ens.download(n)
        want = run_standalone(p, inst, q0[n], n_steps)
        assert rel_err(got, want) <= 2e-6, (case, n, rel_err(got, want))
        assert np.abs(got - q0[n]).max() > 0.0
    ens.close()


def test_ensemble_noise_matches_standalone():
    p, instances = build("weak_L1L2L3_ramp_custom")
    for n, inst in enumerate(instances):
        inst["noise_sigma"] = 2e-3 * (n + 1)
    ens = EnsembleSolver(instances, **p)
    ens.initial_fields(init_mode=1, S0=0.5)
    q0 = [ens.download(n) for n in range(len(instances))]
    ens.step(7)
    ens.step(30)
    for n, inst in enumerate(instances):
        got = ens.download(n)
        want = run_standalone(p, inst, q0[n], 37)
        assert rel_err(got, want) <= 2e-6, (n, rel_err(got, want))
    # distinct seeds give distinct noise: two identical droplets with different seeds diverge
    same = [dict(instances[0], seed=1), dict(instances[0], seed=2)]
    e2 = EnsembleSolver(same, **p)
    e2.initial_fields(init_mode=1, S0=0.5)
    e2.step(3)
    assert np.abs(e2.download(0) - e2.download(1)).max() > 1e-5
    e2.close()
    ens.close()


def test_ensemble_instance_matches_oracle(oracle):
    # constant temperature (step protocol, no pre-equilibration): plain explicit relaxation
    p, instances = build("weak_L1L2L3_ramp_custom", protocol=1)
    inst = dict(instances[1], pre_equil_iters=0)
    ens = EnsembleSolver([instances[0], inst], **p)
    op = make_params(Nx=inst["N"], Ny=inst["N"], Nz=inst["N"], T_star=p["T_star"], L1=p["L1"], L2=p["L2"],
                     L3=p["L3"], W=p["W"], kappa=p["kappa"])
    g, fl = oracle.geometry(op)
    q0 = fp32(oracle.init(op, g, 0, 42, 0.5))
    ens.initial_fields()
    ens.upload(1, q0)
    ens.step(6)
    want = oracle.step_explicit(op, g, fl, q0, inst["T_low"], p["boundary_S"], p["dt"], n=6)
    assert rel_err(ens.download(1), want) <= 2e-6
    ens.close()


def test_ensemble_autotune_restores_state():
    p, instances = build("weak_L1L2L3_ramp_custom")
    ens = EnsembleSolver(instances, **p)
    ens.initial_fields(init_mode=0, S0=0.5)
    ens.step(9)
    before = [ens.download(n) for n in range(len(instances))]
    chunk = ens.autotune(trial_steps=3)
    assert chunk in (8, 12, 16, 24, 32, 48, 64)
    assert ens.step_index == 9
    for n in range(len(instances)):
        assert np.array_equal(ens.download(n), before[n])
    ens.step(20)
    ref = EnsembleSolver(instances, **p)
    ref.initial_fields(init_mode=0, S0=0.5)
    ref.step(29)
    for n in range(len(instances)):
        assert rel_err(ens.download(n), ref.download(n)) <= 2e-6
    ens.close()
    ref.close()


def test_ensemble_observe_defaults_and_counts():
    p, instances = build("strong_L1_step_equilibrium")
    ens = EnsembleSolver(instances, **p)
    ens.initial_fields(init_mode=1, S0=0.5)
    ens.step(12)
    inst = instances[1]
    T = temperature(inst, p["protocol"], 12)
    N = inst["N"]
    a = QsrObserveArgs(T, shell_order(p, T), N // 2, 0.1, 0.25, N // 2, 0.1, 1, 1)
    o_def = ens.observe(1)
    o_exp = ens.observe(1, a)
    for k in ("bulk", "elastic", "anchoring", "total", "avg_S", "max_S", "radiality"):
        assert o_def[k] == o_exp[k], k
    s = standalone(p, inst)
    s.upload(ens.download(1))
    o_one = s.observe(T, shell_order(p, T))
    s.close()
    assert o_def["total"] == pytest.approx(o_one["total"], rel=1e-12)
    c = ens.counts()
    assert c["cells"] == sum(i["N"] ** 3 for i in instances)
    assert 0 < c["written_cells"] <= c["active_cells"] <= c["cells"]
    n0 = ens.launch_count()
    ens.step(40)
    assert ens.launch_count() - n0 == 40
    ens.close()


def test_ensemble_bad_arguments():
    p, instances = build("strong_L1_step_equilibrium")
    with pytest.raises(LdgError):
        EnsembleSolver([dict(instances[0], N=2)], **p)
    with pytest.raises(LdgError):
        EnsembleSolver(instances, **dict(p, protocol=5))
    with pytest.raises(LdgError):
        EnsembleSolver(instances, **dict(p, dt=0.0))
    ens = EnsembleSolver(instances, **p)
    with pytest.raises(LdgError):
        ens.step(1)                      # no field uploaded yet
    ens.initial_fields()
    with pytest.raises(LdgError):
        ens.download(len(instances))     # instance out of range (host side)
    import ctypes
    from lcdrsimulator_b200 import load_library
    buf = np.zeros(5 * 8)
    lib = load_library()
    assert lib.ens_download(ens.handle, len(instances), buf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))) == 1
    assert b"out of range" in lib.ldg_last_error()
    with pytest.raises(LdgError):
        ens.upload(0, np.zeros(7))
    ens.close()


def test_observe_all_matches_per_droplet_observe():
    p, instances = build("weak_L1L2L3_ramp_custom")
    ens = EnsembleSolver(instances, **p)
    ens.initial_fields(init_mode=0, S0=0.5)
    ens.step(17)
    every = ens.observe_all()
    assert len(every) == len(instances)
    for n in range(len(instances)):
        one = ens.observe(n)
        for k, v in one.items():   # checker_rel is NaN when no cell has a checkerboard pattern
            assert every[n][k] == v or (np.isnan(v) and np.isnan(every[n][k])), (n, k)
    ens.close()
