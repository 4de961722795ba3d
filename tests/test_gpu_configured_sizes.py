"""Parity at the workloads' own sizes (default GPU suite), against the reference's FP64 kernels.

* Anisotropic weak-anchoring relaxation at its full size: 256^3 grid, droplet R = 120 cells,
  L1/L2/L3 = 6/3/1e-12 N, W = 1e-5 J/m^2, boundary_S = 0.6, T = 302 K, random directors S0 = 0.5
  (seed 42), dt_max; 1000 explicit steps of this library (plain FP32 and compensated storage)
  against the reference's own FP64 CUDA chain (QSR.cu kernels compiled from the reference sources
  into oracle/_ref/, launched in the order of its time loop, QSR.cu:2713-2753).
* Plain single-temperature relaxation at its full length: 64^3 grid, R = 28 cells, L1 = 6e-12 N,
  strong anchoring with the equilibrium shell order, T = 300 K, 20,000 steps at dt_max, against the
  same reference chain, with the FP64 oracle checked at the 1000-step mark.
* Rounding-sensitivity control at 128^3 (R = 60 cells, the anisotropic physics): the reference's
  FP64 chain is run twice, once from a field moved by one FP64 ulp per value. How far two FP64
  runs that differ only by rounding drift apart at a point is the floor of any pointwise field
  comparison through the defect annihilations of a relaxation from random directors.

Bars (relative to max |Q| for the field, to |F| for the free energy): the configuration's
field error <= 1e-5 and free energy <= 1e-7. Measured rows are written as JSON to
$LDG_ACCURACY_OUT.<name> when that variable is set.
"""
import json
import os

import numpy as np
import pytest

from gpu_helpers import make_pair, fp32, rel_err, rms_rel
from lcdrsimulator_b200.physics import DtRequest, estimate_stable_dt_window, equilibrium_shell_order

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refcuda():
    from oracle.oracle import RefCUDA
    try:
        return RefCUDA()
    except FileNotFoundError:
        pytest.skip("reference CUDA build (oracle/_ref/qsr_cuda_ref.so) not available")


def _dt(d, T):
    r = DtRequest(dx=d["dx"], dy=d["dy"], dz=d["dz"], gamma=d["gamma"], a=d["a"], b=d["b"], c=d["c"],
                  T_star=d["T_star"], modechoice=d["bulk_modechoice"], kappa=d["kappa"], L1=d["L1"], L2=d["L2"],
                  L3=d["L3"], S0=0.5, T_a=T, T_b=T)
    return estimate_stable_dt_window(r)["dt_max"]


def _record(name, payload):
    out = os.environ.get("LDG_ACCURACY_OUT")
    if out:
        with open(f"{out}.{name}", "w") as f:
            json.dump(payload, f)


def _compare(solvers, ref, T, S_shell, Nz):
    want = ref.download()
    o = ref.observe(T, S_shell, Nz // 2)
    F_ref = o["bulk"] + o["elastic"] + o["anchoring"]
    row = dict(F_ref=F_ref)
    for name, s in solvers:
        got = s.download()
        F = s.observe(T, S_shell)["total"]
        row[name] = dict(field_max=rel_err(got, want), field_rms=rms_rel(got, want),
                         energy=abs(F - F_ref) / abs(F_ref))
    return row, want


C2 = dict(Nx=256, Ny=256, Nz=256, kappa=0.0, L1=6e-12, L2=3e-12, L3=1e-12, W=1e-5, droplet_radius_cells=120.0)


def test_anisotropic_weak_256_full_size_1000_steps(refcuda):
    T, S_shell, steps = 302.0, 0.6, 1000
    op, plain, d = make_pair(compensated=0, **C2)
    _, comp, _ = make_pair(compensated=1, **C2)
    dt = _dt(d, T)
    q0 = fp32(plain.initial_field(0, 42, 0.5))
    for s in (plain, comp):
        s.upload(q0)
        s.step(steps, T, S_shell, dt)
    refcuda.create(op)
    refcuda.upload(q0)
    refcuda.time_steps(T, S_shell, dt, steps)
    row, _ = _compare((("fp32", plain), ("compensated", comp)), refcuda, T, S_shell, C2["Nz"])
    refcuda.destroy()
    plain.close()
    comp.close()
    _record("anisotropic_weak_256_1000", dict(case=C2, T=T, S_shell=S_shell, dt=dt, steps=steps, row=row))
    p, c = row["fp32"], row["compensated"]
    assert p["field_max"] <= 1e-5 and p["field_rms"] <= 1e-6 and p["energy"] <= 1e-7, row
    assert c["field_max"] <= 1e-6 and c["field_rms"] <= 1e-7 and c["energy"] <= 1e-8, row


C1 = dict(Nx=64, Ny=64, Nz=64, kappa=0.0, L1=6e-12, droplet_radius_cells=28.0)
C1_CHECKS = [1000, 5000, 10000, 20000]


def test_plain_relaxation_64_full_length_20k_steps(refcuda, oracle):
    T, steps = 300.0, 20000
    op, plain, d = make_pair(compensated=0, **C1)
    _, comp, _ = make_pair(compensated=1, **C1)
    S_shell = equilibrium_shell_order(d["a"], d["b"], d["c"], T, d["T_star"], d["bulk_modechoice"])
    dt = _dt(d, T)
    q0 = fp32(plain.initial_field(0, 42, 0.5))
    for s in (plain, comp):
        s.upload(q0)
    refcuda.create(op)
    refcuda.upload(q0)
    g, fl = oracle.geometry(op)
    rows = []
    done = 0
    for t in C1_CHECKS:
        for s in (plain, comp):
            s.step(t - done, T, S_shell, dt)
        refcuda.time_steps(T, S_shell, dt, t - done)
        done = t
        row, want = _compare((("fp32", plain), ("compensated", comp)), refcuda, T, S_shell, C1["Nz"])
        row["step"] = t
        if t == C1_CHECKS[0]:
            # the FP64 oracle equals the reference chain along the same trajectory
            q_orc = oracle.step_explicit(op, g, fl, q0, T, S_shell, dt, n=t)
            row["oracle_vs_reference"] = rel_err(q_orc, want)
        rows.append(row)
    refcuda.destroy()
    plain.close()
    comp.close()
    _record("plain_relaxation_64_20k", dict(case=C1, T=T, S_shell=S_shell, dt=dt, rows=rows))
    assert rows[0]["oracle_vs_reference"] <= 1e-12, rows[0]
    for row in rows:
        assert np.isfinite(row["F_ref"])
        assert row["compensated"]["energy"] <= 1e-7 and row["fp32"]["energy"] <= 1e-7, row
        assert row["compensated"]["field_rms"] <= 1e-5, row


CTRL = dict(Nx=128, Ny=128, Nz=128, kappa=0.0, L1=6e-12, L2=3e-12, L3=1e-12, W=1e-5, droplet_radius_cells=60.0)
CTRL_CHECKS = [1000, 2500, 5000, 10000, 20000]


def test_rounding_sensitivity_control_128(refcuda):
    """FP64 against FP64 (one ulp apart at the start) beside FP32 and compensated against FP64."""
    T, S_shell = 302.0, 0.6
    op, plain, d = make_pair(compensated=0, **CTRL)
    _, comp, _ = make_pair(compensated=1, **CTRL)
    dt = _dt(d, T)
    q0 = fp32(plain.initial_field(0, 42, 0.5))
    q_ulp = np.nextafter(q0, np.inf)
    for s in (plain, comp):
        s.upload(q0)
    # the perturbed FP64 trajectory first, recorded at every check
    refcuda.create(op)
    refcuda.upload(q_ulp)
    pert = []
    done = 0
    for t in CTRL_CHECKS:
        refcuda.time_steps(T, S_shell, dt, t - done)
        done = t
        pert.append(refcuda.download())
    refcuda.destroy()
    refcuda.create(op)
    refcuda.upload(q0)
    rows = []
    done = 0
    for n, t in enumerate(CTRL_CHECKS):
        for s in (plain, comp):
            s.step(t - done, T, S_shell, dt)
        refcuda.time_steps(T, S_shell, dt, t - done)
        done = t
        row, want = _compare((("fp32", plain), ("compensated", comp)), refcuda, T, S_shell, CTRL["Nz"])
        row["step"] = t
        row["fp64_one_ulp"] = dict(field_max=rel_err(pert[n], want), field_rms=rms_rel(pert[n], want))
        rows.append(row)
    refcuda.destroy()
    plain.close()
    comp.close()
    _record("rounding_control_128", dict(case=CTRL, T=T, S_shell=S_shell, dt=dt, rows=rows))
    for row in rows:
        assert np.isfinite(row["F_ref"])
        assert row["compensated"]["energy"] <= 1e-7, row
        assert row["fp32"]["energy"] <= 1e-6, row


INIT_CASES = [(24, 20, 28, 0.0, 0, 42), (24, 20, 28, 0.0, 1, 42), (24, 20, 28, 0.0, 2, 42),
              (33, 31, 17, 0.0, 0, 7), (64, 64, 64, 28.0, 0, 42), (40, 40, 40, 12.5, 2, 0)]


@pytest.mark.parametrize("case", INIT_CASES, ids=[f"{c[0]}x{c[1]}x{c[2]}_R{c[3]}_mode{c[4]}" for c in INIT_CASES])
def test_initial_field_equals_reference(refcuda, case):
    """qsr_initial_field against the reference's initializeQTensor / initializeIsotropicWithNoise
    (QSR.cu:1841-1904, compiled from the reference sources), byte for byte."""
    import ctypes as C
    Nx, Ny, Nz, R, mode, seed = case
    _, solver, d = make_pair(Nx=Nx, Ny=Ny, Nz=Nz, droplet_radius_cells=R)
    got = solver.initial_field(mode, seed, 0.5, 1e-3)
    solver.close()
    want = np.zeros(Nx * Ny * Nz * 5)
    dp = C.POINTER(C.c_double)
    f = refcuda.L.qref_init
    f.argtypes = [C.c_int] * 3 + [C.c_double] * 4 + [C.c_int, C.c_longlong, C.c_double, C.c_double, dp]
    f(Nx, Ny, Nz, d["dx"], d["dy"], d["dz"], R, mode, seed, 0.5, 1e-3, want.ctypes.data_as(dp))
    assert np.count_nonzero(want) > 0
    assert np.array_equal(got, want)
