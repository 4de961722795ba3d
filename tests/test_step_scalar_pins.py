"""Pins the step scalars and the seeded initial field to the reference's own functions (CPU only).

Three restatements of the reference's host scalars exist: ``lcdrsimulator_b200/physics.py``
(used by the Python driver and bench), ``lcdrsimulator_b200/host/host_common.hpp`` (used by the
drop-in host programs; exported for tests by ``oracle/host_shim.cpp``) and the FP64 oracle's
initialisation. Each is compared with the reference's own code, compiled from its sources into
``oracle/_ref/qsr_cuda_ref.so`` (host functions only; no GPU is used):
estimate_stable_dt_window (QSR.cu:1528-1604), resolve_boundary_shell_order (QSR.cu:1475-1487)
and initializeQTensor / initializeIsotropicWithNoise (QSR.cu:1841-1904). Every value must be
identical, not merely close: a different dt or shell order changes every trajectory.
"""
import ctypes as C
import math
import os

import numpy as np
import pytest

from lcdrsimulator_b200 import physics
from oracle.oracle import BUILD, REF, make_params

_dp = C.POINTER(C.c_double)
FIELDS = ["min_dx", "S_scale", "L_eff_total", "D_total", "dt_diff_total", "L_eff_explicit", "dt_diff", "bulk_rate",
          "dt_bulk", "dt_max", "semi_implicit_active"]


@pytest.fixture(scope="module")
def ref():
    path = os.path.join(REF, "qsr_cuda_ref.so")
    if not os.path.exists(path):
        pytest.skip("reference QSR.cu build (oracle/_ref) not available")
    L = C.CDLL(path)
    L.qref_shell_order.restype = C.c_double
    L.qref_shell_order.argtypes = [C.c_int] + [C.c_double] * 6 + [C.c_int]
    L.qref_dt_window.argtypes = [_dp, _dp]
    L.qref_init.argtypes = [C.c_int] * 3 + [C.c_double] * 4 + [C.c_int, C.c_longlong, C.c_double, C.c_double, _dp]
    return L


@pytest.fixture(scope="module")
def shim(oracle):
    L = C.CDLL(os.path.join(BUILD, "libhost_shim.so"))
    L.hshim_shell_order.restype = C.c_double
    L.hshim_shell_order.argtypes = [C.c_int] + [C.c_double] * 6 + [C.c_int]
    L.hshim_dt_window.argtypes = [_dp, _dp]
    return L


LDG = dict(a=0.044e6, b=1.413e6, c=1.153e6, T_star=307.0)
# (request, label): the five configurations' physics plus edge cases of every branch
DT_CASES = [
    (dict(dx=1e-8, dy=1e-8, dz=1e-8, gamma=0.1, modechoice=1, L1=6e-12, S0=0.5, T_a=300.0, T_b=300.0), "c1"),
    (dict(dx=1e-8, dy=1e-8, dz=1e-8, gamma=0.1, modechoice=1, L1=6e-12, L2=3e-12, L3=1e-12, S0=0.5, T_a=302.0,
          T_b=302.0), "c2"),
    (dict(dx=1e-8, dy=1e-8, dz=1e-8, gamma=0.1, modechoice=1, L1=6e-12, S0=0.5, T_a=315.0, T_b=295.0), "c3"),
    (dict(dx=1e-8, dy=1e-8, dz=1e-8, gamma=0.1, modechoice=1, kappa=6e-12, S0=0.5, T_a=315.0, T_b=295.0), "c5"),
    (dict(dx=1e-8, dy=1.2e-8, dz=9e-9, gamma=0.1, modechoice=2, L1=6e-12, L3=2e-12, S0=0.7, T_a=290.0, T_b=310.0),
     "ravnik_L3"),
    (dict(dx=1e-8, dy=1e-8, dz=1e-8, gamma=0.1, modechoice=1, L1=6e-12, S0=0.5, T_a=300.0, T_b=300.0,
          use_semi_implicit=True, L_stab=6e-12, jacobi_iters=25), "imex_full_stab"),
    (dict(dx=1e-8, dy=1e-8, dz=1e-8, gamma=0.1, modechoice=1, L1=6e-12, L2=-2e-12, S0=0.5, T_a=300.0, T_b=300.0,
          use_semi_implicit=True, L_stab=4e-12, jacobi_iters=10), "imex_partial_negative_L2"),
    (dict(dx=1e-8, dy=1e-8, dz=1e-8, gamma=0.05, modechoice=1, kappa=-6e-12, S0=0.0, T_a=330.0, T_b=330.0,
          use_semi_implicit=True, L_stab=6e-12, jacobi_iters=5), "kappa_negative_isotropic"),
    (dict(dx=2e-8, dy=2e-8, dz=2e-8, gamma=0.1, modechoice=1, L1=6e-12, S_ref_used=0.3, S0=0.5, T_a=300.0,
          T_b=300.0), "S_ref_used"),
    (dict(dx=1e-8, dy=1e-8, dz=1e-8, gamma=0.1, modechoice=1, S0=0.5, T_a=300.0, T_b=300.0), "no_elastic"),
]


def _req_array(r):
    d = physics.DtRequest(**{**LDG, **r})
    return d, np.array([d.dx, d.dy, d.dz, d.gamma, d.a, d.b, d.c, d.T_star, d.modechoice, d.kappa, d.L1, d.L2,
                        d.L3, d.S_ref_used, d.S0, d.T_a, d.T_b, 1.0 if d.use_semi_implicit else 0.0, d.L_stab,
                        d.jacobi_iters], dtype=np.float64)


def _same(a, b):
    return (math.isnan(a) and math.isnan(b)) or a == b


@pytest.mark.parametrize("case", DT_CASES, ids=[c[1] for c in DT_CASES])
def test_dt_window_equals_reference(ref, shim, case):
    d, arr = _req_array(case[0])
    want = np.zeros(11)
    ref.qref_dt_window(arr.ctypes.data_as(_dp), want.ctypes.data_as(_dp))
    got_host = np.zeros(11)
    shim.hshim_dt_window(arr.ctypes.data_as(_dp), got_host.ctypes.data_as(_dp))
    got_py = physics.estimate_stable_dt_window(d)
    for n, f in enumerate(FIELDS):
        assert _same(got_host[n], want[n]), (f, got_host[n], want[n])
        assert _same(float(got_py[f]), want[n]), (f, got_py[f], want[n])


SHELL_CASES = [(custom, S, T, mode) for custom in (0, 1) for S in (0.6, 0.0) for T in (290.0, 300.0, 307.5, 330.0)
               for mode in (1, 2)]


@pytest.mark.parametrize("custom,S,T,mode", SHELL_CASES)
def test_shell_order_equals_reference(ref, shim, custom, S, T, mode):
    args = (custom, S, LDG["a"], LDG["b"], LDG["c"], T, LDG["T_star"], mode)
    want = ref.qref_shell_order(*args)
    assert shim.hshim_shell_order(*args) == want
    policy = "custom" if custom else "equilibrium"
    assert physics.boundary_shell_order(policy, S, LDG["a"], LDG["b"], LDG["c"], T, LDG["T_star"], mode) == want


INIT_CASES = [
    (24, 20, 28, 1e-8, 1e-8, 1e-8, 0.0, 0, 42, 0.5),
    (24, 20, 28, 1e-8, 1e-8, 1e-8, 0.0, 1, 42, 0.5),
    (24, 20, 28, 1e-8, 1e-8, 1e-8, 0.0, 2, 42, 0.5),
    (33, 31, 17, 1e-8, 1.2e-8, 9e-9, 0.0, 0, 7, 0.3),
    (33, 31, 17, 1e-8, 1.2e-8, 9e-9, 0.0, 2, 123456789, 0.3),
    (64, 64, 64, 1e-8, 1e-8, 1e-8, 28.0, 0, 42, 0.5),
    (40, 40, 40, 1e-8, 1e-8, 1e-8, 12.5, 1, 3, 0.6),
    (40, 40, 40, 1e-8, 1e-8, 1e-8, 12.5, 2, 0, 0.6),
]


@pytest.mark.parametrize("case", INIT_CASES, ids=[f"{c[0]}x{c[1]}x{c[2]}_R{c[6]}_mode{c[7]}_seed{c[8]}"
                                                  for c in INIT_CASES])
def test_oracle_init_equals_reference(ref, oracle, case):
    Nx, Ny, Nz, dx, dy, dz, R, mode, seed, S0 = case
    amp = 1e-3
    want = np.zeros(Nx * Ny * Nz * 5)
    ref.qref_init(Nx, Ny, Nz, dx, dy, dz, R, mode, seed, S0, amp, want.ctypes.data_as(_dp))
    op = make_params(Nx=Nx, Ny=Ny, Nz=Nz, dx=dx, dy=dy, dz=dz, droplet_radius_cells=R)
    g, _ = oracle.geometry(op)
    got = oracle.init(op, g, mode, seed, S0, amp)
    assert np.count_nonzero(want) > 0
    assert np.array_equal(got, want)
