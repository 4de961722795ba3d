"""The no-allocation observables entry point against the regular one (GPU).

kzm_observe_device_noalloc serves callers that keep the field in their own device memory and
must not allocate (a framework that owns the device memory pool, or a loop being captured into
a CUDA graph): it reads the caller's device array and uses the library's fixed scratch array.
This file is collected last so that a failure here never hides the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _field(oracle):
    from oracle.oracle import OrcBulkParams
    from lcdrsimulator_b200.physics import bulk_ABC
    bp = OrcBulkParams(24, 20, 16, 1e-8, 1.1e-8, 0.9e-8, 6e-12, 0.1, 1e-10, 0.0, 0.1, 0.25)
    A, B, Cc = bulk_ABC(0.044e6, 1.413e6, 1.153e6, 295.0, 307.0)
    q = oracle.bulk_init(bp, 99, 0.3)
    q = oracle.bulk_step(bp, q, A, B, Cc, n=50)
    return bp, np.asarray(q, np.float32).astype(np.float64), (A, B, Cc)


def test_noalloc_observables_match_regular_entry_point(oracle):
    import torch
    import lcdrsimulator_b200 as L

    bp, q, (A, B, Cc) = _field(oracle)
    solver = L.KZMSolver(bp.Nx, bp.Ny, bp.Nz, bp.dx, bp.dy, bp.dz, bp.kappa, bp.gamma)
    solver.upload(q)
    want = solver.observe(A, B, Cc)
    solver.close()
    assert want["nonzero_defect_plaquettes"] > 0

    lib = L.load_library()
    fn = lib.kzm_observe_device_noalloc
    fn.argtypes = [C.POINTER(L.KzmParams), C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p,
                   C.POINTER(L.KzmObservables)]
    params = L.KzmParams(bp.Nx, bp.Ny, bp.Nz, bp.dx, bp.dy, bp.dz, bp.kappa, bp.gamma, 0.0, 0.1, 0.25)
    q_dev = torch.tensor(q, dtype=torch.float64, device="cuda")  # the caller's own device field
    torch.cuda.synchronize()
    for _ in range(2):  # two calls in a row share the scratch array
        out = L.KzmObservables()
        rc = fn(C.byref(params), C.c_void_p(q_dev.data_ptr()), A, B, Cc, None, C.byref(out))
        assert rc == 0, lib.ldg_last_error()
        got = out.as_dict()
        for k in ("bulk", "elastic", "total", "avg_S", "max_S", "defect_density_per_plaquette",
                  "defect_line_density", "xi_grad_proxy"):
            assert got[k] == pytest.approx(want[k], rel=1e-10), k
        for k in ("defect_plaquettes_used", "nonzero_defect_plaquettes"):
            assert got[k] == want[k], k


def test_noalloc_rejects_grids_beyond_scratch_limit():
    import lcdrsimulator_b200 as L

    lib = L.load_library()
    fn = lib.kzm_observe_device_noalloc
    fn.argtypes = [C.POINTER(L.KzmParams), C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p,
                   C.POINTER(L.KzmObservables)]
    params = L.KzmParams(81, 81, 81, 1e-8, 1e-8, 1e-8, 6e-12, 0.1, 0.0, 0.1, 0.25)  # 531441 > 2^19 sites
    out = L.KzmObservables()
    rc = fn(C.byref(params), C.c_void_p(16), 0.0, 0.0, 0.0, None, C.byref(out))
    assert rc == 1  # LDG_ERR_ARG, before any device access
    assert b"scratch limit" in lib.ldg_last_error()
