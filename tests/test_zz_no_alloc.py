"""The no-allocation observables entry point against the regular one (GPU).

kzm_observe_device_noalloc serves callers that keep the field in their own device memory and
must not allocate: code inside another framework that has reserved the GPU's memory for its own
pool, and step loops that cannot take the device synchronisation of an allocation. It reads the
caller's device array and uses the library's fixed scratch array (at most 2^19 sites). This
file is collected last so that a failure here never hides the other tests.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS_F = ("bulk", "elastic", "total", "avg_S", "max_S", "defect_density_per_plaquette", "defect_line_density",
          "xi_grad_proxy")
KEYS_I = ("defect_plaquettes_used", "nonzero_defect_plaquettes")


def _entry():
    import lcdrsimulator_b200 as L
    lib = L.load_library()
    fn = lib.kzm_observe_device_noalloc
    fn.argtypes = [C.POINTER(L.KzmParams), C.c_void_p, C.c_double, C.c_double, C.c_double, C.c_void_p,
                   C.POINTER(L.KzmObservables)]
    return L, lib, fn


def _field(oracle, shape, d, seed, steps):
    from oracle.oracle import OrcBulkParams
    from lcdrsimulator_b200.physics import bulk_ABC
    bp = OrcBulkParams(*shape, *d, 6e-12, 0.1, 1e-10, 0.0, 0.1, 0.25)
    A, B, Cc = bulk_ABC(0.044e6, 1.413e6, 1.153e6, 295.0, 307.0)
    q = oracle.bulk_init(bp, seed, 0.3)
    q = oracle.bulk_step(bp, q, A, B, Cc, n=steps)
    return bp, np.asarray(q, np.float32).astype(np.float64), (A, B, Cc)


# a small ragged box, and 64 x 64 x 128 = 2^19 sites: the whole scratch array in use
CASES = {"ragged_24x20x16": ((24, 20, 16), (1e-8, 1.1e-8, 0.9e-8), 99, 50),
         "at_limit_64x64x128": ((64, 64, 128), (1e-8, 1e-8, 1e-8), 7, 10)}


@pytest.mark.parametrize("name", list(CASES))
def test_noalloc_observables_match_regular_entry_point(oracle, name):
    import torch
    L, lib, fn = _entry()
    shape, d, seed, steps = CASES[name]
    bp, q, (A, B, Cc) = _field(oracle, shape, d, seed, steps)
    solver = L.KZMSolver(bp.Nx, bp.Ny, bp.Nz, bp.dx, bp.dy, bp.dz, bp.kappa, bp.gamma)
    solver.upload(q)
    want = solver.observe(A, B, Cc)
    solver.close()
    assert want["nonzero_defect_plaquettes"] > 0

    params = L.KzmParams(bp.Nx, bp.Ny, bp.Nz, bp.dx, bp.dy, bp.dz, bp.kappa, bp.gamma, 0.0, 0.1, 0.25)
    q_dev = torch.tensor(q, dtype=torch.float64, device="cuda")  # the caller's own device field
    stream = torch.cuda.current_stream()
    torch.cuda.synchronize()
    free_after = []
    for _ in range(2):  # two calls in a row share the scratch array
        out = L.KzmObservables()
        rc = fn(C.byref(params), C.c_void_p(q_dev.data_ptr()), A, B, Cc, C.c_void_p(stream.cuda_stream),
                C.byref(out))
        assert rc == 0, lib.ldg_last_error()
        free_after.append(torch.cuda.mem_get_info()[0])
        got = out.as_dict()
        for k in KEYS_F:
            assert got[k] == pytest.approx(want[k], rel=1e-10), k
        for k in KEYS_I:
            assert got[k] == want[k], k
    # after the first call (which may load kernels) a call takes no device memory
    assert free_after[1] == free_after[0]


def test_noalloc_rejects_grids_beyond_scratch_limit():
    import torch
    L, lib, fn = _entry()
    n = 81 ** 3  # 531,441 > 2^19 sites
    params = L.KzmParams(81, 81, 81, 1e-8, 1e-8, 1e-8, 6e-12, 0.1, 0.0, 0.1, 0.25)
    # a real field of the full size: were the size guard ever bypassed, the kernels would read
    # valid memory and the test would fail on the return code, not fault
    q_dev = torch.zeros(5 * n, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    out = L.KzmObservables()
    rc = fn(C.byref(params), C.c_void_p(q_dev.data_ptr()), 0.0, 0.0, 0.0, None, C.byref(out))
    assert rc == 1  # LDG_ERR_ARG, before any device access
    assert b"scratch limit" in lib.ldg_last_error()
