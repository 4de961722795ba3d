"""The host programs' text writers and warm-start reader against the reference's own (CPU only).

saveQTensorToFile and saveNematicFieldToFile (QSR.cu:1802-1832) are compiled from the reference
sources into oracle/_ref/qsr_cuda_ref.so (host code); the host programs' parallel writers
(lcdrsimulator_b200/host/host_common.hpp) are exported by oracle/host_shim.cpp. On the same
field both must write the same bytes. The warm-start reader (the init_file key) must read a
Qtensor_output file back to its %.6e precision, and report how far the file is from a
traceless symmetric tensor.
"""
import ctypes as C
import os

import numpy as np
import pytest

from oracle.oracle import BUILD, REF

_dp = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def ref():
    path = os.path.join(REF, "qsr_cuda_ref.so")
    if not os.path.exists(path):
        pytest.skip("reference QSR.cu build (oracle/_ref) not available")
    L = C.CDLL(path)
    for f in (L.qref_save_qtensor, L.qref_save_nematic):
        f.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_char_p]
    return L


@pytest.fixture(scope="module")
def shim(oracle):
    L = C.CDLL(os.path.join(BUILD, "libhost_shim.so"))
    for f in (L.hshim_save_qtensor, L.hshim_save_nematic):
        f.argtypes = [_dp, C.c_int, C.c_int, C.c_int, C.c_char_p]
    L.hshim_load_qtensor.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, _dp, _dp]
    return L


def _field(shape, seed):
    rng = np.random.default_rng(seed)
    n = int(np.prod(shape))
    q = rng.normal(0.0, 0.3, 5 * n)
    q[rng.random(5 * n) < 0.1] = 0.0           # exact zeros (cells outside a droplet)
    q[:5] = [1e-300, -0.0, 1e300, 123456.789, -5e-7]  # extreme exponents and signed zero
    return q


@pytest.mark.parametrize("shape", [(7, 5, 9), (16, 16, 16), (40, 3, 33)])
def test_qtensor_writer_bytes_equal_reference(ref, shim, tmp_path, shape):
    q = _field(shape, sum(shape))
    a, b = tmp_path / "ref.dat", tmp_path / "ours.dat"
    ref.qref_save_qtensor(q.ctypes.data_as(_dp), *shape, str(a).encode())
    assert shim.hshim_save_qtensor(q.ctypes.data_as(_dp), *shape, str(b).encode()) == 0
    assert a.read_bytes() == b.read_bytes()


@pytest.mark.parametrize("shape", [(7, 5, 9), (64, 32, 48)])
def test_nematic_writer_bytes_equal_reference(ref, shim, tmp_path, shape):
    rng = np.random.default_rng(3)
    s_n = rng.normal(0.0, 1.0, 4 * int(np.prod(shape)))
    a, b = tmp_path / "ref.dat", tmp_path / "ours.dat"
    ref.qref_save_nematic(s_n.ctypes.data_as(_dp), *shape, str(a).encode())
    assert shim.hshim_save_nematic(s_n.ctypes.data_as(_dp), *shape, str(b).encode()) == 0
    assert a.read_bytes() == b.read_bytes()


def test_warm_start_reader_round_trip(ref, shim, tmp_path):
    shape = (12, 10, 14)
    n = int(np.prod(shape))
    q = np.random.default_rng(11).normal(0.0, 0.3, 5 * n)
    path = tmp_path / "Qtensor_output_final.dat"
    ref.qref_save_qtensor(q.ctypes.data_as(_dp), *shape, str(path).encode())
    got = np.zeros(5 * n)
    chk = np.zeros(3)
    assert shim.hshim_load_qtensor(str(path).encode(), *shape, got.ctypes.data_as(_dp), chk.ctypes.data_as(_dp)) == 0
    # %.6e keeps 7 significant digits: every value back to half a unit of its last digit
    assert np.all(np.abs(got - q) <= 5.0001e-7 * np.abs(q) + 1e-300)
    # a reference-written file is traceless and symmetric up to that rounding
    assert chk[1] == 0.0
    assert chk[0] <= 3e-6 * chk[2]


def test_warm_start_reader_reports_a_non_traceless_file(shim, tmp_path):
    path = tmp_path / "bad.dat"
    rows = []
    for i in range(2):
        for j in range(2):
            for k in range(2):
                rows.append(f"{i} {j} {k} 0.3 0.1 0 0.1 0.2 0 0 0 0.1\n")  # trace 0.6
    path.write_text("".join(rows))
    got = np.zeros(40)
    chk = np.zeros(3)
    assert shim.hshim_load_qtensor(str(path).encode(), 2, 2, 2, got.ctypes.data_as(_dp), chk.ctypes.data_as(_dp)) == 0
    assert chk[0] == pytest.approx(0.6) and chk[1] == 0.0 and chk[2] == pytest.approx(0.3)
    # malformed files are rejected
    path.write_text("0 0 0 1 2 3\n")
    assert shim.hshim_load_qtensor(str(path).encode(), 1, 1, 1, got.ctypes.data_as(_dp), chk.ctypes.data_as(_dp)) == 1
