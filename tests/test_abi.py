"""The C-ABI library loads on a machine without a GPU and exports every declared symbol."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    src = open(os.path.join(ROOT, "include", "ldg_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z_0-9]*\s*\*?\s*([a-z_][a-z_0-9]*)\s*\(", src, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    for n in ("qsr_create", "qsr_step", "qsr_observe", "qsr_download", "kzm_step", "ldg_last_error"):
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    for n in declared_functions():
        assert hasattr(lib, n), f"libldg_b200.so does not export {n}"


def test_library_exports_with_nm(lib):
    from lcdrsimulator_b200 import library_path
    out = subprocess.run(["nm", "-D", "--defined-only", library_path()], capture_output=True, text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if l.strip())
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing


def test_version_and_error_without_compute(lib):
    lib.ldg_version.restype = ctypes.c_char_p
    assert b"sm_100a" in lib.ldg_version()
    # argument validation happens before any device call
    import lcdrsimulator_b200 as L
    p = L.QsrParams()
    p.Nx, p.Ny, p.Nz = 2, 8, 8
    h = ctypes.c_void_p()
    rc = lib.qsr_create(ctypes.byref(p), ctypes.byref(h))
    assert rc == 1  # LDG_ERR_ARG
    assert b">= 3" in lib.ldg_last_error()


def test_product_does_not_reference_oracle():
    # the product package never imports, loads or links the oracle
    pkg = os.path.join(ROOT, "lcdrsimulator_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".cpp", ".h")):
                text = open(os.path.join(dirpath, f), errors="replace").read()
                assert "oracle" not in text.lower(), f
