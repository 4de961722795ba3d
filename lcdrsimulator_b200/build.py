"""Build recipe of the native library and host programs (nvcc for sm_100a, in-tree outputs).

Outputs under ``lcdrsimulator_b200/_lib/``:
  * ``libldg_b200.so``   - the C-ABI library (include/ldg_b200.h)
  * ``qsr_b200``         - drop-in host program for ``QSR_cuda --config``
  * ``kzm_bulk_ldg_b200``- drop-in host program for ``KZM_bulk_ldg_cuda --config``

Usage: ``python -m lcdrsimulator_b200.build`` (or ``build()`` from Python).
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
HOST = os.path.join(PKG, "host")
LIB = os.path.join(PKG, "_lib")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp"]

LIB_SOURCES = ["ldg_api_common.cu", "qsr.cu", "kzm.cu", "conv3d_tc.cu"]
HOST_PROGRAMS = {"qsr_b200": ["qsr_main.cpp"], "kzm_bulk_ldg_b200": ["kzm_main.cpp"]}


def _host_cxx() -> str:
    for c in ("/usr/bin/g++-13", "/usr/bin/g++"):
        if os.path.exists(c):
            return c
    return shutil.which("g++") or "g++"


def _nvcc() -> str:
    for c in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    return r


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(verbose: bool = False, force: bool = False, ptxas_info: bool = False) -> str:
    """Compile libldg_b200.so and the host programs for sm_100a. Returns the library path."""
    os.makedirs(LIB, exist_ok=True)
    nvcc = _nvcc()
    cxx = _host_cxx()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    headers.append(os.path.join(ROOT, "include", "ldg_b200.h"))
    objs = []
    for src in LIB_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(LIB, src.replace(".cu", ".o"))
        if force or _stale(o, [s] + headers):
            cmd = [nvcc, *ARCH, *NVFLAGS, "-ccbin", cxx, "-c", s, "-o", o]
            if ptxas_info:
                cmd += ["-Xptxas", "-v"]
            r = _run(cmd, verbose)
            if ptxas_info:
                print(r.stderr)
        objs.append(o)
    so = os.path.join(LIB, "libldg_b200.so")
    if force or _stale(so, objs):
        _run([nvcc, *ARCH, "-shared", "-ccbin", cxx, *objs, "-o", so, "-Xcompiler", "-fopenmp", "-lgomp"], verbose)
    for prog, srcs in HOST_PROGRAMS.items():
        paths = [os.path.join(HOST, s) for s in srcs]
        if not all(os.path.exists(p) for p in paths):
            continue
        exe = os.path.join(LIB, prog)
        hdeps = paths + [os.path.join(HOST, f) for f in os.listdir(HOST) if f.endswith((".h", ".hpp"))]
        if force or _stale(exe, hdeps + [so]):
            _run([cxx, "-O2", "-std=c++17", *paths, "-I", os.path.join(ROOT, "include"), "-I", HOST,
                  "-L", LIB, "-lldg_b200", "-Wl,-rpath,$ORIGIN", "-o", exe], verbose)
    return so


if __name__ == "__main__":
    build(verbose=True, force="--force" in sys.argv, ptxas_info="--ptxas" in sys.argv)
