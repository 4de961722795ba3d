"""ctypes bindings for the FP64 CPU oracle and the reference builds -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, by ``__graft_entry__.smoke()`` and by ``bench.py``'s cpu_baseline leg,
always as the checker or the timed CPU baseline, never as the product path.

* ``Oracle``: the FP64 OpenMP restatement in ``ldg_oracle.cpp`` (confined droplet solver of
  QSR.cu and the periodic bulk solver of KZM_bulk_ldg.cu).
* ``RefCPU``: the reference's own QSR.cpp functions (built from the reference sources).
* ``RefCUDA`` / ``RefKZM``: the reference's own FP64 CUDA kernels (QSR.cu, KZM_bulk_ldg.cu)
  compiled for sm_100a; they run only where a GPU is present.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF = os.path.join(HERE, "_ref")

_dp = C.POINTER(C.c_double)
_u8p = C.POINTER(C.c_uint8)


def build(quiet: bool = True) -> None:
    """Compile the oracle (and the reference builds when the reference sources exist)."""
    out = subprocess.run(["make", "-C", HERE, "all"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _ptr(a: np.ndarray, t=_dp):
    return a.ctypes.data_as(t)


class OrcParams(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("a", C.c_double), ("b", C.c_double), ("c", C.c_double), ("T_star", C.c_double),
                ("bulk_modechoice", C.c_int),
                ("kappa", C.c_double), ("L1", C.c_double), ("L2", C.c_double), ("L3", C.c_double),
                ("W", C.c_double), ("gamma", C.c_double), ("droplet_radius_cells", C.c_double)]


class OrcGeometry(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "dx", "dy", "dz", "center_x", "center_y", "center_z", "radius_x", "radius_y", "radius_z",
        "min_spacing", "min_radius", "shell_half_thickness", "core_radius", "delta_eff")] + [
        ("shell_count", C.c_longlong)]


class OrcObservables(C.Structure):
    _fields_ = [("bulk", C.c_double), ("elastic", C.c_double), ("anchoring", C.c_double), ("total", C.c_double),
                ("radiality", C.c_double), ("radiality_count", C.c_longlong),
                ("avg_S", C.c_double), ("max_S", C.c_double), ("core_count", C.c_longlong),
                ("checker_rel", C.c_double),
                ("checker_even_sum", C.c_double), ("checker_odd_sum", C.c_double), ("checker_all_sum", C.c_double),
                ("checker_even_n", C.c_longlong), ("checker_odd_n", C.c_longlong), ("checker_all_n", C.c_longlong),
                ("defect_density", C.c_double), ("defect_count", C.c_longlong), ("defect_plaquettes", C.c_longlong),
                ("xi_grad_proxy", C.c_double), ("xi_sum_sq", C.c_double), ("xi_edges", C.c_longlong)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class OrcBulkParams(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("kappa", C.c_double), ("gamma", C.c_double), ("dt", C.c_double), ("q_norm_cap", C.c_double),
                ("defects_S_threshold", C.c_double), ("defects_charge_cutoff", C.c_double)]


class OrcBulkObservables(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "bulk", "elastic", "total", "avg_S", "max_S", "defect_density_per_plaquette",
        "defect_line_density", "xi_grad_proxy")] + [
        ("defect_plaquettes_used", C.c_longlong), ("nonzero_defect_plaquettes", C.c_longlong)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


DEFAULTS = dict(Nx=32, Ny=32, Nz=32, dx=1e-8, dy=1e-8, dz=1e-8, a=0.044e6, b=1.413e6, c=1.153e6,
                T_star=307.0, bulk_modechoice=1, kappa=6.5e-12, L1=6e-12, L2=0.0, L3=0.0, W=0.0,
                gamma=0.1, droplet_radius_cells=0.0)


def make_params(**kw) -> OrcParams:
    d = dict(DEFAULTS)
    d.update(kw)
    p = OrcParams()
    for k, v in d.items():
        setattr(p, k, v)
    return p


class Oracle:
    """FP64 CPU restatement of the reference step, observables and initialisation."""

    def __init__(self):
        path = os.path.join(BUILD, "libldg_oracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        self.L = L
        L.orc_S_eq.restype = C.c_double
        L.orc_S_eq.argtypes = [C.c_double] * 3
        L.orc_bulk_ABC.argtypes = [C.c_double] * 5 + [C.c_int, _dp, _dp, _dp]

    # -- confined droplet --
    def geometry(self, p: OrcParams):
        g = OrcGeometry()
        n = p.Nx * p.Ny * p.Nz
        flags = np.zeros(n, np.uint8)
        self.L.orc_make_geometry(C.byref(p), C.byref(g))
        self.L.orc_classify(C.byref(p), C.byref(g), _ptr(flags, _u8p))
        return g, flags

    def init(self, p, g, mode, seed, S0, noise_amplitude=1e-3):
        q = np.zeros(p.Nx * p.Ny * p.Nz * 5)
        self.L.orc_init(C.byref(p), C.byref(g), C.c_int(mode), C.c_longlong(seed), C.c_double(S0),
                        C.c_double(noise_amplitude), _ptr(q))
        return q

    def laplacian(self, p, q):
        out = np.zeros_like(q)
        self.L.orc_laplacian(C.byref(p), _ptr(q), _ptr(out))
        return out

    def chem_potential(self, p, g, flags, q, T, S_shell):
        out = np.zeros_like(q)
        self.L.orc_chem_potential(C.byref(p), C.byref(g), _ptr(flags, _u8p), _ptr(q), C.c_double(T),
                                  C.c_double(S_shell), _ptr(out))
        return out

    def step_explicit(self, p, g, flags, q, T, S_shell, dt, q_norm_cap=0.0, n=1):
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        for _ in range(n):
            self.L.orc_step_explicit(C.byref(p), C.byref(g), _ptr(flags, _u8p), _ptr(q), C.c_double(T),
                                     C.c_double(S_shell), C.c_double(dt), C.c_double(q_norm_cap))
        return q

    def step_imex(self, p, g, flags, q, T, S_shell, dt, L_stab, jacobi_iters, n=1):
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        for _ in range(n):
            self.L.orc_step_imex(C.byref(p), C.byref(g), _ptr(flags, _u8p), _ptr(q), C.c_double(T),
                                 C.c_double(S_shell), C.c_double(dt), C.c_double(L_stab), C.c_int(jacobi_iters))
        return q

    def nematic(self, q):
        n = q.size // 5
        out = np.zeros(4 * n)
        self.L.orc_nematic(_ptr(q), C.c_longlong(n), _ptr(out))
        return out.reshape(n, 4)

    def observe(self, p, g, flags, q, T, S_shell, dz_slice=None, dS_thr=0.1, d_cut=0.25, xi_slice=None,
                xi_thr=None):
        dz_slice = p.Nz // 2 if dz_slice is None else dz_slice
        xi_slice = dz_slice if xi_slice is None else xi_slice
        xi_thr = dS_thr if xi_thr is None else xi_thr
        o = OrcObservables()
        self.L.orc_observe(C.byref(p), C.byref(g), _ptr(flags, _u8p), _ptr(q), C.c_double(T), C.c_double(S_shell),
                           C.c_int(dz_slice), C.c_double(dS_thr), C.c_double(d_cut), C.c_int(xi_slice),
                           C.c_double(xi_thr), C.byref(o))
        return o.as_dict()

    def bulk_ABC(self, a, b, c, T, T_star, mode=1):
        A, B, Cc = C.c_double(), C.c_double(), C.c_double()
        self.L.orc_bulk_ABC(a, b, c, T, T_star, mode, C.byref(A), C.byref(B), C.byref(Cc))
        return A.value, B.value, Cc.value

    def S_eq(self, A, B, Cc):
        return self.L.orc_S_eq(A, B, Cc)

    # -- periodic bulk --
    def bulk_init(self, bp: OrcBulkParams, seed, amplitude):
        q = np.zeros(bp.Nx * bp.Ny * bp.Nz * 5)
        self.L.orc_bulk_init(C.byref(bp), C.c_longlong(seed), C.c_double(amplitude), _ptr(q))
        return q

    def bulk_step(self, bp, q, A, B, Cc, n=1):
        cur = np.ascontiguousarray(q, dtype=np.float64).copy()
        nxt = np.zeros_like(cur)
        for _ in range(n):
            self.L.orc_bulk_step(C.byref(bp), _ptr(cur), _ptr(nxt), C.c_double(A), C.c_double(B), C.c_double(Cc))
            cur, nxt = nxt, cur
        return cur

    def bulk_observe(self, bp, q, A, B, Cc):
        o = OrcBulkObservables()
        self.L.orc_bulk_observe(C.byref(bp), _ptr(q), C.c_double(A), C.c_double(B), C.c_double(Cc), C.byref(o))
        return o.as_dict()

    def philox(self, ctr, key, rounds=10):
        c = (C.c_uint32 * 4)(*ctr)
        k = (C.c_uint32 * 2)(*key)
        o = (C.c_uint32 * 4)()
        self.L.orc_philox4x32_rounds(c, k, C.c_int(rounds), o)
        return list(o)


class RefCPU:
    """The reference's own QSR.cpp functions (QSR.cpp:10, 179, 411, 559)."""

    def __init__(self):
        path = os.path.join(REF, "libqsr_cpu_ref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.L = C.CDLL(path)

    @staticmethod
    def _pr(p: OrcParams, T):
        return np.array([p.a, p.b, p.c, T, p.T_star, p.L1, p.L2, p.L3, p.W], dtype=np.float64)

    def laplacian(self, p, q):
        out = np.zeros_like(q)
        self.L.ref_laplacian(_ptr(q), _ptr(out), p.Nx, p.Ny, p.Nz, C.c_double(p.dx), C.c_double(p.dy),
                             C.c_double(p.dz))
        return out

    def chem_potential(self, p, q, T):
        out = np.zeros_like(q)
        self.L.ref_chem_potential(_ptr(q), _ptr(out), p.Nx, p.Ny, p.Nz, C.c_double(p.dx), C.c_double(p.dy),
                                  C.c_double(p.dz), _ptr(self._pr(p, T)), C.c_double(p.kappa),
                                  C.c_int(p.bulk_modechoice))
        return out

    def energy(self, p, q, T):
        b, e = C.c_double(), C.c_double()
        self.L.ref_energy(_ptr(q), p.Nx, p.Ny, p.Nz, C.c_double(p.dx), C.c_double(p.dy), C.c_double(p.dz),
                          _ptr(self._pr(p, T)), C.c_double(p.kappa), C.c_int(p.bulk_modechoice), C.byref(b),
                          C.byref(e))
        return b.value, e.value

    def nematic(self, q5):
        out = np.zeros(4)
        self.L.ref_nematic(_ptr(np.ascontiguousarray(q5, dtype=np.float64)), _ptr(out))
        return out

    def run_steps(self, p, q, T, S_shell, dt, n_steps):
        """n_steps of the reference CPU time step in place (droplet mask of radius
        p.droplet_radius_cells when positive); returns the loop's wall seconds."""
        self.L.ref_run_steps.restype = C.c_double
        return self.L.ref_run_steps(_ptr(q), p.Nx, p.Ny, p.Nz, C.c_double(p.dx), C.c_double(p.dy),
                                    C.c_double(p.dz), _ptr(self._pr(p, T)), C.c_double(p.kappa),
                                    C.c_int(p.bulk_modechoice), C.c_double(p.gamma), C.c_double(dt),
                                    C.c_double(S_shell), C.c_int(n_steps), C.c_double(p.droplet_radius_cells))

    def max_threads(self):
        return self.L.ref_max_threads()


def ref_initial_field(p: OrcParams, mode, seed, S0, noise_amplitude=1e-3) -> np.ndarray:
    """The reference's own seeded initial field: initializeQTensor / initializeIsotropicWithNoise
    (QSR.cu:1841-1904) from the reference build (host code; no GPU needed)."""
    path = os.path.join(REF, "qsr_cuda_ref.so")
    if not os.path.exists(path):
        raise FileNotFoundError(path)
    L = C.CDLL(path)
    L.qref_init.argtypes = [C.c_int] * 3 + [C.c_double] * 4 + [C.c_int, C.c_longlong, C.c_double, C.c_double, _dp]
    q = np.zeros(p.Nx * p.Ny * p.Nz * 5)
    L.qref_init(p.Nx, p.Ny, p.Nz, p.dx, p.dy, p.dz, p.droplet_radius_cells, mode, seed, S0, noise_amplitude, _ptr(q))
    return q


class RefCUDA:
    """The reference's FP64 QSR.cu kernels (GPU only), driven in the reference's launch order."""

    def __init__(self):
        path = os.path.join(REF, "qsr_cuda_ref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = C.CDLL(path)
        self.L = L
        L.qref_delta_eff.restype = C.c_double

    def create(self, p: OrcParams):
        arr = np.array([p.Nx, p.Ny, p.Nz, p.dx, p.dy, p.dz, p.a, p.b, p.c, p.T_star, p.bulk_modechoice,
                        p.kappa, p.L1, p.L2, p.L3, p.W, p.gamma, p.droplet_radius_cells], dtype=np.float64)
        rc = self.L.qref_create(_ptr(arr))
        if rc != 0:
            raise RuntimeError(f"qref_create failed: {rc}")
        self.n = p.Nx * p.Ny * p.Nz

    def upload(self, q):
        assert self.L.qref_upload(_ptr(np.ascontiguousarray(q, dtype=np.float64))) == 0

    def download(self):
        q = np.zeros(self.n * 5)
        assert self.L.qref_download(_ptr(q)) == 0
        return q

    def step(self, T, S_shell, dt, q_norm_cap=0.0, imex=False, L_stab=0.0, jacobi_iters=0):
        rc = self.L.qref_step(C.c_double(T), C.c_double(S_shell), C.c_double(dt), C.c_double(q_norm_cap),
                              C.c_int(int(imex)), C.c_double(L_stab), C.c_int(jacobi_iters))
        assert rc == 0

    def time_steps(self, T, S_shell, dt, n):
        """Device time (ms) of n explicit steps of the reference chain launched back to back."""
        ms = C.c_float(0.0)
        rc = self.L.qref_time_steps(C.c_double(T), C.c_double(S_shell), C.c_double(dt), C.c_int(n), C.byref(ms))
        assert rc == 0, rc
        return ms.value

    def observe(self, T, S_shell, dz_slice, dS_thr=0.1, d_cut=0.25, xi_slice=None, xi_thr=None):
        xi_slice = dz_slice if xi_slice is None else xi_slice
        xi_thr = dS_thr if xi_thr is None else xi_thr
        out = np.zeros(12)
        self.L.qref_observe(C.c_double(T), C.c_double(S_shell), C.c_int(dz_slice), C.c_double(dS_thr),
                            C.c_double(d_cut), C.c_int(xi_slice), C.c_double(xi_thr), _ptr(out))
        keys = ["bulk", "elastic", "anchoring", "radiality", "avg_S", "max_S", "checker_rel", "defect_density",
                "defect_count", "defect_plaquettes", "xi_grad_proxy", "xi_edges"]
        return dict(zip(keys, out.tolist()))

    def destroy(self):
        self.L.qref_destroy()


class RefKZM:
    """The reference's FP64 periodic bulk kernel and host observables (KZM_bulk_ldg.cu)."""

    def __init__(self):
        path = os.path.join(REF, "kzm_cuda_ref.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.L = C.CDLL(path)

    @staticmethod
    def _arr(bp: OrcBulkParams):
        return np.array([bp.Nx, bp.Ny, bp.Nz, bp.dx, bp.dy, bp.dz, bp.kappa, bp.gamma, bp.dt, bp.q_norm_cap,
                         bp.defects_S_threshold, bp.defects_charge_cutoff], dtype=np.float64)

    def run(self, bp, q, n_steps, A, B, Cc, noise_sigma=0.0, seed=0, iter0=0):
        out = np.zeros_like(q)
        rc = self.L.kref_run(_ptr(self._arr(bp)), _ptr(np.ascontiguousarray(q)), _ptr(out), C.c_int(n_steps),
                             C.c_double(A), C.c_double(B), C.c_double(Cc), C.c_double(noise_sigma),
                             C.c_ulonglong(seed), C.c_int(iter0))
        assert rc == 0
        return out

    def time_steps(self, bp, q, n_warm, n_steps, A, B, Cc, noise_sigma=0.0, seed=0):
        """Device time (ms) of n_steps reference updates launched back to back."""
        ms = C.c_float(0.0)
        rc = self.L.kref_time(_ptr(self._arr(bp)), _ptr(np.ascontiguousarray(q)), C.c_int(n_warm), C.c_int(n_steps),
                              C.c_double(A), C.c_double(B), C.c_double(Cc), C.c_double(noise_sigma),
                              C.c_ulonglong(seed), C.byref(ms))
        assert rc == 0, rc
        return ms.value

    def quench(self, bp, q, seed, a, b, c, T_star, T_high, T_low, pre, ramp, total, noise_strength, mode=1):
        """The reference's quench loop (KZM_bulk_ldg.cu:917-970) over total iterations; returns the
        final field and the (A, B, C) of the final temperature."""
        out = np.zeros_like(q)
        r = np.array([a, b, c, T_star, mode, T_high, T_low, pre, ramp, total, noise_strength], dtype=np.float64)
        abc = np.zeros(3)
        rc = self.L.kref_quench(_ptr(self._arr(bp)), _ptr(r), _ptr(np.ascontiguousarray(q)), _ptr(out),
                                C.c_ulonglong(seed), _ptr(abc))
        assert rc == 0
        return out, tuple(abc)

    def observe(self, bp, q, A, B, Cc):
        out = np.zeros(10)
        self.L.kref_observe(_ptr(self._arr(bp)), _ptr(np.ascontiguousarray(q)), C.c_double(A), C.c_double(B),
                            C.c_double(Cc), _ptr(out))
        keys = ["bulk", "elastic", "total", "avg_S", "max_S", "defect_density_per_plaquette",
                "defect_line_density", "xi_grad_proxy", "defect_plaquettes_used", "nonzero_defect_plaquettes"]
        return dict(zip(keys, out.tolist()))
