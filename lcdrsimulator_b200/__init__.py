"""B200-native Landau-de Gennes Q-tensor solver (drop-in for Spectre71/LCDrSimulator's QSR_cuda
and KZM_bulk_ldg_cuda hot path).

The product is the CUDA library ``_lib/libldg_b200.so`` behind the C ABI in
``include/ldg_b200.h``; this module binds it with ctypes. There is no CPU fallback: if the
library or a CUDA device is missing, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from .physics import (bulk_ABC, S_eq, equilibrium_shell_order, estimate_stable_dt_window, DtRequest,
                      boundary_shell_order)

__all__ = ["QSRSolver", "KZMSolver", "EnsembleSolver", "load_library", "library_path", "LdgError", "bulk_ABC", "S_eq",
           "equilibrium_shell_order", "estimate_stable_dt_window", "DtRequest", "boundary_shell_order"]

_PKG = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_PKG, "_lib", "libldg_b200.so")
_lib = None

_dp = C.POINTER(C.c_double)


class LdgError(RuntimeError):
    pass


class QsrParams(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("a", C.c_double), ("b", C.c_double), ("c", C.c_double), ("T_star", C.c_double),
                ("bulk_modechoice", C.c_int),
                ("kappa", C.c_double), ("L1", C.c_double), ("L2", C.c_double), ("L3", C.c_double),
                ("W", C.c_double), ("gamma", C.c_double), ("droplet_radius_cells", C.c_double),
                ("compensated", C.c_int)]


class QsrGeometry(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("center_x", "center_y", "center_z", "radius_x", "radius_y",
                                          "radius_z", "min_spacing", "shell_half_thickness", "delta_eff")] + [
        (n, C.c_longlong) for n in ("shell_cells", "evolving_cells", "active_cells", "written_cells", "box_cells")]


class QsrStepArgs(C.Structure):
    _fields_ = [("T", C.c_double), ("S_shell", C.c_double), ("dt", C.c_double), ("q_norm_cap", C.c_double),
                ("noise_sigma", C.c_double), ("seed", C.c_ulonglong), ("step_index", C.c_longlong),
                ("semi_implicit", C.c_int), ("L_stab", C.c_double), ("jacobi_iters", C.c_int)]


class QsrObserveArgs(C.Structure):
    _fields_ = [("T", C.c_double), ("S_shell", C.c_double), ("defects_z_slice", C.c_int),
                ("defects_S_threshold", C.c_double), ("defects_charge_cutoff", C.c_double),
                ("xi_z_slice", C.c_int), ("xi_S_threshold", C.c_double), ("want_defects", C.c_int),
                ("want_xi", C.c_int)]


class QsrObservables(C.Structure):
    _fields_ = [("bulk", C.c_double), ("elastic", C.c_double), ("anchoring", C.c_double), ("total", C.c_double),
                ("radiality", C.c_double), ("radiality_count", C.c_longlong),
                ("avg_S", C.c_double), ("max_S", C.c_double), ("core_count", C.c_longlong),
                ("checker_rel", C.c_double), ("defect_density", C.c_double),
                ("defect_count", C.c_longlong), ("defect_plaquettes", C.c_longlong),
                ("xi_grad_proxy", C.c_double), ("xi_edges", C.c_longlong),
                ("max_q_norm", C.c_double), ("nonfinite_cells", C.c_longlong)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


class EnsParams(C.Structure):
    _fields_ = [("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("a", C.c_double), ("b", C.c_double), ("c", C.c_double), ("T_star", C.c_double),
                ("bulk_modechoice", C.c_int),
                ("kappa", C.c_double), ("L1", C.c_double), ("L2", C.c_double), ("L3", C.c_double),
                ("W", C.c_double), ("gamma", C.c_double), ("dt", C.c_double), ("q_norm_cap", C.c_double),
                ("boundary_custom", C.c_int), ("boundary_S", C.c_double), ("protocol", C.c_int)]


class EnsInstance(C.Structure):
    _fields_ = [("N", C.c_int), ("droplet_radius_cells", C.c_double), ("T_high", C.c_double),
                ("T_low", C.c_double), ("pre_equil_iters", C.c_longlong), ("ramp_iters", C.c_longlong),
                ("seed", C.c_ulonglong), ("noise_sigma", C.c_double), ("own_material", C.c_int),
                ("W", C.c_double), ("L2", C.c_double), ("L3", C.c_double), ("Ny", C.c_int), ("Nz", C.c_int)]


class KzmParams(C.Structure):
    _fields_ = [("Nx", C.c_int), ("Ny", C.c_int), ("Nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
                ("kappa", C.c_double), ("gamma", C.c_double), ("q_norm_cap", C.c_double),
                ("defects_S_threshold", C.c_double), ("defects_charge_cutoff", C.c_double)]


class KzmStepArgs(C.Structure):
    _fields_ = [("A", C.c_double), ("B", C.c_double), ("C", C.c_double), ("dt", C.c_double),
                ("noise_sigma", C.c_double), ("seed", C.c_ulonglong), ("step_index", C.c_longlong)]


class KzmObservables(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("bulk", "elastic", "total", "avg_S", "max_S",
                                          "defect_density_per_plaquette", "defect_line_density",
                                          "xi_grad_proxy")] + [
        ("defect_plaquettes_used", C.c_longlong), ("nonzero_defect_plaquettes", C.c_longlong)]

    def as_dict(self):
        return {f[0]: getattr(self, f[0]) for f in self._fields_}


def library_path() -> str:
    return _LIB_PATH


def load_library():
    """Load libldg_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(_LIB_PATH):
        raise LdgError(f"{_LIB_PATH} not built; run `python -m lcdrsimulator_b200.build`")
    L = C.CDLL(_LIB_PATH)
    L.ldg_last_error.restype = C.c_char_p
    L.ldg_version.restype = C.c_char_p
    for name in ("qsr_stream", "kzm_stream"):
        getattr(L, name).restype = C.c_void_p
        getattr(L, name).argtypes = [C.c_void_p]
    for name in ("qsr_launch_count", "kzm_launch_count"):
        getattr(L, name).restype = C.c_longlong
        getattr(L, name).argtypes = [C.c_void_p]
    L.qsr_create.argtypes = [C.POINTER(QsrParams), C.POINTER(C.c_void_p)]
    L.qsr_geometry.argtypes = [C.c_void_p, C.POINTER(QsrGeometry)]
    L.qsr_upload.argtypes = [C.c_void_p, _dp]
    L.qsr_download.argtypes = [C.c_void_p, _dp]
    L.qsr_nematic.argtypes = [C.c_void_p, _dp]
    L.qsr_step.argtypes = [C.c_void_p, C.c_int, C.POINTER(QsrStepArgs)]
    L.qsr_observe.argtypes = [C.c_void_p, C.POINTER(QsrObserveArgs), C.POINTER(QsrObservables)]
    L.qsr_sync.argtypes = [C.c_void_p]
    L.qsr_autotune.argtypes = [C.c_void_p, C.POINTER(QsrStepArgs), C.c_int, C.POINTER(C.c_int)]
    L.qsr_destroy.argtypes = [C.c_void_p]
    L.ens_create.argtypes = [C.POINTER(EnsParams), C.c_int, C.POINTER(EnsInstance), C.POINTER(C.c_void_p)]
    L.ens_initial_fields.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_double]
    L.ens_upload.argtypes = [C.c_void_p, C.c_int, _dp]
    L.ens_download.argtypes = [C.c_void_p, C.c_int, _dp]
    L.ens_step.argtypes = [C.c_void_p, C.c_int]
    L.ens_observe.argtypes = [C.c_void_p, C.c_int, C.POINTER(QsrObserveArgs), C.POINTER(QsrObservables)]
    L.ens_autotune.argtypes = [C.c_void_p, C.c_int, C.POINTER(C.c_int)]
    L.ens_geometry.argtypes = [C.c_void_p, C.c_int, C.POINTER(QsrGeometry)]
    L.ens_nematic.argtypes = [C.c_void_p, C.c_int, _dp]
    L.ens_observe_all.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.ens_destroy.argtypes = [C.c_void_p]
    for name in ("ens_step_index", "ens_cells", "ens_active_cells", "ens_written_cells", "ens_launch_count"):
        getattr(L, name).restype = C.c_longlong
        getattr(L, name).argtypes = [C.c_void_p]
    L.ens_stream.restype = C.c_void_p
    L.ens_stream.argtypes = [C.c_void_p]
    L.kzm_create.argtypes = [C.POINTER(KzmParams), C.POINTER(C.c_void_p)]
    L.kzm_upload.argtypes = [C.c_void_p, _dp]
    L.kzm_download.argtypes = [C.c_void_p, _dp]
    L.kzm_step.argtypes = [C.c_void_p, C.c_int, C.POINTER(KzmStepArgs)]
    L.kzm_observe.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double, C.POINTER(KzmObservables)]
    L.kzm_destroy.argtypes = [C.c_void_p]
    _lib = L
    return L


def _check(rc: int, what: str):
    if rc != 0:
        msg = load_library().ldg_last_error().decode(errors="replace")
        raise LdgError(f"{what} failed (status {rc}): {msg}")


def _f64(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


class QSRSolver:
    """Confined droplet solver on one GPU (the QSR_cuda hot path).

    ``params`` keys: Nx Ny Nz dx dy dz a b c T_star bulk_modechoice kappa L1 L2 L3 W gamma
    droplet_radius_cells compensated. Fields cross the boundary as host AoS FP64 arrays of shape
    (Nx*Ny*Nz*5,) in the reference cell order k + Nz*(j + Ny*i).
    """

    DEFAULTS = dict(Nx=100, Ny=100, Nz=100, dx=1e-8, dy=1e-8, dz=1e-8, a=0.044e6, b=1.413e6, c=1.153e6,
                    T_star=308.0, bulk_modechoice=1, kappa=6.5e-12, L1=0.0, L2=0.0, L3=0.0, W=0.0, gamma=0.1,
                    droplet_radius_cells=0.0, compensated=0)

    def __init__(self, **params):
        L = load_library()
        d = dict(self.DEFAULTS)
        d.update(params)
        self.params = d
        p = QsrParams()
        for k, v in d.items():
            setattr(p, k, v)
        self._p = p
        h = C.c_void_p()
        _check(L.qsr_create(C.byref(p), C.byref(h)), "qsr_create")
        self._h = h
        self.n = int(d["Nx"]) * int(d["Ny"]) * int(d["Nz"])
        self.step_index = 0

    @property
    def handle(self):
        return self._h

    def geometry(self) -> dict:
        g = QsrGeometry()
        _check(load_library().qsr_geometry(self._h, C.byref(g)), "qsr_geometry")
        return {f[0]: getattr(g, f[0]) for f in g._fields_}

    def initial_field(self, init_mode=0, random_seed=42, S0=0.5, noise_amplitude=1e-3) -> np.ndarray:
        """The reference's seeded initial field (host AoS FP64)."""
        out = np.empty(5 * self.n)
        L = load_library()
        L.qsr_initial_field.argtypes = [C.c_void_p, C.c_int, C.c_longlong, C.c_double, C.c_double, _dp]
        _check(L.qsr_initial_field(self._h, init_mode, random_seed, S0, noise_amplitude, out.ctypes.data_as(_dp)),
               "qsr_initial_field")
        return out

    def upload(self, q):
        q = _f64(q)
        if q.size != 5 * self.n:
            raise LdgError(f"upload: expected {5 * self.n} doubles, got {q.size}")
        _check(load_library().qsr_upload(self._h, q.ctypes.data_as(_dp)), "qsr_upload")

    def download(self, out=None) -> np.ndarray:
        out = np.empty(5 * self.n) if out is None else out
        _check(load_library().qsr_download(self._h, out.ctypes.data_as(_dp)), "qsr_download")
        return out

    def nematic(self) -> np.ndarray:
        out = np.empty(4 * self.n)
        _check(load_library().qsr_nematic(self._h, out.ctypes.data_as(_dp)), "qsr_nematic")
        return out.reshape(self.n, 4)

    @staticmethod
    def step_args(T, S_shell, dt, q_norm_cap=0.0, noise_sigma=0.0, seed=0, step_index=0, semi_implicit=False,
                  L_stab=0.0, jacobi_iters=0) -> QsrStepArgs:
        return QsrStepArgs(T, S_shell, dt, q_norm_cap, noise_sigma, seed, step_index, int(semi_implicit), L_stab,
                           jacobi_iters)

    def step(self, n_steps, T, S_shell, dt, **kw):
        kw.setdefault("step_index", self.step_index)
        a = self.step_args(T, S_shell, dt, **kw)
        _check(load_library().qsr_step(self._h, int(n_steps), C.byref(a)), "qsr_step")
        self.step_index = kw["step_index"] + n_steps

    def step_raw(self, n_steps, args: QsrStepArgs):
        _check(load_library().qsr_step(self._h, int(n_steps), C.byref(args)), "qsr_step")

    def observe(self, T, S_shell, defects_z_slice=None, defects_S_threshold=0.1, defects_charge_cutoff=0.25,
                xi_z_slice=None, xi_S_threshold=None, want_defects=True, want_xi=True) -> dict:
        dz = int(self.params["Nz"]) // 2 if defects_z_slice is None else defects_z_slice
        xz = dz if xi_z_slice is None else xi_z_slice
        xt = defects_S_threshold if xi_S_threshold is None else xi_S_threshold
        a = QsrObserveArgs(T, S_shell, dz, defects_S_threshold, defects_charge_cutoff, xz, xt, int(want_defects),
                           int(want_xi))
        o = QsrObservables()
        _check(load_library().qsr_observe(self._h, C.byref(a), C.byref(o)), "qsr_observe")
        return o.as_dict()

    def autotune(self, T, S_shell, dt, trial_steps=10, **kw) -> int:
        """Picks the tiled kernel's work-item length for these step arguments (field restored)."""
        a = self.step_args(T, S_shell, dt, **kw)
        c = C.c_int(0)
        _check(load_library().qsr_autotune(self._h, C.byref(a), int(trial_steps), C.byref(c)), "qsr_autotune")
        return c.value

    def sync(self):
        _check(load_library().qsr_sync(self._h), "qsr_sync")

    def stream(self) -> int:
        return load_library().qsr_stream(self._h)

    def launch_count(self) -> int:
        return load_library().qsr_launch_count(self._h)

    def close(self):
        if getattr(self, "_h", None):
            load_library().qsr_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class EnsembleSolver:
    """Many independent droplets advanced together on one GPU (quench-rate / seed sweeps).

    ``params``: the shared material and solver constants (EnsParams fields: dx dy dz a b c
    T_star bulk_modechoice kappa L1 L2 L3 W gamma dt q_norm_cap boundary_custom boundary_S
    protocol). ``instances``: one dict per droplet with keys N droplet_radius_cells T_high
    T_low pre_equil_iters ramp_iters seed noise_sigma. Each step is one persistent kernel
    launch over all droplets; the temperature protocol is evaluated on the device.
    """

    DEFAULTS = dict(dx=1e-8, dy=1e-8, dz=1e-8, a=0.044e6, b=1.413e6, c=1.153e6, T_star=308.0, bulk_modechoice=1,
                    kappa=6.5e-12, L1=0.0, L2=0.0, L3=0.0, W=0.0, gamma=0.1, dt=1e-10, q_norm_cap=0.0,
                    boundary_custom=0, boundary_S=0.5, protocol=2)
    INSTANCE_DEFAULTS = dict(N=64, droplet_radius_cells=0.0, T_high=315.0, T_low=300.0, pre_equil_iters=0,
                             ramp_iters=1000, seed=0, noise_sigma=0.0, own_material=0, W=0.0, L2=0.0, L3=0.0,
                             Ny=0, Nz=0)

    def __init__(self, instances, **params):
        L = load_library()
        d = dict(self.DEFAULTS)
        d.update(params)
        self.params = d
        p = EnsParams()
        for k, v in d.items():
            setattr(p, k, v)
        self.instances = []
        arr = (EnsInstance * len(instances))()
        for n, inst in enumerate(instances):
            e = dict(self.INSTANCE_DEFAULTS)
            e.update(inst)
            self.instances.append(e)
            for k, v in e.items():
                setattr(arr[n], k, v)
        h = C.c_void_p()
        _check(L.ens_create(C.byref(p), len(instances), arr, C.byref(h)), "ens_create")
        self._h = h

    @property
    def handle(self):
        return self._h

    def cells(self, instance) -> int:
        if not 0 <= instance < len(self.instances):
            raise LdgError(f"instance {instance} out of range (0..{len(self.instances) - 1})")
        d = self.instances[instance]
        N = int(d["N"])
        return N * (int(d["Ny"]) or N) * (int(d["Nz"]) or N)

    def initial_fields(self, init_mode=0, S0=0.5, noise_amplitude=1e-3):
        _check(load_library().ens_initial_fields(self._h, init_mode, S0, noise_amplitude), "ens_initial_fields")

    def upload(self, instance, q):
        q = _f64(q)
        if q.size != 5 * self.cells(instance):
            raise LdgError(f"upload: expected {5 * self.cells(instance)} doubles, got {q.size}")
        _check(load_library().ens_upload(self._h, instance, q.ctypes.data_as(_dp)), "ens_upload")

    def download(self, instance, out=None) -> np.ndarray:
        n = 5 * self.cells(instance)
        if out is None:
            out = np.empty(n)
        elif out.dtype != np.float64 or out.size != n or not out.flags["C_CONTIGUOUS"]:
            raise LdgError(f"download: out must be a contiguous float64 array of {n} values")
        _check(load_library().ens_download(self._h, instance, out.ctypes.data_as(_dp)), "ens_download")
        return out

    def nematic(self, instance) -> np.ndarray:
        out = np.empty(4 * self.cells(instance))
        _check(load_library().ens_nematic(self._h, instance, out.ctypes.data_as(_dp)), "ens_nematic")
        return out.reshape(-1, 4)

    def step(self, n_steps):
        _check(load_library().ens_step(self._h, int(n_steps)), "ens_step")

    def observe(self, instance, args: QsrObserveArgs | None = None) -> dict:
        o = QsrObservables()
        _check(load_library().ens_observe(self._h, instance, C.byref(args) if args is not None else None,
                                          C.byref(o)), "ens_observe")
        return o.as_dict()

    def geometry(self, instance) -> dict:
        g = QsrGeometry()
        _check(load_library().ens_geometry(self._h, instance, C.byref(g)), "ens_geometry")
        return {f[0]: getattr(g, f[0]) for f in g._fields_}

    def observe_all(self) -> list[dict]:
        """Observables of every droplet at its protocol temperature, in one pass."""
        out = (QsrObservables * len(self.instances))()
        _check(load_library().ens_observe_all(self._h, None, out), "ens_observe_all")
        return [o.as_dict() for o in out]

    def autotune(self, trial_steps=10) -> int:
        c = C.c_int(0)
        _check(load_library().ens_autotune(self._h, trial_steps, C.byref(c)), "ens_autotune")
        return c.value

    @property
    def step_index(self) -> int:
        return load_library().ens_step_index(self._h)

    def counts(self) -> dict:
        L = load_library()
        return dict(cells=L.ens_cells(self._h), active_cells=L.ens_active_cells(self._h),
                    written_cells=L.ens_written_cells(self._h))

    def stream(self) -> int:
        return load_library().ens_stream(self._h)

    def launch_count(self) -> int:
        return load_library().ens_launch_count(self._h)

    def close(self):
        if getattr(self, "_h", None):
            load_library().ens_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


class KZMSolver:
    """Periodic bulk solver on one GPU (the KZM_bulk_ldg_cuda hot path); x-fastest host order."""

    def __init__(self, Nx, Ny, Nz, dx, dy, dz, kappa, gamma, q_norm_cap=0.0, defects_S_threshold=0.1,
                 defects_charge_cutoff=0.25):
        L = load_library()
        p = KzmParams(Nx, Ny, Nz, dx, dy, dz, kappa, gamma, q_norm_cap, defects_S_threshold, defects_charge_cutoff)
        self._p = p
        h = C.c_void_p()
        _check(L.kzm_create(C.byref(p), C.byref(h)), "kzm_create")
        self._h = h
        self.n = Nx * Ny * Nz

    @property
    def handle(self):
        return self._h

    def upload(self, q):
        q = _f64(q)
        if q.size != 5 * self.n:
            raise LdgError(f"upload: expected {5 * self.n} doubles, got {q.size}")
        _check(load_library().kzm_upload(self._h, q.ctypes.data_as(_dp)), "kzm_upload")

    def download(self, out=None):
        out = np.empty(5 * self.n) if out is None else out
        _check(load_library().kzm_download(self._h, out.ctypes.data_as(_dp)), "kzm_download")
        return out

    def step(self, n_steps, A, B, Cc, dt, noise_sigma=0.0, seed=0, step_index=0):
        a = KzmStepArgs(A, B, Cc, dt, noise_sigma, seed, step_index)
        _check(load_library().kzm_step(self._h, int(n_steps), C.byref(a)), "kzm_step")

    def observe(self, A, B, Cc) -> dict:
        o = KzmObservables()
        _check(load_library().kzm_observe(self._h, A, B, Cc, C.byref(o)), "kzm_observe")
        return o.as_dict()

    def stream(self) -> int:
        return load_library().kzm_stream(self._h)

    def launch_count(self) -> int:
        return load_library().kzm_launch_count(self._h)

    def close(self):
        if getattr(self, "_h", None):
            load_library().kzm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
