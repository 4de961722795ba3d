"""Shared helpers of the GPU parity tests: build matching oracle and library parameter sets."""
import numpy as np

from oracle.oracle import make_params
from lcdrsimulator_b200 import QSRSolver

BASE = dict(dx=1e-8, dy=1e-8, dz=1e-8, a=0.044e6, b=1.413e6, c=1.153e6, T_star=307.0, bulk_modechoice=1,
            kappa=6.5e-12, L1=6e-12, L2=0.0, L3=0.0, W=0.0, gamma=0.1, droplet_radius_cells=0.0)


def make_pair(**kw):
    d = dict(BASE)
    d.update(kw)
    op = make_params(**d)
    solver = QSRSolver(**d)
    return op, solver, d


def fp32(q):
    """Round a field to FP32 (the device storage) and back."""
    return np.asarray(q, dtype=np.float32).astype(np.float64)


def rel_err(a, b):
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def rms_rel(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-300))
