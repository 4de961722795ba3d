"""Host-side scalar physics of the LdG step driver (the reference's QSR.cu host helpers).

Per-step scalars that the step kernels take as arguments: bulk coefficients, the uniaxial
equilibrium order, the shell order policy and the stable-dt estimate.
"""
from __future__ import annotations

import math
from dataclasses import dataclass


def bulk_ABC(a, b, c, T, T_star, mode=1):
    """A, B, C of H = A Q - B (Q^2 - I trQ^2/3) + C trQ^2 Q (QSR.cu:1363-1378)."""
    A = 3.0 * a * (T - T_star)
    if mode == 1:
        return A, (9.0 * b) / 2.0, (9.0 * c) / 2.0
    return A, (27.0 * b) / 2.0, 9.0 * c


def bulk_fS(A, B, C, S):
    """Uniaxial bulk energy f(S) = (A/3) S^2 - (2B/27) S^3 + (C/9) S^4 (QSR.cu:1380-1389)."""
    S2 = S * S
    return (A / 3.0) * S2 - (2.0 * B / 27.0) * (S2 * S) + (C / 9.0) * (S2 * S2)


def S_eq(A, B, C):
    """Lower-energy positive root of 2 C S^2 - B S + 3 A = 0, else 0 (QSR.cu:1391-1418)."""
    if not (C > 0.0):
        return 0.0
    disc = B * B - 24.0 * A * C
    if not (disc > 0.0):
        return 0.0
    sd = math.sqrt(disc)
    best_S, best_f = 0.0, 0.0
    for S in ((B - sd) / (4.0 * C), (B + sd) / (4.0 * C)):
        if not (S > 0.0):
            continue
        f = bulk_fS(A, B, C, S)
        if f < best_f:
            best_f, best_S = f, S
    return best_S


def T_NI(a, b, c, T_star, mode=1):
    """Coexistence temperature T* + B^2/(27 C)/(3a) (QSR.cu:1420-1438)."""
    _, B, C = bulk_ABC(a, b, c, 0.0, 0.0, mode)
    if not (C > 0.0) or not (a > 0.0):
        return float("nan")
    return T_star + (B * B) / (27.0 * C) / (3.0 * a)


def equilibrium_shell_order(a, b, c, T, T_star, mode=1):
    """max(S_eq(T), 0) (QSR.cu:1460-1473)."""
    s = S_eq(*bulk_ABC(a, b, c, T, T_star, mode))
    return s if s > 0.0 else 0.0


def boundary_shell_order(policy, custom_S, a, b, c, T, T_star, mode=1):
    """Shell order policy: 'custom'/'fixed' -> custom_S, else equilibrium (QSR.cu:1440-1487)."""
    p = (policy or "").strip().lower()
    if p in ("custom", "fixed"):
        return custom_S
    return equilibrium_shell_order(a, b, c, T, T_star, mode)


@dataclass
class DtRequest:
    dx: float = 1.0
    dy: float = 1.0
    dz: float = 1.0
    gamma: float = 1.0
    a: float = 0.0
    b: float = 0.0
    c: float = 0.0
    T_star: float = 0.0
    modechoice: int = 1
    kappa: float = 0.0
    L1: float = 0.0
    L2: float = 0.0
    L3: float = 0.0
    S_ref_used: float = float("nan")
    S0: float = 0.0
    T_a: float = 0.0
    T_b: float = 0.0
    use_semi_implicit: bool = False
    L_stab: float = 0.0
    jacobi_iters: int = 0


def estimate_stable_dt_window(r: DtRequest) -> dict:
    """Explicit stability estimate dt_max = min(dt_diff, dt_bulk) (QSR.cu:1528-1604)."""
    min_dx = min(r.dx, r.dy, r.dz)
    S_scale = abs(r.S_ref_used) if math.isfinite(r.S_ref_used) else max(abs(r.S0), 0.5)
    for T in (r.T_a, r.T_b):
        s = abs(equilibrium_shell_order(r.a, r.b, r.c, T, r.T_star, r.modechoice))
        if math.isfinite(s) and s > 0.0:
            S_scale = max(S_scale, s)
    S_scale = max(S_scale, 1.0)
    using_ldg = r.L1 != 0.0 or r.L2 != 0.0 or r.L3 != 0.0
    aniso = r.L2 != 0.0 or r.L3 != 0.0
    if using_ldg:
        L_eff = max(abs(r.L1), abs(r.L2), abs(r.L1 + r.L2), abs(r.L1 + 2.0 * r.L2), abs(r.L3) * S_scale)
    else:
        L_eff = abs(r.kappa)
    if not (L_eff > 0.0):
        L_eff = 1e-12
    D = L_eff / r.gamma
    if not (D > 0.0) or not math.isfinite(D):
        D = 1e-12
    dt_diff_total = 0.5 * (min_dx * min_dx) / (6.0 * D)
    if aniso:
        dt_diff_total *= 0.25
    dt_diff = dt_diff_total
    L_ex = L_eff
    semi = False
    if r.use_semi_implicit and r.L_stab > 0.0 and r.jacobi_iters > 0:
        L_base = r.L1 if using_ldg else r.kappa
        L_stab_signed = r.L_stab if L_base >= 0.0 else -r.L_stab
        L_rem = abs(L_base - L_stab_signed)
        if using_ldg:
            L_ex = max(L_rem, abs(r.L2), abs(r.L1 + r.L2), abs(r.L1 + 2.0 * r.L2), abs(r.L3) * S_scale)
        else:
            L_ex = L_rem
        if L_ex > 0.0:
            dt_diff = 0.5 * (min_dx * min_dx) / (6.0 * (L_ex / r.gamma))
            if aniso:
                dt_diff *= 0.25
        else:
            dt_diff = math.inf
        semi = True

    def rate(T):
        A, B, C = bulk_ABC(r.a, r.b, r.c, T, r.T_star, r.modechoice)
        return abs(A) + abs(B) * S_scale + abs(C) * S_scale * S_scale

    bulk_rate = max(rate(r.T_a), rate(r.T_b))
    dt_bulk = 0.02 * r.gamma / bulk_rate if bulk_rate > 0.0 else math.inf
    dt_max = min(dt_diff, dt_bulk)
    if not (dt_max > 0.0) or not math.isfinite(dt_max):
        dt_max = dt_diff
    return dict(min_dx=min_dx, S_scale=S_scale, L_eff_total=L_eff, D_total=D, dt_diff_total=dt_diff_total,
                L_eff_explicit=L_ex, dt_diff=dt_diff, bulk_rate=bulk_rate, dt_bulk=dt_bulk, dt_max=dt_max,
                semi_implicit_active=semi)
