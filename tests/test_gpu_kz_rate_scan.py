"""Kibble-Zurek rate scan of the periodic bulk quench, this library against the reference's own
FP64 kernel (GPU), compared in distribution.

The reference publishes one number for this path: over a seven-rate scan of its periodic bulk
branch, the final-state defect_line_density falls with the quench time tau_Q with log-log slope
about -0.515 (correlation about -0.990; its Changelog, v0.3.2). Its configurations are not in
the reference tree, so this scan uses the periodic-quench physics of the benchmark (kappa =
6e-12 N, gamma = 0.1, linear ramp 315 K -> 295 K over tau_Q steps, Langevin noise of strength
kT/dx^3 at 300 K, initial |Q| ~ 1e-3) on a 64^3 box at the reference's explicit-limit dt, with
five ramps tau_Q = 500 .. 8000 steps, each followed by a 2000-step hold at 295 K, and eight
seeds per rate (LDG_KZ_SCAN_N=128 runs it on a 128^3 box).

Both sides start from the reference's own initial field (mt19937_64 Gaussian, seed per run) and
follow the reference's temperature schedule; the noise streams differ (Philox4x32-7 here,
splitmix64 in the reference), so single runs differ and the comparison is statistical: the mean
final line density at every rate within 4 combined standard errors, and the two fitted slopes
within 3 combined standard deviations (seed bootstrap). The measured slopes and their spread are
written to $LDG_ACCURACY_OUT.kz_rate_scan when that variable is set.

In this regime (5CB-like constants with B = 6.4e6 J/m^3, thermal noise kT/dx^3 on 10 nm cells)
the final line density rises slightly with tau_Q on both sides (slope about +0.13): ordering is
driven by the cubic term and the noise within a few hundred steps of crossing T*, faster than any
ramp here, so the final state measures the coarsening time left, not a Kibble-Zurek freeze-out.
The reference's published -0.515 comes from its own configurations (its defaults are dt = 1e-11 s
and no thermal noise), which are not in the reference tree.
"""
import json
import math
import os

import numpy as np
import pytest

from oracle.oracle import OrcBulkParams, RefKZM
from lcdrsimulator_b200 import KZMSolver
from lcdrsimulator_b200.physics import bulk_ABC, S_eq

pytestmark = pytest.mark.gpu

# box edge: 64 in the default suite; LDG_KZ_SCAN_N=128 runs the same scan on a 128^3 box
N, D, KAPPA, GAMMA = int(os.environ.get("LDG_KZ_SCAN_N", "64")), 1e-8, 6e-12, 0.1
LDG = dict(a=0.044e6, b=1.413e6, c=1.153e6, T_star=307.0)
T_HIGH, T_LOW, HOLD = 315.0, 295.0, 2000
TAUS = [500, 1000, 2000, 4000, 8000]
SEEDS = list(range(8))
NOISE_STRENGTH = 1.380649e-23 * 300.0 / D ** 3


def explicit_limit_dt():
    """estimate_stable_dt of the periodic program (KZM_bulk_ldg.cu:330-349)."""
    Ah = bulk_ABC(LDG["a"], LDG["b"], LDG["c"], T_HIGH, LDG["T_star"])[0]
    Al, Bl, Cl = bulk_ABC(LDG["a"], LDG["b"], LDG["c"], T_LOW, LDG["T_star"])
    Sl = S_eq(Al, Bl, Cl)
    lap = 2.0 * KAPPA * 3.0 / (D * D)
    local = max(abs(Ah), abs(Al)) + abs(Bl) * abs(Sl) + abs(Cl) * 2.0 * Sl * Sl / 3.0
    return 0.2 / ((1.0 / GAMMA) * (lap + local))


def temperature(it, ramp):
    """compute_temperature (KZM_bulk_ldg.cu:316-327) with pre_equil_iters = 0."""
    if it >= ramp or ramp <= 0:
        return T_LOW
    return T_HIGH + (it / ramp) * (T_LOW - T_HIGH)


def fit_slope(taus, rho_by_rate):
    x = np.log(np.asarray(taus, dtype=np.float64))
    y = np.log(np.asarray([np.mean(r) for r in rho_by_rate]))
    s, _ = np.polyfit(x, y, 1)
    return float(s), float(np.corrcoef(x, y)[0, 1])


def bootstrap_sd(taus, rho_by_rate, draws=400, seed=0):
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(draws):
        res = [np.asarray(r)[rng.integers(0, len(r), len(r))] for r in rho_by_rate]
        if any(np.mean(r) <= 0 for r in res):
            continue
        out.append(fit_slope(taus, res)[0])
    return float(np.std(out, ddof=1))


def test_kz_rate_scan_slope_matches_reference_kernel(oracle):
    ref = RefKZM()
    dt = explicit_limit_dt()
    sigma = math.sqrt(2.0 * (1.0 / GAMMA) * NOISE_STRENGTH * dt)
    bp = OrcBulkParams(N, N, N, D, D, D, KAPPA, GAMMA, dt, 0.0, 0.1, 0.25)
    A_low, B_low, C_low = bulk_ABC(LDG["a"], LDG["b"], LDG["c"], T_LOW, LDG["T_star"])
    ours = {t: [] for t in TAUS}
    theirs = {t: [] for t in TAUS}
    s = KZMSolver(N, N, N, D, D, D, KAPPA, GAMMA)
    for tau in TAUS:
        total = tau + HOLD
        coeffs = [bulk_ABC(LDG["a"], LDG["b"], LDG["c"], temperature(it, tau), LDG["T_star"]) for it in range(total)]
        for seed in SEEDS:
            q0 = oracle.bulk_init(bp, 5000 + seed, 1e-3)
            s.upload(q0)
            for it, (A, B, Cc) in enumerate(coeffs):
                s.step(1, A, B, Cc, dt, noise_sigma=sigma, seed=5000 + seed, step_index=it)
            ours[tau].append(s.observe(A_low, B_low, C_low)["defect_line_density"])
            qr, (A, B, Cc) = ref.quench(bp, q0, 5000 + seed, LDG["a"], LDG["b"], LDG["c"], LDG["T_star"], T_HIGH,
                                        T_LOW, 0, tau, total, NOISE_STRENGTH)
            assert (A, B, Cc) == pytest.approx((A_low, B_low, C_low), rel=1e-15)
            theirs[tau].append(ref.observe(bp, qr, A, B, Cc)["defect_line_density"])
    s.close()
    rows_o = [ours[t] for t in TAUS]
    rows_r = [theirs[t] for t in TAUS]
    slope_o, corr_o = fit_slope(TAUS, rows_o)
    slope_r, corr_r = fit_slope(TAUS, rows_r)
    sd_o, sd_r = bootstrap_sd(TAUS, rows_o), bootstrap_sd(TAUS, rows_r, seed=1)
    rec = dict(box=N, dt=dt, taus=TAUS, hold=HOLD, seeds=len(SEEDS), ours=rows_o, reference=rows_r,
               slope_ours=slope_o, slope_ours_sd=sd_o, corr_ours=corr_o, slope_reference=slope_r,
               slope_reference_sd=sd_r, corr_reference=corr_r, published_slope=-0.515)
    out = os.environ.get("LDG_ACCURACY_OUT")
    if out:
        with open(f"{out}.kz_rate_scan" + ("" if N == 64 else f"_{N}"), "w") as f:
            json.dump(rec, f)
    n = len(SEEDS)
    for t, a, b in zip(TAUS, rows_o, rows_r):
        se = math.sqrt(np.var(a, ddof=1) / n + np.var(b, ddof=1) / n)
        assert abs(np.mean(a) - np.mean(b)) <= 4.0 * se + 1e-3 * abs(np.mean(b)), (t, np.mean(a), np.mean(b), se)
    # the same trend with the quench time on both sides (its sign is the physics of this regime,
    # not a parity property: here the cubic B term and the thermal noise order the box within a few
    # hundred steps of crossing T*, faster than any of these ramps)
    assert abs(slope_o - slope_r) <= 3.0 * math.sqrt(sd_o ** 2 + sd_r ** 2), rec
