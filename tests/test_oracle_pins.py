"""Pins the FP64 CPU oracle to the reference's own code (CPU only).

* Per-cell math against the reference's QSR.cpp functions compiled from its sources
  (Laplacian QSR.cpp:179, chemical potential 559, energy 411, nematic 10).
* Analytic known answers from the reference's formulas (S_eq, uniform nematic stationarity).
* Philox4x32-10 against the published Random123 known-answer vectors.
"""
import math

import numpy as np
import pytest

from oracle.oracle import make_params

CASES = [
    dict(L1=0.0, kappa=6.5e-12),
    dict(L1=6e-12),
    dict(L1=6e-12, L2=3e-12),
    dict(L1=6e-12, L2=3e-12, L3=1e-12),
    dict(L1=6e-12, L3=2e-12, bulk_modechoice=2),
    dict(L1=4e-12, L2=-1e-12, L3=-1e-12, dy=1.3e-8, dz=0.8e-8),
]


@pytest.mark.parametrize("kw", CASES)
def test_chem_potential_matches_reference_cpu(oracle, refcpu, kw):
    p = make_params(Nx=13, Ny=11, Nz=12, **kw)
    g, fl = oracle.geometry(p)
    rng = np.random.default_rng(7)
    q = rng.normal(0, 0.2, p.Nx * p.Ny * p.Nz * 5)
    mo = oracle.chem_potential(p, g, fl, q, 300.0, 0.5)
    mr = refcpu.chem_potential(p, q, 300.0)
    # bit-identical except for the reference CPU's single traceless projection with L3
    assert np.abs(mo - mr).max() <= 1e-14 * np.abs(mr).max()


@pytest.mark.parametrize("kw", CASES)
def test_laplacian_and_energy_match_reference_cpu(oracle, refcpu, kw):
    p = make_params(Nx=10, Ny=9, Nz=12, **kw)
    g, fl = oracle.geometry(p)
    q = np.random.default_rng(3).normal(0, 0.3, p.Nx * p.Ny * p.Nz * 5)
    assert np.array_equal(oracle.laplacian(p, q), refcpu.laplacian(p, q))
    eo = oracle.observe(p, g, fl, q, 301.0, 0.5)
    b, e = refcpu.energy(p, q, 301.0)
    assert eo["bulk"] == pytest.approx(b, rel=1e-13)
    assert eo["elastic"] == pytest.approx(e, rel=1e-13)


def test_nematic_matches_reference_cpu(oracle, refcpu):
    rng = np.random.default_rng(11)
    q = rng.normal(0, 0.3, 5 * 200)
    q[:5] = 0.0  # isotropic cut-off case
    on = oracle.nematic(q)
    for c in range(200):
        assert np.array_equal(on[c], refcpu.nematic(q[5 * c:5 * c + 5]))


def test_uniform_nematic_is_bulk_stationary(oracle):
    # Q = S_eq (n n - I/3) is a bulk stationary point (QSR.cu:1391-1418): mu = 0 in the interior
    # with strong anchoring off.
    p = make_params(Nx=8, Ny=8, Nz=8, L1=6e-12, W=1e-12, droplet_radius_cells=1.0)
    A, B, C = oracle.bulk_ABC(p.a, p.b, p.c, 300.0, p.T_star)
    S = oracle.S_eq(A, B, C)
    assert S > 0.5
    n = np.array([1.0, 2.0, 2.0]) / 3.0
    q5 = S * np.array([n[0] * n[0] - 1 / 3, n[0] * n[1], n[0] * n[2], n[1] * n[1] - 1 / 3, n[1] * n[2]])
    q = np.tile(q5, p.Nx * p.Ny * p.Nz)
    g, fl = oracle.geometry(p)
    mu = oracle.chem_potential(p, g, fl, q, 300.0, S).reshape(-1, 5)
    interior = (fl & 1) == 0  # away from the (tiny) anchoring shell
    assert np.abs(mu[interior]).max() < 1e-9 * abs(A) * S
    # energy density equals f(S) = (A/3)S^2 - (2B/27)S^3 + (C/9)S^4 on interior cells
    o = oracle.observe(p, g, fl, q, 300.0, S)
    fS = (A / 3) * S * S - (2 * B / 27) * S ** 3 + (C / 9) * S ** 4
    dV = p.dx * p.dy * p.dz
    assert o["bulk"] == pytest.approx(fS * dV * (p.Nx - 2) * (p.Ny - 2) * (p.Nz - 2), rel=1e-12)
    assert o["elastic"] == pytest.approx(0.0, abs=1e-30)


def test_S_eq_known_answer(oracle):
    # 2 C S^2 - B S + 3 A = 0 at T = 300 K, T* = 307 K (std convention)
    A, B, C = oracle.bulk_ABC(0.044e6, 1.413e6, 1.153e6, 300.0, 307.0)
    S = oracle.S_eq(A, B, C)
    assert 2 * C * S * S - B * S + 3 * A == pytest.approx(0.0, abs=1e-6 * B)
    # above the spinodal the nematic root disappears
    A2, B2, C2 = oracle.bulk_ABC(0.044e6, 1.413e6, 1.153e6, 330.0, 307.0)
    assert oracle.S_eq(A2, B2, C2) == 0.0


def test_philox_known_answers(oracle):
    # Random123 kat_vectors for philox4x32_10
    assert oracle.philox([0, 0, 0, 0], [0, 0]) == [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]
    assert oracle.philox([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2) == [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]
    assert oracle.philox([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0]) == [
        0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]


def test_geometry_matches_reference_formula(oracle):
    # Default radius 0.5*(min(N)-1)*d centred at (N-1)/2 (QSR.cu:144-162); shell |sd| <= dx.
    p = make_params(Nx=32, Ny=32, Nz=32)
    g, fl = oracle.geometry(p)
    assert g.radius_x == pytest.approx(15.5e-8)
    assert g.center_x == pytest.approx(15.5e-8)
    idx = np.indices((32, 32, 32)).reshape(3, -1).T.astype(float)
    r = np.sqrt(((idx - 15.5) ** 2).sum(1))
    shell = (fl & 1) != 0
    # for a sphere the signed distance is r - R
    assert np.array_equal(shell, np.abs(r - 15.5) <= 1.0 + 1e-12)
    inside = (fl & 4) != 0
    assert np.array_equal(inside, r <= 15.5)
    assert g.shell_count == shell.sum()
    # delta_eff = shell volume / sphere area
    assert g.delta_eff == pytest.approx(shell.sum() * 1e-24 / (4 * math.pi * (15.5e-8) ** 2), rel=1e-12)


def test_init_random_draw_order(oracle):
    # init_mode 0 draws theta, phi from mt19937(seed) in i-j-k order over inside cells
    # (QSR.cu:1841-1878); same seed -> same field, zero outside.
    p = make_params(Nx=12, Ny=12, Nz=12, droplet_radius_cells=4.0)
    g, fl = oracle.geometry(p)
    q1 = oracle.init(p, g, 0, 42, 0.5)
    q2 = oracle.init(p, g, 0, 42, 0.5)
    q3 = oracle.init(p, g, 0, 43, 0.5)
    assert np.array_equal(q1, q2) and not np.array_equal(q1, q3)
    outside = (fl & 4) == 0
    assert np.all(q1.reshape(-1, 5)[outside] == 0.0)
    nf = oracle.nematic(q1)
    idx = np.indices((12, 12, 12)).reshape(3, -1).T.astype(float)
    r = np.sqrt(((idx - 5.5) ** 2).sum(1))
    # S = S0 except inside the core radius (one cell) where it is scaled by r/core_radius
    far = (~outside) & (r >= 1.0)
    near = (~outside) & (r < 1.0)
    assert np.allclose(nf[far, 0], 0.5, atol=1e-6)
    assert np.allclose(nf[near, 0], 0.5 * r[near], atol=1e-6)
