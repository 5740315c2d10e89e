"""CPU tests: the oracle against the reference's own known-answer tests.

  Okada (1985) half-space surface field   test/test_TDvsOkada.jl (<= 1e-13)
  traction-free crack, 5 orientations      test/test_TractionFreeSurface.jl (<= 1e-8)
  Eshelby penny crack slip                 test/test_TDvsEshelbyPennyCrack.jl (<= 11 %)
  Mogi cavity with fixed elements          test/test_TDvsMogi.jl (spread <= 0.05, <= 20 %)
  Savage (1984) gravitational valley       test/test_TDvsSavageGravityValley.jl (mean residual <= 0.15)
plus self-consistency of the oracle (influence matrices + TD_sum == summing
overload; strain == symmetric gradient of displacement at depth, FS and HS).
"""
import os

import numpy as np
import pytest

from helpers import GOLDEN, load_mesh, okada_case, savage_valley_case, savage_valley_check


def test_okada_kat(oracle):
    from oracle import geometry as g
    from oracle import okada85
    c = okada_case()
    _, _, lam, nu, G = g.elastic_constants(1.0, 0.25)
    S, D = oracle.td_sum_eval(c["x"], c["y"], c["z"], c["P1"], c["P2"], c["P3"], [c["Dss"]] * 2, [c["Dds"]] * 2,
                              [c["Dn"]] * 2, nu, G, 1, 1, 1)
    total = np.sqrt(c["Dds"] ** 2 + c["Dss"] ** 2)
    rake = 90 - np.rad2deg(np.arctan(c["Dss"] / c["Dds"]))
    mid_depth = np.sin(np.deg2rad(c["Dip"])) * c["Width"] / 2 + c["TipDepth"]
    ok = okada85.okada85(c["x"], c["y"], mid_depth, c["Strike"], c["Dip"], c["Length"], c["Width"], rake, total,
                         c["Dn"], nu)
    td = list(D) + list(S)
    for a, b in zip(td, ok):
        assert np.max(np.abs(a - b)) <= 1e-13


def _traction_free_max(oracle, P1, P2, P3, bcs, nu, G, lam):
    from oracle import geometry as g
    nrm, mid = g.face_normal_and_midpoint(P1, P2, P3)
    n = len(P1)
    worst = 0.0
    for bc in bcs:
        s = [np.zeros(n) for _ in range(6)]
        s[bc] = np.ones(n)
        Tn, Tds, Tss = oracle.normal_and_shear_tractions(*s, nrm)
        Dn, Dss, Dds, A, b = oracle.slip_calculator(P1, P2, P3, nu, G, lam, mid, nrm, 0, Tn, Tss, Tds)
        S, _ = oracle.td_sum_eval(mid[:, 0], mid[:, 1], mid[:, 2], P1, P2, P3, Dss, Dds, Dn, nu, G, 0, 1, 0)
        st = oracle.hookes_law(S, lam, G)
        st = [st[k] + s[k] for k in range(6)]
        tn, tds, tss = oracle.normal_and_shear_tractions(*st, nrm)
        worst = max(worst, np.abs(tn).max(), np.abs(tds).max(), np.abs(tss).max())
    return worst


def test_traction_free_kat(oracle):
    from oracle import geometry as g
    P = list(load_mesh("squaregrid"))
    for p in P:
        p[:, 2] = 0.0
    _, _, lam, nu, G = g.elastic_constants(5000.0, 0.25)
    # stress component index: xx 0, yy 1, zz 2, xy 3, xz 4, yz 5
    steps = [(lambda p: p, [4, 5, 2]),
             (lambda p: p[:, [1, 0, 2]], [4, 5, 2]),          # flip normal (swap x, y)
             (lambda p: p[:, [0, 2, 1]], [3, 5, 1]),          # vertical (swap y, z)
             (lambda p: p * np.array([-1, 1, 1.0]), [3, 5, 1]),
             (lambda p: p[:, [1, 0, 2]], [3, 4, 0]),          # strike 0 (swap x, y)
             (lambda p: p * np.array([1, -1, 1.0]), [3, 4, 0])]
    for fn, bcs in steps:
        P = [fn(p) for p in P]
        assert _traction_free_max(oracle, *P, bcs, nu, G, lam) <= 1e-8


def test_eshelby_kat(oracle):
    from oracle import geometry as g
    P1, P2, P3 = load_mesh("circle581")
    _, _, lam, nu, G = g.elastic_constants(1.0, 0.25)
    nrm, mid = g.face_normal_and_midpoint(P1, P2, P3)
    n = len(P1)
    rho = np.hypot(mid[:, 0], mid[:, 1])
    good = rho < 0.9
    Dn, Dss, Dds, _, _ = oracle.slip_calculator(P1, P2, P3, nu, G, lam, mid, nrm, 0, np.zeros(n), np.ones(n),
                                                np.zeros(n))
    us = 2 * ((4 * (1 - nu) * 1.0) / (np.pi * (2 - nu) * G)) * np.sqrt(1 - rho ** 2)
    assert np.max(np.abs(np.sqrt(Dss ** 2 + Dds ** 2) / us * 100 - 100)[good]) <= 11
    Dn, _, _, _, _ = oracle.slip_calculator(P1, P2, P3, nu, G, lam, mid, nrm, 0, np.ones(n), np.zeros(n), np.zeros(n))
    un = 2 * ((2 * (1 - nu)) / (np.pi * G)) * np.sqrt(1 - rho ** 2)
    assert np.max(np.abs(Dn / un * 100 - 100)[good]) <= 11


def test_inf_plus_td_sum_equals_summing(oracle):
    rng = np.random.default_rng(3)
    from helpers import random_points, random_triangles
    P1, P2, P3 = random_triangles(rng, 7)
    pts = random_points(rng, 60)
    sl = rng.uniform(-1, 1, (3, 7))
    for hs in (0, 1):
        Si, Di = oracle.td_inf(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, hs)
        S2, D2 = oracle.td_sum(Si, Di)
        S, D = oracle.td_sum_eval(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, hs, nthreads=1)
        assert np.max(np.abs(S2 - S)) <= 1e-12 * np.max(np.abs(S))
        assert np.max(np.abs(D2 - D)) <= 1e-12 * np.max(np.abs(D))


@pytest.mark.parametrize("hs", [0, 1])
def test_strain_is_gradient_of_displacement(oracle, hs):
    rng = np.random.default_rng(1)
    P1 = np.array([[-1.0, 0.2, -1.0], [0.5, -0.3, -2.0]])
    P2 = np.array([[1.0, -0.1, -1.3], [1.2, 0.4, -1.1]])
    P3 = np.array([[0.1, 0.9, -2.2], [-0.2, 0.8, -1.5]])
    sl = rng.uniform(-1, 1, (3, 2))
    pts = rng.uniform([-3, -3, -4], [3, 3, -0.2], (40, 3))
    h = 1e-5
    S, _ = oracle.td_sum_eval(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 0, 1, hs)
    grad = np.zeros((3, 3, len(pts)))
    for k in range(3):
        dp = np.zeros(3)
        dp[k] = h
        _, Up = oracle.td_sum_eval(*(pts + dp).T, P1, P2, P3, *sl, 0.25, 1.0, 1, 0, hs)
        _, Um = oracle.td_sum_eval(*(pts - dp).T, P1, P2, P3, *sl, 0.25, 1.0, 1, 0, hs)
        grad[:, k] = (Up - Um) / (2 * h)
    eps = np.stack([grad[0, 0], grad[1, 1], grad[2, 2], (grad[0, 1] + grad[1, 0]) / 2,
                    (grad[0, 2] + grad[2, 0]) / 2, (grad[1, 2] + grad[2, 1]) / 2])
    assert np.max(np.abs(eps - S)) / np.max(np.abs(S)) < 1e-6


def test_hs_above_surface_raises(oracle):
    P1 = np.array([[0.0, 0.0, -1.0]])
    P2 = np.array([[1.0, 0.0, -1.0]])
    P3 = np.array([[0.0, 1.0, 0.5]])
    with pytest.raises(oracle.OracleError, match="Z coordinates must be negative"):
        oracle.td_inf([0.0], [0.0], [-1.0], P1, P2, P3, [1.0], [1.0], [1.0], 0.25, 1.0, 1, 1, 1)
    with pytest.raises(oracle.OracleError, match="Z coordinates must be negative"):
        oracle.td_inf([0.0], [0.0], [0.1], P1 - [0, 0, 2], P2, P3 - [0, 0, 2], [1.0], [1.0], [1.0], 0.25, 1.0, 1, 1, 1)


def test_dims_error(oracle):
    P = np.zeros((2, 3))
    with pytest.raises(oracle.OracleError, match="Element size inputs must be the same dimensions"):
        oracle.td_inf([0.0], [0.0], [-1.0], P, P, P, [1.0], [1.0, 1.0], [1.0, 1.0], 0.25, 1.0, 1, 1, 0)


def test_mogi_kat(oracle):
    # test/test_TDvsMogi.jl: a 46-face sphere 50 below the free surface, 6
    # fixed elements (SphereFix4 scaled x3) appended, unit pressure; the
    # opening must be near uniform (spread <= 0.05 / G) and the surface
    # displacement within 20 % of Mogi (1958) at x = 0..100
    from oracle import geometry as g
    d = np.load(os.path.join(GOLDEN, "mogi.npz"))
    P1, P2, P3, fixed = d["P1"], d["P2"], d["P3"], d["FixedEls"]
    nrm, mid = g.face_normal_and_midpoint(P1, P2, P3)
    _, _, lam, nu, G = g.elastic_constants(1.0, 0.25)
    n = len(P1)
    Dn, Dss, Dds, A, b = oracle.slip_calculator_fixed(P1, P2, P3, nu, G, lam, mid, nrm, 1, np.ones(n), np.zeros(n),
                                                      np.zeros(n), fixed)
    assert A.shape == (3 * n, 3 * int((fixed == 0).sum()))
    assert Dn.max() - Dn.min() <= 0.05 / G
    free = fixed == 0
    X = np.arange(0.0, 101.0)
    Y, Z = np.zeros_like(X), np.zeros_like(X)
    _, U = oracle.td_sum_eval(X, Y, Z, P1[free], P2[free], P3[free], Dss, Dds, Dn, nu, G, 1, 0, 1)
    An = oracle.mogi_spherical_cavity(50.0, X, Y, 1.0, 1.0, nu, G)
    with np.errstate(divide="ignore", invalid="ignore"):
        for a, u in zip(An, U):
            pct = 100.0 / a * u
            pct[np.isinf(pct)] = np.nan
            assert not np.any(np.abs(pct - 100) > 20)


def test_savage_valley_kat(oracle):
    c = savage_valley_case()
    n = len(c["P1"])
    assert n == 1019
    Tn, Tds, Tss = oracle.normal_and_shear_tractions(*c["sig"], c["nrm"])
    Dn, Dss, Dds, _, _ = oracle.slip_calculator(c["P1"], c["P2"], c["P3"], c["nu"], c["G"], c["lam"], c["mid"],
                                                c["nrm"], 0, Tn, Tss, Tds)
    S, _ = oracle.td_sum_eval(c["X"], c["Y"], c["Z"], c["P1"], c["P2"], c["P3"], Dss, Dds, Dn, c["nu"], c["G"], 1,
                              1, 0)
    means = savage_valley_check(c, S)
    # the oracle's residuals (about -0.040, -0.028, 0.002) are well inside the bound on both sides
    assert max(abs(m) for m in means) < 0.06


def test_oracle_independent_of_thread_count(oracle):
    """Determinism of the oracle: influence matrices, the traction assembly and
    the summing overload give the same bits on 1 and 4 threads."""
    rng = np.random.default_rng(11)
    from helpers import random_points, random_triangles
    P1, P2, P3 = random_triangles(rng, 23)
    pts = random_points(rng, 150)
    sl = rng.uniform(-1, 1, (3, 23))
    for hs in (0, 1):
        a = oracle.td_inf(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, hs, nthreads=1)
        b = oracle.td_inf(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, hs, nthreads=4)
        assert all(np.array_equal(x, y, equal_nan=True) for x, y in zip(a, b))
        a = oracle.td_sum_eval(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, hs, nthreads=1)
        b = oracle.td_sum_eval(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, hs, nthreads=4)
        assert all(np.array_equal(x, y, equal_nan=True) for x, y in zip(a, b))
    from oracle import geometry as g
    P1, P2, P3 = load_mesh("circle581")
    nrm, mid = g.face_normal_and_midpoint(P1, P2, P3)
    A1 = oracle.influence_traction(nrm, mid, P1, P2, P3, 0.25, 1.0, 1.0, 0, nthreads=1, want_A=True)
    A4 = oracle.influence_traction(nrm, mid, P1, P2, P3, 0.25, 1.0, 1.0, 0, nthreads=4, want_A=True)
    assert np.array_equal(A1, A4)
