"""Seeded test geometry shared by the tests (no reference files needed)."""
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_mesh(name):
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    return d["P1"].copy(), d["P2"].copy(), d["P3"].copy()


def random_triangles(rng, n, depth=(-3.0, -0.5), size=1.0, spread=2.0):
    """Random, well-shaped triangles below z=0."""
    c = rng.uniform([-spread, -spread, depth[0]], [spread, spread, depth[1]], (n, 3))
    P = []
    for k in range(3):
        ang = rng.uniform(0, 2 * np.pi, n) + k * 2 * np.pi / 3
        r = size * rng.uniform(0.5, 1.0, n)
        d = np.stack([r * np.cos(ang), r * np.sin(ang), rng.uniform(-0.5, 0.5, n) * size], axis=1)
        P.append(c + d)
    P1, P2, P3 = P
    top = np.maximum(np.maximum(P1[:, 2], P2[:, 2]), P3[:, 2])
    shift = np.where(top > -0.05, top + 0.05, 0.0)[:, None] * np.array([0, 0, 1.0])
    return P1 - shift, P2 - shift, P3 - shift


def random_points(rng, m, lo=(-4, -4, -5), hi=(4, 4, 0)):
    return rng.uniform(lo, hi, (m, 3))


def okada_case():
    """Geometry of the reference's Okada comparison (test/test_TDvsOkada.jl:9-66)."""
    from oracle import geometry as g
    Strike, Dip, Length, Width, TipDepth = 60.0, 45.0, 5.0, 5.0, 1.0
    X = np.array([-1, 1, -1, -1, 1, 1.0]) / 2 * Width
    Y = np.array([1, -1, -1, -1, 1, 1.0]) / 2 * Length
    Z = np.zeros(6)
    ss, ds, fn = g.direction_cosines_from_strike_and_dip(Strike, Dip)
    X, Y, Z = g.rotate_object_3d(X, Y, Z, ds, ss, fn)
    Z = Z - Z.max() - TipDepth
    P1 = np.array([[X[0], Y[0], Z[0]], [X[1], Y[1], Z[1]]])
    P2 = np.array([[X[4], Y[4], Z[4]], [X[3], Y[3], Z[3]]])
    P3 = np.array([[X[2], Y[2], Z[2]], [X[5], Y[5], Z[5]]])
    xx = np.linspace(-10, 10, 50)
    gx, gy = np.meshgrid(xx, xx)
    x = gx.reshape(-1, order="F")
    y = gy.reshape(-1, order="F")
    return dict(P1=P1, P2=P2, P3=P3, x=x, y=y, z=np.zeros_like(x), Dss=0.5, Dds=2.0, Dn=0.6, Strike=Strike,
                Dip=Dip, Length=Length, Width=Width, TipDepth=TipDepth)


# Parity bounds between two FP64 evaluations of the same closed form.  The
# oracle itself sits up to ~1e-12 (per field) from a long-double evaluation in
# half space, because the real, image and free-surface parts cancel; so parity
# is stated norm-wise over each output tensor, and per field with a floor.
TENSOR_TOL = 1e-12
FIELD_TOL = 1e-11
FIELD_FLOOR = 1e-3


def parity(gpu, ref):
    """Norm-wise relative error of a stacked output (fields x ...) and the worst
    per-field error, each field scaled by max(own max, FIELD_FLOOR * tensor max).
    NaN masks must agree."""
    g = np.asarray(gpu, dtype=np.float64)
    r = np.asarray(ref, dtype=np.float64)
    assert g.shape == r.shape
    ng, nr = np.isnan(g), np.isnan(r)
    assert np.array_equal(ng, nr), "NaN masks differ: %d vs %d" % (ng.sum(), nr.sum())
    fin = ~nr
    if not fin.any():
        return 0.0, 0.0
    d = np.where(fin, np.abs(g - r), 0.0)
    a = np.where(fin, np.abs(r), 0.0)
    scale = a.max()
    if scale == 0:
        return float(d.max()), float(d.max())
    tensor = float(d.max() / scale)
    worst = 0.0
    for f in range(g.shape[0]):
        fs = max(a[f].max(), FIELD_FLOOR * scale)
        worst = max(worst, float(d[f].max() / fs))
    return tensor, worst


def assert_parity(gpu, ref, tensor_tol=TENSOR_TOL, field_tol=FIELD_TOL):
    t, f = parity(gpu, ref)
    assert t <= tensor_tol and f <= field_tol, "norm-wise %.2e (tol %.0e), worst field %.2e (tol %.0e)" % (
        t, tensor_tol, f, field_tol)
    return t, f


def rel_inf_err(a, b):
    """max|a-b| / max|b| over entries where b is finite; NaN masks must agree."""
    a = np.asarray(a)
    b = np.asarray(b)
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb), "NaN masks differ: %d vs %d" % (na.sum(), nb.sum())
    m = ~nb
    if not m.any():
        return 0.0
    scale = np.max(np.abs(b[m]))
    if scale == 0:
        return float(np.max(np.abs(a[m])))
    return float(np.max(np.abs(a[m] - b[m])) / scale)


def burgmann_case(half):
    """The two cracks of test/test_TDvsBurgmannLinearFrictionCrack.jl: the 497
    triangle blade fault flattened to y = 0 and scaled to half length 1e-4
    (half 1, driven by sxy, closed by syy) or turned into the z = 0 plane at
    half length 1e4 (half 2, driven by sxz, closed by szz); mu = 0 and
    cohesion Sf = |x| of each collocation point."""
    from oracle.geometry import elastic_constants, face_normal_and_midpoint
    P1, P2, P3 = load_mesh("blade500")
    for P in (P1, P2, P3):
        if half == 1:
            P[:, 1] = 0.0
        else:
            P[:, 1] = P[:, 2]
            P[:, 2] = 0.0
    S = 1e-4 if half == 1 else 1e4
    P1, P2, P3 = P1 * S, P2 * S, P3 * S
    nrm, mid = face_normal_and_midpoint(P1, P2, P3)
    n = len(P1)
    _, _, lam, nu, G = elastic_constants(1.0, 0.25)
    z = np.zeros(n)
    if half == 1:
        sig = (z, np.full(n, -0.05 * S), z, np.full(n, S), z, z)
    else:
        sig = (z, z, np.full(n, -0.05 * S), z, np.full(n, S), z)
    return dict(P1=P1, P2=P2, P3=P3, nrm=nrm, mid=mid, nu=nu, G=G, lam=lam, sig=sig, mu=0.0,
                Sf=np.abs(mid[:, 0]), S=S, n=n)


def burgmann_check(case, half, D_plain, D_fric):
    """The reference's acceptance of test/test_TDvsBurgmannLinearFrictionCrack.jl:
    near the crack centre line, slip within 36 % of the analytic profile on
    |x| < 0.9 a, and the summed percentage deviation at most 1400.  D_*: the
    shear component the case drives (Dss for half 1, Dds for half 2)."""
    from oracle import friction as F
    mid, S, G, nu = case["mid"], case["S"], case["G"], case["nu"]
    good = np.abs(mid[:, 2 if half == 1 else 1]) < S
    x = mid[good, 0]
    ana_u = F.pollard_segall1987_slip(G, nu, 0.0, S, x, S)
    ana_f = F.burgmann1994_slip(G, nu, S, x, S)
    pu = 100.0 / ana_u * np.abs(D_plain[good])
    pf = 100.0 / ana_f * np.abs(D_fric[good])
    pu[np.isinf(pu)] = np.nan
    pf[np.isinf(pf)] = np.nan
    assert np.sum(pu - 100) <= 1400 and np.sum(pf - 100) <= 1400, (np.sum(pu - 100), np.sum(pf - 100))
    inner = np.abs(x) < 0.9 * S
    assert not np.any(np.abs(pu[inner] - 100) > 36), np.nanmax(np.abs(pu[inner] - 100))
    assert not np.any(np.abs(pf[inner] - 100) > 36), np.nanmax(np.abs(pf[inner] - 100))


def random_lcp(rng, n, frac_active=0.5, frac_degenerate=0.0):
    """LCP (M, q) with a known unique solution x*: M = R R^T / n + I is
    positive definite; x* > 0 on a random subset, y* = M x* + q > 0 off it,
    both zero on a further fraction of rows (degenerate)."""
    R = rng.standard_normal((n, n))
    M = R @ R.T / n + np.eye(n)
    u = rng.uniform(size=n)
    act = u < frac_active
    deg = (u >= frac_active) & (u < frac_active + frac_degenerate)
    x = np.where(act, rng.uniform(0.5, 2.0, n), 0.0)
    y = np.where(act | deg, 0.0, rng.uniform(0.5, 2.0, n))
    q = y - M @ x
    return np.asfortranarray(M), q, x


def savage_valley_case():
    """test/test_TDvsSavageGravityValley.jl: the 1019-triangle valley surface
    in full space under gravitational stress (density x g = 1, no tectonic
    stress, nu = 0.25, G = 1), observed on the 50 x 46 grid of the Savage
    (1984) solution mapped under the valley (a = 2, b = -1), shifted to the
    valley centre x = 50."""
    from oracle.geometry import elastic_constants, face_normal_and_midpoint
    from oracle.savage84 import savage1984_gravity_valley_stress
    P1, P2, P3 = load_mesh("valley1000")
    nrm, mid = face_normal_and_midpoint(P1, P2, P3)
    _, _, lam, nu, G = elastic_constants(1.0, 0.25)
    rg = 1.0
    sxx = (nu / (1 - nu)) * rg * mid[:, 2]
    szz = rg * mid[:, 2]
    syy = nu * (sxx + szz)
    z = np.zeros(len(P1))
    u, v = np.meshgrid(np.linspace(0, 4, 50), np.linspace(-0.3265, -4, 46))
    Sxx, Syy, Sxy, Xo, Yo = savage1984_gravity_valley_stress(0.0, rg, nu, 2.0, -1.0, u, v)
    X = Xo.ravel(order="F") + 50
    Z = Yo.ravel(order="F")
    return dict(P1=P1, P2=P2, P3=P3, nrm=nrm, mid=mid, lam=lam, nu=nu, G=G, rg=rg,
                sig=(sxx, syy, szz, z, z, z), X=X, Y=np.zeros_like(X), Z=Z,
                an=(Sxx.ravel(order="F"), Syy.ravel(order="F"), Sxy.ravel(order="F")))


def savage_valley_check(case, strain6):
    """The reference's acceptance: gravity added back to the TD stresses,
    the signed mean residual of sxx, szz and sxz against Savage (NaNs
    dropped) each at most 0.15.  Returns the three means."""
    exx, eyy, ezz, exy, exz, eyz = strain6
    lam, G, nu, rg, Z = case["lam"], case["G"], case["nu"], case["rg"], case["Z"]
    tr = exx + eyy + ezz
    sxx = (nu / (1 - nu)) * rg * Z + 2 * G * exx + lam * tr
    szz = rg * Z + 2 * G * ezz + lam * tr
    sxz = 2 * G * exz
    Sxx, Syy, Sxy = case["an"]
    means = []
    for num, an in ((sxx, Sxx), (szz, Syy), (sxz, Sxy)):
        r = num - an
        means.append(float(np.mean(r[~np.isnan(r)])))
    assert not any(p > 0.15 for p in means), means
    return means


def oracle_system_columns(oracle, sample, P1, P2, P3, nrm, mid, nu, G, lam, hs):
    """Columns [sample; N + sample; 2N + sample] of the system matrix
    A = -[Atn; Atss; Atds] from the oracle's strain influences and traction
    conversion (src/CalculateInfluenceMatrices3D.jl:73-114)."""
    n = len(P1)
    obs = mid - 1e-12 * nrm
    k = len(sample)
    ones = np.ones(k)
    S, _ = oracle.td_inf(obs[:, 0], obs[:, 1], obs[:, 2], P1[sample], P2[sample], P3[sample], ones, ones, ones, nu,
                         G, 0, 1, hs)
    T = oracle.strain_to_traction(S, nrm, lam, G)
    ref = np.empty((3 * n, 3 * k))
    for m in range(3):
        for r in range(3):
            ref[r * n:(r + 1) * n, m * k:(m + 1) * k] = -T[3 * m + r]
    return ref

