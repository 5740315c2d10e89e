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
