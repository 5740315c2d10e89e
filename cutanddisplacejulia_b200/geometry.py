"""Host-side mesh geometry and elastic-constant helpers that feed the TD path:
CreateFaceNormalAndMidPoint (src/CreateFaceNormalAndMidPoint.jl:137-185 with
CreateTriangleNormal! and CreateMidPoint!), CreateP1P2P3
(src/CreateP1P2P3.jl, by direct indexing instead of a search),
CalculateSSandDSDirs (src/CalculateSSandDSDirs.jl), AreaOfTriangle3D and
ElasticConstantsCheck(G, nu) (src/ElasticConstantsCheck.jl:83-95), plus
readers for the reference's mesh formats (ASCII STL, GoCad TSurf, OFF).
O(N) host work; not on the GPU hot path."""
from __future__ import annotations

import numpy as np


def CreateFaceNormalAndMidPoint(P1, P2, P3):
    """Unit normal of (P2-P1)x(P3-P1) and the incentre of every triangle."""
    P1, P2, P3 = (np.asarray(p, dtype=np.float64).reshape(-1, 3) for p in (P1, P2, P3))
    U, V = P2 - P1, P3 - P1
    Nv = np.cross(U, V)
    normal = Nv / np.sqrt((Nv * Nv).sum(1))[:, None]
    c = np.sqrt(((P1 - P2) ** 2).sum(1))
    a = np.sqrt(((P2 - P3) ** 2).sum(1))
    b = np.sqrt(((P1 - P3) ** 2).sum(1))
    if np.any((a == 0) | (b == 0) | (c == 0)):
        raise ValueError("Slither triangles or triangles with no area exist on your surface")
    mid = (P1 * a[:, None] + P2 * b[:, None] + P3 * c[:, None]) / (a + b + c)[:, None]
    return normal, mid


def CreateP1P2P3(Triangles, Points):
    """Vertex lists from a triangle index table (1-based ids in Points[:, 0])."""
    Points = np.asarray(Points, dtype=np.float64)
    ids = Points[:, 0].astype(np.int64)
    lookup = {v: k for k, v in enumerate(ids)}
    T = np.asarray(Triangles, dtype=np.int64)
    rows = np.vectorize(lookup.__getitem__)(T)
    xyz = Points[:, 1:4]
    return xyz[rows[:, 0]], xyz[rows[:, 1]], xyz[rows[:, 2]]


def ss_ds_dirs(cx, cy, cz):
    """Strike-slip and dip-slip direction cosines of element normals."""
    cx, cy, cz = (np.atleast_1d(np.asarray(v, dtype=np.float64)) for v in (cx, cy, cz))
    with np.errstate(invalid="ignore", divide="ignore"):
        nrm = np.sqrt(cx * cx + cy * cy)
        r1, r2 = cx / nrm, cy / nrm
    ss = np.stack([-r2, r1, np.zeros_like(cx)], axis=1)
    dsz = np.cos(np.arccos(cz) - np.pi / 2)
    L = np.sin(np.arccos(dsz))
    L = np.where(cz < 0, -L, L)
    a = np.arctan2(cy, cx)
    ds = np.stack([-np.cos(a) * L, -np.sin(a) * L, dsz], axis=1)
    vert = (cx == 0) & (cy == 0)
    ds[vert] = [-1.0, 0.0, 0.0]
    ss[vert & (cz < 1.0)] = [0.0, -1.0, 0.0]
    ss[vert & ~(cz < 1.0)] = [0.0, 1.0, 0.0]
    return ss, ds


CalculateSSandDSDirs = ss_ds_dirs


def AreaOfTriangle3D(P1, P2, P3):
    """Heron area and half perimeter of every triangle."""
    a = np.sqrt(((P2 - P3) ** 2).sum(1))
    b = np.sqrt(((P1 - P3) ** 2).sum(1))
    c = np.sqrt(((P1 - P2) ** 2).sum(1))
    s = (a + b + c) / 2
    return np.sqrt(s * (s - a) * (s - b) * (s - c)), s


def _elastic_from(vals):
    """(K, E, lambda, nu, G) of an isotropic material from any two of them
    (dict with two of the keys K, E, lam, nu, G), by the standard conversions."""
    from math import sqrt
    k = set(vals)
    K, E, lam, nu, G = (vals.get(x) for x in ("K", "E", "lam", "nu", "G"))
    if k == {"G", "nu"}:
        K, E, lam = 2 * G * (1 + nu) / (3 * (1 - 2 * nu)), 2 * G * (1 + nu), 2 * G * nu / (1 - 2 * nu)
    elif k == {"K", "E"}:
        lam, nu, G = 3 * K * (3 * K - E) / (9 * K - E), (3 * K - E) / (6 * K), 3 * K * E / (9 * K - E)
    elif k == {"K", "lam"}:
        E, nu, G = 9 * K * (K - lam) / (3 * K - lam), lam / (3 * K - lam), 1.5 * (K - lam)
    elif k == {"K", "nu"}:
        E, lam, G = 3 * K * (1 - 2 * nu), 3 * K * nu / (1 + nu), 3 * K * (1 - 2 * nu) / (2 * (1 + nu))
    elif k == {"K", "G"}:
        E, lam, nu = 9 * K * G / (3 * K + G), (3 * K - 2 * G) / 3, (3 * K - 2 * G) / (6 * K + 2 * G)
    elif k == {"E", "lam"}:
        R = sqrt(E * E + 9 * lam * lam + 2 * E * lam)
        K, nu, G = (E + 3 * lam + R) / 6, 2 * lam / (E + lam + R), (E - 3 * lam + R) / 4
    elif k == {"E", "nu"}:
        K, lam, G = E / (3 * (1 - 2 * nu)), E * nu / ((1 + nu) * (1 - 2 * nu)), E / (2 * (1 + nu))
    elif k == {"E", "G"}:
        K, lam, nu = E * G / (3 * (3 * G - E)), G * (E - 2 * G) / (3 * G - E), (E - 2 * G) / (2 * G)
    elif k == {"lam", "nu"}:
        K, E, G = lam * (1 + nu) / (3 * nu), lam * (1 + nu) * (1 - 2 * nu) / nu, lam * (1 - 2 * nu) / (2 * nu)
    elif k == {"lam", "G"}:
        K, E, nu = (3 * lam + 2 * G) / 3, G * (3 * lam + 2 * G) / (lam + G), lam / (2 * (lam + G))
    else:
        raise TypeError("ElasticConstantsCheck needs two different elastic constants")
    return K, E, lam, nu, G


def ElasticConstantsCheck(a, b):
    """(K, E, lambda, nu, G) from any two elastic constants
    (src/ElasticConstantsCheck.jl): typed values (ShearModulus, PoissonsRatio,
    BulkModulus, YoungsModulus, LamesConstant) in either order, or plain
    numbers taken as (G, nu)."""
    from .structs import BulkModulus, LamesConstant, PoissonsRatio, ShearModulus, YoungsModulus
    typed = {ShearModulus: "G", PoissonsRatio: "nu", BulkModulus: "K", YoungsModulus: "E", LamesConstant: "lam"}
    if type(a) in typed and type(b) in typed:
        vals = {}
        for x in (a, b):
            key = typed[type(x)]
            vals[key] = float(getattr(x, key))
        if len(vals) != 2:
            raise TypeError("ElasticConstantsCheck needs two different elastic constants")
        return _elastic_from(vals)
    return _elastic_from({"G": a, "nu": b})


def _rows(c, like):
    """Per-element cosines broadcast along the rows of `like` (element i on row i)."""
    c = np.asarray(c, dtype=np.float64).reshape(-1)
    like = np.asarray(like)
    return c.reshape((-1,) + (1,) * (like.ndim - 1)) if like.ndim > 1 else c


def CalculateNormalTraction3D(Pxx, Pyy, Pzz, Pxy, Pxz, Pyz, CosAx, CosAy, CosAz):
    """Normal traction n.sigma.n of each row's stress on that row's element
    (src/CalculateNormalTraction3D.jl); stresses are vectors or matrices whose
    row i belongs to element i."""
    cx, cy, cz = (_rows(c, Pxx) for c in (CosAx, CosAy, CosAz))
    return (Pxx * (cx * cx) + Pyy * (cy * cy) + Pzz * (cz * cz) + 2 * Pxy * (cx * cy) + 2 * Pyz * (cy * cz)
            + 2 * Pxz * (cz * cx))


def TractionVectorCartesianComponents3D(Pxx, Pyy, Pzz, Pxy, Pxz, Pyz, CosAx, CosAy, CosAz):
    """Traction vector sigma.n (Tx, Ty, Tz) (src/TractionVectorCartesianComponents3D.jl)."""
    cx, cy, cz = (_rows(c, Pxx) for c in (CosAx, CosAy, CosAz))
    return (Pxx * cx + Pxy * cy + Pxz * cz, Pxy * cx + Pyy * cy + Pyz * cz, Pxz * cx + Pyz * cy + Pzz * cz)


def CalculateTractionInChosenDirection3D(Tx, Ty, Tz, CosAx, CosAy, CosAz, ChosenDirectionCos):
    """Shear traction (I - n n^T) t projected on a direction in the element
    plane (src/CalculateTractionInChosenDirection3D.jl); ChosenDirectionCos is
    N x 3, one direction per element."""
    cx, cy, cz = (_rows(c, Tx) for c in (CosAx, CosAy, CosAz))
    D = np.asarray(ChosenDirectionCos, dtype=np.float64).reshape(-1, 3)
    d1, d2, d3 = (_rows(D[:, k], Tx) for k in range(3))
    a = (Tx * (1 - cx * cx) - Ty * (cx * cy) - Tz * (cz * cx)) * d1
    b = (Tx * -(cx * cy) + Ty * (1 - cy * cy) - Tz * (cy * cz)) * d2
    c = (Tx * -(cz * cx) - Ty * (cy * cz) + Tz * (1 - cz * cz)) * d3
    return a + b + c


def TensorTransformation3D(Txx1, Tyy1, Tzz1, Txy1, Txz1, Tyz1, A):
    """Symmetric tensor in the frame whose axes are the rows of the 3 x 3
    direction-cosine matrix A: T2 = A T1 A^T (src/TensorTransformation3D.jl)."""
    A = np.asarray(A, dtype=np.float64).reshape(3, 3)

    def comp(p, q):
        ap, aq = A[p, :], A[q, :]
        return (ap[0] * aq[0] * Txx1 + ap[1] * aq[1] * Tyy1 + ap[2] * aq[2] * Tzz1
                + (ap[0] * aq[1] + ap[1] * aq[0]) * Txy1 + (ap[0] * aq[2] + ap[2] * aq[0]) * Txz1
                + (ap[1] * aq[2] + ap[2] * aq[1]) * Tyz1)
    return comp(0, 0), comp(1, 1), comp(2, 2), comp(0, 1), comp(0, 2), comp(1, 2)


def read_stl(path):
    """ASCII STL (src/STLReader.jl): Points (id, x, y, z), Triangles (1-based)."""
    pts = []
    with open(path) as f:
        for line in f:
            tok = line.split()
            if tok and tok[0] == "vertex":
                pts.append([float(t) for t in tok[1:4]])
    pts = np.asarray(pts, dtype=np.float64)
    n = len(pts)
    Points = np.column_stack([np.arange(1, n + 1, dtype=np.float64), pts])
    Triangles = np.arange(1, n + 1, dtype=np.int64).reshape(-1, 3)
    return Points, Triangles


def read_gocad(path):
    """GoCad ASCII TSurf (src/GoCadAsciiReader.jl): VRTX / ATOM / TRGL records, renumbered 1..n."""
    coords, tris = {}, []
    with open(path) as f:
        for line in f:
            tok = line.split()
            if not tok:
                continue
            if tok[0] == "PROJECTION":
                raise ValueError("More than one Gocad ascii surface in the file, this function can only deal with 1")
            if tok[0] in ("VRTX", "PVRTX"):
                coords[int(tok[1])] = [float(t) for t in tok[2:5]]
            elif tok[0] in ("ATOM", "PATOM"):
                coords[int(tok[1])] = coords[int(tok[2])]
            elif tok[0] == "TRGL":
                tris.append([int(t) for t in tok[1:4]])
    ids = sorted(coords)
    new = {v: k + 1 for k, v in enumerate(ids)}
    Points = np.array([[new[v]] + coords[v] for v in ids], dtype=np.float64)
    Triangles = np.array([[new[v] for v in t] for t in tris], dtype=np.int64)
    return Points, Triangles


def read_off(path):
    """OFF mesh (src/OFFReader.jl): 0-based face indices become 1-based."""
    with open(path) as f:
        tok = [t for line in f for t in line.split("#")[0].split()]
    assert tok[0].upper().endswith("OFF")
    nv, nf = int(tok[1]), int(tok[2])
    k = 4
    pts = np.array(tok[k:k + 3 * nv], dtype=np.float64).reshape(nv, 3)
    k += 3 * nv
    tris = []
    for _ in range(nf):
        c = int(tok[k])
        tris.append([int(t) + 1 for t in tok[k + 1:k + 1 + c]])
        k += 1 + c
    Points = np.column_stack([np.arange(1, nv + 1, dtype=np.float64), pts])
    return Points, np.asarray(tris, dtype=np.int64)


def HookesLaw3DStrain2Stress(*args):
    """Hooke's law, strain -> stress (src/HookesLaw3DStrain2Stress.jl:1-57):
    sigma = 2 G eps + lambda tr(eps) I.  Either (Exx, Eyy, Ezz, Exy, Exz, Eyz,
    lam, G) -> the six components, or (Strains, lam, G) -> Stresses."""
    from .structs import Strains, Stresses
    if len(args) == 3 and isinstance(args[0], Strains):
        S, lam, G = args
        return Stresses(*HookesLaw3DStrain2Stress(*list(S), lam, G))
    Exx, Eyy, Ezz, Exy, Exz, Eyz, lam, G = (np.asarray(a, dtype=np.float64) if k < 6 else a
                                            for k, a in enumerate(args))
    tr = lam * (Exx + Eyy + Ezz)
    return (2 * G * Exx + tr, 2 * G * Eyy + tr, 2 * G * Ezz + tr, 2 * G * Exy, 2 * G * Exz, 2 * G * Eyz)
