"""Host mirror of the reference's influence assembly and plain slip solve:
CalculateInfluenceMatrices3D (src/CalculateInfluenceMatrices3D.jl:2-48),
SlipCalculator3D (src/SlipCalculator3D.jl:1-33), SetupTractionVector
(src/SetupTractionVector.jl), CalculateNormalAndShearTractions3D
(src/CalculateNormalAndShearTractions3D.jl), KnockOutFixedRows
(src/KnockOutFixedRows.jl).  Influence evaluation, traction conversion,
assembly and LU run in libcad_td.so; the per-element boundary-condition
algebra (O(N)) runs on the host as in the reference.
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .geometry import ss_ds_dirs
from .structs import MixedBoundaryConditions, MixedBoundaryConditionsFriction, Stresses, TractionInf, Tractions


def _tri(P):
    return np.asfortranarray(np.asarray(P, dtype=np.float64).reshape(-1, 3))


def _col(a, n):
    a = np.asarray(a, dtype=np.float64).reshape(-1)
    if a.size == 1 and n != 1:
        a = np.full(n, float(a[0]))
    return np.ascontiguousarray(a)


def CalculateNormalAndShearTractions3D(sxx, syy, szz, sxy, sxz, syz, FaceNormalVector):
    """Normal and shear tractions of a stress state on each element: (Tn, Tds, Tss)."""
    n = np.asarray(FaceNormalVector, dtype=np.float64).reshape(-1, 3)
    cx, cy, cz = n[:, 0], n[:, 1], n[:, 2]
    N = n.shape[0]
    sxx, syy, szz, sxy, sxz, syz = (_col(s, N) for s in (sxx, syy, szz, sxy, sxz, syz))
    ss, ds = ss_ds_dirs(cx, cy, cz)
    Tn = sxx * cx * cx + syy * cy * cy + szz * cz * cz + 2 * sxy * cx * cy + 2 * syz * cy * cz + 2 * sxz * cz * cx
    Tx = sxx * cx + sxy * cy + sxz * cz
    Ty = sxy * cx + syy * cy + syz * cz
    Tz = sxz * cx + syz * cy + szz * cz

    def chosen(D):
        a = (Tx * (1 - cx * cx) - Ty * cx * cy - Tz * cz * cx) * D[:, 0]
        b = (Tx * -(cx * cy) + Ty * (1 - cy * cy) - Tz * cy * cz) * D[:, 1]
        c = (Tx * -(cz * cx) - Ty * cy * cz + Tz * (1 - cz * cz)) * D[:, 2]
        return a + b + c

    return Tn, chosen(ds), chosen(ss)


def SetupTractionVector(BoundaryConditions, FaceNormalVector, n, G, lam):
    """(Tn, Tds, Tss) for Stresses, Tractions or MixedBoundaryConditions."""
    bc = BoundaryConditions
    if isinstance(bc, Stresses):
        return CalculateNormalAndShearTractions3D(*bc, FaceNormalVector)
    if isinstance(bc, Tractions):
        return _col(bc.Tn, n), _col(bc.Tds, n), _col(bc.Tss, n)
    if isinstance(bc, MixedBoundaryConditions):
        sTn, sTds, sTss = SetupTractionVector(bc.Stresses, FaceNormalVector, n, G, lam)
        Tn, Tds, Tss = SetupTractionVector(bc.Tractions, FaceNormalVector, n, G, lam)
        return Tn + sTn, Tds + sTds, Tss + sTss
    raise TypeError("unsupported boundary condition type %r" % type(bc).__name__)


def KnockOutFixedRows(FixedEls, Tn, Tds, Tss):
    fixed = np.asarray(FixedEls).reshape(-1) == 1
    if np.any(fixed):
        Tn, Tds, Tss = Tn.copy(), Tds.copy(), Tss.copy()
        Tn[fixed] = 0.0
        Tds[fixed] = 0.0
        Tss[fixed] = 0.0
    return Tn, Tds, Tss


def RemoveFixedElements3D(FixedEls, Triangles, FaceNormalVector, MidPoint, P1, P2, P3):
    """Drop the rows of fixed elements (FixedEls != 0) from the element arrays
    (src/RemoveFixedElements3D.jl); FixedEls itself is returned unchanged, as
    the reference does.  Triangles may be None."""
    keep = np.asarray(FixedEls).reshape(-1) == 0
    pick = (lambda a: None if a is None else np.asarray(a)[keep])
    return (FixedEls, pick(Triangles), pick(FaceNormalVector), pick(MidPoint), pick(P1), pick(P2), pick(P3))


def CalculateInfluenceMatrices3D(FaceNormalVector, MidPoint, P1, P2, P3, nu, G, lam, FixedEls, HSFlag, n,
                                 device=0):
    """Traction influence matrices (TractionInf of nine n x n arrays; with
    elements marked 1 in FixedEls, displacement-influence rows for them and
    only the other elements' columns, n x n_free)."""
    P1, P2, P3 = _tri(P1), _tri(P2), _tri(P3)
    N = P1.shape[0]
    nrm = _tri(FaceNormalVector)
    mid = _tri(MidPoint)
    fixed = None if FixedEls is None else np.ascontiguousarray(np.asarray(FixedEls, dtype=np.float64).reshape(-1))
    nf = N if fixed is None else int(np.sum(fixed != 1))
    out = [np.zeros((N, nf), order="F") for _ in range(9)]
    ctx = _lib.context(device)
    rc = _lib.load().cad_influence_traction(ctx, nrm.ctypes.data, mid.ctypes.data, P1.ctypes.data, P2.ctypes.data,
                                            P3.ctypes.data, N, float(nu), float(G), float(lam),
                                            fixed.ctypes.data if fixed is not None else None, int(HSFlag),
                                            _lib.ptr_array(out))
    _lib.check(rc, ctx)
    return TractionInf(*out)


def SlipCalculator3D(P1, P2, P3, nu, G, lam, MidPoint, FaceNormalVector, HSFlag, BoundaryConditions, FixedEls,
                     device=0, solver="lu64", tol=1e-10, max_iter=200, assembly="fp64", near_factor=3.0):
    """Plain (frictionless) slip solve: returns (Dn, Dss, Dds, A, b).

    solver="lu64" solves A \\ b by FP64 LU as src/SlipCalculator3D.jl:22 does;
    solver="mixed" uses the FP32/TF32 LU + FP64 GMRES path to relative residual tol.
    assembly="mixed" evaluates far-field pairs in FP32 and pairs within
    near_factor mean edge lengths in FP64 (assembly="fp64": all in FP64).

    With MixedBoundaryConditionsFriction boundary conditions this is the
    frictional solve of src/SlipCalculator3D.jl:36-87 and returns
    (Dn, Dss, Dds) only, as the reference does (see SlipCalculator3D_friction)."""
    if isinstance(BoundaryConditions, MixedBoundaryConditionsFriction):
        return SlipCalculator3D_friction(P1, P2, P3, nu, G, lam, MidPoint, FaceNormalVector, HSFlag,
                                         BoundaryConditions, FixedEls, device=device)
    P1, P2, P3 = _tri(P1), _tri(P2), _tri(P3)
    N = P1.shape[0]
    nrm = _tri(FaceNormalVector)
    mid = _tri(MidPoint)
    Tn, Tds, Tss = SetupTractionVector(BoundaryConditions, nrm, N, G, lam)
    fixed = None
    if FixedEls is not None and np.any(np.asarray(FixedEls).reshape(-1) == 1):
        fixed = np.ascontiguousarray(np.asarray(FixedEls, dtype=np.float64).reshape(-1))
        Tn, Tds, Tss = KnockOutFixedRows(FixedEls, _col(Tn, N), _col(Tds, N), _col(Tss, N))
    Tn, Tss, Tds = _col(Tn, N), _col(Tss, N), _col(Tds, N)
    if fixed is not None:
        # fixed elements: displacement rows, no columns, least squares
        nf = int(np.sum(fixed != 1))
        Dn, Dss, Dds = np.zeros(nf), np.zeros(nf), np.zeros(nf)
        A = np.zeros((3 * N, 3 * nf), order="F")
        b = np.zeros(3 * N)
        ctx = _lib.context(device)
        rc = _lib.load().cad_slip_calculator_fixed(ctx, P1.ctypes.data, P2.ctypes.data, P3.ctypes.data, N, float(nu),
                                                   float(G), float(lam), mid.ctypes.data, nrm.ctypes.data,
                                                   int(HSFlag), Tn.ctypes.data, Tss.ctypes.data, Tds.ctypes.data,
                                                   fixed.ctypes.data, Dn.ctypes.data, Dss.ctypes.data,
                                                   Dds.ctypes.data, A.ctypes.data, b.ctypes.data)
        _lib.check(rc, ctx)
        return Dn, Dss, Dds, A, b
    Dn, Dss, Dds = np.zeros(N), np.zeros(N), np.zeros(N)
    A = np.zeros((3 * N, 3 * N), order="F")
    b = np.zeros(3 * N)
    ctx = _lib.context(device)
    with _lib.solver_mode(ctx, solver, tol, max_iter), _lib.assembly_mode(ctx, assembly, near_factor):
        rc = _lib.load().cad_slip_calculator(ctx, P1.ctypes.data, P2.ctypes.data, P3.ctypes.data, N, float(nu),
                                             float(G), float(lam), mid.ctypes.data, nrm.ctypes.data, int(HSFlag),
                                             Tn.ctypes.data, Tss.ctypes.data, Tds.ctypes.data, Dn.ctypes.data,
                                             Dss.ctypes.data, Dds.ctypes.data, A.ctypes.data, b.ctypes.data)
        _lib.check(rc, ctx)
    return Dn, Dss, Dds, A, b


def SlipCalculator3D_friction(P1, P2, P3, nu, G, lam, MidPoint, FaceNormalVector, HSFlag, BoundaryConditions,
                              FixedEls, device=0, tol=1e-10, max_iter=100):
    """Slip with frictional contact (src/SlipCalculator3D.jl:36-238): returns
    (Dn, Dss, Dds).  BoundaryConditions: MixedBoundaryConditionsFriction (the
    remote stress and tractions of its MixedBoundaryConditions, mu and Sf of
    its FrictionParameters, scalars broadcast to every element).  The
    influence matrix is inverted after scaling by Scl = mean half-perimeter / G
    and the 5N-variable complementarity problem is solved by a
    Fischer-Burmeister Newton method on the GPU to max|Phi| <= tol max|q|.
    Prints "Cant overcome frictional strength" and returns zero slip when no
    element can slip, as the reference does.  The reference inverts the square
    influence matrix, so fixed elements are not supported (Julia's inv raises
    on the tall matrix they produce)."""
    if FixedEls is not None and np.any(np.asarray(FixedEls).reshape(-1) == 1):
        raise ValueError("DimensionMismatch: matrix is not square: the frictional solve takes no fixed elements")
    P1, P2, P3 = _tri(P1), _tri(P2), _tri(P3)
    N = P1.shape[0]
    nrm = _tri(FaceNormalVector)
    mid = _tri(MidPoint)
    fp = BoundaryConditions.FrictionParameters
    Tn, Tds, Tss = SetupTractionVector(BoundaryConditions.MixedBoundaryConditions, nrm, N, G, lam)
    Tn, Tss, Tds = _col(Tn, N), _col(Tss, N), _col(Tds, N)
    mu, Sf = _col(fp.mu, N), _col(fp.Sf, N)
    if np.all(-np.abs(Tss) > Tn * mu) and np.all(-np.abs(Tds) > Tn * mu):
        print("Cant overcome frictional strength")
        return np.zeros(N), np.zeros(N), np.zeros(N)
    Dn, Dss, Dds = np.zeros(N), np.zeros(N), np.zeros(N)
    ctx = _lib.context(device)
    rc = _lib.load().cad_slip_calculator_friction(ctx, P1.ctypes.data, P2.ctypes.data, P3.ctypes.data, N, float(nu),
                                                  float(G), float(lam), mid.ctypes.data, nrm.ctypes.data,
                                                  int(HSFlag), Tn.ctypes.data, Tss.ctypes.data, Tds.ctypes.data,
                                                  mu.ctypes.data, Sf.ctypes.data, float(tol), int(max_iter),
                                                  Dn.ctypes.data, Dss.ctypes.data, Dds.ctypes.data)
    _lib.check(rc, ctx)
    return Dn, Dss, Dds


class FrictionSolver:
    """Frictional slip for many loads on one geometry: the set-up of
    src/SlipCalculator3D.jl:56-61 and :90-175 (A assembled, C = inv(A Scl)
    kept on the GPU) once, then `solve` per load (:177-238).  One prepared
    system per device context: preparing another, calling
    SlipCalculator3D_friction or fischer_newton on the same device replaces
    it (solve then raises)."""

    def __init__(self, P1, P2, P3, nu, G, lam, MidPoint, FaceNormalVector, HSFlag, device=0):
        P1, P2, P3 = _tri(P1), _tri(P2), _tri(P3)
        self.N = P1.shape[0]
        self.nrm = _tri(FaceNormalVector)
        self.G, self.lam = float(G), float(lam)
        mid = _tri(MidPoint)
        self.ctx = _lib.context(device)
        rc = _lib.load().cad_friction_prepare(self.ctx, P1.ctypes.data, P2.ctypes.data, P3.ctypes.data, self.N,
                                              float(nu), float(G), float(lam), mid.ctypes.data,
                                              self.nrm.ctypes.data, int(HSFlag))
        _lib.check(rc, self.ctx)

    def solve(self, BoundaryConditions, tol=1e-10, max_iter=100):
        """(Dn, Dss, Dds) for MixedBoundaryConditionsFriction boundary
        conditions (no early exit here: the reference's prepared solve has
        none)."""
        N = self.N
        fp = BoundaryConditions.FrictionParameters
        Tn, Tds, Tss = SetupTractionVector(BoundaryConditions.MixedBoundaryConditions, self.nrm, N, self.G, self.lam)
        Tn, Tss, Tds = _col(Tn, N), _col(Tss, N), _col(Tds, N)
        mu, Sf = _col(fp.mu, N), _col(fp.Sf, N)
        Dn, Dss, Dds = np.zeros(N), np.zeros(N), np.zeros(N)
        rc = _lib.load().cad_friction_solve(self.ctx, N, Tn.ctypes.data, Tss.ctypes.data, Tds.ctypes.data,
                                            mu.ctypes.data, Sf.ctypes.data, float(tol), int(max_iter),
                                            Dn.ctypes.data, Dss.ctypes.data, Dds.ctypes.data)
        _lib.check(rc, self.ctx)
        return Dn, Dss, Dds


def fischer_newton(A, b, device=0, tol=1e-10, max_iter=100):
    """x solving the linear complementarity problem x >= 0, A x + b >= 0,
    x'(A x + b) = 0 -- the FischerNewton.fischer_newton(A, b) call of
    src/SlipCalculator3D.jl:196 -- by the GPU Fischer-Burmeister Newton method
    from x = 0, to max|Phi| <= tol max|b|."""
    A = np.asfortranarray(A, dtype=np.float64)
    b = np.ascontiguousarray(np.asarray(b, dtype=np.float64).reshape(-1))
    n = b.shape[0]
    if A.shape != (n, n):
        raise ValueError("DimensionMismatch: A must be %d x %d" % (n, n))
    x = np.zeros(n)
    ctx = _lib.context(device)
    rc = _lib.load().cad_fischer_newton(ctx, n, A.ctypes.data, b.ctypes.data, float(tol), int(max_iter),
                                        x.ctypes.data)
    _lib.check(rc, ctx)
    return x


def solve(A, B, device=0, solver="lu64", tol=1e-10, max_iter=200):
    """Dense A \\ B on the GPU: FP64 LU with partial pivoting ("lu64"), or the
    FP32/TF32 LU + FP64 GMRES path ("mixed", relative residual tol)."""
    A = np.asfortranarray(A, dtype=np.float64)
    B = np.asarray(B, dtype=np.float64)
    vec = B.ndim == 1
    Bf = np.asfortranarray(B.reshape(B.shape[0], -1))
    n, nrhs = A.shape[0], Bf.shape[1]
    X = np.zeros((n, nrhs), order="F")
    ctx = _lib.context(device)
    with _lib.solver_mode(ctx, solver, tol, max_iter):
        rc = _lib.load().cad_solve(ctx, n, A.ctypes.data, Bf.ctypes.data, nrhs, X.ctypes.data)
        _lib.check(rc, ctx)
    return X[:, 0] if vec else X


BATCH_MODES = {"grouped": 0, "lanes": 1, "lanes_chain": 2}


def SlipCalculator3D_batched(cracks, nu, G, lam, HSFlag, BoundaryConditions, device=0, tol=1e-10,
                             assembly="mixed", near_factor=3.0, mode="grouped"):
    """SlipCalculator3D (src/SlipCalculator3D.jl:1-33) over many independent
    cracks in one batched GPU call.  cracks: list of (P1, P2, P3); one
    boundary condition per crack (or one for all).  Each crack is assembled
    (assembly="mixed": FP32 far field, FP64 near field; "fp64": all FP64) and
    solved by FP32 LU with FP64 refinement to relative residual tol (mode:
    "grouped" -- every crack in each launch; "lanes" / "lanes_chain" -- every
    crack on its own stream lane).  Returns a list of (Dn, Dss, Dds) and the
    final relative residuals."""
    from .geometry import CreateFaceNormalAndMidPoint
    bcs = BoundaryConditions if isinstance(BoundaryConditions, (list, tuple)) else [BoundaryConditions] * len(cracks)
    if len(bcs) != len(cracks):
        raise ValueError("one boundary condition per crack")
    offs = [0]
    blocks = {k: [] for k in ("P1", "P2", "P3", "nrm", "mid", "T")}
    for (P1, P2, P3), bc in zip(cracks, bcs):
        P1, P2, P3 = _tri(P1), _tri(P2), _tri(P3)
        N = P1.shape[0]
        nrm, mid = CreateFaceNormalAndMidPoint(P1, P2, P3)
        Tn, Tds, Tss = SetupTractionVector(bc, nrm, N, G, lam)
        for k, a in (("P1", P1), ("P2", P2), ("P3", P3), ("nrm", _tri(nrm)), ("mid", _tri(mid))):
            blocks[k].append(a.ravel(order="F"))
        blocks["T"].append(np.concatenate([_col(Tn, N), _col(Tss, N), _col(Tds, N)]))
        offs.append(offs[-1] + N)
    cat = {k: np.ascontiguousarray(np.concatenate(v)) if v else np.zeros(0) for k, v in blocks.items()}
    offsets = np.asarray(offs, dtype=np.int64)
    D = np.zeros(3 * offs[-1])
    rel = np.zeros(len(cracks))
    ctx = _lib.context(device)
    L = _lib.load()
    _lib.check(L.cad_set_batch_solve(ctx, BATCH_MODES[mode]), ctx)
    with _lib.solver_mode(ctx, "mixed", tol, 400), _lib.assembly_mode(ctx, assembly, near_factor):
        rc = L.cad_slip_calculator_batched(ctx, len(cracks), offsets.ctypes.data, cat["P1"].ctypes.data,
                                                     cat["P2"].ctypes.data, cat["P3"].ctypes.data,
                                                     cat["nrm"].ctypes.data, cat["mid"].ctypes.data, float(nu),
                                                     float(G), float(lam), int(HSFlag), cat["T"].ctypes.data,
                                                     D.ctypes.data, rel.ctypes.data)
    L.cad_set_batch_solve(ctx, 0)
    _lib.check(rc, ctx)
    out = []
    for c in range(len(cracks)):
        o, N = offs[c], offs[c + 1] - offs[c]
        d = D[3 * o:3 * o + 3 * N]
        out.append((d[:N], d[N:2 * N], d[2 * N:]))
    return out, rel
