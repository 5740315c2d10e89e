"""CPU oracle for the TD hot path (ctypes front end of oracle/libcad_oracle.so).

TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU
baseline use this module as the checker.  The product (the CUDA library and
the `cutanddisplacejulia_b200` package) never imports it.

Every array follows the reference's Julia layout: vertex lists are N x 3,
influence matrices M x N (observation = row, triangle = column), returned
here as numpy views with that shape.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcad_oracle.so")

ERR_HS_ABOVE = 2

_lib = None


def build() -> str:
    """Compile the oracle library (g++, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        d = ctypes.POINTER(ctypes.c_double)
        i64, c_int, dbl = ctypes.c_int64, ctypes.c_int, ctypes.c_double
        L.cado_td_inf.argtypes = [d, d, d, i64, d, d, d, i64, d, d, d, dbl, dbl, c_int, c_int, c_int, c_int, d, d]
        L.cado_td_sum_eval.argtypes = L.cado_td_inf.argtypes
        L.cado_td_inf_ld.argtypes = [d, d, d, i64, d, d, d, i64, d, d, d, dbl, c_int, c_int, c_int, c_int, d, d]
        L.cado_strain_to_traction.argtypes = [d, i64, i64, d, dbl, dbl, c_int, d]
        L.cado_influence_traction.argtypes = [d, d, d, d, d, i64, dbl, dbl, dbl, c_int, c_int, d, d]
        L.cado_normal_shear_tractions.argtypes = [d, d, d, d, d, d, d, i64, d, d, d]
        L.cado_normal_shear_tractions.restype = None
        L.cado_opcount.argtypes = [d, d, d, i64, d, d, d, i64, d, d, d, dbl, c_int, c_int, d]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)) if a is not None else None


def _vec(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))


def _tri(P):
    """N x 3 vertex list -> Fortran-ordered float64 (Julia's N x 3 layout)."""
    P = np.asarray(P, dtype=np.float64)
    if P.ndim == 1:
        P = P.reshape(1, 3)
    return np.asfortranarray(P)


class OracleError(RuntimeError):
    pass


def _check(rc):
    if rc == ERR_HS_ABOVE:
        raise OracleError("Half-space solution: Z coordinates must be negative!")
    if rc != 0:
        raise OracleError(f"oracle error {rc}")


def nthreads_default():
    return os.cpu_count() or 1


def td_inf(X, Y, Z, P1, P2, P3, Dss, Dds, Dn, nu, G, disp, strain, hs, nthreads=None):
    """TD influence-matrix overload (src/TD.jl:77-216).

    Returns (strain, disp): arrays of shape (18, M, N) / (9, M, N) in
    StrainInf / DispInf field order, or None for a disabled flag.
    """
    X, Y, Z = _vec(X), _vec(Y), _vec(Z)
    P1, P2, P3 = _tri(P1), _tri(P2), _tri(P3)
    M, N = X.size, P1.shape[0]
    if not (P2.shape[0] == N and P3.shape[0] == N and np.size(Dss) == N and np.size(Dds) == N and np.size(Dn) == N):
        raise OracleError("Element size inputs must be the same dimensions")
    S = np.empty((18, N, M)) if strain == 1 else None
    D = np.empty((9, N, M)) if disp == 1 else None
    rc = lib().cado_td_inf(_p(X), _p(Y), _p(Z), M, _p(P1), _p(P2), _p(P3), N, _p(_vec(Dss)), _p(_vec(Dds)),
                           _p(_vec(Dn)), float(nu), float(G), int(disp), int(strain), int(hs),
                           nthreads or nthreads_default(), _p(S), _p(D))
    _check(rc)
    return (S.transpose(0, 2, 1) if S is not None else None, D.transpose(0, 2, 1) if D is not None else None)


def td_inf_ld(X, Y, Z, P1, P2, P3, Dss, Dds, Dn, nu, disp, strain, hs, nthreads=None):
    """td_inf evaluated in long double (accuracy referee), rounded to double."""
    X, Y, Z = _vec(X), _vec(Y), _vec(Z)
    P1, P2, P3 = _tri(P1), _tri(P2), _tri(P3)
    M, N = X.size, P1.shape[0]
    S = np.empty((18, N, M)) if strain == 1 else None
    D = np.empty((9, N, M)) if disp == 1 else None
    rc = lib().cado_td_inf_ld(_p(X), _p(Y), _p(Z), M, _p(P1), _p(P2), _p(P3), N, _p(_vec(Dss)), _p(_vec(Dds)),
                              _p(_vec(Dn)), float(nu), int(disp), int(strain), int(hs),
                              nthreads or nthreads_default(), _p(S), _p(D))
    _check(rc)
    return (S.transpose(0, 2, 1) if S is not None else None, D.transpose(0, 2, 1) if D is not None else None)


def td_sum_eval(X, Y, Z, P1, P2, P3, Dss, Dds, Dn, nu, G, disp, strain, hs, nthreads=None):
    """TD summing overload (src/TD.jl:219-410): strain (6, M), disp (3, M)."""
    X, Y, Z = _vec(X), _vec(Y), _vec(Z)
    P1, P2, P3 = _tri(P1), _tri(P2), _tri(P3)
    M, N = X.size, P1.shape[0]
    if not (P2.shape[0] == N and P3.shape[0] == N and np.size(Dss) == N and np.size(Dds) == N and np.size(Dn) == N):
        raise OracleError("Element size inputs must be the same dimensions")
    S = np.empty((6, M)) if strain == 1 else None
    D = np.empty((3, M)) if disp == 1 else None
    rc = lib().cado_td_sum_eval(_p(X), _p(Y), _p(Z), M, _p(P1), _p(P2), _p(P3), N, _p(_vec(Dss)), _p(_vec(Dds)),
                                _p(_vec(Dn)), float(nu), float(G), int(disp), int(strain), int(hs),
                                nthreads or nthreads_default(), _p(S), _p(D))
    _check(rc)
    return S, D


def td_sum(strain_inf, disp_inf):
    """TD_sum (src/TD_sum.jl:1-41): sum the three modes, then over triangles."""
    S = None if strain_inf is None else np.stack(
        [(strain_inf[k] + strain_inf[6 + k] + strain_inf[12 + k]).sum(axis=1) for k in range(6)])
    D = None if disp_inf is None else np.stack(
        [(disp_inf[c] + disp_inf[3 + c] + disp_inf[6 + c]).sum(axis=1) for c in range(3)])
    return S, D


def strain_to_traction(strain_inf, normals, lam, G, nthreads=None):
    """ConvertStrainInfMatsToTraction (src/CalculateInfluenceMatrices3D.jl:73-114): (9, M, N)."""
    _, M, N = strain_inf.shape
    S = np.ascontiguousarray(strain_inf.transpose(0, 2, 1))
    nrm = np.asfortranarray(np.asarray(normals, dtype=np.float64))
    T = np.empty((9, N, M))
    _check(lib().cado_strain_to_traction(_p(S), M, N, _p(nrm), float(lam), float(G), nthreads or nthreads_default(),
                                         _p(T)))
    return T.transpose(0, 2, 1)


def influence_traction(normals, midpoints, P1, P2, P3, nu, G, lam, hs, nthreads=None, want_A=False):
    """CalculateInfluenceMatrices3D without fixed elements, fused per pair.

    Returns the (9, N, N) TractionInf stack, or the 3N x 3N matrix
    A = -[Atn; Atss; Atds] (src/SlipCalculator3D.jl:13-16) when want_A.
    """
    P1, P2, P3 = _tri(P1), _tri(P2), _tri(P3)
    N = P1.shape[0]
    nrm = np.asfortranarray(np.asarray(normals, dtype=np.float64))
    mid = np.asfortranarray(np.asarray(midpoints, dtype=np.float64))
    if want_A:
        A = np.empty((3 * N, 3 * N), order="F")
        rc = lib().cado_influence_traction(_p(nrm), _p(mid), _p(P1), _p(P2), _p(P3), N, float(nu), float(G),
                                           float(lam), int(hs), nthreads or nthreads_default(), None,
                                           A.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
        _check(rc)
        return A
    T = np.empty((9, N, N))
    rc = lib().cado_influence_traction(_p(nrm), _p(mid), _p(P1), _p(P2), _p(P3), N, float(nu), float(G), float(lam),
                                       int(hs), nthreads or nthreads_default(), _p(T), None)
    _check(rc)
    return T.transpose(0, 2, 1)


def assemble_A(trac):
    """A = -[[DnTn DssTn DdsTn]; [DnTss DssTss DdsTss]; [DnTds DssTds DdsTds]]."""
    N = trac.shape[1]
    A = np.empty((3 * N, 3 * N), order="F")
    for r in range(3):        # Tn, Tss, Tds row blocks
        for m in range(3):    # Dn, Dss, Dds column blocks
            A[r * N:(r + 1) * N, m * N:(m + 1) * N] = -trac[3 * m + r]
    return A


def normal_and_shear_tractions(sxx, syy, szz, sxy, sxz, syz, normals):
    """CalculateNormalAndShearTractions3D: returns (Tn, Tds, Tss)."""
    nrm = np.asfortranarray(np.asarray(normals, dtype=np.float64))
    N = nrm.shape[0]
    args = [_vec(np.broadcast_to(np.asarray(s, dtype=np.float64).reshape(-1), (N,)) if np.size(s) in (1, N) else s)
            for s in (sxx, syy, szz, sxy, sxz, syz)]
    Tn, Tds, Tss = np.empty(N), np.empty(N), np.empty(N)
    lib().cado_normal_shear_tractions(*[_p(a) for a in args], _p(nrm), N, _p(Tn), _p(Tds), _p(Tss))
    return Tn, Tds, Tss


def hookes_law(strain6, lam, G):
    """HookesLaw3DStrain2Stress on (6, ...) strains (xx,yy,zz,xy,xz,yz)."""
    exx, eyy, ezz, exy, exz, eyz = strain6
    cons = lam * (exx + eyy + ezz)
    return np.stack([2 * G * exx + cons, 2 * G * eyy + cons, 2 * G * ezz + cons, 2 * G * exy, 2 * G * exz, 2 * G * eyz])


def slip_calculator(P1, P2, P3, nu, G, lam, midpoints, normals, hs, Tn, Tss, Tds, nthreads=None):
    """Plain SlipCalculator3D (src/SlipCalculator3D.jl:1-33), no fixed elements:
    A\\b by LAPACK gesv (numpy).  Returns Dn, Dss, Dds, A, b."""
    A = influence_traction(normals, midpoints, P1, P2, P3, nu, G, lam, hs, nthreads=nthreads, want_A=True)
    b = np.concatenate([_vec(Tn), _vec(Tss), _vec(Tds)])
    D = np.linalg.solve(A, b)
    n = len(b) // 3
    return D[:n], D[n:2 * n], D[2 * n:], A, b


def influence_traction_fixed(normals, midpoints, P1, P2, P3, nu, G, lam, fixed, hs, nthreads=None):
    """CalculateInfluenceMatrices3D with fixed elements
    (src/CalculateInfluenceMatrices3D.jl:10-33, ConcatInfMats and
    PutDispInfsIntoInfMat :145-199): rows of fixed elements hold the
    displacement influence at their collocation points (field f of DispInf in
    place of field f of TractionInf: DnUx for DnTn, DnUy for DnTss, ...), rows
    of the others the traction influence; only the columns of the elements
    that are not fixed are kept.  Returns the (9, N, n_free) stack."""
    fixed = np.asarray(fixed).reshape(-1) == 1
    free = ~fixed
    T = influence_traction(normals, midpoints, P1, P2, P3, nu, G, lam, hs, nthreads=nthreads)
    out = T.copy()
    if fixed.any():
        obs = np.asarray(midpoints, dtype=np.float64) - 1e-12 * np.asarray(normals, dtype=np.float64)
        N = obs.shape[0]
        ones = np.ones(N)
        _, U = td_inf(obs[fixed, 0], obs[fixed, 1], obs[fixed, 2], P1, P2, P3, ones, ones, ones, nu, G, 1, 0, hs,
                      nthreads=nthreads)
        out[:, fixed, :] = U
    return out[:, :, free]


def assemble_A_rect(trac):
    """A = -[[DnTn DssTn DdsTn]; [DnTss DssTss DdsTss]; [DnTds DssTds DdsTds]]
    from (9, N, n_free) fields: 3N x 3 n_free (src/SlipCalculator3D.jl:13-16)."""
    N, nf = trac.shape[1], trac.shape[2]
    A = np.empty((3 * N, 3 * nf), order="F")
    for r in range(3):
        for m in range(3):
            A[r * N:(r + 1) * N, m * nf:(m + 1) * nf] = -trac[3 * m + r]
    return A


def slip_calculator_fixed(P1, P2, P3, nu, G, lam, midpoints, normals, hs, Tn, Tss, Tds, fixed, nthreads=None):
    """SlipCalculator3D with fixed elements (src/SlipCalculator3D.jl:1-33):
    tractions of fixed elements knocked out (src/KnockOutFixedRows.jl), the
    3N x 3 n_free system solved in the least-squares sense as Julia's backslash does
    for a tall matrix (numpy lstsq).  Returns Dn, Dss, Dds (n_free each), A, b."""
    fixed = np.asarray(fixed).reshape(-1) == 1
    Tn, Tss, Tds = (np.where(fixed, 0.0, _vec(t)) for t in (Tn, Tss, Tds))
    A = assemble_A_rect(influence_traction_fixed(normals, midpoints, P1, P2, P3, nu, G, lam, fixed, hs,
                                                 nthreads=nthreads))
    b = np.concatenate([Tn, Tss, Tds])
    D = np.linalg.lstsq(A, b, rcond=None)[0]
    nf = int((~fixed).sum())
    return D[:nf], D[nf:2 * nf], D[2 * nf:], A, b


def mogi_spherical_cavity(D, X, Y, radius, P, nu, G):
    """Surface displacement above a pressurised spherical cavity, Mogi (1958),
    as src/Mogi1958_SphericalCavity.jl states it: returns (Ux, Uy, Uz)."""
    X, Y = np.asarray(X, dtype=np.float64), np.asarray(Y, dtype=np.float64)
    R = np.sqrt(D * D + X * X + Y * Y)
    lsi = radius ** 3 * P * ((1 - nu) / G)
    return X / R ** 3 * lsi, Y / R ** 3 * lsi, D / R ** 3 * lsi


def opcount(X, Y, Z, P1, P2, P3, Dss, Dds, Dn, nu, kind, hs):
    """Literal operation counts per pair (kind 0 strain, 1 displacement)."""
    X, Y, Z = _vec(X), _vec(Y), _vec(Z)
    P1, P2, P3 = _tri(P1), _tri(P2), _tri(P3)
    out = np.zeros(10)
    lib().cado_opcount(_p(X), _p(Y), _p(Z), X.size, _p(P1), _p(P2), _p(P3), P1.shape[0], _p(_vec(Dss)),
                       _p(_vec(Dds)), _p(_vec(Dn)), float(nu), int(kind), int(hs), _p(out))
    keys = ["add", "mul", "div", "sqrt", "transcendental"]
    return dict(zip(keys, out[:5])), dict(zip(keys, out[5:]))
