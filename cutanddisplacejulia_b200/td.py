"""Host mirror of the reference's TD and TD_sum (src/TD.jl:77-410,
src/TD_sum.jl:1-41): same names, argument order and meaning, same error
messages.  All arithmetic runs in libcad_td.so on the GPU.

Dispatch follows the Julia methods:
    TD(X,Y,Z,P1,P2,P3,Dss,Dds,Dn,nu,G,DispFlag,StrainFlag,HSflag)
        -> (StrainInf, DispInf)   allocates M x N influence matrices
    TD(..., StrainInf, DispInf)   fills the given matrices in place
    TD(..., Strains, Disps)       sums over triangles -> (Strains, Disps)
"""
from __future__ import annotations

import numpy as np

from . import _lib
from .structs import DispInf, Disps, StrainInf, Strains

DIMS_MSG = "Element size inputs must be the same dimensions"


def _vec(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float64).reshape(-1))


def _tri(P):
    P = np.asarray(P, dtype=np.float64)
    if P.size == 3:
        P = P.reshape(1, 3)
    return np.asfortranarray(P)


def _scalar(v):
    """Accept PoissonsRatio / ShearModulus-like records or plain numbers."""
    for attr in ("nu", "G", "value"):
        if hasattr(v, attr):
            return float(getattr(v, attr))
    return float(v)


def _prepare(X, Y, Z, P1, P2, P3, Dss, Dds, Dn):
    X, Y, Z = _vec(X), _vec(Y), _vec(Z)
    P1, P2, P3 = _tri(P1), _tri(P2), _tri(P3)
    N = P1.shape[0]
    ok = P2.shape[0] == N and P3.shape[0] == N and np.size(Dds) == N and np.size(Dss) == N and np.size(Dn) == N
    if not ok:
        raise _lib.CadError(_lib.CAD_ERR_DIMS, DIMS_MSG)
    if not (X.size == Y.size == Z.size):
        raise _lib.CadError(_lib.CAD_ERR_DIMS, DIMS_MSG)
    return X, Y, Z, P1, P2, P3, _vec(Dss), _vec(Dds), _vec(Dn)


def _fortran_out(a, M, N):
    a = np.asarray(a)
    if a.dtype != np.float64 or a.shape != (M, N) or not a.flags.f_contiguous:
        raise _lib.CadError(_lib.CAD_ERR_ARG, "influence matrices must be float64, M x N, column-major")
    return a


def TD(X, Y, Z, P1List, P2List, P3List, Dss, Dds, Dn, nu, G, DispFlag, StrainFlag, HSflag, *out, device=0):
    nu, G = _scalar(nu), _scalar(G)
    shape = np.shape(X)
    X, Y, Z, P1, P2, P3, Dss, Dds, Dn = _prepare(X, Y, Z, P1List, P2List, P3List, Dss, Dds, Dn)
    M, N = X.size, P1.shape[0]
    ctx = _lib.context(device)
    L = _lib.load()
    if len(out) == 2 and isinstance(out[0], Strains) and isinstance(out[1], Disps):
        return _td_sum_eval(L, ctx, X, Y, Z, M, P1, P2, P3, N, Dss, Dds, Dn, nu, G, DispFlag, StrainFlag, HSflag, shape)
    if len(out) == 2 and isinstance(out[0], StrainInf) and isinstance(out[1], DispInf):
        S, U = out
    elif len(out) == 0:
        S = StrainInf(*[np.zeros((M, N), order="F") for _ in range(18)]) if StrainFlag == 1 else StrainInf(
            *[np.empty(0)] * 18)
        U = DispInf(*[np.zeros((M, N), order="F") for _ in range(9)]) if DispFlag == 1 else DispInf(
            *[np.empty(0)] * 9)
    else:
        raise TypeError("TD: trailing arguments must be (StrainInf, DispInf) or (Strains, Disps)")
    s_arr = [_fortran_out(a, M, N) for a in S] if StrainFlag == 1 else None
    u_arr = [_fortran_out(a, M, N) for a in U] if DispFlag == 1 else None
    rc = L.cad_td_inf(ctx, X.ctypes.data, Y.ctypes.data, Z.ctypes.data, M, P1.ctypes.data, P2.ctypes.data,
                      P3.ctypes.data, N, Dss.ctypes.data, Dds.ctypes.data, Dn.ctypes.data, nu, G, int(DispFlag),
                      int(StrainFlag), int(HSflag), _lib.ptr_array(s_arr) if s_arr else None,
                      _lib.ptr_array(u_arr) if u_arr else None)
    _lib.check(rc, ctx)
    return S, U


def _td_sum_eval(L, ctx, X, Y, Z, M, P1, P2, P3, N, Dss, Dds, Dn, nu, G, DispFlag, StrainFlag, HSflag, shape):
    s_arr = [np.zeros(M) for _ in range(6)] if StrainFlag == 1 else None
    u_arr = [np.zeros(M) for _ in range(3)] if DispFlag == 1 else None
    rc = L.cad_td_sum_eval(ctx, X.ctypes.data, Y.ctypes.data, Z.ctypes.data, M, P1.ctypes.data, P2.ctypes.data,
                           P3.ctypes.data, N, Dss.ctypes.data, Dds.ctypes.data, Dn.ctypes.data, nu, G,
                           int(DispFlag), int(StrainFlag), int(HSflag),
                           _lib.ptr_array(s_arr) if s_arr else None, _lib.ptr_array(u_arr) if u_arr else None)
    _lib.check(rc, ctx)
    reshape = (lambda a: a.reshape(shape, order="F")) if len(shape) == 2 and shape[1] != 1 else (lambda a: a)
    S = Strains(*[reshape(a) for a in s_arr]) if s_arr else Strains(*[np.empty(0)] * 6)
    U = Disps(*[reshape(a) for a in u_arr]) if u_arr else Disps(*[np.empty(0)] * 3)
    return S, U


def TD_sum(ExxDn, EyyDn, EzzDn, ExyDn, ExzDn, EyzDn, ExxDss, EyyDss, EzzDss, ExyDss, ExzDss, EyzDss,
           ExxDds, EyyDds, EzzDds, ExyDds, ExzDds, EyzDds, UxDn, UyDn, UzDn, UxDss, UyDss, UzDss, UxDds, UyDds,
           UzDds, device=0):
    """Sum influence matrices over modes and triangles -> (Exx, Eyy, Ezz, Exy, Exz, Eyz, Ux, Uy, Uz),
    each an M x 1 column (empty inputs give empty outputs, as in the reference)."""
    strain = [ExxDn, EyyDn, EzzDn, ExyDn, ExzDn, EyzDn, ExxDss, EyyDss, EzzDss, ExyDss, ExzDss, EyzDss,
              ExxDds, EyyDds, EzzDds, ExyDds, ExzDds, EyzDds]
    disp = [UxDn, UyDn, UzDn, UxDss, UyDss, UzDss, UxDds, UyDds, UzDds]
    has_s = np.size(ExxDn) > 0
    has_u = np.size(UxDn) > 0
    ref = ExxDn if has_s else UxDn
    if not (has_s or has_u):
        return tuple(strain[:6]) + (UxDn, UyDn, UzDn)
    M, N = np.shape(ref)
    s_in = [np.asfortranarray(a, dtype=np.float64) for a in strain] if has_s else None
    u_in = [np.asfortranarray(a, dtype=np.float64) for a in disp] if has_u else None
    s_out = [np.zeros((M, 1)) for _ in range(6)] if has_s else None
    u_out = [np.zeros((M, 1)) for _ in range(3)] if has_u else None
    ctx = _lib.context(device)
    rc = _lib.load().cad_td_sum(ctx, M, N, _lib.ptr_array(s_in) if has_s else None,
                                _lib.ptr_array(u_in) if has_u else None,
                                _lib.ptr_array(s_out) if has_s else None, _lib.ptr_array(u_out) if has_u else None)
    _lib.check(rc, ctx)
    so = s_out if has_s else strain[:6]
    uo = u_out if has_u else disp[:3]
    return tuple(so) + tuple(uo)
