"""Oracle-side geometry restatements used to build test inputs.

TEST INFRASTRUCTURE ONLY (tests/, smoke, bench CPU baseline).

  face_normal_and_midpoint   CreateTriangleNormal! (src/CreateTriangleNormal!.jl:51-69) and
                             CreateMidPoint! (src/CreateMidPoint!.jl:23-36): unit normal of
                             (P2-P1) x (P3-P1) and the incentre
  ss_ds_dirs                 CalculateSSandDSDirs (src/CalculateSSandDSDirs.jl:417-481)
  direction_cosines_from_strike_and_dip
                             CreateDirectionCosinesFromStrikeAndDip
                             (src/CreateDirectionCosinesFromStrikeAndDip.jl:1-14) with
                             RotateCosine3D about z (src/RotateCosine3D.jl:82-95)
  rotate_object_3d           RotateObject3DNewCoords (src/RotateObject3DNewCoords.jl:118-129)
  area_half_perimeter        AreaOfTriangle3D (Heron)
  elastic_constants          ElasticConstantsCheck(G, nu) (src/ElasticConstantsCheck.jl:83-95)
"""
from __future__ import annotations

import numpy as np


def face_normal_and_midpoint(P1, P2, P3):
    P1, P2, P3 = (np.asarray(p, dtype=np.float64).reshape(-1, 3) for p in (P1, P2, P3))
    U = P2 - P1
    V = P3 - P1
    Nx = U[:, 1] * V[:, 2] - U[:, 2] * V[:, 1]
    Ny = U[:, 2] * V[:, 0] - U[:, 0] * V[:, 2]
    Nz = U[:, 0] * V[:, 1] - U[:, 1] * V[:, 0]
    mag = np.sqrt(Nx * Nx + Ny * Ny + Nz * Nz)
    normal = np.stack([Nx / mag, Ny / mag, Nz / mag], axis=1)
    c = np.sqrt(((P1 - P2) ** 2).sum(1))
    a = np.sqrt(((P2 - P3) ** 2).sum(1))
    b = np.sqrt(((P1 - P3) ** 2).sum(1))
    if np.any((a == 0) | (b == 0) | (c == 0)):
        raise ValueError("Slither triangles or triangles with no area exist on your surface")
    s = a + b + c
    mid = (P1 * a[:, None] + P2 * b[:, None] + P3 * c[:, None]) / s[:, None]
    return normal, mid


def ss_ds_dirs(cx, cy, cz):
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
    for i in np.nonzero(vert)[0]:
        ds[i] = [-1.0, 0.0, 0.0]
        ss[i] = [0.0, -1.0, 0.0] if cz[i] < 1.0 else [0.0, 1.0, 0.0]
    return ss, ds


def _rot_z(v, ang):
    c, s = np.cos(ang), np.sin(ang)
    R = np.array([[c, -s, 0.0], [s, c, 0.0], [0.0, 0.0, 1.0]])
    return R @ v


def direction_cosines_from_strike_and_dip(strike, dip):
    """Unit (strike-slip, dip-slip, normal) cosines of a plane of given strike and dip (degrees)."""
    c = np.cos(np.deg2rad(dip))
    ss, ds = ss_ds_dirs(c, 0.0, c)
    ang = np.deg2rad(-strike)
    ss = _rot_z(ss[0], ang)
    ds = _rot_z(ds[0], ang)
    fn = np.cross(ss, ds)
    return ss, ds, fn


def rotate_object_3d(X, Y, Z, ax1, ax2, ax3):
    X, Y, Z = (np.asarray(v, dtype=np.float64) for v in (X, Y, Z))
    x = ax1[0] * X + ax2[0] * Y + ax3[0] * Z
    y = ax1[1] * X + ax2[1] * Y + ax3[1] * Z
    z = ax1[2] * X + ax2[2] * Y + ax3[2] * Z
    return x, y, z


def area_half_perimeter(P1, P2, P3):
    a = np.sqrt(((P2 - P3) ** 2).sum(1))
    b = np.sqrt(((P1 - P3) ** 2).sum(1))
    c = np.sqrt(((P1 - P2) ** 2).sum(1))
    s = (a + b + c) / 2
    return np.sqrt(s * (s - a) * (s - b) * (s - c)), s


def elastic_constants(G, nu):
    """(K, E, lambda, nu, G) from shear modulus and Poisson's ratio."""
    K = (2 * G * (1 + nu)) / (3 * (1 - 2 * nu))
    E = 2 * G * (1 + nu)
    lam = (2 * G * nu) / (1 - 2 * nu)
    return K, E, lam, nu, G
