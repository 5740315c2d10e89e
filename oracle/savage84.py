"""Gravitational stresses beneath a long symmetric valley (Savage, Swolfs and
Powers 1985; the plane-strain solution the reference evaluates in
src/Savage1984_GravityValleyStress.jl), for the reference's KAT
test/test_TDvsSavageGravityValley.jl.

TEST INFRASTRUCTURE ONLY: the tests use it as the checker.

The valley is the image of the half plane Im(w) <= 0 under the conformal map
z = w + a b / (w - i a) (b < 0: a valley of depth set by a and b).  The
stress follows from two complex potentials, one for gravity (density x g =
rg, through so = rg b) and one for a horizontal tectonic stress tectxx, plus
the lithostatic terms rg Y / (1 - nu) and rg Y (1 - 2 nu) / (1 - nu).
Returns (Sxx, Syy, Sxy, X, Y) at the mapped points z = X + i Y of the grid
w = u + i v, as the reference does (Syy is the vertical stress).
"""
from __future__ import annotations

import numpy as np


def savage1984_gravity_valley_stress(tectxx, rg, nu, a, b, u, v):
    u = np.asarray(u, dtype=np.float64)
    v = np.asarray(v, dtype=np.float64)
    w = u + 1j * v
    ia = 1j * a
    wm = w - ia                      # w - i a
    wp = w + ia                      # w + i a
    ab = a * b
    so = rg * b
    k1 = 1.0 - nu
    # the map and its derivative
    z = w + ab / wm
    dz = (wm ** 2 - ab) / wm ** 2
    X, Y = z.real, z.imag
    # constants of the potentials at w = -i a (the image of the valley floor)
    phia = -so * ((4 * a + b) * k1 + b) / (8 * k1 * (2 * a + b))
    phiat = -(tectxx * b) / (4 * (2 * a + b))
    d2phia = -(tectxx * b * (4 * a + b) * (b - 12 * a)) / (2 * a * (2 * a + b) * (4 * a + b) ** 3)
    # gravity potential phi and its derivative
    aw = -(1j * (4 * a + b) / (8 * wm)) - ab * (w - 3 * ia) / (8 * k1 * wm ** 3)
    phi = -aw * so / dz + ab * phia / (dz * wm ** 2)
    dlaw = 1j * (4 * a + b) / (8 * wm ** 2) + 2 * ab / (8 * k1 * wm ** 3) - 6j * a ** 2 * b / (8 * k1 * wm ** 4)
    dlphi = -so * dlaw / dz - (2 * ab * (phi + phia)) / (dz * wm ** 3)
    d2phi = -(2 * phi / wm ** 2 + 4 * dlphi / wm + so * 1j * a ** 2 * b / (2 * k1 * wm ** 5)) / dz
    bw = -so * (1j * (4 * a + b) / (8 * wm) + (1 - 2 * nu) * ab * (w - 3 * ia) / (8 * k1 * wm ** 3))
    # tectonic potential
    awt = -(ab * tectxx) / (2 * wm ** 2)
    phit = -awt / dz + ab * phiat / (dz * wm ** 2)
    dlphit = -(ab * tectxx * (4 * a + b) * wm) / (2 * (2 * a + b) * (wm ** 2 - ab) ** 2)
    bwt = -awt
    # psi = -(w phi' + B(w) + phi + psi2) / z', psi2 taken as its limit when a
    # point sits at w = -i a (the reference switches every point when any does)
    r = np.sqrt(u ** 2 + (v + a) ** 2)
    if np.any(r < 1.0e-4):
        psi2 = 0.5 * ab * d2phi
        psi2t = 0.5 * ab * d2phia
    else:
        psi2 = ab * dlphi / wp - ab * (phi - phia) / wp ** 2
        psi2t = ab * dlphit / wp - ab * (phit - phiat) / wp ** 2
    psi = -((w * dlphi + bw + phi) + psi2) / dz
    psit = -((w * dlphit + bwt + phit) + psi2t) / dz
    # Kolosov-Muskhelishvili combinations: sum = Sxx + Syy, dif = Syy - Sxx, Sxy
    zbar = np.conj(z)
    s2 = 2 * (zbar * dlphi / dz + psi)
    s2t = 2 * (zbar * dlphit / dz + psit)
    total = (4 * phit.real + tectxx) + 4 * phi.real + rg * Y / k1
    dif = (s2t.real - tectxx) + s2.real + rg * Y * (1 - 2 * nu) / k1
    Sxy = (s2.imag + s2t.imag) / 2
    Sxx = (total - dif) / 2
    Syy = (total + dif) / 2
    return Sxx, Syy, Sxy, X, Y
