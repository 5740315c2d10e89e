"""Okada (1985) surface displacement and strain of a rectangular dislocation.

TEST INFRASTRUCTURE ONLY: the independent known-answer solution that the
reference's own test (test/test_TDvsOkada.jl) compares its half-space TD
against.  Restated from the published equations (Okada 1985, BSSA 75(4),
eqs. 24-41, Chinnery notation) following the reference's use of them in
src/Okada1985RectangularDislocation.jl:1-153 (geographic rotation and the
conversion to the TD strain convention at :117-150).
"""
from __future__ import annotations

import numpy as np

_EPS = np.finfo(float).eps


def _atan_term(xi, eta, q, R):
    with np.errstate(divide="ignore", invalid="ignore"):
        t = np.arctan(xi * eta / (q * R))
    return np.where(q != 0, t, 0.0)


class _Sub:
    """Auxiliary functions at one corner (xi, eta) for a fixed dip."""

    def __init__(self, xi, eta, q, dip, nu):
        self.xi, self.eta, self.q = xi, eta, q
        self.sd, self.cd = np.sin(dip), np.cos(dip)
        self.nu = nu
        self.R = np.sqrt(xi ** 2 + eta ** 2 + q ** 2)
        self.db = eta * self.sd - q * self.cd
        self.yb = eta * self.cd + q * self.sd
        self.vert = not (self.cd > _EPS)
        self.k = 1 - 2 * nu

    def A(self, x):
        R = self.R
        return (2 * R + x) / (R ** 3 * (R + x) ** 2)

    # displacement I-terms (eqs. 28-29)
    def I5(self):
        xi, eta, q, R, sd, cd, k = self.xi, self.eta, self.q, self.R, self.sd, self.cd, self.k
        if self.vert:
            return -k * xi * sd / (R + self.db)
        X = np.sqrt(xi ** 2 + q ** 2)
        with np.errstate(divide="ignore", invalid="ignore"):
            v = k * 2 / cd * np.arctan((eta * (X + q * cd) + X * (R + X) * sd) / (xi * (R + X) * cd))
        return np.where(xi == 0, 0.0, v)

    def I4(self):
        R, k = self.R, self.k
        if self.vert:
            return -k * self.q / (R + self.db)
        return k * 1 / self.cd * (np.log(R + self.db) - self.sd * np.log(R + self.eta))

    def I3(self):
        R, k, eta = self.R, self.k, self.eta
        if self.vert:
            return k / 2 * (eta / (R + self.db) + self.yb * self.q / (R + self.db) ** 2 - np.log(R + eta))
        return k * (self.yb / (self.cd * (R + self.db)) - np.log(R + eta)) + self.sd / self.cd * self.I4()

    def I2(self):
        return self.k * (-np.log(self.R + self.eta)) - self.I3()

    def I1(self):
        R, k, xi = self.R, self.k, self.xi
        if self.vert:
            return -k / 2 * xi * self.q / (R + self.db) ** 2
        return k * (-xi / (self.cd * (R + self.db))) - self.sd / self.cd * self.I5()

    # tilt K-terms (eqs. 40-41)
    def K3(self):
        R, k, q = self.R, self.k, self.q
        if self.vert:
            return k * self.sd / (R + self.db) * (self.xi ** 2 / (R * (R + self.db)) - 1)
        return k * 1 / self.cd * (q / (R * (R + self.eta)) - self.yb / (R * (R + self.db)))

    def K2(self):
        R = self.R
        return self.k * (-self.sd / R + self.q * self.cd / (R * (R + self.eta))) - self.K3()

    def K1(self):
        R, k, xi = self.R, self.k, self.xi
        if self.vert:
            return k * xi * self.q / (R * (R + self.db) ** 2)
        return k * xi / self.cd * (1 / (R * (R + self.db)) - self.sd / (R * (R + self.eta)))

    # strain J-terms (eqs. 34-35)
    def J1(self):
        R, k, xi, q = self.R, self.k, self.xi, self.q
        if self.vert:
            return k / 2 * q / (R + self.db) ** 2 * (2 * xi ** 2 / (R * (R + self.db)) - 1)
        return k * 1 / self.cd * (xi ** 2 / (R * (R + self.db) ** 2) - 1 / (R + self.db)) - self.sd / self.cd * self.K3()

    def J2(self):
        R, k, xi, q = self.R, self.k, self.xi, self.q
        if self.vert:
            return k / 2 * xi * self.sd / (R + self.db) ** 2 * (2 * q ** 2 / (R * (R + self.db)) - 1)
        return k * 1 / self.cd * xi * self.yb / (R * (R + self.db) ** 2) - self.sd / self.cd * self.K1()

    def J3(self):
        return self.k * -self.xi / (self.R * (self.R + self.eta)) - self.J2()

    def J4(self):
        R = self.R
        return self.k * (-self.cd / R - self.q * self.sd / (R * (R + self.eta))) - self.J1()


def _corner_terms(xi, eta, q, dip, nu):
    """All 27 Chinnery integrands at one corner, keyed 'ux_ss' ... 'uyy_tf'."""
    s = _Sub(xi, eta, q, dip, nu)
    R, sd, cd, db, yb = s.R, s.sd, s.cd, s.db, s.yb
    at = _atan_term(xi, eta, q, R)
    Ae, Ax = s.A(eta), s.A(xi)
    I1, I2, I3, I4, I5 = s.I1(), s.I2(), s.I3(), s.I4(), s.I5()
    K1, K2, K3 = s.K1(), s.K2(), s.K3()
    J1, J2, J3, J4 = s.J1(), s.J2(), s.J3(), s.J4()
    t = {}
    # displacements (eqs. 25-27)
    t["ux_ss"] = xi * q / (R * (R + eta)) + I1 * sd + at
    t["uy_ss"] = (eta * cd + q * sd) * q / (R * (R + eta)) + q * cd / (R + eta) + I2 * sd
    t["uz_ss"] = (eta * sd - q * cd) * q / (R * (R + eta)) + q * sd / (R + eta) + I4 * sd
    t["ux_ds"] = q / R - I3 * sd * cd
    t["uy_ds"] = (eta * cd + q * sd) * q / (R * (R + xi)) - I1 * sd * cd + cd * at
    t["uz_ds"] = db * q / (R * (R + xi)) - I5 * sd * cd + sd * at
    t["ux_tf"] = q ** 2 / (R * (R + eta)) - I3 * sd ** 2
    t["uy_tf"] = -(eta * sd - q * cd) * q / (R * (R + xi)) - sd * xi * q / (R * (R + eta)) - I1 * sd ** 2 + sd * at
    t["uz_tf"] = (eta * cd + q * sd) * q / (R * (R + xi)) + cd * xi * q / (R * (R + eta)) - I5 * sd ** 2 - cd * at
    # tilts (eqs. 37-39)
    t["uzx_ss"] = -xi * q ** 2 * Ae * cd + ((xi * q) / R ** 3 - K1) * sd
    t["uzy_ss"] = (db * q / R ** 3) * cd + (xi ** 2 * q * Ae * cd - sd / R + yb * q / R ** 3 - K2) * sd
    t["uzx_ds"] = db * q / R ** 3 + q * sd / (R * (R + eta)) + K3 * sd * cd
    t["uzy_ds"] = yb * db * q * Ax - (2 * db / (R * (R + xi)) + xi * sd / (R * (R + eta))) * sd + K1 * sd * cd
    t["uzx_tf"] = q ** 2 / R ** 3 * sd - q ** 3 * Ae * cd + K3 * sd ** 2
    t["uzy_tf"] = (yb * sd + db * cd) * q ** 2 * Ax + xi * q ** 2 * Ae * sd * cd - (2 * q / (R * (R + xi)) - K1) * sd ** 2
    # strains (eqs. 31-33)
    t["uxx_ss"] = xi ** 2 * q * Ae - J1 * sd
    t["uxy_ss"] = xi ** 3 * db / (R ** 3 * (eta ** 2 + q ** 2)) - (xi ** 3 * Ae + J2) * sd
    t["uyx_ss"] = xi * q / R ** 3 * cd + (xi * q ** 2 * Ae - J2) * sd
    t["uyy_ss"] = yb * q / R ** 3 * cd + (q ** 3 * Ae * sd - 2 * q * sd / (R * (R + eta)) - (xi ** 2 + eta ** 2) / R ** 3 * cd - J4) * sd
    t["uxx_ds"] = xi * q / R ** 3 + J3 * sd * cd
    t["uxy_ds"] = yb * q / R ** 3 - sd / R + J1 * sd * cd
    t["uyx_ds"] = yb * q / R ** 3 + q * cd / (R * (R + eta)) + J1 * sd * cd
    t["uyy_ds"] = yb ** 2 * q * Ax - (2 * yb / (R * (R + xi)) + xi * cd / (R * (R + eta))) * sd + J2 * sd * cd
    t["uxx_tf"] = xi * q ** 2 * Ae + J3 * sd ** 2
    t["uxy_tf"] = -db * q / R ** 3 - xi ** 2 * q * Ae * sd + J1 * sd ** 2
    t["uyx_tf"] = q ** 2 / R ** 3 * cd + q ** 3 * Ae * sd + J1 * sd ** 2
    t["uyy_tf"] = (yb * cd - db * sd) * q ** 2 * Ax - q * np.sin(2 * dip) / (R * (R + xi)) - (xi * q ** 2 * Ae - J2) * sd ** 2
    return t


def okada85(e, n, depth, strike, dip, L, W, rake, slip, opening, nu):
    """Surface (z = 0) field of a rectangular dislocation whose centroid lies at
    (0, 0, -depth).  Angles in degrees.  Returns (ue, un, uz, exx, eyy, ezz,
    exy, exz, eyz) in the TD strain convention of the reference."""
    e = np.asarray(e, dtype=np.float64).reshape(-1)
    n = np.asarray(n, dtype=np.float64).reshape(-1)
    st, dp, rk = np.deg2rad(strike), np.deg2rad(dip), np.deg2rad(rake)
    U1, U2, U3 = np.cos(rk) * slip, np.sin(rk) * slip, opening
    d = depth + np.sin(dp) * W / 2
    ec = e + np.cos(st) * np.cos(dp) * W / 2
    nc = n - np.sin(st) * np.cos(dp) * W / 2
    x = np.cos(st) * nc + np.sin(st) * ec + L / 2
    y = np.sin(st) * nc - np.cos(st) * ec + np.cos(dp) * W
    p = y * np.cos(dp) + d * np.sin(dp)
    q = y * np.sin(dp) - d * np.cos(dp)
    corners = [(x, p, 1.0), (x, p - W, -1.0), (x - L, p, -1.0), (x - L, p - W, 1.0)]
    acc = {}
    for xi, eta, sgn in corners:
        t = _corner_terms(xi, eta, q, dp, nu)
        for k, v in t.items():
            acc[k] = acc.get(k, 0.0) + sgn * v

    def comb(base):
        return (-U1 / (2 * np.pi) * acc[base + "_ss"] - U2 / (2 * np.pi) * acc[base + "_ds"]
                + U3 / (2 * np.pi) * acc[base + "_tf"])

    ux, uy, uz = comb("ux"), comb("uy"), comb("uz")
    uxx, uxy, uyx, uyy = comb("uxx"), comb("uxy"), comb("uyx"), comb("uyy")
    uzx, uzy = comb("uzx"), comb("uzy")
    s, c = np.sin(st), np.cos(st)
    ue = s * ux - c * uy
    un = c * ux + s * uy
    unn = c ** 2 * uxx + np.sin(2 * st) * (uxy + uyx) / 2 + s ** 2 * uyy
    une = np.sin(2 * st) * (uxx - uyy) / 2 + s ** 2 * uyx - c ** 2 * uxy
    uen = np.sin(2 * st) * (uxx - uyy) / 2 - c ** 2 * uyx + s ** 2 * uxy
    uee = s ** 2 * uxx - np.sin(2 * st) * (uyx + uxy) / 2 + c ** 2 * uyy
    uze = -s * uzx + c * uzy
    uzn = -c * uzx - s * uzy
    unz, uez = -uzn, -uze
    uzz = -(uee + unn) * nu / (1 - nu)
    exy = -(uen + une) / 2
    uyz = -(uzn + unz) / 2
    uxz = -(uze + uez) / 2
    return ue, un, uz, -uee, -unn, -uzz, exy, -uxz, -uyz
