"""CPU oracle for the frictional slip solve (numpy).

TEST INFRASTRUCTURE ONLY: tests/ use this module as the checker.  The product
never imports it.

What it restates:
  * SlipCalculator3D with MixedBoundaryConditionsFriction
    (src/SlipCalculator3D.jl:36-87): the early exit when no element can
    overcome its frictional resistance (:47-55), A and b of the plain solve,
    Scl = mean(HalfPerimeter)/G (:58-60), C = inv(A*Scl) (:61);
  * the 5n x 5n linear complementarity problem (src/SlipCalculator3D.jl:90-175)
    and the read-out of slip from its solution (:177-238);
  * Burgmann (1994) slip of a 2D crack with linearly increasing cohesion
    (src/Burgmann1994_FractureLinearFrictionSlipProfile.jl) and the
    Pollard-Segall (1987) profile (src/PollardSegall1987_FractureSlipProfile.jl),
    the analytic solutions test/test_TDvsBurgmannLinearFrictionCrack.jl checks
    against.

The reference solves the LCP with FischerNewton.fischer_newton (package
FischerNewton 0.1.4, git-tree-sha1 d1eea50f5d0dbcc5967a974fff06d9e7b1c16637,
Manifest.toml:275-281), which is not part of the reference checkout.  Its
source is not restated; `fischer_newton` below is the published method it is
named for, written from the mathematics: the Fischer-Burmeister NCP function
phi(a, b) = sqrt(a^2 + b^2) - a - b (Fischer 1992) turns the LCP
x >= 0, y = M x + q >= 0, x'y = 0 into Phi(x) = 0, solved by a semismooth
Newton method with an Armijo backtracking line search on psi = |Phi|^2 / 2;
at points where x_i = y_i = 0 the generalized Jacobian row is taken along
z = e_beta as De Luca, Facchinei and Kanzow (1996) construct it.  The LCP
solution it converges to is what is compared, not its iterates.
"""
from __future__ import annotations

import numpy as np

from . import oracle as _orc
from .geometry import area_half_perimeter


def fb_phi(a, b):
    """Fischer-Burmeister function, in the cancellation-free form
    -2ab / (sqrt(a^2+b^2) + a + b) where a + b > 0."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    r = np.sqrt(a * a + b * b)
    s = a + b
    with np.errstate(divide="ignore", invalid="ignore"):
        stable = -2.0 * a * b / (r + s)
    return np.where(s > 0, stable, r - s)


def fb_jacobian_diag(x, y, z, w):
    """Diagonals (Da, Db) of a generalized Jacobian J = diag(Da) + diag(Db) M.
    Rows with x_i = y_i = 0 use (z_i, w_i) = (1, (M e_beta)_i) instead."""
    deg = z != 0
    a = np.where(deg, z, x)
    b = np.where(deg, w, y)
    r = np.sqrt(a * a + b * b)
    return a / r - 1.0, b / r - 1.0


def fischer_newton(M, q, tol=1e-10, max_iter=100, sigma=1e-4, halvings=40):
    """Solve the LCP (M, q) from x = 0.  Returns (x, iterations, rel), rel =
    max|Phi(x)| / max(|q|) at exit (converged when rel <= tol)."""
    M = np.asarray(M, dtype=np.float64)
    q = np.asarray(q, dtype=np.float64).reshape(-1)
    n = q.shape[0]
    x = np.zeros(n)
    qscale = float(np.max(np.abs(q))) if n else 0.0
    if qscale == 0.0:
        qscale = 1.0
    it = 0
    while True:
        y = M @ x + q
        phi = fb_phi(x, y)
        rel = float(np.max(np.abs(phi))) / qscale if n else 0.0
        if rel <= tol or it >= max_iter:
            return x, it, rel
        z = ((x == 0.0) & (y == 0.0)).astype(np.float64)
        w = M @ z if z.any() else np.zeros(n)
        Da, Db = fb_jacobian_diag(x, y, z, w)
        J = Db[:, None] * M
        J[np.diag_indices(n)] += Da
        psi = 0.5 * float(phi @ phi)
        try:
            d = np.linalg.solve(J, -phi)
            slope = -2.0 * psi
            ok = bool(np.all(np.isfinite(d)))
        except np.linalg.LinAlgError:
            ok = False
        if not ok:   # steepest descent on psi
            g = Da * phi + M.T @ (Db * phi)
            d = -g
            slope = -float(g @ g)
        Md = M @ d
        step = 0.0
        t = 1.0
        for _ in range(halvings):
            if 0.5 * float(np.sum(fb_phi(x + t * d, y + t * Md) ** 2)) <= psi + sigma * t * slope:
                step = t
                break
            t *= 0.5
        it += 1
        if step == 0.0:   # no decrease left at rounding level
            y = M @ x + q
            rel = float(np.max(np.abs(fb_phi(x, y)))) / qscale
            return x, it, rel
        x = x + step * d


def friction_lcp(C, b, mu, Sf):
    """(M, q) of src/SlipCalculator3D.jl:90-175 and :190-193: C = inv(A*Scl)
    (3n x 3n), b the traction vector [Tn; Tss; Tds], mu and Sf per element
    (scalars broadcast as `zeros(n).+mu` does)."""
    C = np.asarray(C, dtype=np.float64)
    n = C.shape[0] // 3
    mu = np.zeros(n) + mu
    Sf = np.zeros(n) + Sf
    L = [slice(k * n, (k + 1) * n) for k in range(5)]
    dmu = np.diag(mu)
    ID = np.eye(n)
    M = np.zeros((5 * n, 5 * n))
    for r in range(3):
        Cr1, Cr2, Cr3 = C[L[r], L[0]], C[L[r], L[1]], C[L[r], L[2]]
        M[L[r], L[0]] = Cr1 - Cr2 @ dmu - Cr3 @ dmu
        M[L[r], L[1]] = Cr2
        M[L[r], L[2]] = Cr3
    M[L[1], L[3]] = ID
    M[L[2], L[4]] = ID
    M[L[3], L[0]] = 2 * dmu
    M[L[3], L[1]] = -ID
    M[L[4], L[0]] = 2 * dmu
    M[L[4], L[2]] = -ID
    D = C @ np.asarray(b, dtype=np.float64)
    q = np.zeros(5 * n)
    for r in range(3):
        q[L[r]] = -C[L[r], L[1]] @ Sf - C[L[r], L[2]] @ Sf + D[L[r]]
    q[L[3]] = 2 * Sf
    q[L[4]] = 2 * Sf
    return M, q


def friction_slip_from_lcp(M, q, x, n, Scl):
    """Dn, Dss, Dds (scaled back by Scl) and Tn, Tss, Tds of an LCP solution
    (src/SlipCalculator3D.jl:197-237)."""
    y = M @ x + q
    L = [slice(k * n, (k + 1) * n) for k in range(5)]
    Dn = y[L[0]] * Scl
    Dss = (y[L[1]] - x[L[3]]) * Scl
    Dds = (y[L[2]] - x[L[4]]) * Scl
    Tn = -x[L[0]]
    Tss = y[L[3]] - x[L[1]]
    Tds = y[L[4]] - x[L[2]]
    return Dn, Dss, Dds, Tn, Tss, Tds


def slip_calculator_friction(P1, P2, P3, nu, G, lam, midpoints, normals, hs, Tn, Tss, Tds, mu, Sf, tol=1e-10,
                             max_iter=100, nthreads=None):
    """SlipCalculator3D with friction (src/SlipCalculator3D.jl:36-87).
    Tn, Tss, Tds: the element tractions of the boundary conditions (remote
    stress resolved plus applied tractions).  Returns (Dn, Dss, Dds, info)
    with info = dict(iterations, rel, exit) where exit is True when the early
    return of :47-55 was taken."""
    Tn, Tss, Tds = (np.asarray(t, dtype=np.float64).reshape(-1) for t in (Tn, Tss, Tds))
    n = Tn.shape[0]
    fric_res = Tn * mu
    if np.all(-np.abs(Tss) > fric_res) and np.all(-np.abs(Tds) > fric_res):
        return np.zeros(n), np.zeros(n), np.zeros(n), dict(iterations=0, rel=0.0, exit=True)
    A = _orc.influence_traction(normals, midpoints, P1, P2, P3, nu, G, lam, hs, nthreads=nthreads, want_A=True)
    b = np.concatenate([Tn, Tss, Tds])
    _, half = area_half_perimeter(np.asarray(P1, float), np.asarray(P2, float), np.asarray(P3, float))
    Scl = float(np.mean(half)) / G
    C = np.linalg.inv(A * Scl)
    M, q = friction_lcp(C, b, mu, Sf)
    x, it, rel = fischer_newton(M, q, tol=tol, max_iter=max_iter)
    Dn, Dss, Dds, *_ = friction_slip_from_lcp(M, q, x, n, Scl)
    return Dn, Dss, Dds, dict(iterations=it, rel=rel, exit=False, x=x, M=M, q=q)


def burgmann1994_slip(G, nu, Ts, x, a):
    """Slip of a 2D crack under remote shear Ts with cohesion growing linearly
    with |x| (src/Burgmann1994_FractureLinearFrictionSlipProfile.jl)."""
    x = np.abs(np.asarray(x, dtype=np.float64))
    out = np.zeros_like(x)
    for i, xi in enumerate(x):
        s = np.sqrt(complex(a * a - xi * xi)).real
        term = (xi * xi / a) * np.arccosh(a / xi) if a / xi >= 1 else (xi * xi / a)
        out[i] = ((1 - nu) / G) * (2 * ((Ts * s) - ((Ts * (1 / np.pi)) * (s + term))))
    return out


def pollard_segall1987_slip(G, nu, syy, sxy, x, a):
    """Opening/sliding of a 2D crack under uniform remote load
    (src/PollardSegall1987_FractureSlipProfile.jl, first output)."""
    x = np.asarray(x, dtype=np.float64)
    return (2 * (1 - nu) / G) * np.sqrt(a ** 2 - x ** 2) * (syy + sxy)
