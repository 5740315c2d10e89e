"""Seeded synthetic workloads with the shapes of the benchmark configurations.

There is no public dataset for this path; every mesh, slip and boundary
condition below is generated from a seed.

  fault_grid      planar rectangular fault on y = 0, split into triangles, with
                  an observation grid on a parallel plane (forward evaluation)
  penny           circular crack on z = 0: Delaunay triangulation of a jittered
                  hexagonal lattice (full-space assembly + solve)
  dipping_rect    rectangle dipping at a given angle below the free surface:
                  jittered regular triangulation (half-space assembly + solve)
  remote_stress   seeded uniform remote stress tensor
  surface_grid    observation grid on the free surface z = 0
"""
from __future__ import annotations

import numpy as np


def _orient_up(P1, P2, P3, up=np.array([0.0, 0.0, 1.0])):
    n = np.cross(P2 - P1, P3 - P1)
    flip = (n @ up) < 0
    P2, P3 = np.where(flip[:, None], P3, P2), np.where(flip[:, None], P2, P3)
    return P1, P2, P3


def fault_grid(seed=0, nx=10, nz=5, ngrid=50, x=(-1.0, 1.0), z=(-1.5, -0.5), obs_y=0.1, obs_extent=2.0,
               slip_scale=1e-3):
    """Fault on y = 0 cut into nx x nz rectangles, each split into 2 triangles;
    slips U[-slip_scale, slip_scale]; ngrid x ngrid observation points on y = obs_y."""
    rng = np.random.default_rng(seed)
    xs = np.linspace(x[0], x[1], nx + 1)
    zs = np.linspace(z[0], z[1], nz + 1)
    P1, P2, P3 = [], [], []
    for i in range(nx):
        for k in range(nz):
            a = [xs[i], 0.0, zs[k]]
            b = [xs[i + 1], 0.0, zs[k]]
            c = [xs[i + 1], 0.0, zs[k + 1]]
            d = [xs[i], 0.0, zs[k + 1]]
            P1 += [a, a]
            P2 += [b, c]
            P3 += [c, d]
    P1, P2, P3 = (np.array(p, dtype=np.float64) for p in (P1, P2, P3))
    n = len(P1)
    Dss, Dds, Dn = rng.uniform(-slip_scale, slip_scale, (3, n))
    g = np.linspace(-obs_extent, obs_extent, ngrid)
    gx, gz = np.meshgrid(g, g)
    X = gx.reshape(-1, order="F")
    Z = gz.reshape(-1, order="F")
    Y = np.full_like(X, obs_y)
    return dict(P1=P1, P2=P2, P3=P3, Dss=Dss, Dds=Dds, Dn=Dn, X=X, Y=Y, Z=Z)


def penny(seed=0, radius=1.0, spacing=0.06, jitter=0.1, z=0.0):
    """Circular crack: Delaunay of a hexagonal lattice inside the circle (interior
    points jittered by +-jitter*spacing) plus points on the rim."""
    from scipy.spatial import Delaunay

    rng = np.random.default_rng(seed)
    h = spacing * np.sqrt(3) / 2
    pts = []
    nrow = int(np.ceil(radius / h)) + 1
    ncol = int(np.ceil(radius / spacing)) + 1
    for j in range(-nrow, nrow + 1):
        for i in range(-ncol, ncol + 1):
            px = i * spacing + (spacing / 2 if j % 2 else 0.0)
            py = j * h
            if np.hypot(px, py) < radius - 0.5 * spacing:
                pts.append((px, py))
    pts = np.array(pts)
    pts = pts + rng.uniform(-jitter * spacing, jitter * spacing, pts.shape)
    nrim = int(np.round(2 * np.pi * radius / spacing))
    th = np.linspace(0, 2 * np.pi, nrim, endpoint=False)
    rim = radius * np.stack([np.cos(th), np.sin(th)], 1)
    pts = np.vstack([pts, rim])
    tri = Delaunay(pts).simplices
    P = np.column_stack([pts, np.full(len(pts), z)])
    P1, P2, P3 = P[tri[:, 0]], P[tri[:, 1]], P[tri[:, 2]]
    area = 0.5 * np.abs(np.cross(P2 - P1, P3 - P1)[:, 2])
    keep = area > 1e-3 * spacing * spacing
    return _orient_up(P1[keep], P2[keep], P3[keep])


def dipping_rect(seed=0, ntri=10000, length=2.0, width=1.0, dip=60.0, top_depth=2.0, jitter=0.1):
    """Rectangle (length along strike x, width down dip) dipping `dip` degrees,
    top edge at z = -top_depth; regular grid of ~ntri/2 cells jittered by
    +-jitter of a cell at interior nodes, each cell split into 2 triangles."""
    rng = np.random.default_rng(seed)
    ncell = ntri // 2
    nw = max(1, int(round(np.sqrt(ncell * width / length))))
    nl = max(1, ncell // nw)
    u = np.linspace(-length / 2, length / 2, nl + 1)
    w = np.linspace(0.0, width, nw + 1)
    U, W = np.meshgrid(u, w, indexing="ij")
    du, dw = length / nl, width / nw
    interior = np.zeros_like(U, dtype=bool)
    interior[1:-1, 1:-1] = True
    U = U + np.where(interior, rng.uniform(-jitter * du, jitter * du, U.shape), 0.0)
    W = W + np.where(interior, rng.uniform(-jitter * dw, jitter * dw, W.shape), 0.0)
    d = np.deg2rad(dip)
    X = U
    Y = W * np.cos(d)
    Z = -top_depth - W * np.sin(d)
    node = np.stack([X, Y, Z], -1)
    P1, P2, P3 = [], [], []
    for i in range(nl):
        for k in range(nw):
            a, b, c, e = node[i, k], node[i + 1, k], node[i + 1, k + 1], node[i, k + 1]
            P1 += [a, a]
            P2 += [b, c]
            P3 += [c, e]
    P1, P2, P3 = (np.array(p) for p in (P1, P2, P3))
    return P1, P2, P3


def remote_stress(seed=0, scale=1e-3):
    """Six remote stress components (sxx, syy, szz, sxy, sxz, syz) ~ U[-scale, scale]."""
    return np.random.default_rng(seed).uniform(-scale, scale, 6)


def surface_grid(n=100, extent=4.0):
    g = np.linspace(-extent, extent, n)
    gx, gy = np.meshgrid(g, g)
    X = gx.reshape(-1, order="F")
    Y = gy.reshape(-1, order="F")
    return X, Y, np.zeros_like(X)


def ellipse_crack(seed=0, a=1.0, b=1.0, ntri=800, jitter=0.1):
    """Elliptical crack with semi-axes a (x) and b (y) on z = 0, ~ntri triangles:
    the unit penny mesh at the lattice spacing that gives ntri, stretched."""
    # a penny of radius 1 at spacing s has ~ 2 pi / (sqrt(3) s^2 / 2) lattice
    # points, about twice as many triangles
    s = np.sqrt(4 * np.pi / (np.sqrt(3) * max(ntri, 8)))
    P1, P2, P3 = penny(seed=seed, radius=1.0, spacing=s, jitter=jitter)
    scale = np.array([a, b, 1.0])
    return P1 * scale, P2 * scale, P3 * scale


def crack_batch(seed=0, count=512, n_range=(200, 2000), radius_range=(0.5, 2.0), aspect_range=(0.3, 1.0)):
    """`count` independent full-space cracks: semi-major axis U[radius_range],
    aspect ratio U[aspect_range] (1: penny), random orientation (uniform on
    the sphere) and centre, triangle count log-uniform in n_range.  Returns a
    list of (P1, P2, P3) and the seeded remote stress (6 components) of each."""
    rng = np.random.default_rng(seed)
    out, stresses = [], []
    for k in range(count):
        n = int(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]))))
        a = rng.uniform(*radius_range)
        b = a * rng.uniform(*aspect_range)
        P1, P2, P3 = ellipse_crack(seed=int(rng.integers(1 << 30)), a=a, b=b, ntri=n)
        q = rng.standard_normal(4)
        q /= np.linalg.norm(q)
        w, x, y, z = q
        R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                      [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                      [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])
        c = rng.uniform(-5, 5, 3)
        out.append(tuple(P @ R.T + c for P in (P1, P2, P3)))
        stresses.append(rng.uniform(-1e-3, 1e-3, 6))
    return out, stresses
