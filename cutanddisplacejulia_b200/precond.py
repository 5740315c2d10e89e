"""Learned sparse-approximate-inverse preconditioner for the influence system
(an addition to the reference, whose only solver is the dense A\\b of
src/SlipCalculator3D.jl:22).

For element i, a small network (csrc/mlp.cu; trained and evaluated by the
library's own BF16 kernels) reads the geometry of i's 16 nearest elements --
centroid offsets and normals in i's own (normal, strike, dip) frame, scaled by
i's size, and area ratios -- and predicts the 16 3x3 blocks (A^-1)[i, j] of
the inverse system matrix between i and those neighbours, in units of
h_i / G (h_i = sqrt(2 area_i)).  Those blocks form a block-sparse right
preconditioner M ~ A^-1 for FP64 GMRES (cad_set_preconditioner,
CAD_SOLVER_GMRES_SPAI).  Training targets are the same blocks of exact
inverses that the library computes (FP64 LU with the identity as right-hand
side) on small seeded meshes.

Device buffers are torch tensors (memory plumbing only); every computation
on them is a libcad_td.so kernel.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .geometry import CreateFaceNormalAndMidPoint, ss_ds_dirs

K = 16          # neighbours per element (the element itself first)
N_IN = 7 * K    # offset (3), normal (3), area ratio (1) per neighbour
N_OUT = 9 * K


def element_frames(P1, P2, P3):
    """Centroids, normals, strike and dip directions, areas of the triangles."""
    P1, P2, P3 = (np.asarray(p, dtype=np.float64).reshape(-1, 3) for p in (P1, P2, P3))
    nrm, _ = CreateFaceNormalAndMidPoint(P1, P2, P3)
    ss, ds = ss_ds_dirs(nrm[:, 0], nrm[:, 1], nrm[:, 2])
    cen = (P1 + P2 + P3) / 3.0
    area = 0.5 * np.linalg.norm(np.cross(P2 - P1, P3 - P1), axis=1)
    return cen, nrm, ss, ds, area


def features(P1, P2, P3):
    """(X, nbr, h): network inputs (N x 112, float32), the 16 nearest
    elements of each element (N x 16, int32, itself first) and the element
    sizes h = sqrt(2 area) that scale offsets and the predicted blocks."""
    from scipy.spatial import cKDTree
    cen, nrm, ss, ds, area = element_frames(P1, P2, P3)
    n = len(cen)
    k = min(K, n)
    nbr = cKDTree(cen).query(cen, k=k)[1].reshape(n, k)
    if k < K:   # tiny meshes: repeat the farthest neighbour (its blocks are trained to share)
        nbr = np.concatenate([nbr, np.repeat(nbr[:, -1:], K - k, axis=1)], axis=1)
    h = np.sqrt(2.0 * area)
    R = np.stack([nrm, ss, ds], axis=1)                       # N x 3 x 3, rows = local axes
    off = np.einsum("iab,ikb->ika", R, cen[nbr] - cen[:, None, :]) / h[:, None, None]
    nloc = np.einsum("iab,ikb->ika", R, nrm[nbr])
    arat = (area[nbr] / area[:, None])[..., None]
    X = np.concatenate([off, nloc, arat], axis=2).reshape(n, N_IN)
    return X.astype(np.float32), nbr.astype(np.int32), h


def inverse_blocks(Ainv, nbr, h, G):
    """Training targets: (A^-1)[i, nbr[i, q]] as 3x3 blocks (rows: unknowns
    i, N + i, 2N + i; columns the neighbour's), divided by h_i / G; N x 144."""
    n = nbr.shape[0]
    rows = np.stack([np.arange(n), n + np.arange(n), 2 * n + np.arange(n)], axis=1)     # N x 3
    cols = np.stack([nbr, n + nbr, 2 * n + nbr], axis=2)                                  # N x K x 3
    T = Ainv[rows[:, None, :, None], cols[:, :, None, :]]                                # N x K x 3 x 3
    return (T / (h / G)[:, None, None, None]).reshape(n, N_OUT).astype(np.float32)


def training_meshes(seed=0, count=24, n_range=(250, 700)):
    """Seeded small meshes: full-space penny / elliptical cracks and
    half-space dipping rectangles (depth and dip varied)."""
    from . import workloads
    rng = np.random.default_rng(seed)
    out = []
    for c in range(count):
        n = int(np.exp(rng.uniform(np.log(n_range[0]), np.log(n_range[1]))))
        if c % 2 == 0:
            a = rng.uniform(0.5, 2.0)
            P = workloads.ellipse_crack(seed=int(rng.integers(1 << 30)), a=a, b=a * rng.uniform(0.3, 1.0), ntri=n)
            out.append((P, 0))
        else:
            P = workloads.dipping_rect(seed=int(rng.integers(1 << 30)), ntri=n, length=rng.uniform(1.0, 3.0),
                                       width=rng.uniform(0.5, 1.5), dip=rng.uniform(20, 90),
                                       top_depth=rng.uniform(0.3, 3.0))
            out.append((P, 1))
    return out


def training_set(meshes, G=1.0, nu=0.25, device=0):
    """(X, T): features and exact-inverse targets of every element of every
    mesh; the inverses come from the library's FP64 LU (A X = I)."""
    from .assembly import SlipCalculator3D, solve
    from .geometry import ElasticConstantsCheck
    from .structs import Tractions
    _, _, lam, nu, G = ElasticConstantsCheck(G, nu)
    Xs, Ts = [], []
    for (P1, P2, P3), hs in meshes:
        n = len(P1)
        nrm, mid = CreateFaceNormalAndMidPoint(P1, P2, P3)
        A = SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, hs, Tractions(np.ones(n), np.zeros(n), np.zeros(n)),
                             np.zeros(n), device=device)[3]
        Ainv = solve(A, np.eye(3 * n), device=device)
        X, nbr, h = features(P1, P2, P3)
        Xs.append(X)
        Ts.append(inverse_blocks(Ainv, nbr, h, G))
    return np.concatenate(Xs), np.concatenate(Ts)


class Network:
    """The preconditioner network's FP32 master weights on the device, trained
    and evaluated by cad_lpc_step."""

    def __init__(self, seed=0, device=0, params=None):
        import torch
        self.dev = torch.device("cuda", device)
        self.ctx = _lib.context(device)
        self.L = _lib.load()
        npar = self.L.cad_lpc_param_count()
        if params is None:
            params = init_params(seed)
        assert params.size == npar
        self.params = torch.tensor(params, dtype=torch.float32, device=self.dev)
        self.m = torch.zeros_like(self.params)
        self.v = torch.zeros_like(self.params)
        self.t = 0

    def _step(self, X, T=None, out=None, grads=None, loss=None, adam=False, lr=1e-3):
        P = ctypes.c_void_p
        ptr = (lambda a: None if a is None else P(a.data_ptr()))
        rc = self.L.cad_lpc_step(self.ctx, ptr(self.params), ptr(X), ptr(T), X.shape[0], ptr(out), ptr(grads),
                                 ptr(loss), ptr(self.m) if adam else None, ptr(self.v) if adam else None, self.t,
                                 ctypes.c_float(lr))
        _lib.check(rc, self.ctx)

    def gradients(self, X, T):
        """(sum of squared errors, gradient of the mean squared error) of one
        pass over X (rows x 112), T (rows x 144) -- numpy in, numpy out."""
        import torch
        Xd = torch.tensor(X, dtype=torch.float32, device=self.dev)
        Td = torch.tensor(T, dtype=torch.float32, device=self.dev)
        g = torch.zeros_like(self.params)
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        self._step(Xd, Td, grads=g, loss=loss)
        torch.cuda.synchronize(self.dev)
        return float(loss.item()), g.cpu().numpy()

    def train(self, X, T, steps=2000, batch=4096, lr=1e-3, seed=0):
        """Adam on minibatches drawn (seeded) from X, T; returns the loss
        (mean squared error) of every 100th step's minibatch."""
        import torch
        Xd = torch.tensor(X, dtype=torch.float32, device=self.dev)
        Td = torch.tensor(T, dtype=torch.float32, device=self.dev)
        g = torch.zeros_like(self.params)
        loss = torch.zeros(1, dtype=torch.float32, device=self.dev)
        rng = np.random.default_rng(seed)
        n = X.shape[0]
        hist = []
        for s in range(steps):
            idx = torch.tensor(rng.integers(0, n, min(batch, n)), device=self.dev)
            xb, tb = Xd[idx].contiguous(), Td[idx].contiguous()
            self.t += 1
            lr_s = lr * 0.5 * (1 + np.cos(np.pi * s / steps))
            self._step(xb, tb, grads=g, loss=loss if s % 100 == 0 else None, adam=True, lr=lr_s)
            if s % 100 == 0:
                hist.append(float(loss.item()) / (xb.shape[0] * N_OUT))
        torch.cuda.synchronize(self.dev)
        return hist

    def predict(self, X):
        """Network outputs (rows x 144) for X (rows x 112): numpy in, torch (device) out."""
        import torch
        Xd = torch.tensor(X, dtype=torch.float32, device=self.dev)
        out = torch.empty((X.shape[0], N_OUT), dtype=torch.float32, device=self.dev)
        self._step(Xd, out=out)
        return out


def init_params(seed=0):
    """He-initialised weights, zero biases (FP32, the library's layout)."""
    rng = np.random.default_rng(seed)
    parts = []
    for fi, fo in ((N_IN, 256), (256, 256), (256, N_OUT)):
        parts.append(rng.standard_normal((fi, fo)).astype(np.float32) * np.float32(np.sqrt(2.0 / fi)))
        parts.append(np.zeros(fo, dtype=np.float32))
    return np.concatenate([p.ravel() for p in parts])


class LearnedPreconditioner:
    """The trained network applied to one mesh: device neighbour indices and
    blocks (in the system's units), set on the context with .install()."""

    def __init__(self, net, P1, P2, P3, G=1.0):
        import torch
        X, nbr, h = features(P1, P2, P3)
        out = net.predict(X)
        scale = torch.tensor((h / G).astype(np.float32), device=net.dev)[:, None]
        self.blocks = (out * scale).contiguous()
        self.nbr = torch.tensor(nbr, device=net.dev)
        self.N = len(nbr)
        self.ctx = net.ctx

    def install(self):
        _lib.check(_lib.load().cad_set_preconditioner(self.ctx, self.N, K, ctypes.c_void_p(self.nbr.data_ptr()),
                                                      ctypes.c_void_p(self.blocks.data_ptr())), self.ctx)
        return self


def solve_preconditioned(A, b, precond=None, block_jacobi=False, device=0, tol=1e-10, max_iter=2000):
    """A x = b by FP64 GMRES right-preconditioned by `precond` (a
    LearnedPreconditioner), by block Jacobi, or by nothing (identity blocks);
    host arrays.  Returns (x, iterations)."""
    import torch
    dev = torch.device("cuda", device)
    n3 = A.shape[0]
    N = n3 // 3
    ctx = _lib.context(device)
    L = _lib.load()
    Ad = torch.tensor(np.asfortranarray(A).ravel(order="F"), device=dev)
    xd = torch.tensor(np.asarray(b, dtype=np.float64), device=dev)
    keep = None
    if precond is not None:
        precond.install()
    else:
        nbr = torch.arange(N, dtype=torch.int32, device=dev)
        if block_jacobi:
            blocks = torch.empty((N, 9), dtype=torch.float32, device=dev)
            _lib.check(L.cad_block_jacobi_dev(ctx, N, Ad.data_ptr(), n3, nbr.data_ptr(), blocks.data_ptr()), ctx)
        else:
            blocks = torch.tensor(np.tile(np.eye(3, dtype=np.float32).ravel(), (N, 1)), device=dev)
        keep = (nbr, blocks)
        _lib.check(L.cad_set_preconditioner(ctx, N, 1, nbr.data_ptr(), blocks.data_ptr()), ctx)
    with _lib.solver_mode(ctx, "gmres_spai", tol, max_iter):
        rc = L.cad_solve_dev(ctx, n3, Ad.data_ptr(), n3, xd.data_ptr(), n3, 1)
        it, rr = _lib.last_solve_stats(ctx)
    L.cad_set_preconditioner(ctx, 0, 0, None, None)
    del keep
    _lib.check(rc, ctx)
    return xd.cpu().numpy(), it
