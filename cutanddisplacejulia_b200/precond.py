"""Learned sparse-approximate-inverse preconditioner for the influence system
(an addition to the reference, whose only solver is the dense A\\b of
src/SlipCalculator3D.jl:22).

For element i, a small network (csrc/mlp.cu) reads the geometry of i's 16
nearest elements -- centroid offsets and normals in i's own (normal, strike,
dip) frame, offsets scaled by i's size, and area ratios -- and predicts the 16
3x3 blocks (A^-1)[i, j] of the inverse system matrix between i and those
neighbours, in units of h_i / G (h_i = sqrt(2 area_i)).  Those blocks form a
block-sparse right preconditioner M ~ A^-1 for FP64 GMRES
(CAD_SOLVER_GMRES_SPAI / CAD_SOLVER_GMRES_LEARNED).  Training targets are the
same blocks of exact inverses that the library computes (FP64 LU with the
identity as right-hand side) on small seeded meshes.

Everything numerical runs in libcad_td.so behind its C ABI -- neighbour
search and features (csrc/lpc.cu), the training set (kept on the device),
training, prediction and the preconditioned solve; this module passes host
numpy arrays and holds the network's weights between calls.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .geometry import CreateFaceNormalAndMidPoint, ElasticConstantsCheck

K = 16          # neighbours per element (the element itself first)
N_IN = 7 * K    # offset (3), normal (3), area ratio (1) per neighbour
N_OUT = 9 * K

_F = ctypes.POINTER(ctypes.c_float)


def _fptr(a):
    return a.ctypes.data_as(_F)


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _col(a):
    return np.ascontiguousarray(np.asfortranarray(np.asarray(a, dtype=np.float64).reshape(-1, 3)).ravel(order="F"))


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


class TrainingSet:
    """The context's training set, kept on the device: features and exact-
    inverse targets of every element of every added mesh."""

    def __init__(self, device=0, G=1.0, nu=0.25):
        self.L = _lib.load()
        self.ctx = _lib.context(device)
        _, _, self.lam, self.nu, self.G = ElasticConstantsCheck(G, nu)
        _lib.check(self.L.cad_lpc_dataset_clear(self.ctx), self.ctx)

    def add(self, P1, P2, P3, hs):
        nrm, mid = CreateFaceNormalAndMidPoint(P1, P2, P3)
        n = len(nrm)
        a = [_col(x) for x in (P1, P2, P3, mid, nrm)]
        _lib.check(self.L.cad_lpc_dataset_add(self.ctx, *[_dptr(x) for x in a[:3]], n, self.nu, self.G, self.lam,
                                              _dptr(a[3]), _dptr(a[4]), int(hs)), self.ctx)

    @property
    def rows(self):
        return int(self.L.cad_lpc_dataset_rows(self.ctx))


def training_set(meshes, G=1.0, nu=0.25, device=0):
    """The training set of `meshes` ([((P1, P2, P3), hs), ...]) on the device."""
    ts = TrainingSet(device=device, G=G, nu=nu)
    for (P1, P2, P3), hs in meshes:
        ts.add(P1, P2, P3, hs)
    return ts


class Network:
    """The preconditioner network: FP32 master weights held here (host),
    trained and evaluated by the library's kernels on the context's device."""

    def __init__(self, seed=0, device=0, params=None):
        self.ctx = _lib.context(device)
        self.L = _lib.load()
        npar = self.L.cad_lpc_param_count()
        self.params = np.ascontiguousarray(init_params(seed) if params is None else params, dtype=np.float32)
        assert self.params.size == npar

    def _load(self):
        _lib.check(self.L.cad_lpc_set_network(self.ctx, _fptr(self.params)), self.ctx)

    def gradients(self, X, T):
        """(sum of squared errors, gradient of the mean squared error) of one
        pass over X (rows x 112), T (rows x 144) -- numpy in, numpy out."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        T = np.ascontiguousarray(T, dtype=np.float32)
        self._load()
        g = np.zeros_like(self.params)
        loss = np.zeros(1, dtype=np.float32)
        _lib.check(self.L.cad_lpc_forward_backward(self.ctx, _fptr(X), _fptr(T), X.shape[0], None, _fptr(g),
                                                   _fptr(loss)), self.ctx)
        return float(loss[0]), g

    def train(self, data, T=None, steps=2000, batch=4096, lr=1e-3, seed=0):
        """Adam (cosine step size) on minibatches of a TrainingSet, or of host
        arrays (data = X rows x 112, T rows x 144); returns the mean squared
        error of every 100th minibatch."""
        if T is not None:
            X = np.ascontiguousarray(data, dtype=np.float32)
            T = np.ascontiguousarray(T, dtype=np.float32)
            _lib.check(self.L.cad_lpc_dataset_set(self.ctx, _fptr(X), _fptr(T), X.shape[0]), self.ctx)
        self._load()
        hist = np.zeros((steps + 99) // 100, dtype=np.float32)
        _lib.check(self.L.cad_lpc_train(self.ctx, steps, batch, ctypes.c_float(lr), seed, _fptr(hist)), self.ctx)
        _lib.check(self.L.cad_lpc_get_network(self.ctx, _fptr(self.params)), self.ctx)
        return [float(h) for h in hist]

    def predict(self, X):
        """Network outputs (rows x 144) for X (rows x 112), numpy in and out."""
        X = np.ascontiguousarray(X, dtype=np.float32)
        self._load()
        out = np.empty((X.shape[0], N_OUT), dtype=np.float32)
        _lib.check(self.L.cad_lpc_forward_backward(self.ctx, _fptr(X), None, X.shape[0], _fptr(out), None, None),
                   self.ctx)
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
    """The trained network applied to one mesh: .install() runs features,
    network and scaling on the device and sets the blocks as the context's
    preconditioner (CAD_SOLVER_GMRES_SPAI)."""

    def __init__(self, net, P1, P2, P3, G=1.0):
        self.net = net
        self.P = [_col(p) for p in (P1, P2, P3)]
        self.N = len(self.P[0]) // 3
        self.G = float(G)
        self.ctx = net.ctx

    def install(self):
        self.net._load()
        _lib.check(_lib.load().cad_lpc_install(self.ctx, *[_dptr(p) for p in self.P], self.N, self.G), self.ctx)
        return self


def solve_preconditioned(A, b, precond=None, block_jacobi=False, device=0, tol=1e-10, max_iter=2000):
    """A x = b by FP64 GMRES right-preconditioned by `precond` (a
    LearnedPreconditioner), by block Jacobi, or by nothing; host arrays in and
    out.  Returns (x, iterations)."""
    ctx = _lib.context(device)
    L = _lib.load()
    n3 = A.shape[0]
    Af = np.asfortranarray(np.asarray(A, dtype=np.float64))
    bb = np.ascontiguousarray(b, dtype=np.float64)
    x = np.empty(n3, dtype=np.float64)
    if precond is not None:
        precond.install()
        mode = "gmres_spai"
    else:
        mode = "gmres_block_jacobi" if block_jacobi else "gmres"
    with _lib.solver_mode(ctx, mode, tol, max_iter):
        rc = L.cad_solve(ctx, n3, Af.ctypes.data, bb.ctypes.data, 1, x.ctypes.data)
        it, _ = _lib.last_solve_stats(ctx)
    _lib.check(rc, ctx)
    return x, it
