"""GPU tests of the learned preconditioner (an addition to the reference):
the library's BF16 training kernels against the CPU reference of the same
network (oracle/mlp_ref.py: float64 with BF16 rounding at the kernels'
rounding points); the device features, neighbour lists and training targets
against their CPU reference (oracle/lpc_ref.py); and the trained
preconditioner against block Jacobi and no preconditioning on held-out meshes
(GMRES iterations to relative residual 1e-10, solution against the FP64 LU).
The product path (cutanddisplacejulia_b200.precond) passes host arrays to the
C ABI only."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRAD_TOL = 5e-3      # norm-wise relative, per parameter tensor


def test_gradients_match_cpu_reference(cad):
    from cutanddisplacejulia_b200 import precond
    from oracle import mlp_ref
    rng = np.random.default_rng(3)
    params = precond.init_params(seed=5)
    params[-(256 * 144 + 144):] *= 0.3
    X = rng.standard_normal((96, precond.N_IN)).astype(np.float32)
    T = rng.standard_normal((96, precond.N_OUT)).astype(np.float32)
    net = precond.Network(params=params)
    loss, g = net.gradients(X, T)
    loss_o, g_o = mlp_ref.forward_backward(params, X.astype(np.float64), T.astype(np.float64))
    assert abs(loss - loss_o) <= 1e-3 * loss_o
    o = 0
    for shape in [(112, 256), (256,), (256, 256), (256,), (256, 144), (144,)]:
        n = int(np.prod(shape))
        a, b = g[o:o + n], g_o[o:o + n]
        assert np.linalg.norm(a - b) <= GRAD_TOL * np.linalg.norm(b), shape
        o += n


def test_training_reduces_loss(cad):
    from cutanddisplacejulia_b200 import precond
    rng = np.random.default_rng(0)
    X = rng.standard_normal((2048, precond.N_IN)).astype(np.float32)
    W = rng.standard_normal((precond.N_IN, precond.N_OUT)).astype(np.float32) / 10
    T = np.tanh(X @ W).astype(np.float32)
    net = precond.Network(seed=1)
    hist = net.train(X, T, steps=600, batch=512, lr=2e-3)
    assert hist[-1] < 0.2 * hist[0]


def test_learned_preconditioner_beats_block_jacobi(cad):
    from cutanddisplacejulia_b200 import precond, workloads
    meshes = precond.training_meshes(seed=0, count=16, n_range=(250, 600))
    ts = precond.training_set(meshes)
    assert ts.rows == sum(len(P[0]) for P, _ in meshes)
    net = precond.Network(seed=0)
    net.train(ts, steps=1500, batch=4096, lr=1e-3)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    for (P1, P2, P3), hs in ((workloads.ellipse_crack(seed=101, a=1.3, b=0.8, ntri=700), 0),
                             (workloads.dipping_rect(seed=102, ntri=700, dip=45.0, top_depth=1.0), 1)):
        n = len(P1)
        nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
        bc = cad.Stresses(*workloads.remote_stress(seed=7))
        Dn, Dss, Dds, A, b = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, hs, bc, np.zeros(n))
        D = np.concatenate([Dn, Dss, Dds])
        _, it_none = precond.solve_preconditioned(A, b)
        _, it_bj = precond.solve_preconditioned(A, b, block_jacobi=True)
        M = precond.LearnedPreconditioner(net, P1, P2, P3, G)
        x, it_lp = precond.solve_preconditioned(A, b, precond=M)
        assert np.linalg.norm(A @ x - b) <= 2e-10 * np.linalg.norm(b)
        assert np.linalg.norm(x - D) <= 1e-8 * np.linalg.norm(D)
        print("GMRES iterations: learned %d, block Jacobi %d, none %d" % (it_lp, it_bj, it_none))
        assert it_lp < it_bj <= it_none + 2, (it_lp, it_bj, it_none)


def test_device_features_match_cpu_reference(cad):
    from cutanddisplacejulia_b200 import _lib, workloads
    from oracle import lpc_ref
    L = _lib.load()
    ctx = _lib.context(0)
    for P, n in ((workloads.dipping_rect(seed=11, ntri=900, dip=50.0, top_depth=1.0), 900),
                 (workloads.ellipse_crack(seed=12, a=1.2, b=0.7, ntri=400), 400),
                 (workloads.ellipse_crack(seed=13, a=1.0, b=1.0, ntri=12), 12)):
        P1, P2, P3 = P
        N = len(P1)
        X0, nbr0, h0 = lpc_ref.features(P1, P2, P3)
        cols = [np.ascontiguousarray(np.asfortranarray(p).ravel(order="F")) for p in (P1, P2, P3)]
        X = np.empty((N, lpc_ref.N_IN), dtype=np.float32)
        nbr = np.empty((N, lpc_ref.K), dtype=np.int32)
        h = np.empty(N)
        _gpu_features(L, ctx, cols, N, X, nbr, h)
        assert np.allclose(h, h0, rtol=1e-14, atol=0)
        # the same neighbour distances, itself first; neighbours at equal
        # distances (symmetric meshes) may come in either order
        cen = (P1 + P2 + P3) / 3.0
        dist = lambda nb: np.linalg.norm(cen[nb] - cen[:, None, :], axis=2)
        assert np.array_equal(nbr[:, 0], np.arange(N))
        assert np.allclose(dist(nbr), dist(nbr0), rtol=1e-12, atol=1e-14)
        same = np.all(nbr == nbr0, axis=1)
        if N >= 400:   # jittered meshes: ties are rare
            assert same.mean() >= 0.99
        assert np.max(np.abs(X[same] - X0[same])) <= 1e-5 * max(1.0, np.max(np.abs(X0)))


def _gpu_features(L, ctx, cols, N, X, nbr, h):
    """cad_lpc_features_dev on device copies of the vertex lists (torch
    tensors as test plumbing)."""
    import torch
    dev = torch.device("cuda", 0)
    dP = [torch.tensor(c, device=dev) for c in cols]
    dX = torch.empty(X.shape, dtype=torch.float32, device=dev)
    dn = torch.empty(nbr.shape, dtype=torch.int32, device=dev)
    dh = torch.empty(N, dtype=torch.float64, device=dev)
    _lib_check(L, ctx, L.cad_lpc_features_dev(ctx, *[p.data_ptr() for p in dP], N, dX.data_ptr(), dn.data_ptr(),
                                              dh.data_ptr()))
    torch.cuda.synchronize()
    X[:] = dX.cpu().numpy()
    nbr[:] = dn.cpu().numpy()
    h[:] = dh.cpu().numpy()


def _lib_check(L, ctx, rc):
    from cutanddisplacejulia_b200 import _lib
    _lib.check(rc, ctx)


def test_training_targets_match_exact_inverse(cad):
    from cutanddisplacejulia_b200 import _lib, precond, workloads
    from oracle import lpc_ref
    L = _lib.load()
    ctx = _lib.context(0)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    (P1, P2, P3) = workloads.dipping_rect(seed=21, ntri=300, dip=70.0, top_depth=0.8)
    n = len(P1)
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    A = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 1,
                             cad.Tractions(np.ones(n), np.zeros(n), np.zeros(n)), np.zeros(n))[3]
    X0, nbr0, h0 = lpc_ref.features(P1, P2, P3)
    T0 = lpc_ref.inverse_blocks(np.linalg.inv(A), nbr0, h0, G)
    ts = precond.TrainingSet()
    ts.add(P1, P2, P3, 1)
    assert ts.rows == n
    X = np.empty((n, lpc_ref.N_IN), dtype=np.float32)
    T = np.empty((n, lpc_ref.N_OUT), dtype=np.float32)
    _lib.check(L.cad_lpc_dataset_get(ctx, 0, n, X.ctypes.data, T.ctypes.data), ctx)
    assert np.max(np.abs(X - X0)) <= 1e-5 * np.max(np.abs(X0))
    assert np.max(np.abs(T - T0)) <= 1e-5 * np.max(np.abs(T0))
