"""GPU tests of the learned preconditioner (an addition to the reference):
the library's BF16 training kernels against the CPU reference of the same
network (oracle/mlp_ref.py: float64 with BF16 rounding at the kernels'
rounding points), and the trained preconditioner against block Jacobi and
no preconditioning on held-out meshes (GMRES iterations to relative residual
1e-10, solution against the FP64 LU)."""
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
    X, T = precond.training_set(meshes)
    net = precond.Network(seed=0)
    net.train(X, T, steps=1500, batch=4096, lr=1e-3)
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
