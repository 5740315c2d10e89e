"""GPU tests of the mixed-precision solve (FP32 LU with TF32 tensor-core
updates preconditioning FP64 GMRES): the solution must reach the requested
FP64 relative residual and agree with the FP64 LU solution (the plain path,
src/SlipCalculator3D.jl:22) to 1e-8 relative, on general matrices and on the
influence systems of a full-space penny crack and a half-space dipping crack."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SLIP_TOL = 1e-8   # relative slip error vs the FP64 LU solution
RESID_TOL = 1e-10


def _rel(a, b):
    return np.max(np.abs(a - b)) / np.max(np.abs(b))


@pytest.mark.parametrize("n,nrhs", [(37, 1), (129, 2), (700, 3), (1500, 1)])
def test_mixed_solve_general_matrix(cad, n, nrhs):
    from cutanddisplacejulia_b200 import _lib
    rng = np.random.default_rng(1000 + n)
    A = rng.standard_normal((n, n)) + 2.0 * np.sqrt(n) * np.eye(n)
    B = rng.standard_normal((n, nrhs))
    X = cad.solve(A, B, solver="mixed", tol=RESID_TOL)
    Xo = np.linalg.solve(A, B)
    assert _rel(X, Xo) <= SLIP_TOL
    for c in range(nrhs):
        assert np.linalg.norm(A @ X[:, c] - B[:, c]) <= 2 * RESID_TOL * np.linalg.norm(B[:, c])
    it, rr = _lib.last_solve_stats(_lib.context(0))
    assert 1 <= it <= 200 and rr <= RESID_TOL


def _geom(P1, P2, P3):
    from oracle import geometry as g
    nrm, mid = g.face_normal_and_midpoint(P1, P2, P3)
    _, _, lam, nu, G = g.elastic_constants(1.0, 0.25)
    return nrm, mid, lam, nu, G


def test_mixed_slip_calculator_penny_matches_fp64(cad):
    from cutanddisplacejulia_b200 import workloads
    P1, P2, P3 = workloads.penny(seed=3, spacing=0.12)
    nrm, mid, lam, nu, G = _geom(P1, P2, P3)
    n = len(P1)
    bc = cad.Tractions(np.full(n, -1e-3), np.zeros(n), np.zeros(n))
    ref = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 0, bc, np.zeros(n))
    mix = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 0, bc, np.zeros(n), solver="mixed", tol=RESID_TOL)
    D, Dm = np.concatenate(ref[:3]), np.concatenate(mix[:3])
    assert _rel(Dm, D) <= SLIP_TOL
    A, b = mix[3], mix[4]
    assert np.linalg.norm(A @ Dm - b) <= 2 * RESID_TOL * np.linalg.norm(b)


def test_mixed_slip_calculator_halfspace_dipping_matches_fp64(cad):
    from cutanddisplacejulia_b200 import workloads
    P1, P2, P3 = workloads.dipping_rect(seed=5, ntri=400)
    nrm, mid, lam, nu, G = _geom(P1, P2, P3)
    n = len(P1)
    s = workloads.remote_stress(seed=5)
    bc = cad.Stresses(*[np.full(n, v) for v in s])
    ref = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 1, bc, np.zeros(n))
    mix = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 1, bc, np.zeros(n), solver="mixed", tol=RESID_TOL)
    D, Dm = np.concatenate(ref[:3]), np.concatenate(mix[:3])
    assert _rel(Dm, D) <= SLIP_TOL


@pytest.mark.parametrize("solver", ["mixed", "gmres_block_jacobi"])
def test_mixed_and_gmres_slip_against_lapack_on_oracle_matrix(cad, oracle, solver):
    # anchored on the oracle, not on the GPU's own FP64 path: numpy LAPACK on
    # the oracle's system matrix of a half-space crack
    from cutanddisplacejulia_b200 import workloads
    P1, P2, P3 = workloads.dipping_rect(seed=8, ntri=300)
    nrm, mid, lam, nu, G = _geom(P1, P2, P3)
    n = len(P1)
    s = workloads.remote_stress(seed=8)
    bc = cad.Stresses(*[np.full(n, v) for v in s])
    got = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 1, bc, np.zeros(n), solver=solver, tol=RESID_TOL)
    Ao = oracle.influence_traction(nrm, mid, P1, P2, P3, nu, G, lam, 1, want_A=True)
    Tn, Tds, Tss = cad.CalculateNormalAndShearTractions3D(*s, nrm)
    Do = np.linalg.solve(Ao, np.concatenate([Tn, Tss, Tds]))
    assert np.linalg.norm(np.concatenate(got[:3]) - Do) <= SLIP_TOL * np.linalg.norm(Do)


def test_mixed_solve_dev_leaves_matrix_unchanged(cad):
    torch = pytest.importorskip("torch")
    from cutanddisplacejulia_b200 import _lib
    L = _lib.load()
    ctx = _lib.context(0)
    n = 300
    rng = np.random.default_rng(7)
    A = rng.standard_normal((n, n)) + 40.0 * np.eye(n)
    b = rng.standard_normal(n)
    dev = torch.device("cuda", 0)
    Ad = torch.tensor(A.T.copy(), dtype=torch.float64, device=dev)   # row-major A^T = column-major A
    bd = torch.tensor(b, dtype=torch.float64, device=dev)
    with _lib.solver_mode(ctx, "mixed", RESID_TOL):
        _lib.check(L.cad_solve_dev(ctx, n, Ad.data_ptr(), n, bd.data_ptr(), n, 1), ctx)
    torch.cuda.synchronize()
    assert np.array_equal(Ad.cpu().numpy(), A.T)
    assert _rel(bd.cpu().numpy(), np.linalg.solve(A, b)) <= SLIP_TOL


def test_mixed_reports_not_converged(cad):
    from cutanddisplacejulia_b200 import _lib
    rng = np.random.default_rng(11)
    n = 200
    A = rng.standard_normal((n, n)) + 3.0 * np.eye(n)
    with pytest.raises(_lib.CadError) as e:
        cad.solve(A, rng.standard_normal(n), solver="mixed", tol=1e-30, max_iter=1)
    assert e.value.args and "GMRES" in str(e.value)


def test_set_solver_rejects_bad_arguments(cad):
    from cutanddisplacejulia_b200 import _lib
    L = _lib.load()
    ctx = _lib.context(0)
    assert L.cad_set_solver(ctx, 7, 1e-10, 10) == _lib.CAD_ERR_ARG
    assert L.cad_set_solver(ctx, _lib.CAD_SOLVER_MIXED, 0.0, 10) == _lib.CAD_ERR_ARG
    assert L.cad_set_solver(ctx, _lib.CAD_SOLVER_MIXED, 1e-10, 0) == _lib.CAD_ERR_ARG
    assert L.cad_set_solver(ctx, _lib.CAD_SOLVER_LU64, 1e-10, 200) == _lib.CAD_OK
    it, rr = ctypes.c_int(-1), ctypes.c_double(-1.0)
    assert L.cad_last_solve_stats(ctx, ctypes.byref(it), ctypes.byref(rr)) == _lib.CAD_OK


def test_mixed_repeated_solves_same_size(cad):
    # the FP32 factorisation of one call signature runs eagerly, then is
    # captured as a CUDA graph and replayed; new contents on every call
    rng = np.random.default_rng(77)
    n = 900
    for rep in range(4):
        A = rng.standard_normal((n, n)) + 2.0 * np.sqrt(n) * np.eye(n)
        B = rng.standard_normal((n, 1))
        X = cad.solve(A, B, solver="mixed", tol=RESID_TOL)
        assert _rel(X, np.linalg.solve(A, B)) <= SLIP_TOL, rep


def _near_pairs(P1, P2, P3, mid, nrm, factor=3.0, tile=128):
    """(i, j) pairs the mixed assembly evaluates in FP64: every point i of a
    128-element tile holding some point within factor x mean edge length of
    triangle j's centroid."""
    cen = (P1 + P2 + P3) / 3.0
    edges = (np.linalg.norm(P2 - P1, axis=1) + np.linalg.norm(P3 - P2, axis=1) + np.linalg.norm(P1 - P3, axis=1))
    r = factor * edges.sum() / (3.0 * len(P1))
    obs = mid - 1e-12 * nrm
    d2 = ((obs[:, None, :] - cen[None, :, :]) ** 2).sum(-1)
    near = d2 < r * r
    n = len(P1)
    tiles = np.zeros_like(near)
    for t0 in range(0, n, tile):
        tiles[t0:t0 + tile] = near[t0:t0 + tile].any(axis=0)[None, :]
    return tiles


@pytest.mark.parametrize("kind", ["penny", "dipping"])
def test_mixed_assembly_matrix(cad, kind):
    from cutanddisplacejulia_b200 import workloads
    from oracle import oracle
    if kind == "penny":
        P1, P2, P3 = workloads.penny(seed=3, spacing=0.12)
        hs = 0
    else:
        P1, P2, P3 = workloads.dipping_rect(seed=5, ntri=500)
        hs = 1
    nrm, mid, lam, nu, G = _geom(P1, P2, P3)
    n = len(P1)
    bc = cad.Tractions(np.full(n, -1e-3), np.zeros(n), np.zeros(n))
    Am = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, hs, bc, np.zeros(n), assembly="mixed")[3]
    Ao = oracle.influence_traction(nrm, mid, P1, P2, P3, nu, G, lam, hs, want_A=True)
    near = np.tile(_near_pairs(P1, P2, P3, mid, nrm), (3, 3))
    scale = np.max(np.abs(Ao))
    assert near.any() and (~near).any()
    # near-field pairs: FP64, as the plain path (normwise 1e-12)
    assert np.max(np.abs(Am[near] - Ao[near])) <= 1e-12 * scale
    # far-field pairs: FP32 arithmetic (normwise 1e-6 of the matrix)
    assert np.max(np.abs(Am[~near] - Ao[~near])) <= 1e-6 * scale


def test_mixed_assembly_and_solve_slip_error(cad):
    from cutanddisplacejulia_b200 import workloads
    P1, P2, P3 = workloads.dipping_rect(seed=5, ntri=800)
    nrm, mid, lam, nu, G = _geom(P1, P2, P3)
    n = len(P1)
    s = workloads.remote_stress(seed=0)
    bc = cad.Stresses(*s)
    ref = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 1, bc, np.zeros(n))
    mix = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 1, bc, np.zeros(n), solver="mixed", tol=RESID_TOL,
                               assembly="mixed")
    D, Dm = np.concatenate(ref[:3]), np.concatenate(mix[:3])
    # the system itself differs from the FP64 one by the far field's FP32
    # rounding; the slip follows it to about that level
    assert np.linalg.norm(Dm - D) / np.linalg.norm(D) <= 1e-5
    Am, b = mix[3], mix[4]
    assert np.linalg.norm(Am @ Dm - b) <= 2 * RESID_TOL * np.linalg.norm(b)


def test_mixed_many_rhs_influence_system(cad):
    # 48 remote stress states on one half-space crack: batched refinement on
    # the FP32 factors, every column to the residual tolerance
    from cutanddisplacejulia_b200 import assembly, workloads
    P1, P2, P3 = workloads.dipping_rect(seed=9, ntri=600)
    nrm, mid, lam, nu, G = _geom(P1, P2, P3)
    n = len(P1)
    bc = cad.Tractions(np.full(n, -1e-3), np.zeros(n), np.zeros(n))
    A = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 1, bc, np.zeros(n))[3]
    rng = np.random.default_rng(4)
    B = np.empty((3 * n, 48))
    for c in range(48):
        Tn, Tds, Tss = assembly.CalculateNormalAndShearTractions3D(*rng.uniform(-1e-3, 1e-3, 6), nrm)
        B[:, c] = np.concatenate([Tn, Tss, Tds])
    X = cad.solve(A, B, solver="mixed", tol=RESID_TOL)
    Xo = np.linalg.solve(A, B)
    for c in range(48):
        assert np.linalg.norm(A @ X[:, c] - B[:, c]) <= 2 * RESID_TOL * np.linalg.norm(B[:, c])
        assert np.linalg.norm(X[:, c] - Xo[:, c]) <= SLIP_TOL * np.linalg.norm(Xo[:, c])


def test_mixed_many_rhs_general_matrix(cad):
    # condition number 1e3, no structure: every column must reach the residual
    # tolerance (refinement, GMRES for any column it leaves).  The TF32
    # trailing updates make the FP32 factors accurate to ~1e-3 relative, so
    # the mixed solve is meant for condition numbers up to ~1e3-1e4 (the
    # influence systems are ~1e2); ill-conditioned systems take the FP64 LU.
    from cutanddisplacejulia_b200 import _lib
    rng = np.random.default_rng(5)
    n = 400
    Q1, _ = np.linalg.qr(rng.standard_normal((n, n)))
    Q2, _ = np.linalg.qr(rng.standard_normal((n, n)))
    A = (Q1 * np.logspace(0, -3, n)) @ Q2.T
    B = rng.standard_normal((n, 3))
    X = cad.solve(A, B, solver="mixed", tol=RESID_TOL, max_iter=400)
    for c in range(3):
        assert np.linalg.norm(A @ X[:, c] - B[:, c]) <= 2 * RESID_TOL * np.linalg.norm(B[:, c])
    it, rr = _lib.last_solve_stats(_lib.context(0))
    assert rr <= RESID_TOL and it >= 1


@pytest.mark.parametrize("solver", ["lu64", "mixed"])
def test_repeated_solves_on_cuda_default_stream(cad, solver):
    # the same call signature three times on CUDA's legacy default stream,
    # which cannot be captured: the solves run eagerly every time
    from cutanddisplacejulia_b200 import _lib
    L = _lib.load()
    ctx = _lib.context(0)
    own = L.cad_get_stream(ctx)
    rng = np.random.default_rng(77)
    n = 600
    A = rng.standard_normal((n, n)) + 2.0 * np.sqrt(n) * np.eye(n)
    B = rng.standard_normal((n, 1))
    Xo = np.linalg.solve(A, B)
    _lib.check(L.cad_set_stream(ctx, None), ctx)
    try:
        for _ in range(3):
            X = cad.solve(A, B, solver=solver, tol=RESID_TOL)
            assert _rel(X, Xo) <= SLIP_TOL
    finally:
        _lib.check(L.cad_set_stream(ctx, own), ctx)


def test_gmres_restart_setting(cad):
    from cutanddisplacejulia_b200 import _lib
    L = _lib.load()
    ctx = _lib.context(0)
    assert L.cad_set_gmres_restart(ctx, 64) == _lib.CAD_ERR_ARG
    assert L.cad_set_gmres_restart(ctx, -1) == _lib.CAD_ERR_ARG
    rng = np.random.default_rng(91)
    n = 450
    A = rng.standard_normal((n, n)) + 3.0 * np.sqrt(n) * np.eye(n)
    B = rng.standard_normal((n, 1))
    Xo = np.linalg.solve(A, B)
    try:
        for m in (5, 30, 63):
            _lib.check(L.cad_set_gmres_restart(ctx, m), ctx)
            X = cad.solve(A, B, solver="gmres_block_jacobi", tol=RESID_TOL, max_iter=2000)
            assert np.linalg.norm(A @ X[:, 0] - B[:, 0]) <= 2 * RESID_TOL * np.linalg.norm(B[:, 0])
            assert _rel(X, Xo) <= SLIP_TOL
    finally:
        _lib.check(L.cad_set_gmres_restart(ctx, 0), ctx)
