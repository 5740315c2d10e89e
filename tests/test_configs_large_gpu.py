"""GPU parity at the benchmark configurations' own sizes, each anchored on the
oracle (the CPU restatement of the reference) or on LAPACK through it:

* C5 -- the 60000-unknown half-space crack: sampled element columns of the
  system matrix against the oracle's TD strain + traction conversion
  (src/TD.jl, src/CalculateInfluenceMatrices3D.jl:73-114), and the
  learned-preconditioner GMRES slip against the FP64 LU's (relative
  residual <= 1e-10, slip within 1e-8).
* C4b -- a seeded subset of the 512-crack batch that spans its 200-2000
  triangle range: every crack's batched slip against numpy LAPACK on the
  oracle's own matrix (src/SlipCalculator3D.jl:1-33).
* C4a -- 256 seeded remote stresses on the 30000-unknown half-space system:
  the mixed solve of all columns against the FP64 LU, worst column.
* The incremental re-assembly (fracture-propagation loop,
  test/test_PropagationTest.jl:398) against the oracle's assembly of the
  moved mesh.
"""
import numpy as np
import pytest

from helpers import assert_parity, oracle_system_columns

pytestmark = pytest.mark.gpu


def _col(torch, dev, a):
    return torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device=dev)


def test_c5_sampled_columns_and_learned_gmres(cad, oracle):
    import torch

    from cutanddisplacejulia_b200 import _lib, precond, workloads
    P1, P2, P3 = workloads.dipping_rect(seed=0, ntri=20000, length=3.0, width=1.5, dip=45.0, top_depth=2.0)
    n = len(P1)
    n3 = 3 * n
    assert 19000 < n <= 20000
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    dev = torch.device("cuda", 0)
    L = _lib.load()
    ctx = _lib.context(0)
    g = [_col(torch, dev, a) for a in (nrm, mid, P1, P2, P3)]
    A = torch.empty(n3 * n3, dtype=torch.float64, device=dev)
    _lib.check(L.cad_assemble_dev(ctx, *[x.data_ptr() for x in g], n, nu, G, lam, 1, A.data_ptr(), n3), ctx)
    torch.cuda.synchronize()
    At = A.view(n3, n3)
    sample = np.sort(np.random.default_rng(7).choice(n, 16, replace=False))
    cols = np.concatenate([sample, n + sample, 2 * n + sample])
    got = At[torch.tensor(cols, device=dev)].cpu().numpy().T
    ref = oracle_system_columns(oracle, sample, P1, P2, P3, nrm, mid, nu, G, lam, 1)
    assert_parity(got[None], ref[None])
    # learned preconditioner (trained here on seeded 500-2000-triangle meshes)
    net = precond.Network(seed=0)
    net.train(precond.training_set(precond.training_meshes(seed=0, count=12, n_range=(500, 2000))), steps=1500,
              batch=4096, lr=1e-3)
    Tn, Tds, Tss = cad.CalculateNormalAndShearTractions3D(*workloads.remote_stress(seed=0), nrm)
    b = torch.tensor(np.concatenate([Tn, Tss, Tds]), device=dev)
    F = A.clone()
    xl = b.clone()
    _lib.check(L.cad_lpc_install_dev(ctx, g[2].data_ptr(), g[3].data_ptr(), g[4].data_ptr(), n, G), ctx)
    with _lib.solver_mode(ctx, "gmres_spai", 1e-10, 3000):
        _lib.check(L.cad_solve_dev(ctx, n3, A.data_ptr(), n3, xl.data_ptr(), n3, 1), ctx)
        its, rr = _lib.last_solve_stats(ctx)
    x = b.clone()
    with _lib.solver_mode(ctx, "lu64"):
        _lib.check(L.cad_solve_dev(ctx, n3, F.data_ptr(), n3, x.data_ptr(), n3, 1), ctx)
    torch.cuda.synchronize()
    del F
    res = float(torch.linalg.vector_norm(At.t() @ xl - b) / torch.linalg.vector_norm(b))
    err = float(torch.linalg.vector_norm(xl - x) / torch.linalg.vector_norm(x))
    print("C5 learned GMRES: %d iterations, residual %.2e, slip error vs FP64 LU %.2e" % (its, res, err))
    assert res <= 1e-10
    assert err <= 1e-8


@pytest.mark.parametrize("assembly,tol", [("fp64", 1e-8), ("mixed", 1e-4)])
def test_c4b_batch_subset_against_lapack_on_oracle_matrix(cad, oracle, assembly, tol):
    from cutanddisplacejulia_b200 import workloads
    cracks, stresses = workloads.crack_batch(seed=0, count=512)
    sizes = np.array([len(c[0]) for c in cracks])
    order = np.argsort(sizes)
    # the smallest, the largest and four seeded others in between
    pick = [int(order[0]), int(order[-1])] + [int(i) for i in np.random.default_rng(2).choice(order[1:-1], 4,
                                                                                               replace=False)]
    sub = [cracks[i] for i in pick]
    assert sizes[pick].min() < 260 and sizes[pick].max() > 1700
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    bcs = [cad.Stresses(*stresses[i]) for i in pick]
    out, rel = cad.SlipCalculator3D_batched(sub, nu, G, lam, 0, bcs, tol=1e-10, assembly=assembly)
    assert np.all(rel <= 1e-10)
    for (P1, P2, P3), bc, D in zip(sub, bcs, out):
        nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
        Ao = oracle.influence_traction(nrm, mid, P1, P2, P3, nu, G, lam, 0, want_A=True)
        Tn, Tds, Tss = cad.CalculateNormalAndShearTractions3D(bc.sxx, bc.syy, bc.szz, bc.sxy, bc.sxz, bc.syz, nrm)
        Do = np.linalg.solve(Ao, np.concatenate([Tn, Tss, Tds]))
        Dg = np.concatenate(D)
        assert np.linalg.norm(Dg - Do) <= tol * np.linalg.norm(Do), len(P1)


def test_c4a_256_right_hand_sides_on_c3(cad):
    import torch

    from cutanddisplacejulia_b200 import _lib, assembly, workloads
    P1, P2, P3 = workloads.dipping_rect(seed=0, ntri=10000)
    n = len(P1)
    n3 = 3 * n
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    dev = torch.device("cuda", 0)
    L = _lib.load()
    ctx = _lib.context(0)
    g = [_col(torch, dev, a) for a in (nrm, mid, P1, P2, P3)]
    A = torch.empty(n3 * n3, dtype=torch.float64, device=dev)
    _lib.check(L.cad_assemble_dev(ctx, *[x.data_ptr() for x in g], n, nu, G, lam, 1, A.data_ptr(), n3), ctx)
    rng = np.random.default_rng(12)
    B = np.empty((256, n3))
    for c in range(256):
        Tn, Tds, Tss = assembly.CalculateNormalAndShearTractions3D(*rng.uniform(-1e-3, 1e-3, 6), nrm)
        B[c] = np.concatenate([Tn, Tss, Tds])
    Bd = torch.tensor(B, device=dev)          # row c = column c of the column-major 3N x 256 block
    Xm = Bd.clone()
    torch.cuda.synchronize()
    with _lib.solver_mode(ctx, "mixed", 1e-10, 400):
        _lib.check(L.cad_solve_dev(ctx, n3, A.data_ptr(), n3, Xm.data_ptr(), n3, 256), ctx)
    F = A.clone()
    X64 = Bd.clone()
    torch.cuda.synchronize()
    with _lib.solver_mode(ctx, "lu64"):
        _lib.check(L.cad_solve_dev(ctx, n3, F.data_ptr(), n3, X64.data_ptr(), n3, 256), ctx)
    torch.cuda.synchronize()
    del F
    At = A.view(n3, n3).t()
    res = torch.linalg.vector_norm(Xm @ At.t() - Bd, dim=1) / torch.linalg.vector_norm(Bd, dim=1)
    err = torch.linalg.vector_norm(Xm - X64, dim=1) / torch.linalg.vector_norm(X64, dim=1)
    print("C4a: worst residual %.2e, worst slip error vs FP64 LU %.2e" % (float(res.max()), float(err.max())))
    assert float(res.max()) <= 2e-10
    assert float(err.max()) <= 1e-8


@pytest.mark.parametrize("hs", [0, 1])
def test_incremental_update_against_oracle(cad, oracle, hs):
    import torch

    from cutanddisplacejulia_b200 import _lib, workloads
    dev = torch.device("cuda", 0)
    L, ctx = _lib.load(), _lib.context(0)
    P1, P2, P3 = workloads.dipping_rect(seed=4, ntri=500, top_depth=1.0)
    n = len(P1)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    g = [_col(torch, dev, a) for a in (nrm, mid, P1, P2, P3)]
    A = torch.empty(9 * n * n, dtype=torch.float64, device=dev)
    _lib.check(L.cad_assemble_dev(ctx, *[x.data_ptr() for x in g], n, nu, G, lam, hs, A.data_ptr(), 3 * n), ctx)
    # a propagation step: a few tip elements move
    rng = np.random.default_rng(19)
    changed = np.sort(rng.choice(n, 12, replace=False)).astype(np.int64)
    P3n = P3.copy()
    P3n[changed] += rng.uniform(-0.02, 0.02, (12, 3)) * [1, 1, 0.5]
    nrm2, mid2 = cad.CreateFaceNormalAndMidPoint(P1, P2, P3n)
    g2 = [_col(torch, dev, a) for a in (nrm2, mid2, P1, P2, P3n)]
    torch.cuda.synchronize()
    _lib.check(L.cad_assemble_update_dev(ctx, *[x.data_ptr() for x in g2], n, nu, G, lam, hs, changed.ctypes.data,
                                         len(changed), A.data_ptr(), 3 * n), ctx)
    torch.cuda.synchronize()
    Au = A.view(3 * n, 3 * n).t().cpu().numpy()
    Ao = oracle.influence_traction(nrm2, mid2, P1, P2, P3n, nu, G, lam, hs, want_A=True)
    assert_parity(Au[None], Ao[None])
