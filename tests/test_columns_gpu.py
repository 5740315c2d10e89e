"""GPU test of the column-block assembly (cad_assemble_columns_dev): the
system matrix sharded by element columns as dist.column_block splits it for
3 ranks (run one after another on this GPU; the blocks need no exchange)
must reproduce the columns of the full assembly (cad_assemble_dev) exactly,
in full space and half space (the full assembly with per-side free-surface
corrections, as the block computes them; within the parity tolerance of the
default shared-edge one), and seeded columns of each block must match the
oracle's restatement of the assembly."""
import numpy as np
import pytest

from helpers import assert_parity, oracle_system_columns

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("hs", [0, 1])
def test_column_blocks_equal_full_assembly(cad, oracle, hs):
    import torch

    from cutanddisplacejulia_b200 import _lib, dist, workloads
    P1, P2, P3 = workloads.dipping_rect(seed=5, ntri=700, top_depth=1.0)
    if not hs:
        P1, P2, P3 = P1 + [0, 0, 4.0], P2 + [0, 0, 4.0], P3 + [0, 0, 4.0]
    n = len(P1)
    n3 = 3 * n
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    dev = torch.device("cuda", 0)
    L = _lib.load()
    ctx = _lib.context(0)
    col = (lambda a: torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device=dev))
    g = [col(nrm), col(mid), col(P1), col(P2), col(P3)]
    A = torch.empty(n3 * n3, dtype=torch.float64, device=dev)
    _lib.check(L.cad_assemble_dev(ctx, *[x.data_ptr() for x in g], n, nu, G, lam, hs, A.data_ptr(), n3), ctx)
    torch.cuda.synchronize()
    shared = A.view(n3, n3).cpu().numpy().T   # column-major 3N x 3N
    _lib.check(L.cad_set_shared_edges(ctx, 0), ctx)
    try:
        _lib.check(L.cad_assemble_dev(ctx, *[x.data_ptr() for x in g], n, nu, G, lam, hs, A.data_ptr(), n3), ctx)
        torch.cuda.synchronize()
    finally:
        _lib.check(L.cad_set_shared_edges(ctx, 1), ctx)
    full = A.view(n3, n3).cpu().numpy().T
    assert_parity(shared[None], full[None])
    for rank in range(3):
        j0, j1 = dist.column_block(n, rank, 3)
        nb = j1 - j0
        B = torch.full((3 * nb * n3,), float("nan"), dtype=torch.float64, device=dev)
        _lib.check(L.cad_assemble_columns_dev(ctx, *[x.data_ptr() for x in g], n, nu, G, lam, hs, j0, j1,
                                              B.data_ptr(), n3), ctx)
        torch.cuda.synchronize()
        block = B.view(3 * nb, n3).cpu().numpy().T
        cols = np.concatenate([m * n + np.arange(j0, j1) for m in range(3)])
        assert np.array_equal(block, full[:, cols])
        # four seeded element columns of the block against the oracle
        pick = np.sort(np.random.default_rng(rank).choice(nb, 4, replace=False))
        ref = oracle_system_columns(oracle, j0 + pick, P1, P2, P3, nrm, mid, nu, G, lam, hs)
        got = block[:, np.concatenate([m * nb + pick for m in range(3)])]
        assert_parity(got[None], ref[None])


def test_column_block_argument_checks(cad):
    from cutanddisplacejulia_b200 import _lib
    L = _lib.load()
    ctx = _lib.context(0)
    n = 10
    z = np.zeros(3 * n)
    rc = L.cad_assemble_columns_dev(ctx, z.ctypes.data, z.ctypes.data, z.ctypes.data, z.ctypes.data, z.ctypes.data,
                                    n, 0.25, 1.0, 1.0, 0, 4, 11, None, 3 * n)
    assert rc == _lib.CAD_ERR_ARG
