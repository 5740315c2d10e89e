"""Incremental re-assembly (cad_assemble_update_dev): after the geometry of a
few elements changes, recomputing only their rows and columns of the system
matrix must give the matrix a full re-assembly gives (FP64 parity 1e-12
normwise), and leave every other entry untouched."""
import ctypes

import numpy as np
import pytest

from helpers import assert_parity

pytestmark = pytest.mark.gpu


def _assemble(L, ctx, dev, P1, P2, P3, hs, A=None):
    import torch

    from cutanddisplacejulia_b200 import _lib, geometry
    nrm, mid = geometry.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, nu, G = geometry.ElasticConstantsCheck(1.0, 0.25)
    col = (lambda a: torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device=dev))
    g = [col(a) for a in (nrm, mid, P1, P2, P3)]
    n = len(P1)
    if A is None:
        A = torch.empty(9 * n * n, dtype=torch.float64, device=dev)
        _lib.check(L.cad_assemble_dev(ctx, *[x.data_ptr() for x in g], n, nu, G, lam, hs, A.data_ptr(), 3 * n), ctx)
    torch.cuda.synchronize()   # the library's stream is not torch's: finish before torch reads A
    return A, g, (nu, G, lam)


@pytest.mark.parametrize("hs", [0, 1])
def test_update_matches_full_reassembly(cad, hs):
    import torch

    from cutanddisplacejulia_b200 import _lib, workloads
    dev = torch.device("cuda", 0)
    L, ctx = _lib.load(), _lib.context(0)
    P1, P2, P3 = workloads.dipping_rect(seed=4, ntri=400, top_depth=1.0)
    n = len(P1)
    A_old, _, _ = _assemble(L, ctx, dev, P1, P2, P3, hs)
    A_keep = A_old.clone()
    rng = np.random.default_rng(9)
    changed = np.sort(rng.choice(n, 9, replace=False)).astype(np.int64)
    P1n = P1.copy()
    P1n[changed] += rng.uniform(-0.01, 0.01, (9, 3)) * [1, 1, 0.5]
    A_full, g, (nu, G, lam) = _assemble(L, ctx, dev, P1n, P2, P3, hs)
    _lib.check(L.cad_assemble_update_dev(ctx, *[x.data_ptr() for x in g], n, nu, G, lam, hs,
                                         changed.ctypes.data, len(changed), A_old.data_ptr(), 3 * n), ctx)
    torch.cuda.synchronize()
    Au = A_old.view(3 * n, 3 * n).t().cpu().numpy()
    Af = A_full.view(3 * n, 3 * n).t().cpu().numpy()
    Ak = A_keep.view(3 * n, 3 * n).t().cpu().numpy()
    assert_parity(Au[None], Af[None])
    idx = np.concatenate([changed, n + changed, 2 * n + changed])
    keep = np.ones(3 * n, dtype=bool)
    keep[idx] = False
    assert np.array_equal(Au[np.ix_(keep, keep)], Ak[np.ix_(keep, keep)])
    assert not np.array_equal(Au[idx], Ak[idx])


def test_update_rejects_bad_index(cad):
    import torch

    from cutanddisplacejulia_b200 import _lib, workloads
    dev = torch.device("cuda", 0)
    L, ctx = _lib.load(), _lib.context(0)
    P1, P2, P3 = workloads.dipping_rect(seed=4, ntri=50)
    n = len(P1)
    A, g, (nu, G, lam) = _assemble(L, ctx, dev, P1, P2, P3, 0)
    bad = np.array([3, n], dtype=np.int64)
    rc = L.cad_assemble_update_dev(ctx, *[x.data_ptr() for x in g], n, nu, G, lam, 0, bad.ctypes.data, 2,
                                   A.data_ptr(), 3 * n)
    assert rc == _lib.CAD_ERR_ARG
