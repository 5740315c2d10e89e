"""The autotuner: with a cache file it times the candidate launch shapes the
first time a (kernel, size class, precision) key is met, stores the winner,
and a later context reads the file instead of timing again.  Tuned shapes
change no result: the system matrix is bit for bit the untuned one, and the
solves agree with the untuned FP64 LU to rounding."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(L, ctx, torch, dev, n_tri, hs):
    from cutanddisplacejulia_b200 import _lib, geometry, workloads
    P1, P2, P3 = workloads.dipping_rect(seed=8, ntri=n_tri, top_depth=1.0)
    nrm, mid = geometry.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, nu, G = geometry.ElasticConstantsCheck(1.0, 0.25)
    col = (lambda a: torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device=dev))
    g = [col(a) for a in (nrm, mid, P1, P2, P3)]
    n = len(P1)
    A = torch.empty(9 * n * n, dtype=torch.float64, device=dev)
    _lib.check(L.cad_assemble_dev(ctx, *[x.data_ptr() for x in g], n, nu, G, lam, hs, A.data_ptr(), 3 * n), ctx)
    torch.cuda.synchronize()
    return A, n


def test_autotune_cache_round_trip(cad, tmp_path):
    import ctypes

    import torch

    from cutanddisplacejulia_b200 import _lib
    dev = torch.device("cuda", 0)
    L = _lib.load()
    ctx = _lib.context(0)
    cache = str(tmp_path / "tune.txt")
    A0, n = _system(L, ctx, torch, dev, 600, 1)            # untuned (shared-edge half-space path)
    b = torch.linspace(-1e-3, 1e-3, 3 * n, dtype=torch.float64, device=dev)
    F = A0.clone()
    x0 = b.clone()
    _lib.check(L.cad_solve_dev(ctx, 3 * n, F.data_ptr(), 3 * n, x0.data_ptr(), 3 * n, 1), ctx)
    try:
        _lib.check(L.cad_set_autotune(ctx, 1, cache.encode()), ctx)
        A1, _ = _system(L, ctx, torch, dev, 600, 1)        # times the pair-kernel shapes
        assert torch.equal(A0, A1)
        F = A1.clone()
        x1 = b.clone()
        _lib.check(L.cad_solve_dev(ctx, 3 * n, F.data_ptr(), 3 * n, x1.data_ptr(), 3 * n, 1), ctx)   # the leaf
        torch.cuda.synchronize()
        assert float(torch.linalg.vector_norm(x1 - x0) / torch.linalg.vector_norm(x0)) <= 1e-12
        tuned = ctypes.c_int64(0)
        entries = L.cad_autotune_entries(ctx, ctypes.byref(tuned))
        assert entries >= 2 and tuned.value >= 2
        text = open(cache).read()
        assert "pair_amat_f64_hs1_edge_N1024" in text and "pair_amat_f64_hs1_edge_minblocks_N1024" in text
        assert "lu_leaf_f64_n2048" in text
        # a fresh load of the file in cached-only mode: nothing is timed again
        _lib.check(L.cad_set_autotune(ctx, 2, cache.encode()), ctx)
        before = ctypes.c_int64(0)
        L.cad_autotune_entries(ctx, ctypes.byref(before))
        A2, _ = _system(L, ctx, torch, dev, 600, 1)
        assert torch.equal(A0, A2)
        after = ctypes.c_int64(0)
        assert L.cad_autotune_entries(ctx, ctypes.byref(after)) == entries
        assert after.value == before.value
    finally:
        _lib.check(L.cad_set_autotune(ctx, 0, None), ctx)
    assert os.path.exists(cache)


def test_autotune_arguments(cad):
    from cutanddisplacejulia_b200 import _lib
    L = _lib.load()
    ctx = _lib.context(0)
    assert L.cad_set_autotune(ctx, 3, None) == _lib.CAD_ERR_ARG
