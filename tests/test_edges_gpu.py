"""GPU tests of the shared-edge half-space assembly (cad_set_shared_edges):
the free-surface correction of each mesh edge is evaluated once per point and
reused, with the sign of the side's direction, by the triangles that share
the edge.  The matrix must agree with the per-side assembly (the reference's
order of work, src/TDstressHS.jl) and with the oracle's sampled columns to the
parity tolerance, on meshes that reach the free surface, with triangles whose
orientation disagrees with their neighbours' (shared sides running the same
way) and after the geometry changes (the cached edge table is rebuilt)."""
import numpy as np
import pytest

from helpers import assert_parity, oracle_system_columns, rel_inf_err

pytestmark = pytest.mark.gpu


def _assemble(cad, P1, P2, P3, shared):
    import torch

    from cutanddisplacejulia_b200 import _lib
    dev = torch.device("cuda", 0)
    L, ctx = _lib.load(), _lib.context(0)
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    col = (lambda a: torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device=dev))
    g = [col(a) for a in (nrm, mid, P1, P2, P3)]
    n = len(P1)
    A = torch.full((9 * n * n,), float("nan"), dtype=torch.float64, device=dev)
    _lib.check(L.cad_set_shared_edges(ctx, int(shared)), ctx)
    try:
        _lib.check(L.cad_assemble_dev(ctx, *[x.data_ptr() for x in g], n, nu, G, lam, 1, A.data_ptr(), 3 * n), ctx)
        torch.cuda.synchronize()
    finally:
        _lib.check(L.cad_set_shared_edges(ctx, 1), ctx)
    return A.view(3 * n, 3 * n).t().cpu().numpy(), (nrm, mid, nu, G, lam)


@pytest.mark.parametrize("top_depth", [0.0, 0.05, 1.0])
def test_shared_edges_match_per_side_and_oracle(cad, oracle, top_depth):
    from cutanddisplacejulia_b200 import workloads
    P1, P2, P3 = workloads.dipping_rect(seed=11, ntri=900, top_depth=top_depth)
    # highest vertex at z = -top_depth exactly (top_depth 0: an edge row on
    # the free surface, its z values -0.0)
    zmax = max(P[:, 2].max() for P in (P1, P2, P3))
    P1, P2, P3 = (P - [0.0, 0.0, zmax + top_depth] for P in (P1, P2, P3))
    A_e, (nrm, mid, nu, G, lam) = _assemble(cad, P1, P2, P3, True)
    A_s, _ = _assemble(cad, P1, P2, P3, False)
    assert np.isfinite(A_e).all()
    assert_parity(A_e[None], A_s[None])
    assert rel_inf_err(A_e, A_s) < 1e-13
    pick = np.sort(np.random.default_rng(3).choice(len(P1), 6, replace=False))
    ref = oracle_system_columns(oracle, pick, P1, P2, P3, nrm, mid, nu, G, lam, 1)
    n = len(P1)
    got = A_e[:, np.concatenate([m * n + pick for m in range(3)])]
    assert_parity(got[None], ref[None])


def test_shared_edges_mixed_orientation_and_geometry_change(cad):
    from cutanddisplacejulia_b200 import workloads
    P1, P2, P3 = workloads.dipping_rect(seed=12, ntri=600, top_depth=0.2)
    flip = np.random.default_rng(5).random(len(P1)) < 0.3
    P2f, P3f = np.where(flip[:, None], P3, P2), np.where(flip[:, None], P2, P3)
    A_e, _ = _assemble(cad, P1, P2f, P3f, True)
    A_s, _ = _assemble(cad, P1, P2f, P3f, False)
    assert_parity(A_e[None], A_s[None])
    # the same context, new vertices: the edge table must follow them
    P1m = P1.copy()
    P1m[::7] += np.array([0.003, -0.002, -0.001])
    A_e2, _ = _assemble(cad, P1m, P2f, P3f, True)
    A_s2, _ = _assemble(cad, P1m, P2f, P3f, False)
    assert_parity(A_e2[None], A_s2[None])
    assert not np.array_equal(A_e2, A_e)


def test_shared_edges_argument_check(cad):
    from cutanddisplacejulia_b200 import _lib
    L, ctx = _lib.load(), _lib.context(0)
    assert L.cad_set_shared_edges(ctx, 2) == _lib.CAD_ERR_ARG
    assert L.cad_set_shared_edges(ctx, -1) == _lib.CAD_ERR_ARG
    _lib.check(L.cad_set_shared_edges(ctx, 1), ctx)
