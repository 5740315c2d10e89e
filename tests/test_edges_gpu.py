"""GPU tests of the shared-edge half-space paths (cad_set_shared_edges).

System matrix: the free-surface correction of each mesh edge is evaluated
once per point and reused, with the sign of the side's direction, by the
triangles that share the edge.  Sums (TD with Strains/Disps): each edge's
correction is evaluated once for the net Burgers vector of the sides on it.
Both must agree with the per-side evaluation (the reference's order of work,
src/TD.jl:1831-1866 and 1222-1262) and with the oracle to the parity
tolerance, on meshes that reach the free surface, with triangles whose
orientation disagrees with their neighbours' (shared sides running the same
way) and after the geometry changes (the cached edge table is rebuilt).
Unconnected triangles (no shared edges) stay on the per-side kernels."""
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


def _td_sum(cad, pts, P1, P2, P3, sl, shared, disp=1, strain=1):
    from cutanddisplacejulia_b200 import _lib
    L, ctx = _lib.load(), _lib.context(0)
    _lib.check(L.cad_set_shared_edges(ctx, int(shared)), ctx)
    try:
        S, U = cad.TD(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, disp, strain, 1, cad.Strains(), cad.Disps())
    finally:
        _lib.check(L.cad_set_shared_edges(ctx, 1), ctx)
    return np.stack(list(S)), np.stack(list(U))


def _sum_case(seed, top_depth, ntri=300, m=500, flip_frac=0.0):
    from cutanddisplacejulia_b200 import workloads
    P1, P2, P3 = workloads.dipping_rect(seed=seed, ntri=ntri, top_depth=top_depth)
    zmax = max(P[:, 2].max() for P in (P1, P2, P3))
    P1, P2, P3 = (P - [0.0, 0.0, zmax + top_depth] for P in (P1, P2, P3))
    rng = np.random.default_rng(seed)
    if flip_frac:
        flip = rng.random(len(P1)) < flip_frac
        P2, P3 = np.where(flip[:, None], P3, P2), np.where(flip[:, None], P2, P3)
    n = len(P1)
    mid = (P1 + P2 + P3) / 3.0
    # smooth slip plus noise: interior edges carry small net Burgers vectors
    sl = np.stack([1e-3 * np.cos(mid[:, 0] + k) * np.sin(2 * mid[:, 2] - k) for k in range(3)])
    sl += rng.uniform(-1e-4, 1e-4, (3, n))
    pts = np.column_stack([rng.uniform(-2.0, 2.0, m), rng.uniform(-1.5, 1.5, m), rng.uniform(-3.0, -0.02, m)])
    return pts, (P1, P2, P3), sl


@pytest.mark.parametrize("top_depth", [0.0, 0.3])
def test_shared_edges_td_sum_matches_per_side_and_oracle(cad, oracle, top_depth):
    pts, P, sl = _sum_case(21, top_depth)
    S_e, U_e = _td_sum(cad, pts, *P, sl, True)
    S_s, U_s = _td_sum(cad, pts, *P, sl, False)
    assert_parity(S_e, S_s)
    assert_parity(U_e, U_s)
    So, Uo = oracle.td_sum_eval(*pts.T, *P, *sl, 0.25, 1.0, 1, 1, 1)
    assert_parity(S_e, So)
    assert_parity(U_e, Uo)


def test_shared_edges_td_sum_flags_and_mixed_orientation(cad, oracle):
    pts, P, sl = _sum_case(22, 0.1, ntri=240, m=300, flip_frac=0.3)
    So, Uo = oracle.td_sum_eval(*pts.T, *P, *sl, 0.25, 1.0, 1, 1, 1)
    S, U = _td_sum(cad, pts, *P, sl, True, disp=0, strain=1)
    assert_parity(S, So)
    assert not U.any()
    S, U = _td_sum(cad, pts, *P, sl, True, disp=1, strain=0)
    assert_parity(U, Uo)
    assert not S.any()


def test_unconnected_triangles_stay_per_side(cad):
    from helpers import random_points, random_triangles
    rng = np.random.default_rng(23)
    P1, P2, P3 = random_triangles(rng, 30)
    pts = random_points(rng, 200)
    sl = rng.uniform(-1e-3, 1e-3, (3, 30))
    S_e, U_e = _td_sum(cad, pts, P1, P2, P3, sl, True)
    S_s, U_s = _td_sum(cad, pts, P1, P2, P3, sl, False)
    assert np.array_equal(S_e, S_s) and np.array_equal(U_e, U_s)


def test_shared_edges_traction_fields_match_per_side(cad):
    from cutanddisplacejulia_b200 import _lib, workloads
    P1, P2, P3 = workloads.dipping_rect(seed=13, ntri=500, top_depth=0.1)
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    n = len(P1)
    L, ctx = _lib.load(), _lib.context(0)
    out = []
    for shared in (1, 0):
        _lib.check(L.cad_set_shared_edges(ctx, shared), ctx)
        try:
            T = cad.CalculateInfluenceMatrices3D(nrm, mid, P1, P2, P3, nu, G, lam, np.zeros(n), 1, n)
        finally:
            _lib.check(L.cad_set_shared_edges(ctx, 1), ctx)
        out.append(np.stack(list(T)))
    assert_parity(out[0], out[1])
    assert rel_inf_err(out[0], out[1]) < 1e-13


def _td_inf(cad, pts, P1, P2, P3, sl, shared, disp=1, strain=1):
    from cutanddisplacejulia_b200 import _lib
    L, ctx = _lib.load(), _lib.context(0)
    _lib.check(L.cad_set_shared_edges(ctx, int(shared)), ctx)
    try:
        S, U = cad.TD(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, disp, strain, 1)
    finally:
        _lib.check(L.cad_set_shared_edges(ctx, 1), ctx)
    return (np.stack(list(S)) if strain else None), (np.stack(list(U)) if disp else None)


@pytest.mark.parametrize("top_depth", [0.0, 0.2])
def test_shared_edges_influence_fields_match_per_side_and_oracle(cad, oracle, top_depth):
    pts, P, sl = _sum_case(24, top_depth, ntri=260, m=240, flip_frac=0.2)
    S_e, U_e = _td_inf(cad, pts, *P, sl, True)
    S_s, U_s = _td_inf(cad, pts, *P, sl, False)
    assert_parity(S_e, S_s)
    assert_parity(U_e, U_s)
    So, Uo = oracle.td_inf(*pts.T, *P, *sl, 0.25, 1.0, 1, 1, 1)
    assert_parity(S_e, So)
    assert_parity(U_e, Uo)
    # one output at a time
    S1, _ = _td_inf(cad, pts, *P, sl, True, disp=0, strain=1)
    _, U1 = _td_inf(cad, pts, *P, sl, True, disp=1, strain=0)
    assert_parity(S1, So)
    assert_parity(U1, Uo)
