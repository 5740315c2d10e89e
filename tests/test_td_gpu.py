"""GPU parity of the TD kernels against the CPU oracle, through the C ABI.

Tolerance (helpers.assert_parity): max|gpu - oracle| / max|oracle| <= 1e-12
over each output tensor (all 18 strain, 9 displacement or 9 traction fields
together), and <= 1e-11 per field (scaled by the larger of the field's own
maximum and 1e-3 of the tensor maximum); NaN masks (observation points on a
triangle side, in the triangle plane) must be identical.
"""
import numpy as np
import pytest

from helpers import assert_parity, load_mesh, okada_case, random_points, random_triangles

pytestmark = pytest.mark.gpu


def _inf(cad, pts, P1, P2, P3, sl, hs, disp=1, strain=1):
    S, U = cad.TD(pts[:, 0], pts[:, 1], pts[:, 2], P1, P2, P3, sl[0], sl[1], sl[2], 0.25, 1.0, disp, strain, hs)
    return (np.stack(list(S)) if strain else None), (np.stack(list(U)) if disp else None)


@pytest.mark.parametrize("hs", [0, 1])
def test_td_inf_parity_random(cad, oracle, hs):
    rng = np.random.default_rng(10 + hs)
    P1, P2, P3 = random_triangles(rng, 24)
    pts = random_points(rng, 300)
    sl = rng.uniform(-1e-3, 1e-3, (3, 24))
    S, U = _inf(cad, pts, P1, P2, P3, sl, hs)
    So, Uo = oracle.td_inf(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, hs)
    assert_parity(S, So)
    assert_parity(U, Uo)


def test_td_inf_on_edge_points_are_nan(cad, oracle):
    # points exactly on the sides of flat triangles in their own plane
    P1 = np.array([[0.0, 0.0, -1.0], [2.0, 0.0, -2.0]])
    P2 = np.array([[1.0, 0.0, -1.0], [3.0, 0.0, -2.0]])
    P3 = np.array([[0.0, 1.0, -1.0], [2.0, 1.0, -2.0]])
    pts = np.array([[0.5, 0.0, -1.0], [0.0, 0.5, -1.0], [0.5, 0.5, -1.0], [0.25, 0.25, -1.0], [2.5, 0.0, -2.0],
                    [0.3, 0.1, -1.5], [1.0, 1.0, -1.0]])
    sl = np.ones((3, 2))
    for hs in (0, 1):
        S, U = _inf(cad, pts, P1, P2, P3, sl, hs)
        So, Uo = oracle.td_inf(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, hs)
        assert np.isnan(So).any()
        assert_parity(S, So)
        assert_parity(U, Uo)


def test_td_inf_flat_surface_triangle_matches_reference_semantics(cad, oracle):
    # half-space triangle lying on z = 0 (the reference's flat-image branch)
    P1 = np.array([[0.0, 0.0, 0.0]])
    P2 = np.array([[1.0, 0.2, 0.0]])
    P3 = np.array([[0.3, 1.1, 0.0]])
    rng = np.random.default_rng(5)
    pts = random_points(rng, 64, lo=(-2, -2, -2), hi=(2, 2, -0.1))
    sl = np.array([[0.3], [-0.7], [0.5]])
    S, U = _inf(cad, pts, P1, P2, P3, sl, 1)
    So, Uo = oracle.td_inf(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, 1)
    assert_parity(S, So)
    assert_parity(U, Uo)


def test_td_inf_zero_slip_modes_skip(cad, oracle):
    rng = np.random.default_rng(7)
    P1, P2, P3 = random_triangles(rng, 5)
    pts = random_points(rng, 40)
    sl = np.zeros((3, 5))
    sl[1] = rng.uniform(-1, 1, 5)
    for hs in (0, 1):
        S, U = _inf(cad, pts, P1, P2, P3, sl, hs)
        So, Uo = oracle.td_inf(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, hs)
        assert_parity(S, So)
        assert_parity(U, Uo)


@pytest.mark.parametrize("hs", [0, 1])
def test_td_summing_parity(cad, oracle, hs):
    rng = np.random.default_rng(20 + hs)
    P1, P2, P3 = random_triangles(rng, 37)
    pts = random_points(rng, 515)
    sl = rng.uniform(-1e-3, 1e-3, (3, 37))
    S, U = cad.TD(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, hs, cad.Strains(), cad.Disps())
    So, Uo = oracle.td_sum_eval(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, hs)
    assert_parity(np.stack(list(S)), So)
    assert_parity(np.stack(list(U)), Uo)


def test_td_sum_reduces_influence_matrices(cad, oracle):
    rng = np.random.default_rng(30)
    P1, P2, P3 = random_triangles(rng, 11)
    pts = random_points(rng, 90)
    sl = rng.uniform(-1, 1, (3, 11))
    S, U = cad.TD(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, 0)
    out = cad.TD_sum(*list(S), *list(U))
    So, Uo = oracle.td_sum(oracle.td_inf(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, 0)[0],
                           oracle.td_inf(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, 0)[1])
    assert_parity(np.stack([o.ravel() for o in out[:6]]), So)
    assert_parity(np.stack([o.ravel() for o in out[6:]]), Uo)


def test_okada_kat_on_gpu(cad):
    from oracle import okada85
    c = okada_case()
    S, U = cad.TD(c["x"], c["y"], c["z"], c["P1"], c["P2"], c["P3"], [c["Dss"]] * 2, [c["Dds"]] * 2,
                  [c["Dn"]] * 2, 0.25, 1.0, 1, 1, 1, cad.Strains(), cad.Disps())
    total = np.sqrt(c["Dds"] ** 2 + c["Dss"] ** 2)
    rake = 90 - np.rad2deg(np.arctan(c["Dss"] / c["Dds"]))
    mid_depth = np.sin(np.deg2rad(c["Dip"])) * c["Width"] / 2 + c["TipDepth"]
    ok = okada85.okada85(c["x"], c["y"], mid_depth, c["Strike"], c["Dip"], c["Length"], c["Width"], rake, total,
                         c["Dn"], 0.25)
    for a, b in zip(list(U) + list(S), ok):
        assert np.max(np.abs(a - b)) <= 1e-13


def test_hs_above_surface_error(cad):
    P1 = np.array([[0.0, 0.0, -1.0]])
    P2 = np.array([[1.0, 0.0, -1.0]])
    P3 = np.array([[0.0, 1.0, 0.5]])
    with pytest.raises(cad.CadError, match="Half-space solution: Z coordinates must be negative!"):
        cad.TD([0.0], [0.0], [-1.0], P1, P2, P3, [1.0], [1.0], [1.0], 0.25, 1.0, 1, 1, 1)


def test_empty_inputs(cad):
    P = np.zeros((0, 3))
    S, U = cad.TD(np.zeros(0), np.zeros(0), np.zeros(0), P, P, P, [], [], [], 0.25, 1.0, 1, 1, 0)
    assert S.exxDn.shape == (0, 0)
    S, U = cad.TD([0.0, 1.0], [0.0, 1.0], [-1.0, -1.0], P, P, P, [], [], [], 0.25, 1.0, 1, 1, 0, cad.Strains(),
                  cad.Disps())
    assert np.all(S.exx == 0) and np.all(U.Ux == 0)


@pytest.mark.parametrize("hs", [0, 1])
def test_influence_traction_parity(cad, oracle, hs):
    P1, P2, P3 = load_mesh("circle581")
    if hs:
        P1, P2, P3 = (p - np.array([0, 0, 1.5]) for p in (P1, P2, P3))
    from oracle import geometry as g
    nrm, mid = g.face_normal_and_midpoint(P1, P2, P3)
    _, _, lam, nu, G = g.elastic_constants(1.0, 0.25)
    T = cad.CalculateInfluenceMatrices3D(nrm, mid, P1, P2, P3, nu, G, lam, np.zeros(len(P1)), hs, len(P1))
    To = oracle.influence_traction(nrm, mid, P1, P2, P3, nu, G, lam, hs)
    assert_parity(np.stack(list(T)), To)


def test_slip_calculator_parity(cad, oracle):
    from oracle import geometry as g
    P1, P2, P3 = load_mesh("circle581")
    nrm, mid = g.face_normal_and_midpoint(P1, P2, P3)
    _, _, lam, nu, G = g.elastic_constants(1.0, 0.25)
    n = len(P1)
    bc = cad.Tractions(np.ones(n), np.zeros(n), np.zeros(n))
    Dn, Dss, Dds, A, b = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 0, bc, np.zeros(n))
    Dno, Dsso, Ddso, Ao, bo = oracle.slip_calculator(P1, P2, P3, nu, G, lam, mid, nrm, 0, np.ones(n), np.zeros(n),
                                                     np.zeros(n))
    assert_parity(A[None], Ao[None])
    assert np.array_equal(b, bo)
    D = np.concatenate([Dn, Dss, Dds])
    Do = np.concatenate([Dno, Dsso, Ddso])
    assert np.max(np.abs(D - Do)) / np.max(np.abs(Do)) <= 1e-10


def test_traction_free_kat_on_gpu(cad):
    from oracle import geometry as g
    P = list(load_mesh("squaregrid"))
    for p in P:
        p[:, 2] = 0.0
    _, _, lam, nu, G = g.elastic_constants(5000.0, 0.25)
    nrm, mid = cad.CreateFaceNormalAndMidPoint(*P)
    n = len(P[0])
    for bc_index in (4, 5, 2):
        s = [np.zeros(n) for _ in range(6)]
        s[bc_index] = np.ones(n)
        Dn, Dss, Dds, _, _ = cad.SlipCalculator3D(*P, nu, G, lam, mid, nrm, 0, cad.Stresses(*s), np.zeros(n))
        S, _ = cad.TD(mid[:, 0], mid[:, 1], mid[:, 2], *P, Dss, Dds, Dn, nu, G, 0, 1, 0, cad.Strains(), cad.Disps())
        e = np.stack(list(S))
        cons = lam * (e[0] + e[1] + e[2])
        st = [2 * G * e[0] + cons, 2 * G * e[1] + cons, 2 * G * e[2] + cons, 2 * G * e[3], 2 * G * e[4], 2 * G * e[5]]
        st = [st[k] + s[k] for k in range(6)]
        Tn, Tds, Tss = cad.CalculateNormalAndShearTractions3D(*st, nrm)
        assert max(np.abs(Tn).max(), np.abs(Tds).max(), np.abs(Tss).max()) <= 1e-8


def test_solve_matches_lapack(cad):
    rng = np.random.default_rng(40)
    A = rng.standard_normal((300, 300)) + 300 * np.eye(300)
    B = rng.standard_normal((300, 4))
    X = cad.solve(A, B)
    assert np.max(np.abs(X - np.linalg.solve(A, B))) <= 1e-12 * np.max(np.abs(X))


@pytest.mark.parametrize("n,nrhs", [(1, 1), (37, 2), (700, 3), (2111, 1)])
def test_solve_with_pivoting_matches_lapack(cad, n, nrhs):
    # general matrices (no diagonal dominance): partial pivoting is exercised
    rng = np.random.default_rng(n)
    A = rng.standard_normal((n, n))
    B = rng.standard_normal((n, nrhs))
    X = cad.solve(A, B)
    Xo = np.linalg.solve(A, B)
    cond = np.linalg.cond(A)
    assert np.max(np.abs(X - Xo)) <= 1e-14 * cond * np.max(np.abs(Xo)) + 1e-300
    assert np.linalg.norm(A @ X - B) <= 1e-12 * np.linalg.norm(A) * np.linalg.norm(X)


def test_solve_singular_raises(cad):
    A = np.eye(50)
    A[:, 7] = 0.0
    with pytest.raises(cad.CadError, match="singular"):
        cad.solve(A, np.ones(50))


@pytest.mark.parametrize("n", [700, 1149, 2111])
def test_repeated_solves_same_size(cad, n):
    # one call signature four times (first eager, then captured as a CUDA
    # graph, then replayed), with new matrix contents on every call
    rng = np.random.default_rng(7 * n)
    for rep in range(4):
        A = rng.standard_normal((n, n))
        B = rng.standard_normal((n, 2))
        X = cad.solve(A, B)
        Xo = np.linalg.solve(A, B)
        cond = np.linalg.cond(A)
        assert np.max(np.abs(X - Xo)) <= 1e-14 * cond * np.max(np.abs(Xo)), rep


def test_savage_valley_kat_on_gpu(cad, oracle):
    """test/test_TDvsSavageGravityValley.jl through the GPU: the plain solve of
    the valley surface under gravity, the summed strain at the Savage grid,
    the reference's residual bound, and agreement with the oracle's run."""
    from helpers import savage_valley_case, savage_valley_check
    c = savage_valley_case()
    Dn, Dss, Dds, _, _ = cad.SlipCalculator3D(c["P1"], c["P2"], c["P3"], c["nu"], c["G"], c["lam"], c["mid"],
                                              c["nrm"], 0, cad.Stresses(*c["sig"]), np.zeros(len(c["P1"])))
    S, _ = cad.TD(c["X"], c["Y"], c["Z"], c["P1"], c["P2"], c["P3"], Dss, Dds, Dn, c["nu"], c["G"], 1, 1, 0,
                  cad.Strains(), cad.Disps())
    means = savage_valley_check(c, np.stack(list(S)))
    Tn, Tds, Tss = oracle.normal_and_shear_tractions(*c["sig"], c["nrm"])
    Dno, Dsso, Ddso, _, _ = oracle.slip_calculator(c["P1"], c["P2"], c["P3"], c["nu"], c["G"], c["lam"], c["mid"],
                                                   c["nrm"], 0, Tn, Tss, Tds)
    So, _ = oracle.td_sum_eval(c["X"], c["Y"], c["Z"], c["P1"], c["P2"], c["P3"], Dsso, Ddso, Dno, c["nu"], c["G"],
                               1, 1, 0)
    means_o = savage_valley_check(c, So)
    assert np.allclose(means, means_o, rtol=0, atol=1e-8)


def test_results_are_reproducible(cad):
    """Run-to-run determinism: the summing evaluation (fixed-order partial
    sums, no floating-point atomics) gives the same bits on repeated calls,
    and so does the assembly + FP64 solve once its factorisation replays."""
    from cutanddisplacejulia_b200 import workloads
    rng = np.random.default_rng(21)
    P1, P2, P3 = random_triangles(rng, 40)
    pts = random_points(rng, 3000)
    sl = rng.uniform(-1, 1, (3, 40))
    runs = [cad.TD(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, 1, cad.Strains(), cad.Disps()) for _ in range(2)]
    for a, b in zip(runs[0], runs[1]):
        assert all(np.array_equal(x, y, equal_nan=True) for x, y in zip(a, b))
    P1, P2, P3 = workloads.penny(seed=0, spacing=0.1)
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    n = len(P1)
    bc = cad.Tractions(np.full(n, -1e-3), np.full(n, 2e-4), np.zeros(n))
    sols = [np.concatenate(cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 0, bc, np.zeros(n))[:3])
            for _ in range(3)]
    assert np.array_equal(sols[1], sols[2])
    assert np.linalg.norm(sols[0] - sols[1]) <= 1e-13 * np.linalg.norm(sols[1])
