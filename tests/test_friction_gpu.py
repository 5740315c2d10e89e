"""GPU tests of the frictional slip solve (src/SlipCalculator3D.jl:36-238):
C = inv(A Scl), the 5N-variable complementarity problem and its
Fischer-Burmeister Newton solve on the device, through the public API.
Against the oracle (oracle/friction.py: the same problem and method in
numpy; slip norm-wise within 1e-8), the reference's acceptance test
test/test_TDvsBurgmannLinearFrictionCrack.jl (36 % / 1400), and LCPs with
known unique solutions for the dense entry point."""
import numpy as np
import pytest

from helpers import burgmann_case, burgmann_check, random_lcp

pytestmark = pytest.mark.gpu

SLIP_TOL = 1e-8   # norm-wise, GPU slip vs oracle slip (both to max|Phi| <= 1e-10 max|q|)


def _bc(cad, c):
    return cad.MixedBoundaryConditionsFriction(
        cad.MixedBoundaryConditions(cad.Stresses(*c["sig"]), cad.Tractions(0.0, 0.0, 0.0)),
        cad.FrictionParameters(c["mu"], c["Sf"]))


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("half", [1, 2])
def test_friction_burgmann_vs_oracle_and_kat(cad, oracle, half):
    from oracle import friction as F
    c = burgmann_case(half)
    args = (c["P1"], c["P2"], c["P3"], c["nu"], c["G"], c["lam"], c["mid"], c["nrm"], 0)
    DnF, DssF, DdsF = cad.SlipCalculator3D(*args, _bc(cad, c), np.zeros(c["n"]))
    it, rel = cad._lib.last_solve_stats(cad.context(0))
    assert rel <= 1e-10 and 1 <= it <= 30
    Tn, Tds, Tss = oracle.normal_and_shear_tractions(*c["sig"], c["nrm"])
    Dno, Dsso, Ddso, info = F.slip_calculator_friction(*args, Tn, Tss, Tds, c["mu"], c["Sf"])
    # the GPU solves each Newton system in reduced form (3N unknowns), the
    # oracle in full (5N): the same directions up to rounding, so the same path
    assert abs(it - info["iterations"]) <= 1, (it, info["iterations"])
    for g, o in ((DnF, Dno), (DssF, Dsso), (DdsF, Ddso)):
        assert _rel(g, o) <= SLIP_TOL * max(1.0, np.linalg.norm(np.concatenate([Dno, Dsso, Ddso])) /
                                            max(np.linalg.norm(o), 1e-300))
    Dn, Dss, Dds, _, _ = cad.SlipCalculator3D(*args, cad.Stresses(*c["sig"]), np.zeros(c["n"]))
    if half == 1:
        burgmann_check(c, half, Dss, DssF)
    else:
        burgmann_check(c, half, Dds, DdsF)


def test_friction_with_friction_coefficient(cad, oracle):
    """mu > 0 and constant cohesion on the first crack: the slip, the contact
    set and the residual against the oracle."""
    from oracle import friction as F
    c = burgmann_case(1)
    c["mu"] = 0.6
    c["Sf"] = np.full(c["n"], 0.2 * c["S"])
    args = (c["P1"], c["P2"], c["P3"], c["nu"], c["G"], c["lam"], c["mid"], c["nrm"], 0)
    DnF, DssF, DdsF = cad.SlipCalculator3D(*args, _bc(cad, c), None)
    Tn, Tds, Tss = oracle.normal_and_shear_tractions(*c["sig"], c["nrm"])
    Dno, Dsso, Ddso, info = F.slip_calculator_friction(*args, Tn, Tss, Tds, c["mu"], c["Sf"])
    ref = np.concatenate([Dno, Dsso, Ddso])
    got = np.concatenate([DnF, DssF, DdsF])
    assert np.linalg.norm(got - ref) <= SLIP_TOL * np.linalg.norm(ref)
    assert np.abs(DssF).max() > 0   # some elements slip


def test_friction_early_exit(cad):
    c = burgmann_case(1)
    n = c["n"]
    bc = cad.MixedBoundaryConditionsFriction(
        cad.MixedBoundaryConditions(cad.Stresses(0.0, 0.0, 0.0, 0.0, 0.0, 0.0),
                                    cad.Tractions(np.full(n, -10.0), np.full(n, 0.1), np.full(n, -0.1))),
        cad.FrictionParameters(0.6, 0.0))
    Dn, Dss, Dds = cad.SlipCalculator3D(c["P1"], c["P2"], c["P3"], c["nu"], c["G"], c["lam"], c["mid"], c["nrm"],
                                        0, bc, None)
    assert not Dn.any() and not Dss.any() and not Dds.any()


@pytest.mark.parametrize("n,deg", [(300, 0.0), (1000, 0.0), (500, 0.1)])
def test_fischer_newton_dense_known_solution(cad, n, deg):
    rng = np.random.default_rng(11 + n)
    M, q, xs = random_lcp(rng, n, frac_degenerate=deg)
    x = cad.fischer_newton(M, q, tol=1e-12, max_iter=200)
    assert np.max(np.abs(x - xs)) <= 1e-9 * max(1.0, np.abs(xs).max())


def test_fischer_newton_matches_oracle_iterates(cad):
    """Same method, same start: the GPU and the oracle take the same number
    of Newton steps on a well-conditioned problem."""
    from oracle import friction as F
    rng = np.random.default_rng(5)
    M, q, xs = random_lcp(rng, 400)
    x = cad.fischer_newton(M, q, tol=1e-12, max_iter=200)
    it_g, rel_g = cad._lib.last_solve_stats(cad.context(0))
    xo, it_o, rel_o = F.fischer_newton(M, q, tol=1e-12, max_iter=200)
    assert it_g == it_o
    assert np.max(np.abs(x - xo)) <= 1e-10 * np.abs(xo).max()


def test_fischer_newton_not_converged(cad):
    rng = np.random.default_rng(3)
    M, q, xs = random_lcp(rng, 200)
    with pytest.raises(cad.CadError) as e:
        cad.fischer_newton(M, q, tol=1e-14, max_iter=1)
    assert e.value.code == cad._lib.CAD_ERR_NOT_CONVERGED
    assert "Fischer-Newton" in str(e.value)


def test_friction_half_space_dipping_crack(cad, oracle):
    """Friction in half space: a 60-degree dipping crack 1 below the surface
    under a compressive remote stress with shear, mu = 0.7 and cohesion
    growing with depth (about 45 % of the elements slip, the rest stick);
    slip against the oracle's frictional solve (the half-space influence
    matrix on both sides)."""
    from oracle import friction as F

    from cutanddisplacejulia_b200 import workloads
    P1, P2, P3 = workloads.dipping_rect(seed=4, ntri=320, top_depth=1.0)
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    n = len(P1)
    sig = (-2e-3, -1e-3, -3e-3, 1e-3, 1.5e-3, -0.5e-3)
    Sf = 2e-4 * np.abs(mid[:, 2])
    bc = cad.MixedBoundaryConditionsFriction(
        cad.MixedBoundaryConditions(cad.Stresses(*sig), cad.Tractions(0.0, 0.0, 0.0)),
        cad.FrictionParameters(0.7, Sf))
    args = (P1, P2, P3, nu, G, lam, mid, nrm, 1)
    DnF, DssF, DdsF = cad.SlipCalculator3D(*args, bc, None)
    it, rel = cad._lib.last_solve_stats(cad.context(0))
    assert rel <= 1e-10
    Tn, Tds, Tss = oracle.normal_and_shear_tractions(*[np.full(n, s) for s in sig], nrm)
    Dno, Dsso, Ddso, info = F.slip_calculator_friction(*args, Tn, Tss, Tds, 0.7, Sf)
    ref = np.concatenate([Dno, Dsso, Ddso])
    got = np.concatenate([DnF, DssF, DdsF])
    slipping = np.abs(Dsso) > 1e-9
    assert 0 < slipping.sum() < n
    assert np.linalg.norm(got - ref) <= SLIP_TOL * np.linalg.norm(ref)
    assert np.array_equal(np.abs(DssF) > 1e-9, slipping)


def test_fischer_newton_rank_deficient_complementarity(cad):
    """A positive semi-definite, rank-deficient M (solutions not unique): the
    returned x must satisfy the complementarity conditions x >= 0,
    y = M x + q >= 0, x'y = 0 to the tolerance's scale."""
    rng = np.random.default_rng(0)
    n = 400
    B = rng.standard_normal((n, 120))
    M = np.asfortranarray(B @ B.T / 120)
    xs = np.where(rng.uniform(size=n) < 0.3, rng.uniform(0.5, 1.0, n), 0.0)
    ys = np.where(xs > 0, 0.0, rng.uniform(0.5, 1.0, n))
    q = ys - M @ xs
    x = cad.fischer_newton(M, q, tol=1e-12, max_iter=200)
    y = M @ x + q
    s = np.abs(q).max()
    assert x.min() >= -1e-10 * s and y.min() >= -1e-10 * s
    assert np.abs(x * y).max() <= 1e-10 * s * max(1.0, np.abs(x).max())


def test_prepared_friction_solver_many_loads(cad):
    """One prepared system (C = inv(A Scl) kept on the GPU), three loads: each
    equals the one-shot frictional solve of the same load (the same device
    code path; 1e-12 norm-wise leaves room for a captured replay of the
    factorisation picking other library kernels than its eager first run);
    solving after the prepared system was replaced raises."""
    c = burgmann_case(1)
    args = (c["P1"], c["P2"], c["P3"], c["nu"], c["G"], c["lam"], c["mid"], c["nrm"], 0)
    S = c["S"]
    loads = []
    for k, (syy, sxy, mu) in enumerate(((-0.05, 1.0, 0.0), (-0.1, 0.7, 0.2), (-0.2, -1.2, 0.4))):
        sig = (0.0, syy * S, 0.0, sxy * S, 0.0, 0.0)
        loads.append(cad.MixedBoundaryConditionsFriction(
            cad.MixedBoundaryConditions(cad.Stresses(*sig), cad.Tractions(0.0, 0.0, 0.0)),
            cad.FrictionParameters(mu, c["Sf"] * (1 + k))))
    solver = cad.FrictionSolver(*args)
    prepared = [solver.solve(bc) for bc in loads]
    for bc, got in zip(loads, prepared):
        ref = np.concatenate(cad.SlipCalculator3D(*args, bc, None))
        assert np.linalg.norm(np.concatenate(got) - ref) <= 1e-12 * np.linalg.norm(ref)
    assert np.abs(prepared[1][1]).max() > 0
    M = np.asfortranarray(np.eye(4) + 0.1)
    cad.fischer_newton(M, -np.ones(4))   # replaces the prepared system on this device
    with pytest.raises(cad.CadError) as e:
        solver.solve(loads[0])
    assert e.value.code == cad._lib.CAD_ERR_ARG
