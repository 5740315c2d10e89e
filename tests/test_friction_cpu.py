"""CPU checks of the frictional slip oracle (oracle/friction.py) against the
reference's own acceptance test, test/test_TDvsBurgmannLinearFrictionCrack.jl
(Burgmann 1994 linearly increasing cohesion, Pollard-Segall 1987 uniform
load: per-element deviation <= 36 % on |x| < 0.9 a, summed deviation
<= 1400), plus the complementarity conditions of its LCP solutions and the
Fischer-Newton method on LCPs with known unique solutions."""
import numpy as np
import pytest

from helpers import burgmann_case, burgmann_check, random_lcp


@pytest.mark.parametrize("half", [1, 2])
def test_oracle_friction_burgmann_kat(oracle, half):
    from oracle import friction as F
    c = burgmann_case(half)
    Tn, Tds, Tss = oracle.normal_and_shear_tractions(*c["sig"], c["nrm"])
    args = (c["P1"], c["P2"], c["P3"], c["nu"], c["G"], c["lam"], c["mid"], c["nrm"], 0, Tn, Tss, Tds)
    DnF, DssF, DdsF, info = F.slip_calculator_friction(*args, c["mu"], c["Sf"])
    assert not info["exit"] and info["rel"] <= 1e-10 and info["iterations"] <= 30
    Dn, Dss, Dds, _, _ = oracle.slip_calculator(*args)
    if half == 1:
        burgmann_check(c, half, Dss, DssF)
    else:
        burgmann_check(c, half, Dds, DdsF)
    # complementarity of the LCP solution
    x, M, q = info["x"], info["M"], info["q"]
    y = M @ x + q
    scale = np.abs(q).max()
    assert x.min() >= -1e-9 * scale and y.min() >= -1e-9 * scale
    assert np.max(np.abs(x * y)) <= 1e-9 * scale * scale


@pytest.mark.parametrize("n,deg", [(40, 0.0), (200, 0.0), (120, 0.1)])
def test_oracle_fischer_newton_known_solution(n, deg):
    from oracle import friction as F
    rng = np.random.default_rng(7 + n)
    M, q, xs = random_lcp(rng, n, frac_degenerate=deg)
    x, it, rel = F.fischer_newton(M, q, tol=1e-12, max_iter=200)
    assert rel <= 1e-12
    assert np.max(np.abs(x - xs)) <= 1e-9 * max(1.0, np.abs(xs).max())


def test_oracle_friction_early_exit(oracle):
    """All elements held by friction: zero slip without assembling
    (src/SlipCalculator3D.jl:47-55)."""
    from oracle import friction as F
    c = burgmann_case(1)
    n = c["n"]
    Tn = np.full(n, -10.0)
    Tss = np.full(n, 0.1)
    Tds = np.full(n, -0.1)
    Dn, Dss, Dds, info = F.slip_calculator_friction(c["P1"], c["P2"], c["P3"], c["nu"], c["G"], c["lam"], c["mid"],
                                                    c["nrm"], 0, Tn, Tss, Tds, 0.6, 0.0)
    assert info["exit"] and not Dn.any() and not Dss.any() and not Dds.any()


def test_friction_wrapper_rejects_fixed_elements():
    import cutanddisplacejulia_b200 as cad
    c = burgmann_case(1)
    bc = cad.MixedBoundaryConditionsFriction(
        cad.MixedBoundaryConditions(cad.Stresses(*c["sig"]), cad.Tractions(0.0, 0.0, 0.0)),
        cad.FrictionParameters(0.0, c["Sf"]))
    fixed = np.zeros(c["n"])
    fixed[3] = 1
    with pytest.raises(ValueError, match="DimensionMismatch"):
        cad.SlipCalculator3D(c["P1"], c["P2"], c["P3"], c["nu"], c["G"], c["lam"], c["mid"], c["nrm"], 0, bc, fixed)
