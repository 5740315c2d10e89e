"""GPU tests of fixed elements (src/CalculateInfluenceMatrices3D.jl:10-33,
:145-199; src/SlipCalculator3D.jl with FixedEls): displacement rows for fixed
elements, their columns dropped, the tall system solved in the least-squares
sense.  Against the oracle (1e-12 normwise for the matrices, 1e-8 for the slip
against numpy's lstsq) and the reference's Mogi test (test/test_TDvsMogi.jl)."""
import os

import numpy as np
import pytest

from helpers import GOLDEN, assert_parity

pytestmark = pytest.mark.gpu


def _mogi():
    d = np.load(os.path.join(GOLDEN, "mogi.npz"))
    return d["P1"], d["P2"], d["P3"], d["FixedEls"]


def _dipping_with_fixed(seed, hs):
    from cutanddisplacejulia_b200 import workloads
    P1, P2, P3 = workloads.dipping_rect(seed=seed, ntri=300, top_depth=1.0)
    fixed = np.zeros(len(P1))
    fixed[np.random.default_rng(seed).choice(len(P1), 17, replace=False)] = 1
    if not hs:
        P1, P2, P3 = P1 + [0, 0, 5.0], P2 + [0, 0, 5.0], P3 + [0, 0, 5.0]
    return P1, P2, P3, fixed


@pytest.mark.parametrize("case", ["mogi", "dipping_hs", "dipping_fs"])
def test_influence_and_slip_with_fixed_elements(cad, oracle, case):
    if case == "mogi":
        P1, P2, P3, fixed = _mogi()
        hs = 1
    else:
        hs = 1 if case == "dipping_hs" else 0
        P1, P2, P3, fixed = _dipping_with_fixed(3, hs)
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    n = len(P1)
    T = cad.CalculateInfluenceMatrices3D(nrm, mid, P1, P2, P3, nu, G, lam, fixed, hs, n)
    To = oracle.influence_traction_fixed(nrm, mid, P1, P2, P3, nu, G, lam, fixed, hs)
    assert_parity(np.stack(list(T)), To)
    rng = np.random.default_rng(1)
    Tn, Tss, Tds = rng.uniform(-1, 1, (3, n))
    bc = cad.Tractions(Tn, Tss, Tds)
    Dn, Dss, Dds, A, b = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, hs, bc, fixed)
    Dno, Dsso, Ddso, Ao, bo = oracle.slip_calculator_fixed(P1, P2, P3, nu, G, lam, mid, nrm, hs, Tn, Tss, Tds, fixed)
    assert A.shape == Ao.shape and np.array_equal(b, bo)
    assert_parity(A[None], Ao[None])
    D, Do = np.concatenate([Dn, Dss, Dds]), np.concatenate([Dno, Dsso, Ddso])
    assert np.linalg.norm(D - Do) <= 1e-8 * np.linalg.norm(Do)


def test_mogi_kat_on_gpu(cad):
    P1, P2, P3, fixed = _mogi()
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    n = len(P1)
    bc = cad.Tractions(np.ones(n), np.zeros(n), np.zeros(n))
    Dn, Dss, Dds, _, _ = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 1, bc, fixed)
    assert Dn.max() - Dn.min() <= 0.05 / G
    free = fixed == 0
    X = np.arange(0.0, 101.0)
    Y, Z = np.zeros_like(X), np.zeros_like(X)
    _, U = cad.TD(X, Y, Z, P1[free], P2[free], P3[free], Dss, Dds, Dn, nu, G, 1, 0, 1, cad.Strains(), cad.Disps())
    R = np.sqrt(50.0 ** 2 + X ** 2 + Y ** 2)
    lsi = 1.0 * 1.0 * (1 - nu) / G
    An = (X / R ** 3 * lsi, Y / R ** 3 * lsi, 50.0 / R ** 3 * lsi)
    with np.errstate(divide="ignore", invalid="ignore"):
        for a, u in zip(An, U):
            pct = 100.0 / a * np.asarray(u)
            pct[np.isinf(pct)] = np.nan
            assert not np.any(np.abs(pct - 100) > 20)
