"""GPU parity at the full sizes of the benchmark configurations, against the
oracle (the CPU restatement of the reference, src/TD.jl and
src/CalculateInfluenceMatrices3D.jl) on the same seeded inputs:

  C1  full-space fault (10 x 5 rectangles, 100 triangles) seen from a 50 x 50
      grid on y = 0.1: the summing TD overload, 6 stresses (Hooke's law on the
      strain, src/HookesLaw3DStrain2Stress.jl) and 3 displacements;
  C2  pressurised penny crack (lattice spacing 0.06, 2013 triangles): the
      3N x 3N system matrix and its FP64 LU solution.
Tolerances: 1e-12 normwise for the FP64 evaluations, 1e-10 relative for the
slip against numpy's LAPACK solve of the oracle's matrix."""
import numpy as np
import pytest

from helpers import assert_parity

pytestmark = pytest.mark.gpu


def test_c1_fault_grid_stress_and_displacement(cad, oracle):
    from cutanddisplacejulia_b200 import workloads
    f = workloads.fault_grid(seed=0)            # 100 triangles, 2500 points
    assert len(f["P1"]) == 100 and len(f["X"]) == 2500
    nu, G, lam = 0.25, 1.0, 1.0                 # mu = 1, lambda = 1
    S, U = cad.TD(f["X"], f["Y"], f["Z"], f["P1"], f["P2"], f["P3"], f["Dss"], f["Dds"], f["Dn"], nu, G, 1, 1, 0,
                  cad.Strains(), cad.Disps())
    So, Uo = oracle.td_sum_eval(f["X"], f["Y"], f["Z"], f["P1"], f["P2"], f["P3"], f["Dss"], f["Dds"], f["Dn"], nu,
                                G, 1, 1, 0)
    stress = np.stack(list(cad.HookesLaw3DStrain2Stress(S, lam, G)))
    stress_o = np.stack(cad.HookesLaw3DStrain2Stress(*So, lam, G))
    assert_parity(stress, stress_o)
    assert_parity(np.stack(list(U)), Uo)


def test_c2_penny_matrix_and_solve(cad, oracle):
    from cutanddisplacejulia_b200 import workloads
    P1, P2, P3 = workloads.penny(seed=0, spacing=0.06)
    n = len(P1)
    assert 1900 < n < 2200
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    bc = cad.Tractions(np.full(n, -1e-3), np.zeros(n), np.zeros(n))
    Dn, Dss, Dds, A, b = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 0, bc, np.zeros(n))
    Ao = oracle.influence_traction(nrm, mid, P1, P2, P3, nu, G, lam, 0, want_A=True)
    assert_parity(A[None], Ao[None])
    D = np.concatenate([Dn, Dss, Dds])
    Do = np.linalg.solve(Ao, b)
    assert np.max(np.abs(D - Do)) / np.max(np.abs(Do)) <= 1e-10
