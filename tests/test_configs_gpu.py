"""GPU parity at the full sizes of the benchmark configurations, against the
oracle (the CPU restatement of the reference, src/TD.jl and
src/CalculateInfluenceMatrices3D.jl) on the same seeded inputs:

  C1  full-space fault (10 x 5 rectangles, 100 triangles) seen from a 50 x 50
      grid on y = 0.1: the summing TD overload, 6 stresses (Hooke's law on the
      strain, src/HookesLaw3DStrain2Stress.jl) and 3 displacements;
  C2  pressurised penny crack (lattice spacing 0.06, 2013 triangles): the
      3N x 3N system matrix and its FP64 LU solution;
  C3  half-space dipping crack (10 000 triangles, 3N = 30 000): the full
      system matrix on the GPU, checked against the oracle on a seeded sample
      of element columns (the oracle's whole matrix takes minutes of CPU),
      and its FP64 LU solution through the size-independent residual.
Tolerances: 1e-12 normwise for the FP64 evaluations, 1e-10 relative for the
slip against numpy's LAPACK solve of the oracle's matrix, 1e-12 for the
relative residual of the C3 solve."""
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


def test_c3_dipping_half_space_sampled_columns_and_residual(cad, oracle):
    import torch

    from cutanddisplacejulia_b200 import _lib, workloads
    P1, P2, P3 = workloads.dipping_rect(seed=0, ntri=10000)
    n = len(P1)
    n3 = 3 * n
    assert 9000 < n <= 10000
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    dev = torch.device("cuda", 0)
    L = _lib.load()
    ctx = _lib.context(0)
    col = (lambda a: torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device=dev))
    g = [col(nrm), col(mid), col(P1), col(P2), col(P3)]
    A = torch.empty(n3 * n3, dtype=torch.float64, device=dev)
    _lib.check(L.cad_assemble_dev(ctx, *[x.data_ptr() for x in g], n, nu, G, lam, 1, A.data_ptr(), n3), ctx)
    torch.cuda.synchronize()   # the library's stream is not torch's
    At = A.view(n3, n3)        # row j of this view is column j of the column-major matrix
    sample = np.sort(np.random.default_rng(3).choice(n, 24, replace=False))
    cols = np.concatenate([sample, n + sample, 2 * n + sample])
    got = At[torch.tensor(cols, device=dev)].cpu().numpy().T   # (3N, 72)
    obs = mid - 1e-12 * nrm
    k = len(sample)
    ones = np.ones(k)
    S, _ = oracle.td_inf(obs[:, 0], obs[:, 1], obs[:, 2], P1[sample], P2[sample], P3[sample], ones, ones, ones, nu,
                         G, 0, 1, 1)
    T = oracle.strain_to_traction(S, nrm, lam, G)   # (9, N, k), TractionInf field order
    ref = np.empty((n3, 3 * k))
    for m in range(3):          # slip mode Dn, Dss, Dds (column block)
        for r in range(3):      # traction Tn, Tss, Tds (row block)
            ref[r * n:(r + 1) * n, m * k:(m + 1) * k] = -T[3 * m + r]
    assert_parity(got[None], ref[None])
    # the FP64 LU solution of the full system, through its residual
    Tn, Tds, Tss = cad.CalculateNormalAndShearTractions3D(*workloads.remote_stress(seed=0), nrm)
    b = torch.tensor(np.concatenate([Tn, Tss, Tds]), device=dev)
    F = A.clone()
    x = b.clone()
    with _lib.solver_mode(ctx, "lu64"):
        _lib.check(L.cad_solve_dev(ctx, n3, F.data_ptr(), n3, x.data_ptr(), n3, 1), ctx)
    torch.cuda.synchronize()
    del F
    res = At.t() @ x - b
    assert float(torch.linalg.vector_norm(res) / torch.linalg.vector_norm(b)) <= 1e-12
