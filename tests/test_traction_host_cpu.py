"""CPU tests of the host traction helpers (cutanddisplacejulia_b200/geometry.py:
CalculateNormalTraction3D, TractionVectorCartesianComponents3D,
CalculateTractionInChosenDirection3D, TensorTransformation3D, restating the
reference files of the same names): composed with Hooke's law as
ConvertStrainInfMatsToTraction does (src/CalculateInfluenceMatrices3D.jl:73-114),
they reproduce the oracle's traction influence fields; the tensor rotation
agrees with A T A^T."""
import numpy as np


def test_helpers_compose_to_the_oracle_traction_conversion(oracle):
    import cutanddisplacejulia_b200 as cad
    from helpers import random_points, random_triangles
    rng = np.random.default_rng(4)
    P1, P2, P3 = random_triangles(rng, 9)
    pts = random_points(rng, 40)
    normals = rng.standard_normal((40, 3))
    normals /= np.linalg.norm(normals, axis=1)[:, None]
    ones = np.ones(9)
    S, _ = oracle.td_inf(*pts.T, P1, P2, P3, ones, ones, ones, 0.25, 1.0, 0, 1, 1)   # (18, 40, 9)
    lam, G = 1.0, 1.0
    T = oracle.strain_to_traction(S, normals, lam, G)                             # (9, 40, 9)
    ss, ds = cad.CalculateSSandDSDirs(normals[:, 0], normals[:, 1], normals[:, 2])
    cx, cy, cz = normals.T
    for m in range(3):                       # slip modes Dn, Dss, Dds
        sig = cad.HookesLaw3DStrain2Stress(*S[6 * m:6 * m + 6], lam, G)
        Tn = cad.CalculateNormalTraction3D(*sig, cx, cy, cz)
        Tx, Ty, Tz = cad.TractionVectorCartesianComponents3D(*sig, cx, cy, cz)
        Tss = cad.CalculateTractionInChosenDirection3D(Tx, Ty, Tz, cx, cy, cz, ss)
        Tds = cad.CalculateTractionInChosenDirection3D(Tx, Ty, Tz, cx, cy, cz, ds)
        for k, t in enumerate((Tn, Tss, Tds)):
            ref = T[3 * m + k]
            assert np.max(np.abs(t - ref)) <= 1e-12 * np.max(np.abs(ref))


def test_tensor_transformation_is_a_t_at():
    import cutanddisplacejulia_b200 as cad
    rng = np.random.default_rng(2)
    A, _ = np.linalg.qr(rng.standard_normal((3, 3)))
    t = rng.standard_normal(6)
    T1 = np.array([[t[0], t[3], t[4]], [t[3], t[1], t[5]], [t[4], t[5], t[2]]])
    T2 = A @ T1 @ A.T
    got = cad.TensorTransformation3D(*t, A)
    want = (T2[0, 0], T2[1, 1], T2[2, 2], T2[0, 1], T2[0, 2], T2[1, 2])
    assert np.allclose(got, want, rtol=0, atol=1e-14)
