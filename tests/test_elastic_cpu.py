"""CPU tests of host utilities: ElasticConstantsCheck (src/ElasticConstantsCheck.jl)
as the reference's test/test_ElasticConstantsCheck.jl runs it (G = 50, nu = 0.01
passed through every pair of constants in turn must come back unchanged; every
pair, in either order, agrees with the (G, nu) conversion), and
RemoveFixedElements3D (src/RemoveFixedElements3D.jl)."""
import itertools

import numpy as np


def test_round_trip_through_every_pair():
    import cutanddisplacejulia_b200 as cad
    K, E, lam, nu, G = cad.ElasticConstantsCheck(cad.ShearModulus(50.0), cad.PoissonsRatio(0.01))
    K, E, lam, nu, G = cad.ElasticConstantsCheck(cad.BulkModulus(K), cad.YoungsModulus(E))
    K, E, lam, nu, G = cad.ElasticConstantsCheck(cad.BulkModulus(K), cad.LamesConstant(lam))
    K, E, lam, nu, G = cad.ElasticConstantsCheck(cad.BulkModulus(K), cad.PoissonsRatio(nu))
    K, E, lam, nu, G = cad.ElasticConstantsCheck(cad.BulkModulus(K), cad.ShearModulus(G))
    K, E, lam, nu, G = cad.ElasticConstantsCheck(cad.YoungsModulus(E), cad.LamesConstant(lam))
    K, E, lam, nu, G = cad.ElasticConstantsCheck(cad.YoungsModulus(E), cad.PoissonsRatio(nu))
    K, E, lam, nu, G = cad.ElasticConstantsCheck(cad.YoungsModulus(E), cad.ShearModulus(G))
    K, E, lam, nu, G = cad.ElasticConstantsCheck(cad.LamesConstant(lam), cad.PoissonsRatio(nu))
    K, E, lam, nu2, G2 = cad.ElasticConstantsCheck(cad.LamesConstant(lam), cad.ShearModulus(G))
    assert np.isclose(G2, 50.0, rtol=1e-12) and np.isclose(nu2, 0.01, rtol=1e-10)


def test_every_pair_either_order():
    import cutanddisplacejulia_b200 as cad
    ref = cad.ElasticConstantsCheck(1.7, 0.27)          # plain numbers: (G, nu)
    K, E, lam, nu, G = ref
    vals = [cad.BulkModulus(K), cad.YoungsModulus(E), cad.LamesConstant(lam), cad.PoissonsRatio(nu),
            cad.ShearModulus(G)]
    for a, b in itertools.permutations(vals, 2):
        assert np.allclose(cad.ElasticConstantsCheck(a, b), ref, rtol=1e-12, atol=0)


def test_remove_fixed_elements():
    """RemoveFixedElements3D (src/RemoveFixedElements3D.jl) on the Mogi mesh
    with its 6 fixed elements: the other 46 rows remain, in order."""
    import os

    import cutanddisplacejulia_b200 as cad
    from helpers import GOLDEN
    d = np.load(os.path.join(GOLDEN, "mogi.npz"))
    P1, P2, P3, fixed = d["P1"], d["P2"], d["P3"], d["FixedEls"]
    nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
    tris = np.arange(3 * len(P1)).reshape(-1, 3)
    F, T, N, M, Q1, Q2, Q3 = cad.RemoveFixedElements3D(fixed, tris, nrm, mid, P1, P2, P3)
    keep = fixed == 0
    assert F is fixed and len(Q1) == 46
    for a, b in ((T, tris), (N, nrm), (M, mid), (Q1, P1), (Q2, P2), (Q3, P3)):
        assert np.array_equal(a, np.asarray(b)[keep])
