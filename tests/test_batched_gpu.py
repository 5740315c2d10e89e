"""GPU tests of the batched slip solve over independent cracks (FP32 LU with
FP64 refinement inside one captured CUDA graph): every crack's slip against
the plain per-crack FP64 path (src/SlipCalculator3D.jl:1-33), with FP64 and
with mixed-precision assembly; replay of the captured graph; the half-space
argument check."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RESID_TOL = 1e-10


def _cracks(count, seed=11):
    from cutanddisplacejulia_b200 import workloads
    cracks, stresses = workloads.crack_batch(seed=seed, count=count, n_range=(60, 500))
    return cracks, stresses


def _reference(cad, cracks, bcs, nu, G, lam):
    out = []
    for (P1, P2, P3), bc in zip(cracks, bcs):
        nrm, mid = cad.CreateFaceNormalAndMidPoint(P1, P2, P3)
        r = cad.SlipCalculator3D(P1, P2, P3, nu, G, lam, mid, nrm, 0, bc, np.zeros(len(P1)))
        out.append(np.concatenate(r[:3]))
    return out


@pytest.mark.parametrize("mode", ["grouped", "lanes", "lanes_chain"])
@pytest.mark.parametrize("assembly,tol", [("fp64", 1e-8), ("mixed", 1e-4)])
def test_batched_matches_per_crack(cad, assembly, tol, mode):
    cracks, stresses = _cracks(14)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    bcs = [cad.Stresses(*s) for s in stresses]
    ref = _reference(cad, cracks, bcs, nu, G, lam)
    for rep in range(2):   # the second call replays the captured graph
        out, rel = cad.SlipCalculator3D_batched(cracks, nu, G, lam, 0, bcs, tol=RESID_TOL, assembly=assembly,
                                                mode=mode)
        assert np.all(rel <= RESID_TOL)
        for c in range(len(cracks)):
            D = np.concatenate(out[c])
            assert np.linalg.norm(D - ref[c]) <= tol * np.linalg.norm(ref[c]), (rep, c)


@pytest.mark.parametrize("mode", ["grouped", "lanes"])
def test_batched_sweeps_converge_without_fallback(cad, mode):
    # tol = 1 leaves every crack to the fixed refinement sweeps (no GMRES
    # finish): four sweeps alone bring every crack to about the residual the
    # batch promises (the finish takes any crack the last step short)
    cracks, stresses = _cracks(20, seed=7)
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    bcs = [cad.Stresses(*s) for s in stresses]
    out, rel = cad.SlipCalculator3D_batched(cracks, nu, G, lam, 0, bcs, tol=1.0, assembly="fp64", mode=mode)
    assert np.all(rel <= 10 * RESID_TOL), rel.max()
    ref = _reference(cad, cracks, bcs, nu, G, lam)
    for c in range(len(cracks)):
        D = np.concatenate(out[c])
        assert np.linalg.norm(D - ref[c]) <= 1e-8 * np.linalg.norm(ref[c]), c


def test_batched_empty_and_single(cad):
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    out, rel = cad.SlipCalculator3D_batched([], nu, G, lam, 0, [], assembly="fp64")
    assert out == [] and len(rel) == 0
    cracks, stresses = _cracks(1, seed=3)
    bc = cad.Stresses(*stresses[0])
    out, rel = cad.SlipCalculator3D_batched(cracks, nu, G, lam, 0, [bc], assembly="fp64")
    ref = _reference(cad, cracks, [bc], nu, G, lam)[0]
    assert np.linalg.norm(np.concatenate(out[0]) - ref) <= 1e-8 * np.linalg.norm(ref)


def test_batched_halfspace_above_surface_raises(cad):
    cracks, stresses = _cracks(3, seed=5)
    # lift the second crack above the free surface
    P1, P2, P3 = cracks[1]
    cracks[1] = (P1 + [0, 0, 20.0], P2 + [0, 0, 20.0], P3 + [0, 0, 20.0])
    _, _, lam, nu, G = cad.ElasticConstantsCheck(1.0, 0.25)
    with pytest.raises(cad.CadError, match="Z coordinates must be negative"):
        cad.SlipCalculator3D_batched(cracks, nu, G, lam, 1, [cad.Stresses(*s) for s in stresses], assembly="fp64")
