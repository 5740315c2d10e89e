"""Generate the committed fixtures under tests/golden/ from the reference's own
test meshes.  Runs only where the reference checkout is present (it is not on
GPU machines); the resulting .npz files are what the tests read.

  squaregrid.npz   test/SquareGrid.stl          (STLReader, src/STLReader.jl)
  circle581.npz    test/CircleMesh_1a_500Faces.ts (GoCadAsciiReader, src/GoCadAsciiReader.jl)
  mogi.npz         test/SphereUniformDistributionON_46Faces.ts with test/SphereFix4.ts (scaled x3)
                   appended as fixed elements (DataAppender3D), 50 below the surface, as
                   test/test_TDvsMogi.jl:6-20 builds it; also holds FixedEls
  blade500.npz     test/BladeFaultShort_500Tris_Vertical_NorthDip_0.5.ts (GoCadAsciiReader), as read;
                   test/test_TDvsBurgmannLinearFrictionCrack.jl flattens and scales it itself
  valley1000.npz   test/ValleySurface_ProperEq_1000Faces.ts (GoCadAsciiReader), as read
                   (test/test_TDvsSavageGravityValley.jl)

Each file holds P1, P2, P3 (N x 3 float64), built as CreateP1P2P3 does
(src/CreateP1P2P3.jl): vertex k of triangle i is the point whose index the
triangle row names.

Usage:  python tests/golden/make_golden.py <path of the CutAndDisplaceJulia checkout>
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def read_stl_ascii(path):
    """ASCII STL: every 'vertex' line is a point, consecutive triples are triangles."""
    pts = []
    with open(path) as f:
        for line in f:
            tok = line.split()
            if tok and tok[0] == "vertex":
                pts.append([float(t) for t in tok[1:4]])
    pts = np.array(pts, dtype=np.float64)
    tris = np.arange(len(pts)).reshape(-1, 3)
    return pts, tris


def read_gocad_ts(path):
    """GoCad ASCII TSurf with VRTX / ATOM / TRGL records (one surface)."""
    coords = {}
    tris = []
    with open(path) as f:
        for line in f:
            tok = line.split()
            if not tok:
                continue
            if tok[0] == "PROJECTION":
                raise ValueError("More than one Gocad ascii surface in the file, this function can only deal with 1")
            if tok[0] in ("VRTX", "PVRTX"):
                coords[int(tok[1])] = [float(t) for t in tok[2:5]]
            elif tok[0] in ("ATOM", "PATOM"):
                coords[int(tok[1])] = coords[int(tok[2])]
            elif tok[0] == "TRGL":
                tris.append([int(t) for t in tok[1:4]])
    ids = sorted(coords)
    index = {v: k for k, v in enumerate(ids)}
    pts = np.array([coords[v] for v in ids], dtype=np.float64)
    tris = np.array([[index[v] for v in t] for t in tris], dtype=np.int64)
    return pts, tris


def p1p2p3(pts, tris):
    return pts[tris[:, 0]].copy(), pts[tris[:, 1]].copy(), pts[tris[:, 2]].copy()


def main(ref):
    test_dir = os.path.join(ref, "test")
    pts, tris = read_stl_ascii(os.path.join(test_dir, "SquareGrid.stl"))
    P1, P2, P3 = p1p2p3(pts, tris)
    np.savez_compressed(os.path.join(HERE, "squaregrid.npz"), P1=P1, P2=P2, P3=P3)
    pts, tris = read_gocad_ts(os.path.join(test_dir, "CircleMesh_1a_500Faces.ts"))
    P1, P2, P3 = p1p2p3(pts, tris)
    np.savez_compressed(os.path.join(HERE, "circle581.npz"), P1=P1, P2=P2, P3=P3)
    print("wrote squaregrid.npz (%d tris), circle581.npz (%d tris)" % (len(read_stl_ascii(
        os.path.join(test_dir, "SquareGrid.stl"))[1]), len(tris)))
    pts, tris = read_gocad_ts(os.path.join(test_dir, "SphereUniformDistributionON_46Faces.ts"))
    ptsf, trisf = read_gocad_ts(os.path.join(test_dir, "SphereFix4.ts"))
    ptsf = ptsf * 3.0
    allp = np.vstack([pts, ptsf])
    allt = np.vstack([tris, trisf + len(pts)])
    fixed = np.concatenate([np.zeros(len(tris)), np.ones(len(trisf))])
    allp[:, 2] -= 50.0
    P1, P2, P3 = p1p2p3(allp, allt)
    np.savez_compressed(os.path.join(HERE, "mogi.npz"), P1=P1, P2=P2, P3=P3, FixedEls=fixed)
    print("wrote mogi.npz (%d tris, %d fixed)" % (len(allt), int(fixed.sum())))
    pts, tris = read_gocad_ts(os.path.join(test_dir, "BladeFaultShort_500Tris_Vertical_NorthDip_0.5.ts"))
    P1, P2, P3 = p1p2p3(pts, tris)
    np.savez_compressed(os.path.join(HERE, "blade500.npz"), P1=P1, P2=P2, P3=P3)
    print("wrote blade500.npz (%d tris)" % len(tris))
    pts, tris = read_gocad_ts(os.path.join(test_dir, "ValleySurface_ProperEq_1000Faces.ts"))
    P1, P2, P3 = p1p2p3(pts, tris)
    np.savez_compressed(os.path.join(HERE, "valley1000.npz"), P1=P1, P2=P2, P3=P3)
    print("wrote valley1000.npz (%d tris)" % len(tris))


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python make_golden.py <path of the CutAndDisplaceJulia checkout>")
    main(sys.argv[1])
