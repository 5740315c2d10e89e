"""CPU tests of the host mesh readers and CreateP1P2P3 (cutanddisplacejulia_b200/geometry.py,
restating src/STLReader.jl, src/GoCadAsciiReader.jl, src/OFFReader.jl, src/CreateP1P2P3.jl):
the committed reference meshes are written out in each format (shared vertices,
non-contiguous GoCad vertex ids, an ATOM record, comments in the OFF file), read back, and the
vertex lists must come back exactly."""
import numpy as np
import pytest

from helpers import load_mesh


def _shared(P1, P2, P3):
    """Unique points and a 0-based triangle table of a vertex-list mesh."""
    allp = np.vstack([P1, P2, P3])
    pts, inv = np.unique(allp, axis=0, return_inverse=True)
    n = len(P1)
    return pts, np.stack([inv[:n], inv[n:2 * n], inv[2 * n:]], axis=1)


def test_stl_round_trip(tmp_path):
    from cutanddisplacejulia_b200 import geometry as g
    P1, P2, P3 = load_mesh("squaregrid")
    path = tmp_path / "m.stl"
    with open(path, "w") as f:
        f.write("solid test\n")
        for a, b, c in zip(P1, P2, P3):
            f.write("facet normal 0 0 1\nouter loop\n")
            for v in (a, b, c):
                f.write("vertex %.17g %.17g %.17g\n" % tuple(v))
            f.write("endloop\nendfacet\n")
        f.write("endsolid test\n")
    Points, Tris = g.read_stl(str(path))
    Q1, Q2, Q3 = g.CreateP1P2P3(Tris, Points)
    for a, b in ((P1, Q1), (P2, Q2), (P3, Q3)):
        assert np.array_equal(a, b)


def test_gocad_round_trip_with_atoms_and_sparse_ids(tmp_path):
    from cutanddisplacejulia_b200 import geometry as g
    P1, P2, P3 = load_mesh("circle581")
    pts, tri = _shared(P1, P2, P3)
    ids = 5 + 2 * np.arange(len(pts))          # non-contiguous vertex ids
    atom_id = int(ids[-1]) + 7                 # an ATOM that repeats vertex 0
    tri = tri.copy()
    tri[0, 0] = -1                             # triangle 0 uses the ATOM instead
    path = tmp_path / "m.ts"
    with open(path, "w") as f:
        f.write("GOCAD TSurf 1\nHEADER {\nname:test\n}\nTFACE\n")
        for i, p in zip(ids, pts):
            f.write("VRTX %d %.17g %.17g %.17g\n" % (i, *p))
        f.write("ATOM %d %d\n" % (atom_id, ids[0]))
        for t in tri:
            f.write("TRGL %d %d %d\n" % tuple(atom_id if k < 0 else ids[k] for k in t))
        f.write("END\n")
    Points, Tris = g.read_gocad(str(path))
    Q1, Q2, Q3 = g.CreateP1P2P3(Tris, Points)
    E1 = P1.copy()
    E1[0] = pts[0]
    for a, b in ((E1, Q1), (P2, Q2), (P3, Q3)):
        assert np.array_equal(a, b)


def test_gocad_rejects_several_surfaces(tmp_path):
    from cutanddisplacejulia_b200 import geometry as g
    path = tmp_path / "two.ts"
    path.write_text("GOCAD TSurf 1\nPROJECTION Unknown\nVRTX 1 0 0 0\n")
    with pytest.raises(ValueError, match="More than one Gocad ascii surface"):
        g.read_gocad(str(path))


def test_off_round_trip_with_comments(tmp_path):
    from cutanddisplacejulia_b200 import geometry as g
    P1, P2, P3 = load_mesh("blade500")
    pts, tri = _shared(P1, P2, P3)
    path = tmp_path / "m.off"
    with open(path, "w") as f:
        f.write("OFF\n# a comment line\n%d %d 0\n" % (len(pts), len(tri)))
        for p in pts:
            f.write("%.17g %.17g %.17g\n" % tuple(p))
        for t in tri:
            f.write("3 %d %d %d  # face\n" % tuple(t))
    Points, Tris = g.read_off(str(path))
    Q1, Q2, Q3 = g.CreateP1P2P3(Tris, Points)
    for a, b in ((P1, Q1), (P2, Q2), (P3, Q3)):
        assert np.array_equal(a, b)
