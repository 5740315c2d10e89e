"""CPU test of the kernels' arithmetic: csrc/td_device.cuh (the per-pair code
the CUDA kernels inline) compiled for the host with fused multiply-add
contraction enabled, run against the oracle on the same cases the GPU tests
use.  Catches formula and branch errors without a GPU.

The shared-edge half-space paths are mirrored on the host as the kernels lay
them out: per-edge strain and displacement maps read with the side's sign
(influence fields), and one correction per edge for the net Burgers vector
of its sides (sums).  The edge table follows the library's numbering rules.
They are checked against the per-side code and the oracle, on connected
meshes that reach the free surface, with a quarter of the triangles flipped."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from helpers import assert_parity, random_points, random_triangles

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "cutanddisplacejulia_b200", "csrc")


@pytest.fixture(scope="module")
def host_lib(tmp_path_factory):
    cxx = shutil.which("g++")
    if cxx is None:
        pytest.skip("no C++ compiler")
    out = tmp_path_factory.mktemp("hostdev") / "libdevice_host.so"
    flags = ["-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=fast", "-Wno-unknown-pragmas"]
    probe = subprocess.run([cxx, "-mfma", "-x", "c++", "-fsyntax-only", "-"], input=b"int main(){}",
                           capture_output=True)
    if probe.returncode == 0:
        flags.append("-mfma")
    subprocess.run([cxx, *flags, "-I", CSRC, "-o", str(out), os.path.join(ROOT, "tests", "device_host_harness.cpp")],
                   check=True)
    return ctypes.CDLL(str(out))


def run(lib, pts, P1, P2, P3, sl, hs):
    M, N = len(pts), len(P1)
    X, Y, Z = [np.ascontiguousarray(pts[:, k]) for k in range(3)]
    P = [np.asfortranarray(p, dtype=np.float64) for p in (P1, P2, P3)]
    s = [np.ascontiguousarray(v, dtype=np.float64) for v in sl]
    S = np.zeros((18, N, M))
    D = np.zeros((9, N, M))
    c = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    lib.host_td_inf(c(X), c(Y), c(Z), ctypes.c_int64(M), c(P[0]), c(P[1]), c(P[2]), ctypes.c_int64(N), c(s[0]),
                    c(s[1]), c(s[2]), ctypes.c_double(0.25), 1, 1, hs, c(S), c(D))
    return S.transpose(0, 2, 1), D.transpose(0, 2, 1)


@pytest.mark.parametrize("seed", [10, 11, 20, 21])
@pytest.mark.parametrize("hs", [0, 1])
def test_device_code_matches_oracle(host_lib, oracle, seed, hs):
    rng = np.random.default_rng(seed)
    P1, P2, P3 = random_triangles(rng, 24)
    pts = random_points(rng, 300)
    sl = rng.uniform(-1e-3, 1e-3, (3, 24))
    S, D = run(host_lib, pts, P1, P2, P3, sl, hs)
    So, Do = oracle.td_inf(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, hs)
    assert_parity(S, So)
    assert_parity(D, Do)


def test_device_code_edge_and_flat_cases(host_lib, oracle):
    P1 = np.array([[0.0, 0.0, -1.0], [2.0, 0.0, -2.0], [0.0, 0.0, 0.0]])
    P2 = np.array([[1.0, 0.0, -1.0], [3.0, 0.0, -2.0], [1.0, 0.2, 0.0]])
    P3 = np.array([[0.0, 1.0, -1.0], [2.0, 1.0, -2.0], [0.3, 1.1, 0.0]])
    pts = np.array([[0.5, 0.0, -1.0], [0.0, 0.5, -1.0], [0.5, 0.5, -1.0], [0.25, 0.25, -1.0], [2.5, 0.0, -2.0],
                    [0.3, 0.1, -1.5], [1.0, 1.0, -1.0], [0.4, 0.3, -0.5]])
    sl = np.array([[0.3, 1.0, -0.2], [-0.7, 0.0, 0.4], [0.5, 1.0, 0.0]])
    for hs in (0, 1):
        S, D = run(host_lib, pts, P1, P2, P3, sl, hs)
        So, Do = oracle.td_inf(*pts.T, P1, P2, P3, *sl, 0.25, 1.0, 1, 1, hs)
        assert np.isnan(So).any()
        assert_parity(S, So)
        assert_parity(D, Do)


def edge_table(P1, P2, P3):
    """The mesh's distinct triangle sides as the library numbers them: side s
    of triangle j runs P1->P2, P2->P3, P3->P1; code +(e + 1) when it runs the
    way edge e was first seen, -(e + 1) when reversed (-0.0 taken as 0.0).
    Also each edge's sides as +-(triangle + 1), in triangle order."""
    N = len(P1)
    V = (P1, P2, P3)
    seen, pts = {}, []
    code = np.zeros(3 * N, dtype=np.int32)
    for j in range(N):
        for sd in range(3):
            a = tuple(float(v) + 0.0 for v in V[sd][j])
            b = tuple(float(v) + 0.0 for v in V[(sd + 1) % 3][j])
            if (a, b) in seen:
                c = seen[(a, b)] + 1
            elif (b, a) in seen:
                c = -(seen[(b, a)] + 1)
            else:
                seen[(a, b)] = len(pts)
                pts.append(a + b)
                c = len(pts)
            code[3 * j + sd] = c
    E = len(pts)
    ptr = np.zeros(E + 1, dtype=np.int32)
    for c in code:
        ptr[abs(c)] += 1
    ptr = np.cumsum(ptr).astype(np.int32)
    fill = ptr[:-1].copy()
    tris = np.zeros(3 * N, dtype=np.int32)
    for k, c in enumerate(code):
        t = k // 3 + 1
        tris[fill[abs(c) - 1]] = t if c > 0 else -t
        fill[abs(c) - 1] += 1
    return code, np.array(pts, dtype=np.float64).reshape(E, 6), ptr, tris


def _edge_case(seed, top_depth, ntri=120, m=80, flip_frac=0.25):
    from cutanddisplacejulia_b200 import workloads
    P1, P2, P3 = workloads.dipping_rect(seed=seed, ntri=ntri, top_depth=top_depth)
    zmax = max(P[:, 2].max() for P in (P1, P2, P3))
    P1, P2, P3 = (P - [0.0, 0.0, zmax + top_depth] for P in (P1, P2, P3))
    rng = np.random.default_rng(seed)
    flip = rng.random(len(P1)) < flip_frac
    P2, P3 = np.where(flip[:, None], P3, P2), np.where(flip[:, None], P2, P3)
    sl = rng.uniform(-1e-3, 1e-3, (3, len(P1)))
    pts = np.column_stack([rng.uniform(-2.0, 2.0, m), rng.uniform(-1.5, 1.5, m), rng.uniform(-2.5, -0.02, m)])
    return pts, (P1, P2, P3), sl


@pytest.mark.parametrize("top_depth", [0.0, 0.2])
def test_shared_edge_influence_matches_per_side_and_oracle(host_lib, oracle, top_depth):
    pts, P, sl = _edge_case(31, top_depth)
    code, epts, _, _ = edge_table(*P)
    assert len(epts) < 0.9 * 3 * len(P[0])
    M, N = len(pts), len(P[0])
    X, Y, Z = [np.ascontiguousarray(pts[:, k]) for k in range(3)]
    Pf = [np.asfortranarray(p, dtype=np.float64) for p in P]
    s = [np.ascontiguousarray(v) for v in sl]
    S, D = np.zeros((18, N, M)), np.zeros((9, N, M))
    c = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    host_lib.host_td_inf_edges(c(X), c(Y), c(Z), ctypes.c_int64(M), c(Pf[0]), c(Pf[1]), c(Pf[2]), ctypes.c_int64(N),
                               c(s[0]), c(s[1]), c(s[2]), ctypes.c_double(0.25), c(code), c(np.ascontiguousarray(epts)),
                               ctypes.c_int64(len(epts)), c(S), c(D))
    S, D = S.transpose(0, 2, 1), D.transpose(0, 2, 1)
    Ss, Ds = run(host_lib, pts, *P, sl, 1)
    assert_parity(S, Ss)
    assert_parity(D, Ds)
    So, Do = oracle.td_inf(*pts.T, *P, *sl, 0.25, 1.0, 1, 1, 1)
    assert_parity(S, So)
    assert_parity(D, Do)


@pytest.mark.parametrize("top_depth", [0.0, 0.2])
def test_shared_edge_sums_match_oracle(host_lib, oracle, top_depth):
    pts, P, sl = _edge_case(32, top_depth)
    _, epts, ptr, tris = edge_table(*P)
    M, N = len(pts), len(P[0])
    X, Y, Z = [np.ascontiguousarray(pts[:, k]) for k in range(3)]
    Pf = [np.asfortranarray(p, dtype=np.float64) for p in P]
    s = [np.ascontiguousarray(v) for v in sl]
    S, D = np.zeros((6, M)), np.zeros((3, M))
    c = lambda a: a.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
    host_lib.host_td_sum_edges(c(X), c(Y), c(Z), ctypes.c_int64(M), c(Pf[0]), c(Pf[1]), c(Pf[2]), ctypes.c_int64(N),
                               c(s[0]), c(s[1]), c(s[2]), ctypes.c_double(0.25), c(ptr), c(tris),
                               c(np.ascontiguousarray(epts)), ctypes.c_int64(len(epts)), c(S), c(D))
    So, Do = oracle.td_sum_eval(*pts.T, *P, *sl, 0.25, 1.0, 1, 1, 1)
    assert_parity(S, So)
    assert_parity(D, Do)
