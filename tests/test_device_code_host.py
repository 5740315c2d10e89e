"""CPU test of the kernels' arithmetic: csrc/td_device.cuh (the per-pair code
the CUDA kernels inline) compiled for the host with fused multiply-add
contraction enabled, run against the oracle on the same cases the GPU tests
use.  Catches formula and branch errors without a GPU."""
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
