"""Build libcad_td.so in-tree with nvcc for sm_100a (no GPU needed to build)."""
from __future__ import annotations

import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB = os.path.join(HERE, "libcad_td.so")
OBJDIR = os.path.join(HERE, "_build")
SOURCES = ["capi.cu", "td_kernels.cu", "probe.cu", "noalloc.cu", "lu.cu", "mixed.cu", "mlp.cu", "trsv.cu", "lcp.cu", "gemm.cu", "lpc.cu", "krylov.cu", "tune.cu"]
HEADERS = ["td_device.cuh", "tde_closed_form.cuh", "td_kernels.h", "lu.h", "mixed.h", "mlp.h", "lcp.h", "gemm.h", "sm100.cuh", "lpc.h", "krylov.h", "tune.h",
           os.path.join("..", "..", "include", "cad_td.h")]

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-lineinfo", "-std=c++17",
    "-Xcompiler", "-fPIC",
]
LIBS: list = []


def _nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _obj(src):
    return os.path.join(OBJDIR, os.path.splitext(src)[0] + ".o")


def _stale_objects(force):
    """Sources whose object is missing or older than the source or any header."""
    hdr_t = max((os.path.getmtime(os.path.join(CSRC, h)) for h in HEADERS if os.path.exists(os.path.join(CSRC, h))),
                default=0.0)
    out = []
    for s in SOURCES:
        o = _obj(s)
        if force or not os.path.exists(o) or os.path.getmtime(o) < max(hdr_t, os.path.getmtime(os.path.join(CSRC, s))):
            out.append(s)
    return out


def build(force: bool = False, verbose: bool = False) -> str:
    """Compile csrc/*.cu (one nvcc per source, in parallel; only stale ones)
    and link cutanddisplacejulia_b200/libcad_td.so."""
    stale = _stale_objects(force)
    if not stale and os.path.exists(LIB) and all(os.path.getmtime(_obj(s)) <= os.path.getmtime(LIB) for s in SOURCES):
        return LIB
    nvcc = _nvcc()
    os.makedirs(OBJDIR, exist_ok=True)

    def compile_one(src):
        cmd = [nvcc, *NVCC_FLAGS, "-c", os.path.join(CSRC, src), "-o", _obj(src) + ".tmp"]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        subprocess.run(cmd, check=True)
        os.replace(_obj(src) + ".tmp", _obj(src))

    with ThreadPoolExecutor(max_workers=max(1, min(len(stale), os.cpu_count() or 1))) as ex:
        list(ex.map(compile_one, stale))
    cuda_lib = os.path.join(os.path.dirname(os.path.dirname(nvcc)), "lib64")
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", LIB + ".tmp",
           *[_obj(s) for s in SOURCES], *LIBS, "-Xlinker", "-rpath," + cuda_lib]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force=True, verbose=True))
