#!/usr/bin/env python3
"""Benchmark of the TD hot path on B200.

Workload (one step): the plain-FP64 pressurised penny crack in full space --
traction influence assembly of a ~2000-triangle crack (every triangle on every
collocation point, the 3N x 3N system A = -[Atn;Atss;Atds]) followed by the
dense LU solve A D = b with uniform normal traction -1e-3 (mu = 1, nu = 0.25).
The mesh is seeded synthetic data (Delaunay of a jittered hexagonal lattice).

Metric: TD pair-evaluations per second over the whole step (pairs per step /
step time), FP64.  Also reported: the split between assembly and solve, the
roofline of the TD pair kernel and of the solve, an end-to-end number through
the host C ABI (pinned host buffers in and out), the CPU baseline, clocks.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): every rank solves its own replica (the dense LU does not
shard without an exchange step); value = all ranks' pairs / max step time.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

from cutanddisplacejulia_b200 import dist as cdist  # noqa: E402

# Algorithmic FP64 operations per pair-evaluation of the assembly kernel:
# full-space strain of all three unit slip modes (2960, counted with the
# oracle's counting scalar on this mesh's collocation pairs) plus the strain ->
# traction epilogue (288 = 3 modes x 96).  Frozen values: kernel-side common
# subexpressions count as speed-up, not as fewer operations.
FALG_ASSEMBLY_FS = 2960.0 + 288.0
# Half-space strain of all three unit modes (43867 on the dipping-crack
# collocation pairs) plus the same traction epilogue.
FALG_ASSEMBLY_HS = 43867.0 + 288.0
# DRAM bytes (read + write) of one assembly from the committed ncu captures
# (profiles/td_pair_kernel_*.md, profiles/fsc_edge_kernel_*.md): (triangles
# captured, bytes).  Both scale as N^2.  Half space: the shared-edge path's two
# kernels, fsc_edge_kernel (17.75 MB + 1.0328 GB) and the edge pair kernel
# built for three blocks per SM (1.0982 GB + 307.38 MB), at 1980 triangles and
# 3037 edges.
PAIR_TRAFFIC = {"penny": (2013, 2.49e6 + 233.84e6), "dipping": (1980, 17.75e6 + 1.0328e9 + 1.0982e9 + 307.38e6)}
# FP64-pipe activity (fraction of peak, ncu sm__pipe_fp64_cycles_active) of the
# shared-edge half-space assembly's kernels, from the committed capture at 1980
# triangles (profiles/fsc_edge_kernel_*.md)
FP64_PIPE_ACTIVE_HS = {"fsc_edge_kernel": 0.538, "td_pair_kernel_edge": 0.591}
# share of the step's (serialised) device time taken by the LU panel leaf, from
# the committed launch list (profiles/launches_penny2013_fp64_and_mixed_step.md)
DOMINANT_SHARE = {"penny": 0.532}
SPACING = 0.06          # lattice spacing of the penny crack (~2013 triangles)
NU, G = 0.25, 1.0
TRACTION = -1e-3
MIXED_TOL = 1e-10       # relative residual the mixed-precision solve iterates to
NEAR_FACTOR = 3.0       # near field of the mixed assembly, in mean edge lengths

UNIT = "pair-evals/s"
# the headline metric as the benchmark's definition names it
BASELINE_METRIC = "TD pair-evals/s vs FP64 peak; solve time at rel-residual 1e-10, mixed vs FP64"
WORKLOADS = {
    "penny": ("TD pair-evals/s (FS penny crack: influence assembly + FP64 LU solve)",
              "penny crack, full space, %d triangles, 3N=%d unknowns, FP64 assembly + LU"),
    "dipping": (BASELINE_METRIC,
                "2x1 crack dipping 60 deg, top at depth 2, half space, %d triangles, 3N=%d unknowns"),
    "learned": ("TD pair-evals/s (HS dipping crack: FP64 assembly + learned-preconditioner GMRES to 1e-10)",
                "3x1.5 crack dipping 45 deg, top at depth 2, half space, %d triangles, 3N=%d unknowns"),
    "friction": ("frictional slip solve time (assembly + inverse + Fischer-Newton LCP), FS penny crack",
                 "penny crack, full space, %d triangles, 5N=%d LCP unknowns, Tn=-2e-3 Tss=1e-3, mu=0.3, "
                 "cohesion 2e-4 r/R, Fischer-Newton to max|Phi| <= 1e-10 max|q|"),
    "batch": ("TD pair-evals/s (batch of independent FS cracks: assembly + solve)",
              "%d full-space penny/elliptical cracks, semi-axis U[0.5,2], aspect U[0.3,1], random orientation, "
              "200-2000 triangles each (log-uniform), %d triangles in all"),
}
WORKLOADS["tdsum"] = ("TD pair-evals/s (HS summed strain + displacement of a slipping crack at observation points)",
                      "2x1 crack dipping 60 deg, top at depth 2, half space, %d triangles with smooth seeded slip; "
                      "%d observation points (a %d x %d grid on the free surface z = 0, x, y in [-4, 4])")
WORKLOADS["gemm"] = ("LU trailing-update GEMM TFLOP/s (C -= A B, column-major)",
                     "%d x %d x %d, FP64 DMMA (each instruction shape) and TF32 tcgen05")
METRIC = WORKLOADS["penny"][0]


def _hbm_peak():
    """Measured HBM copy bandwidth of this pool's B200s when the peaks file
    exists, else the earlier measurement on the same pool."""
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            v = float(json.load(f)["hbm_gbs"])
        return v, "measured HBM copy bandwidth (MEASURED_PEAKS.json hbm_gbs), of measured"
    except (OSError, KeyError, ValueError, TypeError):
        return 6650.0, "6.65 TB/s, an earlier copy-bandwidth measurement on this pool (of fallback)"


HBM_PEAK_GBS = _hbm_peak()


def workload(kind="penny", ntri=10000):
    """Geometry, Lame lambda, half-space flag and the traction vector (Tn, Tss, Tds)."""
    import numpy as np

    from cutanddisplacejulia_b200 import assembly, geometry, workloads
    _, _, lam, _, _ = geometry.ElasticConstantsCheck(G, NU)
    if kind == "penny":
        P1, P2, P3 = workloads.penny(seed=0, spacing=SPACING)
        nrm, mid = geometry.CreateFaceNormalAndMidPoint(P1, P2, P3)
        n = len(P1)
        return P1, P2, P3, nrm, mid, lam, 0, (np.full(n, TRACTION), np.zeros(n), np.zeros(n))
    P1, P2, P3 = workloads.dipping_rect(seed=0, ntri=ntri)
    nrm, mid = geometry.CreateFaceNormalAndMidPoint(P1, P2, P3)
    s = workloads.remote_stress(seed=0)
    Tn, Tds, Tss = assembly.CalculateNormalAndShearTractions3D(*s, nrm)
    return P1, P2, P3, nrm, mid, lam, 1, (Tn, Tss, Tds)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_reference_step(wl, nthreads):
    """One step on the CPU: the oracle (restatement of the reference, all
    threads) assembles A, LAPACK (numpy, all threads) solves it."""
    import numpy as np
    from oracle import oracle as O
    P1, P2, P3, nrm, mid, lam, hs, T = wl
    t0 = time.perf_counter()
    A = O.influence_traction(nrm, mid, P1, P2, P3, NU, G, lam, hs, nthreads=nthreads, want_A=True)
    t1 = time.perf_counter()
    np.linalg.solve(A, np.concatenate(T))
    t2 = time.perf_counter()
    return t1 - t0, t2 - t1


def cpu_reference_c3(wl, nthreads, cols=24, seed=3):
    """Bounded CPU sample of the 30000-unknown half-space step: the oracle
    (restatement of the reference, all threads) assembles the tractions of
    `cols` seeded element columns on every collocation point, scaled by N /
    cols to the whole matrix; numpy LAPACK gesv solves a seeded system of the
    full size (3N x 3N) once.  Returns (assembly s, solve s, description)."""
    import numpy as np
    n = len(wl[0])
    rng = np.random.default_rng(seed)
    asm_s = _c3_assembly_sample(wl, nthreads, cols=cols, seed=seed)
    m = 3 * n
    M = rng.standard_normal((m, m))
    M[np.diag_indices(m)] += m
    rhs = rng.standard_normal(m)
    t1 = time.perf_counter()
    np.linalg.solve(M, rhs)
    sol_s = time.perf_counter() - t1
    del M
    desc = ("oracle HS assembly of %d seeded element columns on all %d collocation points (%d threads), scaled by "
            "N/%d to the full matrix; numpy LAPACK gesv of a seeded %d x %d system (full size, once)"
            % (cols, n, nthreads, cols, m, m))
    return asm_s, sol_s, desc


def _c3_assembly_sample(wl, nthreads, cols=24, seed=3):
    """Seconds the oracle takes for the full half-space assembly, estimated from
    `cols` seeded element columns (scaled by N / cols)."""
    import numpy as np
    from oracle import oracle as O
    P1, P2, P3, nrm, mid, lam, hs, T = wl
    n = len(P1)
    sample = np.sort(np.random.default_rng(seed).choice(n, cols, replace=False))
    obs = mid - 1e-12 * nrm
    ones = np.ones(cols)
    t0 = time.perf_counter()
    S, _ = O.td_inf(obs[:, 0], obs[:, 1], obs[:, 2], P1[sample], P2[sample], P3[sample], ones, ones, ones, NU, G, 0,
                    1, hs, nthreads=nthreads)
    O.strain_to_traction(S, nrm, lam, G, nthreads=nthreads)
    return (time.perf_counter() - t0) * n / cols


def reference_line(args, metric, value, unit, higher, ms, workload_desc, sample, nthreads, extra=None):
    line = {
        "impl": "reference", "metric": metric, "value": value, "unit": unit, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": higher,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload_desc, "inputs": "host memory"},
        "cpu_baseline": {"value": value, "unit": unit, "cores": nthreads, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    line.update(extra or {})
    return line


def run_reference_tdsum(args, nthreads):
    """Reference arm of the tdsum workload: the oracle's half-space sums of all
    triangles at a seeded sample of 300 grid points per step (all host
    threads), scaled to pair-evals/s."""
    import numpy as np
    from oracle import oracle as O
    P1, P2, P3, sl, X, Y, Z = tdsum_case(args.ntri)
    n, m = len(P1), X.size

    def step(seed):
        pick = np.random.default_rng(seed).choice(m, 300, replace=False)
        t0 = time.perf_counter()
        O.td_sum_eval(X[pick], Y[pick], Z[pick], P1, P2, P3, *sl, NU, G, 1, 1, 1)
        return time.perf_counter() - t0
    for w in range(args.warmup):
        step(100 + w)
    ts = [step(k) for k in range(args.steps)]
    sec = sum(ts) / len(ts)
    value = 300.0 * n / sec
    return reference_line(args, WORKLOADS["tdsum"][0], value, UNIT, True, sec * 1e3 * m / 300.0,
                          WORKLOADS["tdsum"][1] % (n, m, TDSUM_GRID, TDSUM_GRID),
                          "oracle HS sums of all %d triangles at 300 seeded grid points per step (%d threads), "
                          "%.2f s per sample; ms_per_step scaled to all %d points" % (n, nthreads, sec, m),
                          nthreads)


def run_reference_friction(args, nthreads):
    """Reference arm of the friction workload: the oracle's frictional solve
    (assembly, numpy inverse, numpy Fischer-Newton on the full 5N system) of
    the first (smallest) penny crack, per step."""
    from oracle import friction as F
    c = friction_case(max(args.friction_spacing))

    def step():
        t0 = time.perf_counter()
        F.slip_calculator_friction(c["P1"], c["P2"], c["P3"], NU, G, c["lam"], c["mid"], c["nrm"], 0, c["Tn"],
                                   c["Tss"], c["Tds"], c["mu"], c["Sf"])
        return time.perf_counter() - t0
    for _ in range(args.warmup):
        step()
    ms = 1e3 * sum(step() for _ in range(args.steps)) / args.steps
    return reference_line(args, WORKLOADS["friction"][0], ms, "ms", False, ms,
                          WORKLOADS["friction"][1] % (c["n"], 5 * c["n"]),
                          "one full frictional solve of the %d-triangle crack per step: oracle assembly, numpy "
                          "inverse and Fischer-Newton (LAPACK, %d threads)" % (c["n"], nthreads), nthreads)


def run_reference_batch(args, nthreads, sample=8):
    """Reference arm of the batch workload on a bounded sample: the first
    `sample` cracks of the same seeded batch, each assembled by the oracle and
    solved by numpy LAPACK, one after the other; pairs per second of the
    sample."""
    import numpy as np
    from oracle import oracle as O

    from cutanddisplacejulia_b200 import assembly, geometry, workloads
    cracks, stresses = workloads.crack_batch(seed=0, count=args.cracks * world)
    # weak scaling over ranks: a batch of --cracks cracks per rank, the seeded
    # batch of cracks x world split by crack (balanced by factorisation work)
    all_pairs = float(sum(len(c[0]) ** 2 for c in cracks))
    if world > 1:
        mine = cdist.crack_shard([len(c[0]) for c in cracks], rank, world)
        cracks, stresses = [cracks[i] for i in mine], [stresses[i] for i in mine]
    _, _, lam, _, _ = geometry.ElasticConstantsCheck(G, NU)
    wls = []
    for (P1, P2, P3), st in list(zip(cracks, stresses))[:sample]:
        nrm, mid = geometry.CreateFaceNormalAndMidPoint(P1, P2, P3)
        Tn, Tds, Tss = assembly.CalculateNormalAndShearTractions3D(*st, nrm)
        wls.append((P1, P2, P3, nrm, mid, lam, 0, (Tn, Tss, Tds)))
    pairs = float(sum(len(w[0]) ** 2 for w in wls))

    def step():
        t = 0.0
        for wl in wls:
            a, b = cpu_reference_step(wl, nthreads)
            t += a + b
        return t
    for _ in range(args.warmup):
        step()
    step_s = sum(step() for _ in range(args.steps)) / args.steps
    ntot = sum(len(w[0]) for w in wls)
    return reference_line(args, WORKLOADS["batch"][0], pairs / step_s, UNIT, True, step_s * 1e3,
                          WORKLOADS["batch"][1] % (args.cracks, sum(len(c[0]) for c in cracks)),
                          "the first %d cracks of the batch (%d triangles, %.3g pairs) per step: oracle assembly "
                          "+ numpy LAPACK gesv, %d threads" % (len(wls), ntot, pairs, nthreads), nthreads)


def run_reference(args, rank):
    if rank != 0:
        return
    import numpy as np  # noqa: F401
    from oracle import oracle as O
    O.build()
    nthreads = os.cpu_count() or 1
    if args.workload in ("friction", "batch"):
        fn = run_reference_friction if args.workload == "friction" else run_reference_batch
        print(json.dumps(fn(args, nthreads)), flush=True)
        return
    if args.workload == "tdsum":
        print(json.dumps(run_reference_tdsum(args, nthreads)), flush=True)
        return
    if args.workload == "learned":
        print(json.dumps({"impl": "reference", "unavailable": "the CPU restatement needs well over an hour per "
                          "step at N = 20000 in half space; the reference arm covers penny, dipping, friction and "
                          "batch"}), flush=True)
        return
    wl = workload(args.workload, args.ntri)
    n = len(wl[0])
    if args.workload == "dipping":
        # bounded sample per step (the full CPU step takes minutes)
        asm_s, sol_s, desc = cpu_reference_c3(wl, nthreads)
        for w in range(max(0, args.warmup - 1)):
            _c3_assembly_sample(wl, nthreads, seed=50 + w)
        ta = 0.0
        for k in range(args.steps):
            # a fresh seeded column sample each step; the full-size solve is timed once
            ta += _c3_assembly_sample(wl, nthreads, seed=100 + k)
        asm_s = ta / args.steps
        step_s = asm_s + sol_s
        value = n * n / step_s
        line = {
            "impl": "reference", "metric": WORKLOADS["dipping"][0], "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS["dipping"][1] % (n, 3 * n), "inputs": "host memory",
                       "step": "FP64 assembly + FP64 LU (the reference's A\\b), CPU"},
            "breakdown_ms": {"assembly_scaled": asm_s * 1e3, "solve": sol_s * 1e3},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port", "sample": desc},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    for _ in range(args.warmup):
        cpu_reference_step(wl, nthreads)
    ta, ts = 0.0, 0.0
    for _ in range(args.steps):
        a, s = cpu_reference_step(wl, nthreads)
        ta += a
        ts += s
    step_s = (ta + ts) / args.steps
    value = n * n / step_s
    line = {
        "impl": "reference", "metric": WORKLOADS[args.workload][0], "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload][1] % (n, 3 * n), "inputs": "host memory"},
        "breakdown_ms": {"assembly": ta / args.steps * 1e3, "solve": ts / args.steps * 1e3},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": nthreads, "kind": "port",
                         "sample": "full workload per step: oracle assembly (%d threads) + numpy LAPACK gesv" % nthreads},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def surface_grid(hs, n=100, extent=4.0):
    """Observation grid of the displacement check: n x n on z = 0 (half space)
    or z = 0.5 (full space), x, y in [-extent, extent]."""
    import numpy as np
    g = np.linspace(-extent, extent, n)
    X, Y = np.meshgrid(g, g, indexing="ij")
    return X.ravel(), Y.ravel(), np.full(X.size, 0.0 if hs else 0.5)


def near_field_study(ctx, L, stream, step_asm_args, A, b0, x64, factors):
    """Mixed assembly with the FP64 near field widened: per near-field radius
    (in mean edge lengths), the assembly time, the mixed solve's slip error
    against the FP64 LU and the system matrix's largest entry error (A is
    overwritten)."""
    import torch

    from cutanddisplacejulia_b200 import _lib
    dN, dM, dP1, dP2, dP3, n, lam, hs = step_asm_args
    n3 = 3 * n
    A64 = torch.empty_like(A)
    _lib.check(L.cad_assemble_dev(ctx, dN.data_ptr(), dM.data_ptr(), dP1.data_ptr(), dP2.data_ptr(), dP3.data_ptr(),
                                  n, NU, G, lam, hs, A64.data_ptr(), n3), ctx)
    scale = float(A64.abs().max())
    out = []
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    for f in factors:
        with _lib.solver_mode(ctx, "mixed", tol=MIXED_TOL, max_iter=200), _lib.assembly_mode(ctx, "mixed", f):
            for rep in range(2):   # the second assembly is timed
                torch.cuda.synchronize()
                ev[0].record(stream)
                _lib.check(L.cad_assemble_dev(ctx, dN.data_ptr(), dM.data_ptr(), dP1.data_ptr(), dP2.data_ptr(),
                                              dP3.data_ptr(), n, NU, G, lam, hs, A.data_ptr(), n3), ctx)
                ev[1].record(stream)
                torch.cuda.synchronize()
            asm_ms = ev[0].elapsed_time(ev[1])
            mat_err = float((A - A64).abs().max()) / scale
            x = b0.clone()
            _lib.check(L.cad_solve_dev(ctx, n3, A.data_ptr(), n3, x.data_ptr(), n3, 1), ctx)
            torch.cuda.synchronize()
        out.append({"near_factor": f, "assembly_ms": asm_ms, "matrix_max_rel_err": mat_err,
                    "slip_rel_err_vs_fp64_lu": float(torch.linalg.vector_norm(x - x64) / torch.linalg.vector_norm(x64))})
    del A64
    return out


def mixed_solve_timing(args, ctx, L, stream, step_asm_args, A, b0, x64, ms_fp64, world, dev):
    """The mixed-precision step on the same workload: far-field pairs assembled
    in FP32 (near field -- within 3 mean edge lengths -- in FP64), then FP32 LU
    (TF32 tensor-core updates) preconditioning FP64 GMRES to relative residual
    1e-10 (A is left unchanged).  Timed like the FP64 step (CUDA events on the
    context stream, warm-up first).  Errors against the FP64 path: system matrix
    (the tractions of unit slips), slip, and the surface displacement the slip
    produces on a 100 x 100 grid."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from cutanddisplacejulia_b200 import _lib
    dN, dM, dP1, dP2, dP3, n, lam, hs = step_asm_args
    n3 = 3 * n
    xm = torch.empty_like(x64)

    def assemble(into):
        _lib.check(L.cad_assemble_dev(ctx, dN.data_ptr(), dM.data_ptr(), dP1.data_ptr(), dP2.data_ptr(),
                                      dP3.data_ptr(), n, NU, G, lam, hs, into.data_ptr(), n3), ctx)

    def step(evs=None):
        if evs:
            evs[0].record(stream)
        assemble(A)
        if evs:
            evs[1].record(stream)
        xm.copy_(b0)
        _lib.check(L.cad_solve_dev(ctx, n3, A.data_ptr(), n3, xm.data_ptr(), n3, 1), ctx)
        if evs:
            evs[2].record(stream)

    with _lib.solver_mode(ctx, "mixed", tol=MIXED_TOL, max_iter=200), _lib.assembly_mode(ctx, "mixed", NEAR_FACTOR):
        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        for k in range(args.steps):
            step(evs[k])
        t1.record(stream)
        torch.cuda.synchronize()
        iters, relres = _lib.last_solve_stats(ctx)
        factor_ms = L.cad_last_time_ms(ctx, 2)   # the last step's cast + FP32 LU + block inverses
    ms = t0.elapsed_time(t1) / args.steps
    ms = cdist.max_over_ranks(ms, dev)
    asm_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    sol_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)
    Am = A.view(n3, n3).t()
    resid = float(torch.linalg.vector_norm(Am @ xm - b0) / torch.linalg.vector_norm(b0))
    slip_err = float(torch.linalg.vector_norm(xm - x64) / torch.linalg.vector_norm(x64))
    # the FP64 matrix beside the mixed one: traction error of unit slips
    A64 = torch.empty_like(A)
    assemble(A64)
    trac_err = float((A64 - A).abs().max() / A64.abs().max())
    del A64
    # surface displacement of both slips (summing TD overload, FP64)
    gx, gy, gz = (torch.tensor(v, dtype=torch.float64, device=dev) for v in surface_grid(hs))
    M = gx.numel()

    def surface(x):
        Dn, Dss, Dds = x[:n].contiguous(), x[n:2 * n].contiguous(), x[2 * n:].contiguous()
        U = torch.empty(3 * M, dtype=torch.float64, device=dev)
        _lib.check(L.cad_td_sum_eval_dev(ctx, gx.data_ptr(), gy.data_ptr(), gz.data_ptr(), M, dP1.data_ptr(),
                                         dP2.data_ptr(), dP3.data_ptr(), n, Dss.data_ptr(), Dds.data_ptr(),
                                         Dn.data_ptr(), NU, 1, 0, hs, None, U.data_ptr()), ctx)
        return U
    U64, Um = surface(x64), surface(xm)
    disp_err = float(torch.linalg.vector_norm(Um - U64) / torch.linalg.vector_norm(U64))
    return {"solver": "FP32 LU (TF32 tensor-core trailing updates) preconditioning FP64 restarted GMRES",
            "assembly": "FP32 far field, FP64 within %g mean edge lengths of the source centroid" % NEAR_FACTOR,
            "tol": MIXED_TOL, "ms_per_step": ms,
            "breakdown_ms": {"assembly": asm_ms, "solve": sol_ms, "solve_fp32_factorisation": factor_ms,
                             "solve_gmres": sol_ms - factor_ms},
            "gmres_iterations": iters, "rel_residual": resid,
            "errors_vs_fp64": {"traction_matrix_max_rel": trac_err, "slip_rel_l2": slip_err,
                               "surface_disp_rel_l2": disp_err, "surface_grid": "100 x 100, x,y in [-4, 4], z = %g"
                               % (0.0 if hs else 0.5)},
            "step_speedup_vs_fp64": ms_fp64 / ms}


def batch_rhs_timing(args, ctx, L, stream, asm_args, nrm, A, dev):
    """K right-hand sides (seeded remote stress tensors, six components
    U[-1e-3, 1e-3], resolved onto the element tractions) on the same system:
    assembly + FP64 LU with K columns, and mixed assembly + FP32 LU + batched
    FP64 refinement (GMRES for any column it leaves).  One timed pass each
    after one warm-up pass; errors of the mixed solutions against the FP64 LU
    ones (largest column relative L2)."""
    import numpy as np
    import torch

    from cutanddisplacejulia_b200 import _lib, assembly
    dN, dM, dP1, dP2, dP3, n, lam, hs = asm_args
    n3, K = 3 * n, args.batch_rhs
    rng = np.random.default_rng(7)
    B = np.empty((n3, K))
    for c in range(K):
        Tn, Tds, Tss = assembly.CalculateNormalAndShearTractions3D(*rng.uniform(-1e-3, 1e-3, 6), nrm)
        B[:, c] = np.concatenate([Tn, Tss, Tds])
    B0 = torch.tensor(np.asfortranarray(B).ravel(order="F"), device=dev)
    X = torch.empty_like(B0)

    def run(mode):
        with _lib.solver_mode(ctx, "lu64" if mode == "fp64" else "mixed", tol=MIXED_TOL, max_iter=400), \
                _lib.assembly_mode(ctx, mode, NEAR_FACTOR):
            ms = []
            for rep in range(2):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                _lib.check(L.cad_assemble_dev(ctx, dN.data_ptr(), dM.data_ptr(), dP1.data_ptr(), dP2.data_ptr(),
                                              dP3.data_ptr(), n, NU, G, lam, hs, A.data_ptr(), n3), ctx)
                X.copy_(B0)
                _lib.check(L.cad_solve_dev(ctx, n3, A.data_ptr(), n3, X.data_ptr(), n3, K), ctx)
                e1.record(stream)
                torch.cuda.synchronize()
                ms.append(e0.elapsed_time(e1))
            its = _lib.last_solve_stats(ctx)[0] if mode == "mixed" else 0
        return ms[-1], X.view(K, n3).clone(), its
    ms64, X64, _ = run("fp64")
    msm, Xm, its = run("mixed")
    err = float(((Xm - X64).norm(dim=1) / X64.norm(dim=1)).max())
    return {"rhs": K, "fp64_ms": ms64, "mixed_ms": msm, "speedup": ms64 / msm, "mixed_iterations": its,
            "max_col_slip_rel_err_vs_fp64": err,
            "what": "assembly + factorisation + K-column solve; mixed = FP32 far field, FP32 LU, batched FP64 "
                    "refinement to relative residual %g" % MIXED_TOL}


def run_batch(args, rank, world, local_rank):
    """Many independent cracks (the batching configuration): every crack
    assembled (FP32 far field / FP64 near field) and solved by FP32 LU with
    FP64 refinement to relative residual 1e-10, all cracks in one captured
    CUDA graph over 32 stream lanes (cad_slip_calculator_batched_dev).  Beside
    it: the plain per-crack FP64 path (assembly + FP64 LU, one crack after the
    other) on the same cracks, and the slip error against it."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from cutanddisplacejulia_b200 import _lib, assembly, geometry, workloads
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    cracks, stresses = workloads.crack_batch(seed=0, count=args.cracks * world)
    # weak scaling over ranks: a batch of --cracks cracks per rank, the seeded
    # batch of cracks x world split by crack (balanced by factorisation work)
    all_pairs = float(sum(len(c[0]) ** 2 for c in cracks))
    if world > 1:
        mine = cdist.crack_shard([len(c[0]) for c in cracks], rank, world)
        cracks, stresses = [cracks[i] for i in mine], [stresses[i] for i in mine]
    _, _, lam, _, _ = geometry.ElasticConstantsCheck(G, NU)
    offs = [0]
    blocks = {k: [] for k in ("P1", "P2", "P3", "nrm", "mid", "T")}
    for (P1, P2, P3), st in zip(cracks, stresses):
        N = len(P1)
        nrm, mid = geometry.CreateFaceNormalAndMidPoint(P1, P2, P3)
        Tn, Tds, Tss = assembly.CalculateNormalAndShearTractions3D(*st, nrm)
        for k, a in (("P1", P1), ("P2", P2), ("P3", P3), ("nrm", nrm), ("mid", mid)):
            blocks[k].append(np.asfortranarray(a).ravel(order="F"))
        blocks["T"].append(np.concatenate([Tn, Tss, Tds]))
        offs.append(offs[-1] + N)
    host = {k: np.ascontiguousarray(np.concatenate(v)) for k, v in blocks.items()}
    d = {k: torch.tensor(v, device=dev) for k, v in host.items()}
    ntot = offs[-1]
    offsets = np.asarray(offs, dtype=np.int64)
    pairs = float(sum((offs[c + 1] - offs[c]) ** 2 for c in range(len(cracks))))
    D = torch.zeros(3 * ntot, dtype=torch.float64, device=dev)
    rel = np.zeros(len(cracks))
    L = _lib.load()
    ctx = _lib.context(local_rank)
    if args.eager:   # CUDA's default stream: the batch is issued directly, not captured
        _lib.check(L.cad_set_stream(ctx, None), ctx)
        stream = torch.cuda.default_stream(dev)
    else:
        stream = torch.cuda.ExternalStream(L.cad_get_stream(ctx), device=dev)
    torch.cuda.set_stream(stream)

    def batched():
        _lib.check(L.cad_slip_calculator_batched_dev(ctx, len(cracks), offsets.ctypes.data, d["P1"].data_ptr(),
                                                     d["P2"].data_ptr(), d["P3"].data_ptr(), d["nrm"].data_ptr(),
                                                     d["mid"].data_ptr(), NU, G, lam, 0, d["T"].data_ptr(),
                                                     D.data_ptr(), rel.ctypes.data), ctx)

    with _lib.solver_mode(ctx, "mixed", MIXED_TOL, 400), _lib.assembly_mode(ctx, "mixed", NEAR_FACTOR):
        t0 = time.perf_counter()
        batched()                                   # captures the batch graph
        torch.cuda.synchronize()
        capture_s = time.perf_counter() - t0
        for _ in range(max(0, args.warmup - 1)):
            batched()
        torch.cuda.synchronize()
        clocks = ClockSampler(local_rank)
        clocks.start()
        time.sleep(0.3)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = L.cad_kernel_launches(ctx)
        e0.record(stream)
        for _ in range(args.steps):
            batched()
        e1.record(stream)
        torch.cuda.synchronize()
        clk = clocks.stop()
        launches = L.cad_kernel_launches(ctx) - l0
    ms = e0.elapsed_time(e1) / args.steps
    ms = cdist.max_over_ranks(ms, dev)
    Dm = D.clone()
    # plain per-crack FP64 path on the same cracks: assembly + FP64 LU
    A = torch.empty(9 * max(offs[c + 1] - offs[c] for c in range(len(cracks))) ** 2, dtype=torch.float64,
                    device=dev)
    D64 = torch.empty_like(D)

    def plain():
        for c in range(len(cracks)):
            o, N = offs[c], offs[c + 1] - offs[c]
            n3 = 3 * N
            _lib.check(L.cad_assemble_dev(ctx, d["nrm"].data_ptr() + 24 * o, d["mid"].data_ptr() + 24 * o,
                                          d["P1"].data_ptr() + 24 * o, d["P2"].data_ptr() + 24 * o,
                                          d["P3"].data_ptr() + 24 * o, N, NU, G, lam, 0, A.data_ptr(), n3), ctx)
            D64[3 * o:3 * o + n3].copy_(d["T"][3 * o:3 * o + n3])
            _lib.check(L.cad_solve_dev(ctx, n3, A.data_ptr(), n3, D64.data_ptr() + 24 * o, n3, 1), ctx)
    plain()
    torch.cuda.synchronize()
    e0.record(stream)
    plain()
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1)
    errs = [float(torch.linalg.vector_norm(Dm[3 * offs[c]:3 * offs[c + 1]] - D64[3 * offs[c]:3 * offs[c + 1]]) /
                  torch.linalg.vector_norm(D64[3 * offs[c]:3 * offs[c + 1]])) for c in range(len(cracks))]
    # end to end through the host C ABI (host arrays in, slips back to the host)
    Dh = np.zeros(3 * ntot)
    with _lib.solver_mode(ctx, "mixed", MIXED_TOL, 400), _lib.assembly_mode(ctx, "mixed", NEAR_FACTOR):
        def e2e_call():
            _lib.check(L.cad_slip_calculator_batched(ctx, len(cracks), offsets.ctypes.data, host["P1"].ctypes.data,
                                                     host["P2"].ctypes.data, host["P3"].ctypes.data,
                                                     host["nrm"].ctypes.data, host["mid"].ctypes.data, NU, G, lam, 0,
                                                     host["T"].ctypes.data, Dh.ctypes.data, rel.ctypes.data), ctx)
        e2e_call()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_call()
        e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    line = {
        "metric": WORKLOADS["batch"][0], "value": all_pairs / (ms * 1e-3), "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 + f64 refinement", "data": "synthetic",
        "config": {"workload": WORKLOADS["batch"][1] % (len(cracks), ntot), "pairs_per_step": pairs,
                   "pairs_all_ranks": all_pairs, "parallelism": "cracks split over %d ranks" % world,
                   "system_matrices_gb": 9 * pairs * 8 / 1e9, "l2": "inputs larger than L2"},
        "breakdown_ms": {"batched_graph": ms, "graph_capture_first_call_s": capture_s},
        "plain_fp64_per_crack_ms": plain_ms, "speedup_vs_plain_fp64": plain_ms / ms,
        "max_crack_slip_rel_err_vs_fp64": max(errs), "max_rel_residual": float(rel.max()),
        "clocks": clk, "gpu_launches": int(launches),
        "e2e": {"value": all_pairs / (cdist.max_over_ranks(e2e_ms, dev) * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": int(18 * ntot * 8),
                "d2h_bytes_per_step": int(3 * ntot * 8), "ms_per_step": e2e_ms,
                "api": "cad_slip_calculator_batched (host C ABI)"},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_learned(args, rank, world, local_rank):
    """The learned-preconditioner configuration: a network trained (by the
    library's BF16 kernels) on exact inverse blocks of small seeded meshes,
    applied to a large half-space crack as a block-sparse right
    preconditioner of FP64 GMRES; beside it block-Jacobi GMRES and the FP64
    dense LU (the fallback, and the reference for the solution error)."""
    import numpy as np
    import torch

    from cutanddisplacejulia_b200 import _lib, assembly, geometry, precond, workloads
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    L = _lib.load()
    ctx = _lib.context(local_rank)
    stream = torch.cuda.ExternalStream(L.cad_get_stream(ctx), device=dev)
    torch.cuda.set_stream(stream)
    # training
    net, training = train_network(args, local_rank)
    # the system
    P1, P2, P3 = workloads.dipping_rect(seed=0, ntri=args.ntri, length=3.0, width=1.5, dip=45.0, top_depth=2.0)
    n = len(P1)
    n3 = 3 * n
    nrm, mid = geometry.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, _, _ = geometry.ElasticConstantsCheck(G, NU)
    Tn, Tds, Tss = assembly.CalculateNormalAndShearTractions3D(*workloads.remote_stress(seed=0), nrm)
    b = torch.tensor(np.concatenate([Tn, Tss, Tds]), device=dev)

    def col(a):
        return torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device=dev)
    dP1, dP2, dP3, dN, dM = col(P1), col(P2), col(P3), col(nrm), col(mid)
    A = torch.empty(n3 * n3, dtype=torch.float64, device=dev)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]

    def timed(fn):
        torch.cuda.synchronize()
        ev[0].record(stream)
        fn()
        ev[1].record(stream)
        torch.cuda.synchronize()
        return ev[0].elapsed_time(ev[1])

    asm_ms = timed(lambda: _lib.check(L.cad_assemble_dev(ctx, dN.data_ptr(), dM.data_ptr(), dP1.data_ptr(),
                                                         dP2.data_ptr(), dP3.data_ptr(), n, NU, G, lam, 1,
                                                         A.data_ptr(), n3), ctx))
    solves = {}
    xs = {}
    nbr1 = torch.arange(n, dtype=torch.int32, device=dev)
    bj = torch.empty((n, 9), dtype=torch.float32, device=dev)
    setup_ms = {}
    for name in ("learned", "block_jacobi"):
        if name == "learned":   # features, network and blocks on the device
            setup_ms[name] = timed(lambda: _lib.check(L.cad_lpc_install_dev(ctx, dP1.data_ptr(), dP2.data_ptr(),
                                                                            dP3.data_ptr(), n, G), ctx))
        else:
            setup_ms[name] = timed(lambda: _lib.check(L.cad_block_jacobi_dev(ctx, n, A.data_ptr(), n3,
                                                                             nbr1.data_ptr(), bj.data_ptr()), ctx))
            _lib.check(L.cad_set_preconditioner(ctx, n, 1, nbr1.data_ptr(), bj.data_ptr()), ctx)
        x = b.clone()
        with _lib.solver_mode(ctx, "gmres_spai", MIXED_TOL, args.max_iter):
            rc = []
            ms = timed(lambda: rc.append(L.cad_solve_dev(ctx, n3, A.data_ptr(), n3, x.data_ptr(), n3, 1)))
            its, rr = _lib.last_solve_stats(ctx)
        L.cad_set_preconditioner(ctx, 0, 0, None, None)
        xs[name] = x
        solves[name] = {"ms": ms, "iterations": its, "rel_residual": rr, "converged": rc[0] == 0,
                        "setup_ms": setup_ms[name]}
    # FP64 dense LU (overwrites A)
    x = b.clone()
    with _lib.solver_mode(ctx, "lu64"):
        lu_ms = timed(lambda: _lib.check(L.cad_solve_dev(ctx, n3, A.data_ptr(), n3, x.data_ptr(), n3, 1), ctx))
    solves["fp64_lu"] = {"ms": lu_ms}
    for name in ("learned", "block_jacobi"):
        solves[name]["slip_rel_err_vs_fp64_lu"] = float(torch.linalg.vector_norm(xs[name] - x) /
                                                         torch.linalg.vector_norm(x))
    pairs = float(n) * n
    step_ms = asm_ms + setup_ms["learned"] + solves["learned"]["ms"]
    line = {
        "metric": WORKLOADS["learned"][0], "value": world * pairs / (step_ms * 1e-3), "unit": UNIT, "n_gpus": world,
        "steps": 1, "warmup": 0, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 (network bf16)", "data": "synthetic",
        "config": {"workload": WORKLOADS["learned"][1] % (n, n3), "pairs_per_step": pairs},
        "breakdown_ms": {"assembly_fp64": asm_ms, "learned_setup": setup_ms["learned"],
                         "learned_gmres": solves["learned"]["ms"]},
        "solves_to_rel_residual_1e-10": solves,
        "speedup_learned_vs_fp64_lu": lu_ms / solves["learned"]["ms"],
        "training": training,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


TUNE_CACHE = os.path.join(ROOT, "cutanddisplacejulia_b200", "autotune_b200.txt")


def _autotune_summary(L, ctx, args):
    if args.no_autotune:
        return None
    tuned = ctypes.c_int64(0)
    entries = L.cad_autotune_entries(ctx, ctypes.byref(tuned))
    return {"cache": os.path.relpath(TUNE_CACHE, ROOT), "entries": int(entries), "timed_in_this_run": tuned.value}


def train_network(args, device):
    """The learned preconditioner's network, trained on this GPU by the
    library's kernels on exact inverse blocks of seeded meshes (outside every
    timed region: a one-time cost, the network serves any mesh)."""
    from cutanddisplacejulia_b200 import precond
    t0 = time.perf_counter()
    meshes = precond.training_meshes(seed=0, count=args.train_meshes, n_range=(args.train_min, args.train_max))
    ts = precond.training_set(meshes, device=device)
    t1 = time.perf_counter()
    net = precond.Network(seed=0, device=device)
    hist = net.train(ts, steps=args.train_steps, batch=4096, lr=1e-3)
    t2 = time.perf_counter()
    return net, {"meshes": len(meshes), "triangles_per_mesh": [args.train_min, args.train_max], "samples": ts.rows,
                 "data_generation_s": t1 - t0, "train_s": t2 - t1, "steps": args.train_steps,
                 "loss_first_last": [hist[0], hist[-1]]}


def run_c3(args, rank, world, local_rank):
    """The 30000-unknown half-space crack (C3): the headline step is FP64
    assembly + GMRES right-preconditioned by the learned sparse approximate
    inverse to relative residual 1e-10; beside it the plain FP64 step
    (assembly + dense LU, the reference's path) and the mixed-precision step
    (FP32 far field + FP32 LU preconditioning FP64 GMRES), each timed the same
    way and compared with the FP64 LU's slip."""
    import numpy as np
    import torch
    import torch.distributed as dist

    from cutanddisplacejulia_b200 import _lib
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = workload("dipping", args.ntri)
    P1, P2, P3, nrm, mid, lam, hs, T = wl
    n = len(P1)
    n3 = 3 * n

    def col(a):
        return torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device=dev)

    dP1, dP2, dP3, dN, dM = col(P1), col(P2), col(P3), col(nrm), col(mid)
    b0 = torch.tensor(np.concatenate(T), dtype=torch.float64, device=dev)
    A = torch.empty(n3 * n3, dtype=torch.float64, device=dev)
    L = _lib.load()
    ctx = _lib.context(local_rank)
    stream = torch.cuda.ExternalStream(L.cad_get_stream(ctx), device=dev)
    torch.cuda.set_stream(stream)
    peak = ctypes.c_double(0.0)
    _lib.check(L.cad_fp64_fma_probe(ctx, 20000, ctypes.byref(peak)), ctx)
    fp64_peak = peak.value
    pairs = float(n) * n
    # launch shapes from the autotune cache (keys missing from it are timed
    # during the warm-up steps and added)
    if not args.no_autotune:
        _lib.check(L.cad_set_autotune(ctx, 1, TUNE_CACHE.encode()), ctx)

    def assemble():
        _lib.check(L.cad_assemble_dev(ctx, dN.data_ptr(), dM.data_ptr(), dP1.data_ptr(), dP2.data_ptr(),
                                      dP3.data_ptr(), n, NU, G, lam, hs, A.data_ptr(), n3), ctx)

    def timed_steps(step, nmarks, clocks=None):
        """W warm-up steps, then K steps bracketed by barrier + synchronize;
        per-step phase times from CUDA events on the library's stream."""
        for _ in range(args.warmup):
            step(None)
        torch.cuda.synchronize()
        evs = [[torch.cuda.Event(enable_timing=True) for _ in range(nmarks)] for _ in range(args.steps)]
        if clocks:
            clocks.start()
            time.sleep(0.3)
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        l0 = L.cad_kernel_launches(ctx)
        t0.record(stream)
        for k in range(args.steps):
            step(evs[k])
        t1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        clk = clocks.stop() if clocks else None
        launches = L.cad_kernel_launches(ctx) - l0
        ms = cdist.max_over_ranks(t0.elapsed_time(t1) / args.steps, dev)
        phases = [statistics.mean(e[i].elapsed_time(e[i + 1]) for e in evs) for i in range(nmarks - 1)]
        return ms, phases, launches, clk

    # the plain FP64 step: assembly + dense LU (the reference's A\b)
    x64 = torch.empty(n3, dtype=torch.float64, device=dev)

    def fp64_step(ev):
        if ev:
            ev[0].record(stream)
        assemble()
        if ev:
            ev[1].record(stream)
        x64.copy_(b0)
        _lib.check(L.cad_solve_dev(ctx, n3, A.data_ptr(), n3, x64.data_ptr(), n3, 1), ctx)
        if ev:
            ev[2].record(stream)
    with _lib.solver_mode(ctx, "lu64"):
        ms64, (asm64, sol64), _, _ = timed_steps(fp64_step, 3)
    assemble()
    Am = A.view(n3, n3).t()
    resid64 = float(torch.linalg.vector_norm(Am @ x64 - b0) / torch.linalg.vector_norm(b0))

    # the learned network (one-time training, not timed)
    net, training = train_network(args, local_rank)

    # the headline step: FP64 assembly + learned preconditioner (features,
    # network, blocks on the device) + FP64 GMRES to relative residual 1e-10
    xl = torch.empty(n3, dtype=torch.float64, device=dev)

    # the preconditioner depends on the geometry only: it is built on a second
    # stream (the context pointed at it for that call) while the matrix is
    # assembled; the solve waits for both
    side = torch.cuda.Stream(device=dev)
    fork, join = torch.cuda.Event(), torch.cuda.Event()

    def learned_step(ev):
        if ev:
            ev[0].record(stream)
        fork.record(stream)
        side.wait_event(fork)
        _lib.check(L.cad_set_stream(ctx, ctypes.c_void_p(side.cuda_stream)), ctx)
        rc = L.cad_lpc_install_dev(ctx, dP1.data_ptr(), dP2.data_ptr(), dP3.data_ptr(), n, G)
        _lib.check(L.cad_set_stream(ctx, ctypes.c_void_p(stream.cuda_stream)), ctx)
        _lib.check(rc, ctx)
        join.record(side)
        assemble()
        if ev:
            ev[1].record(stream)
        stream.wait_event(join)
        if ev:
            ev[2].record(stream)
        xl.copy_(b0)
        _lib.check(L.cad_solve_dev(ctx, n3, A.data_ptr(), n3, xl.data_ptr(), n3, 1), ctx)
        if ev:
            ev[3].record(stream)
    clocks = ClockSampler(local_rank)
    with _lib.solver_mode(ctx, "gmres_spai", MIXED_TOL, args.max_iter):
        ms, (asm_ms, setup_ms, gmres_ms), launches, clk = timed_steps(learned_step, 4, clocks)
        its, _ = _lib.last_solve_stats(ctx)
    resid = float(torch.linalg.vector_norm(Am @ xl - b0) / torch.linalg.vector_norm(b0))
    slip_err = float(torch.linalg.vector_norm(xl - x64) / torch.linalg.vector_norm(x64))
    pair_kernel_ms = L.cad_last_time_ms(ctx, 0)

    # the mixed-precision step beside it
    mixed = None if args.no_mixed else mixed_solve_timing(args, ctx, L, stream, (dN, dM, dP1, dP2, dP3, n, lam, hs),
                                                          A=A, b0=b0, x64=x64, ms_fp64=ms64, world=world, dev=dev)
    batch = None if args.batch_rhs <= 0 else batch_rhs_timing(args, ctx, L, stream, (dN, dM, dP1, dP2, dP3, n, lam,
                                                                                      hs), nrm, A, dev)
    near = None if not args.near_study else near_field_study(ctx, L, stream, (dN, dM, dP1, dP2, dP3, n, lam, hs), A,
                                                             b0, x64, [3.0, 6.0, 12.0, 24.0, 48.0])

    # end to end through the host C ABI: cad_slip_calculator in the learned
    # mode (assembly, preconditioner and GMRES inside the call), pinned host
    # geometry and tractions in, slips out
    def pinned(a):
        return torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    hP1, hP2, hP3 = (pinned(np.asfortranarray(p).ravel(order="F")) for p in (P1, P2, P3))
    hN, hM = pinned(np.asfortranarray(nrm).ravel(order="F")), pinned(np.asfortranarray(mid).ravel(order="F"))
    hTn, hTss, hTds = (pinned(t) for t in T)
    hD = [torch.zeros(n, dtype=torch.float64).pin_memory() for _ in range(3)]

    def e2e_call():
        _lib.check(L.cad_slip_calculator(ctx, hP1.data_ptr(), hP2.data_ptr(), hP3.data_ptr(), n, NU, G, lam,
                                         hM.data_ptr(), hN.data_ptr(), hs, hTn.data_ptr(), hTss.data_ptr(),
                                         hTds.data_ptr(), hD[0].data_ptr(), hD[1].data_ptr(), hD[2].data_ptr(),
                                         None, None), ctx)
    with _lib.solver_mode(ctx, "gmres_learned", MIXED_TOL, args.max_iter):
        for _ in range(max(1, args.warmup)):
            e2e_call()
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_call()
        e2e_ms = cdist.max_over_ranks((time.perf_counter() - t0) * 1e3 / args.steps, dev)
    e2e_slip = torch.cat([d.to(dev) for d in hD])
    e2e_err = float(torch.linalg.vector_norm(e2e_slip - x64) / torch.linalg.vector_norm(x64))

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        nth = os.cpu_count() or 1
        a_s, s_s, desc = cpu_reference_c3(wl, nth)
        cpu = {"value": pairs / (a_s + s_s), "unit": UNIT, "cores": nth, "kind": "port",
               "sample": desc + ": assembly %.1f s (scaled), solve %.1f s" % (a_s, s_s)}

    falg = FALG_ASSEMBLY_HS
    asm_tflops = falg * pairs / (asm_ms * 1e-3) / 1e12
    # algorithmic bytes of the solve: the FP32 copy of A (read 8, write 4
    # bytes per entry), one FP32 pass per Arnoldi product, and one FP64 pass
    # per true residual (each restart cycle and the final check)
    fp64_passes = -(-its // 30) + 1
    gmres_bytes = n3 * n3 * (12.0 + 4.0 * its + 8.0 * fp64_passes)
    gmres_gbs = gmres_bytes / (gmres_ms * 1e-3) / 1e9
    line = {
        "metric": BASELINE_METRIC, "value": cdist.replica_throughput(pairs, ms, world), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64 (network bf16)", "data": "synthetic",
        "config": {"workload": WORKLOADS["dipping"][1] % (n, n3), "pairs_per_step": pairs,
                   "step": "FP64 assembly + learned-preconditioner FP64 GMRES to relative residual 1e-10 (the "
                           "preconditioner built on a second stream during the assembly; preconditioner_setup is "
                           "the part of it left after the assembly)",
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs larger than L2 (A is %.0f MB per step)" % (n3 * n3 * 8 / 1e6)},
        "breakdown_ms": {"assembly": asm_ms, "assembly_kernels_last": pair_kernel_ms,
                         "preconditioner_setup": setup_ms, "gmres": gmres_ms},
        "gmres_iterations": its, "rel_residual": resid, "slip_rel_err_vs_fp64_lu": slip_err,
        "solve_ms_to_rel_residual_1e-10": {"learned_gmres": setup_ms + gmres_ms, "fp64_lu": sol64,
                                           "mixed": mixed["breakdown_ms"]["solve"] if mixed else None},
        "fp64": {"ms_per_step": ms64, "breakdown_ms": {"assembly": asm64, "solve_lu": sol64},
                 "rel_residual": resid64, "lu_tflops": ((2.0 / 3.0) * n3 ** 3 + 2.0 * n3 * n3) / (sol64 * 1e-3) / 1e12,
                 "step": "FP64 assembly + FP64 LU (own DMMA GEMMs, cluster panel leaves) + chained triangular solves"},
        "step_speedup_vs_fp64": ms64 / ms,
        "clocks": clk,
        "e2e": {"value": world * pairs / (e2e_ms * 1e-3), "unit": UNIT,
                "h2d_bytes_per_step": (5 * 3 * n + 3 * n) * 8, "d2h_bytes_per_step": 3 * n * 8,
                "ms_per_step": e2e_ms, "slip_rel_err_vs_fp64_lu": e2e_err,
                "api": "cad_slip_calculator, solver CAD_SOLVER_GMRES_LEARNED (host C ABI, pinned host buffers)"},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "fsc_edge_kernel + td_pair_kernel<HS, strain, A-matrix, EDGE> (the step's dominant "
                               "phase: the FP64 shared-edge half-space assembly)",
                     "bound": "fp64", "achieved": asm_tflops, "peak": fp64_peak, "unit": "TFLOP/s",
                     "frac": asm_tflops / fp64_peak,
                     "peak_source": "measured FP64 FMA throughput (cad_fp64_fma_probe, this run); "
                                    "MEASURED_PEAKS.json has no FP64 figure",
                     "falg_per_pair": falg,
                     "traffic": PAIR_TRAFFIC["dipping"][1] * (n / PAIR_TRAFFIC["dipping"][0]) ** 2,
                     "traffic_source": "ncu DRAM bytes (read + write) of the assembly's two kernels at N=%d, "
                                       "scaled by (N/%d)^2; the edge maps (18 doubles per edge and point) are "
                                       "written once and read by the triangles sharing each edge, the rest is "
                                       "the matrix" % (PAIR_TRAFFIC["dipping"][0], PAIR_TRAFFIC["dipping"][0]),
                     "falg_note": "F_alg is the reference's literal count per pair, which evaluates each "
                                  "side's free-surface correction per triangle and slip mode; the shared-edge "
                                  "path evaluates it once per edge, so the algorithmic rate exceeds the FP64 "
                                  "pipe's peak while the pipe itself is about half busy (fp64_pipe_active_ncu)",
                     "fp64_pipe_active_ncu": FP64_PIPE_ACTIVE_HS,
                     "step_share": asm_ms / ms},
        "roofline_gmres": {"kernel": "GMRES(30): FP32 copy of A, one FP32 pass over A per Arnoldi product, "
                                     "one FP64 pass per restart residual",
                           "bound": "hbm", "achieved": gmres_gbs, "peak": HBM_PEAK_GBS[0], "unit": "GB/s",
                           "frac": gmres_gbs / HBM_PEAK_GBS[0], "peak_source": HBM_PEAK_GBS[1],
                           "algorithmic_bytes": gmres_bytes, "fp64_residual_passes": fp64_passes,
                           "step_share": gmres_ms / ms},
        "cpu_baseline": cpu,
        "mixed": mixed,
        "batch_rhs": batch,
        "near_field_study": near,
        "training": training,
        "autotune": _autotune_summary(L, ctx, args),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import numpy as np
    import torch
    import torch.distributed as dist

    import cutanddisplacejulia_b200 as cad
    from cutanddisplacejulia_b200 import _lib

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    wl = workload(args.workload, args.ntri)
    P1, P2, P3, nrm, mid, lam, hs, T = wl
    n = len(P1)
    n3 = 3 * n

    def col(a):   # N x 3 -> column-major flat device array (Julia layout)
        return torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device=dev)

    dP1, dP2, dP3, dN, dM = col(P1), col(P2), col(P3), col(nrm), col(mid)
    b0 = torch.tensor(np.concatenate(T), dtype=torch.float64, device=dev)
    A = torch.empty(n3 * n3, dtype=torch.float64, device=dev)
    x = torch.empty(n3, dtype=torch.float64, device=dev)
    L = _lib.load()
    ctx = _lib.context(local_rank)
    # the library's own stream (high priority: the LU's panel chain goes ahead
    # of its look-ahead GEMMs), shared with torch for the timing events
    stream = torch.cuda.ExternalStream(L.cad_get_stream(ctx), device=dev)
    torch.cuda.set_stream(stream)

    peak = ctypes.c_double(0.0)
    _lib.check(L.cad_fp64_fma_probe(ctx, 20000, ctypes.byref(peak)), ctx)
    fp64_peak_tflops = peak.value

    def step(evs=None):
        if evs:
            evs[0].record(stream)
        _lib.check(L.cad_assemble_dev(ctx, dN.data_ptr(), dM.data_ptr(), dP1.data_ptr(), dP2.data_ptr(),
                                      dP3.data_ptr(), n, NU, G, lam, hs, A.data_ptr(), n3), ctx)
        if evs:
            evs[1].record(stream)
        x.copy_(b0)
        _lib.check(L.cad_solve_dev(ctx, n3, A.data_ptr(), n3, x.data_ptr(), n3, 1), ctx)
        if evs:
            evs[2].record(stream)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()

    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(3)] for _ in range(args.steps)]
    clocks = ClockSampler(local_rank)
    clocks.start()
    time.sleep(0.3)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    launches0 = L.cad_kernel_launches(ctx)
    t_start.record(stream)
    for k in range(args.steps):
        step(evs[k])
    t_end.record(stream)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    clk = clocks.stop()
    launches = L.cad_kernel_launches(ctx) - launches0
    ms_total = t_start.elapsed_time(t_end)
    asm_ms = statistics.mean(e[0].elapsed_time(e[1]) for e in evs)
    sol_ms = statistics.mean(e[1].elapsed_time(e[2]) for e in evs)
    pair_kernel_ms = L.cad_last_time_ms(ctx, 0)   # last pair-kernel launch alone (library events)
    ms_step = ms_total / args.steps
    ms_step = cdist.max_over_ranks(ms_step, dev)

    # solution quality: relative residual of the last solve against a fresh A
    _lib.check(L.cad_assemble_dev(ctx, dN.data_ptr(), dM.data_ptr(), dP1.data_ptr(), dP2.data_ptr(), dP3.data_ptr(),
                                  n, NU, G, lam, hs, A.data_ptr(), n3), ctx)
    Am = A.view(n3, n3).t()      # column-major storage
    resid = float(torch.linalg.vector_norm(Am @ x - b0) / torch.linalg.vector_norm(b0))

    mixed = None if args.no_mixed else mixed_solve_timing(args, ctx, L, stream, step_asm_args=(
        dN, dM, dP1, dP2, dP3, n, lam, hs), A=A, b0=b0, x64=x, ms_fp64=ms_step, world=world, dev=dev)
    batch = None if args.batch_rhs <= 0 else batch_rhs_timing(args, ctx, L, stream, (dN, dM, dP1, dP2, dP3, n, lam,
                                                                                      hs), nrm, A, dev)

    # end to end through the host C ABI: pinned host inputs, slips back to host
    def pinned(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        return t
    hP1, hP2, hP3 = (pinned(np.asfortranarray(p).ravel(order="F")) for p in (P1, P2, P3))
    hN, hM = pinned(np.asfortranarray(nrm).ravel(order="F")), pinned(np.asfortranarray(mid).ravel(order="F"))
    hTn, hTss, hTds = (pinned(t) for t in T)
    hDn, hDss, hDds = (torch.zeros(n, dtype=torch.float64).pin_memory() for _ in range(3))

    def e2e_call():
        _lib.check(L.cad_slip_calculator(ctx, hP1.data_ptr(), hP2.data_ptr(), hP3.data_ptr(), n, NU, G, lam,
                                         hM.data_ptr(), hN.data_ptr(), hs, hTn.data_ptr(), hTss.data_ptr(),
                                         hTds.data_ptr(), hDn.data_ptr(), hDss.data_ptr(), hDds.data_ptr(), None,
                                         None), ctx)

    for _ in range(max(1, args.warmup)):
        e2e_call()
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_call()
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    e2e_ms = cdist.max_over_ranks(e2e_ms, dev)
    h2d = (5 * 3 * n + 3 * n) * 8
    d2h = 3 * n * 8

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        nth = os.cpu_count() or 1
        a_s, s_s = cpu_reference_step(wl, nth)
        cpu = {"value": n * n / (a_s + s_s), "unit": UNIT, "cores": nth, "kind": "port",
               "sample": "one full step (oracle assembly + numpy LAPACK gesv) on %d host threads: "
                         "assembly %.3f s, solve %.3f s" % (nth, a_s, s_s)}

    pairs = float(n) * n
    # assembly time per step over the timed region (pair kernel + the two small
    # per-element prep kernels, all on this stream): the launch duration used
    falg = FALG_ASSEMBLY_HS if hs else FALG_ASSEMBLY_FS
    achieved = falg * pairs / (asm_ms * 1e-3) / 1e12
    lu_flops = (2.0 / 3.0) * n3 ** 3 + 2.0 * n3 * n3
    solve_tflops = lu_flops / (sol_ms * 1e-3) / 1e12
    line = {
        "metric": WORKLOADS[args.workload][0], "value": cdist.replica_throughput(pairs, ms_step, world), "unit": UNIT,
        "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload][1] % (n, n3),
                   "pairs_per_step": pairs, "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs larger than L2 (A is %.0f MB per step)" % (n3 * n3 * 8 / 1e6)},
        "breakdown_ms": {"assembly": asm_ms, "td_pair_kernel_last": pair_kernel_ms, "solve": sol_ms},
        "residual": resid,
        "clocks": clk,
        "e2e": {"value": world * pairs / (e2e_ms * 1e-3), "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "api": "cad_slip_calculator (host C ABI, pinned host buffers)"},
        "gpu_launches": int(launches),
        # the step's dominant phase is the dense solve (its largest kernel, the
        # LU panel leaf, is latency-bound: one cluster-wide pivot exchange per
        # column); the TD pair kernel is the assembly's
        "roofline": {"kernel": "dense FP64 solve: blocked LU with look-ahead (cluster leaf_lu_kernel, own row-swap "
                               "and triangular kernels, own DMMA trailing-update products) + chained triangular "
                               "solves",
                     "bound": "fp64", "achieved": solve_tflops, "peak": fp64_peak_tflops, "unit": "TFLOP/s",
                     "frac": solve_tflops / fp64_peak_tflops,
                     "peak_source": "measured FP64 FMA throughput (cad_fp64_fma_probe, this run)",
                     "work": "(2/3)(3N)^3 + 2(3N)^2 flops per solve", "traffic": None,
                     "step_share": sol_ms / ms_step},
        "dominant_kernel": {"name": "leaf_lu_kernel<double, 32, 1>",
                            "share_of_step_ncu": DOMINANT_SHARE.get(args.workload),
                            "bound": "latency: one pivot search and row exchange across a 12-16 CTA cluster per "
                                     "column (about 1.7 us per column)",
                            "source": "profiles/launches_penny2013_fp64_and_mixed_step.md",
                            "ncu_full": "profiles/leaf_lu_kernel_penny2013.md",
                            # from that capture (4856 x 32 panel): the panel read once, issue 12.8 %,
                            # FP64 pipe 2.2 %, DRAM 0.17 % of peak
                            "ncu_dram_bytes_per_launch": 1.46e6, "ncu_issue_active": 0.128,
                            "ncu_fp64_pipe": 0.022},
        "roofline_assembly": {"kernel": "td_pair_kernel<%s, strain, A-matrix>" % ("HS" if hs else "FS"),
                              "bound": "fp64", "achieved": achieved, "peak": fp64_peak_tflops, "unit": "TFLOP/s",
                              "frac": achieved / fp64_peak_tflops,
                              "peak_source": "measured FP64 FMA throughput (cad_fp64_fma_probe, this run)",
                              "falg_per_pair": falg,
                              "traffic": PAIR_TRAFFIC[args.workload][1] * (n / PAIR_TRAFFIC[args.workload][0]) ** 2,
                              "traffic_source": "ncu DRAM bytes (read + write) of one launch at "
                                                "N=%d, scaled by (N/%d)^2" % (PAIR_TRAFFIC[args.workload][0],
                                                                               PAIR_TRAFFIC[args.workload][0]),
                              "step_share": asm_ms / ms_step},
        "cpu_baseline": cpu,
        "mixed": mixed,
        "batch_rhs": batch,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


FRICTION_SPACINGS = (0.12, 0.06)   # 496 and 2013 triangles


def friction_case(spacing):
    """Penny crack under compression and shear with friction: host arrays of
    the C-ABI call (P1, P2, P3, normals, midpoints column-major; Tn, Tss, Tds,
    mu, Sf per element)."""
    import numpy as np

    from cutanddisplacejulia_b200 import geometry, workloads
    P1, P2, P3 = workloads.penny(seed=0, spacing=spacing)
    nrm, mid = geometry.CreateFaceNormalAndMidPoint(P1, P2, P3)
    _, _, lam, _, _ = geometry.ElasticConstantsCheck(G, NU)
    n = len(P1)
    r = np.hypot(mid[:, 0], mid[:, 1])
    return dict(n=n, lam=lam, P1=P1, P2=P2, P3=P3, nrm=nrm, mid=mid, Tn=np.full(n, -2e-3), Tss=np.full(n, 1e-3),
                Tds=np.zeros(n), mu=np.full(n, 0.3), Sf=2e-4 * r)


def friction_call(L, ctx, c, out):
    import numpy as np

    def f(a):
        return np.asfortranarray(a, dtype=np.float64)
    keep = [f(c[k]) for k in ("P1", "P2", "P3", "mid", "nrm")] + \
        [np.ascontiguousarray(c[k], dtype=np.float64) for k in ("Tn", "Tss", "Tds", "mu", "Sf")]
    P1, P2, P3, mid, nrm, Tn, Tss, Tds, mu, Sf = keep
    n = c["n"]
    return L.cad_slip_calculator_friction(ctx, P1.ctypes.data, P2.ctypes.data, P3.ctypes.data, n, NU, G, c["lam"],
                                          mid.ctypes.data, nrm.ctypes.data, 0, Tn.ctypes.data, Tss.ctypes.data,
                                          Tds.ctypes.data, mu.ctypes.data, Sf.ctypes.data, 1e-10, 100,
                                          out[0].ctypes.data, out[1].ctypes.data, out[2].ctypes.data)


def run_gemm(args, rank, world, local_rank):
    """The dense LU's own trailing-update product on its own: C (m x m) -= A
    (m x k) B (k x m) with k = 256 (the LU's block width), FP64 on DMMA tensor
    cores (library default and each instruction shape) and FP32 on TF32
    tcgen05 tensor cores; per-launch time from CUDA events on the library's
    stream, inputs larger than L2 (C alone is m^2 x 8 bytes)."""
    import torch

    from cutanddisplacejulia_b200 import _lib
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    L = _lib.load()
    ctx = _lib.context(local_rank)
    stream = torch.cuda.ExternalStream(L.cad_get_stream(ctx), device=dev)
    torch.cuda.set_stream(stream)
    m, k = args.gemm_m, 256
    peak = ctypes.c_double(0.0)
    _lib.check(L.cad_fp64_fma_probe(ctx, 20000, ctypes.byref(peak)), ctx)
    res = {}
    for name, prec, dt in (("fp64", 0, torch.float64), ("fp64_m8n8k4", 2, torch.float64),
                           ("fp64_m16n8k8", 3, torch.float64), ("fp64_m16n8k16", 4, torch.float64),
                           ("tf32", 1, torch.float32)):
        g = torch.Generator(device=dev).manual_seed(0)
        A = torch.rand(m * k, dtype=dt, device=dev, generator=g)
        B = torch.rand(k * m, dtype=dt, device=dev, generator=g)
        C = torch.rand(m * m, dtype=dt, device=dev, generator=g)

        def call():
            _lib.check(L.cad_gemm_sub_dev(ctx, prec, m, m, k, A.data_ptr(), m, B.data_ptr(), k, C.data_ptr(), m),
                       ctx)
        for _ in range(args.warmup):
            call()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            call()
        e1.record(stream)
        torch.cuda.synchronize()
        ms = cdist.max_over_ranks(e0.elapsed_time(e1) / args.steps, dev)
        res[name] = {"ms": ms, "tflops": 2.0 * m * m * k / (ms * 1e-3) / 1e12}
        del A, B, C
    line = {"metric": WORKLOADS["gemm"][0], "value": res["fp64"]["tflops"], "unit": "TFLOP/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["fp64"]["ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOADS["gemm"][1] % (m, m, k), "l2": "inputs larger than L2"},
            "fp64_fma_peak_tflops": peak.value, "frac_fp64": res["fp64"]["tflops"] / peak.value, "variants": res}
    if rank == 0:
        print(json.dumps(line), flush=True)


# Half-space strain + displacement per pair, both frozen oracle counts (the
# summing TD overload evaluates all three slip modes of each).
FALG_SUM_HS = 43867.0 + 6780.0
TDSUM_GRID = 100


def tdsum_case(ntri, grid=TDSUM_GRID):
    """The dipping crack with smooth seeded slip, and a grid of surface points."""
    import numpy as np

    from cutanddisplacejulia_b200 import workloads
    P1, P2, P3 = workloads.dipping_rect(seed=0, ntri=ntri)
    mid = (P1 + P2 + P3) / 3.0
    rng = np.random.default_rng(1)
    sl = np.stack([1e-3 * np.cos(0.7 * mid[:, 0] + k) * np.cos(0.9 * mid[:, 2] - k) for k in range(3)])
    sl += rng.uniform(-1e-4, 1e-4, sl.shape)
    g = np.linspace(-4.0, 4.0, grid)
    X, Y = np.meshgrid(g, g)
    return P1, P2, P3, sl, X.ravel(), Y.ravel(), np.zeros(X.size)


def run_tdsum(args, rank, world, local_rank):
    """The summing TD overload (src/TD.jl:219-410) in half space: strain and
    displacement at the free surface of a slipping dipping crack.  One step =
    one cad_td_sum_eval_dev call on device-resident inputs (the shared-edge
    path: each mesh edge's free-surface correction once, for the net Burgers
    vector of its sides); the per-side path and the host API (cad.TD with
    Strains/Disps, host arrays) are timed beside it."""
    import numpy as np
    import torch

    import cutanddisplacejulia_b200 as cad
    from cutanddisplacejulia_b200 import _lib
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    L = _lib.load()
    ctx = _lib.context(local_rank)
    stream = torch.cuda.ExternalStream(L.cad_get_stream(ctx), device=dev)
    P1, P2, P3, sl, X, Y, Z = tdsum_case(args.ntri)
    n, m = len(P1), X.size
    pairs = float(n) * m
    col = (lambda a: torch.tensor(np.asfortranarray(a).ravel(order="F"), dtype=torch.float64, device=dev))
    Xd, Yd, Zd = col(X), col(Y), col(Z)
    Pd = [col(P) for P in (P1, P2, P3)]
    Sd = [col(v) for v in sl]   # Dss, Dds, Dn
    S = torch.empty(6 * m, dtype=torch.float64, device=dev)
    U = torch.empty(3 * m, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    peak = ctypes.c_double(0.0)
    _lib.check(L.cad_fp64_fma_probe(ctx, 20000, ctypes.byref(peak)), ctx)

    def call():
        _lib.check(L.cad_td_sum_eval_dev(ctx, Xd.data_ptr(), Yd.data_ptr(), Zd.data_ptr(), m,
                                         *[p.data_ptr() for p in Pd], n, *[v.data_ptr() for v in Sd], NU, 1, 1, 1,
                                         S.data_ptr(), U.data_ptr()), ctx)

    def timed(shared, steps, clocks=None):
        _lib.check(L.cad_set_shared_edges(ctx, shared), ctx)
        for _ in range(args.warmup):
            call()
        if clocks:
            clocks.start()
            time.sleep(0.3)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()
        l0 = L.cad_kernel_launches(ctx)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            call()
        e1.record(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        clk = clocks.stop() if clocks else None
        ms = cdist.max_over_ranks(e0.elapsed_time(e1) / steps, dev)
        return ms, (L.cad_kernel_launches(ctx) - l0), torch.cat([S, U]).cpu().numpy(), clk

    ms_side, _, out_side, _ = timed(0, max(1, args.steps // 2))
    ms, launches, out, clk = timed(1, args.steps, ClockSampler(local_rank))
    kern_ms = L.cad_last_time_ms(ctx, 0)
    rel = float(np.abs(out - out_side).max() / np.abs(out_side).max())
    # end to end through the public API with host arrays
    Xh, Yh, Zh = X.copy(), Y.copy(), Z.copy()
    cad.TD(Xh, Yh, Zh, P1, P2, P3, *sl, NU, G, 1, 1, 1, cad.Strains(), cad.Disps())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        Sh, Uh = cad.TD(Xh, Yh, Zh, P1, P2, P3, *sl, NU, G, 1, 1, 1, cad.Strains(), cad.Disps())
    e2e_ms = (time.perf_counter() - t0) * 1e3 / args.steps
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import oracle as O
        O.build()
        nthreads = os.cpu_count() or 1
        pick = np.random.default_rng(7).choice(m, 300, replace=False)
        t0 = time.perf_counter()
        So, Uo = O.td_sum_eval(X[pick], Y[pick], Z[pick], P1, P2, P3, *sl, NU, G, 1, 1, 1)
        cpu_s = time.perf_counter() - t0
        got_s = out[:6 * m].reshape(6, m)[:, pick]
        got_u = out[6 * m:].reshape(3, m)[:, pick]
        err = max(float(np.abs(got_s - So).max() / np.abs(So).max()), float(np.abs(got_u - Uo).max() / np.abs(Uo).max()))
        cpu = {"value": 300.0 * n / cpu_s, "unit": UNIT, "cores": nthreads, "kind": "port",
               "sample": "oracle HS sums of all %d triangles at 300 seeded grid points (%d threads): %.1f s; "
                         "max rel err of the GPU result there %.2e" % (n, nthreads, cpu_s, err)}
    achieved = pairs * FALG_SUM_HS / (ms * 1e-3) / 1e12
    line = {
        "metric": WORKLOADS["tdsum"][0], "value": cdist.replica_throughput(pairs, ms, world), "unit": UNIT,
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS["tdsum"][1] % (n, m, TDSUM_GRID, TDSUM_GRID), "pairs_per_step": pairs,
                   "parallelism": "replicas" if world > 1 else "single",
                   "l2": "inputs and partial sums fit in L2; the step is FP64-bound, not memory-bound"},
        "breakdown_ms": {"kernels_last": kern_ms},
        "per_side": {"ms_per_step": ms_side, "value": pairs / (ms_side * 1e-3), "max_rel_diff": rel},
        "speedup_vs_per_side": ms_side / ms,
        "clocks": clk,
        "e2e": {"value": world * pairs / (e2e_ms * 1e-3), "unit": UNIT, "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": (3 * m + 9 * n + 3 * n) * 8, "d2h_bytes_per_step": 9 * m * 8,
                "api": "cad.TD(..., Strains(), Disps()) with host arrays (cad_td_sum_eval, host C ABI)"},
        "gpu_launches": int(launches),
        "roofline": {"kernel": "td_pair_kernel<HS, sum, EDGE> + fsc_sum_kernel (shared-edge half-space sums)",
                     "bound": "fp64", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                     "frac": achieved / peak.value, "falg_per_pair": FALG_SUM_HS,
                     "peak_source": "measured FP64 FMA throughput (cad_fp64_fma_probe, this run)",
                     "falg_note": "the reference's literal count per pair; the shared-edge path evaluates each "
                                  "edge's free-surface correction once instead of per side and mode",
                     "traffic": None},
        "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def run_friction(args, rank, world, local_rank):
    """Frictional slip (src/SlipCalculator3D.jl:36-238) through the C ABI with
    host buffers: one step = assembly of A, C = inv(A Scl) by the FP64 LU,
    the 5N LCP by Fischer-Burmeister Newton (one FP64 LU of the Newton
    system, reduced to 3N unknowns, per step).  Two sizes: 496 triangles (the size of the
    reference's friction test) and 2013 (the penny workload); the CPU
    baseline (oracle + numpy, all threads) on the 496-triangle case."""
    import numpy as np
    import torch

    from cutanddisplacejulia_b200 import _lib
    torch.cuda.set_device(local_rank)
    L = _lib.load()
    ctx = _lib.context(local_rank)
    sizes = []
    for sp in args.friction_spacing:
        c = friction_case(sp)
        n = c["n"]
        out = [np.zeros(n), np.zeros(n), np.zeros(n)]
        for _ in range(args.warmup):
            _lib.check(friction_call(L, ctx, c, out), ctx)
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        stream = torch.cuda.ExternalStream(L.cad_get_stream(ctx), device=torch.device("cuda", local_rank))
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        torch.cuda.synchronize()
        ev[0].record(stream)
        l0 = L.cad_kernel_launches(ctx)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            _lib.check(friction_call(L, ctx, c, out), ctx)
        wall = time.perf_counter() - t0
        ev[1].record(stream)
        torch.cuda.synchronize()
        launches = (L.cad_kernel_launches(ctx) - l0) // args.steps
        its, rel = _lib.last_solve_stats(ctx)
        dev = torch.device("cuda", local_rank)
        ms = cdist.max_over_ranks(ev[0].elapsed_time(ev[1]) / args.steps, dev)
        wall_ms = cdist.max_over_ranks(1e3 * wall / args.steps, dev)
        n3, n5 = 3 * n, 5 * n
        # inverse (LU + 3N-column solve) and one LU of the reduced 3N x 3N Newton system per step
        flops = (8.0 / 3.0) * n3 ** 3 + its * (2.0 / 3.0) * n3 ** 3
        sizes.append({"triangles": n, "lcp_unknowns": n5, "ms_per_solve": ms, "e2e_wall_ms": wall_ms,
                      "newton_steps": its, "gpu_launches_per_solve": launches,
                      "final_rel_phi": rel, "slip_max": [float(np.abs(o).max()) for o in out],
                      "fp64_lu_tflops": flops / (ms * 1e-3) / 1e12})
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import friction as F
        from oracle import oracle as O
        O.build()
        c = friction_case(max(args.friction_spacing))
        t0 = time.perf_counter()
        F.slip_calculator_friction(c["P1"], c["P2"], c["P3"], NU, G, c["lam"], c["mid"], c["nrm"], 0, c["Tn"],
                                   c["Tss"], c["Tds"], c["mu"], c["Sf"])
        cpu_s = time.perf_counter() - t0
        cpu = {"value": cpu_s * 1e3, "unit": "ms", "cores": os.cpu_count(), "kind": "port",
               "sample": "the %d-triangle case, one full solve: oracle assembly + numpy inv + numpy "
                         "Fischer-Newton (LAPACK, all threads)" % c["n"]}
    head = sizes[0]
    line = {
        "metric": WORKLOADS["friction"][0], "value": head["ms_per_solve"], "unit": "ms", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_solve"], "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS["friction"][1] % (head["triangles"], head["lcp_unknowns"]),
                   "inputs": "host memory (C ABI, copies inside the timed region)"},
        "sizes": sizes, "cpu_baseline": cpu, "gpu_launches": head["gpu_launches_per_solve"] * args.steps,
        "e2e": {"value": head["e2e_wall_ms"], "unit": "ms", "h2d_bytes_per_step": 8 * 25 * head["triangles"],
                "d2h_bytes_per_step": 8 * 3 * head["triangles"]},
    }
    if rank == 0:
        print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-precision solve of the same system")
    ap.add_argument("--no-autotune", action="store_true", help="fixed launch shapes instead of the autotune cache")
    ap.add_argument("--near-study", action="store_true",
                    help="dipping: mixed assembly with the FP64 near field at 3-48 mean edge lengths (slip errors)")
    ap.add_argument("--batch-rhs", type=int, default=0,
                    help="also time K seeded remote-stress right-hand sides on the same system (FP64 LU and mixed)")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="dipping",
                    help="dipping (default): the 30000-unknown half-space crack, learned-preconditioner step with "
                         "the FP64 and mixed steps beside it; penny: the full-space penny crack (N~2000)")
    ap.add_argument("--ntri", type=int, default=10000, help="triangles of the dipping crack")
    ap.add_argument("--friction-spacing", type=float, nargs="+", default=list(FRICTION_SPACINGS),
                    help="lattice spacings of the friction workload's penny cracks (0.12: 496 triangles)")
    ap.add_argument("--cracks", type=int, default=512, help="cracks of the batch workload")
    ap.add_argument("--gemm-m", type=int, default=16384, help="rows and columns of the gemm workload's C")
    ap.add_argument("--eager", action="store_true",
                    help="batch: issue every launch directly instead of replaying the captured graph (for profilers)")
    ap.add_argument("--train-meshes", type=int, default=32, help="training meshes of the learned preconditioner")
    ap.add_argument("--train-min", type=int, default=500, help="smallest training mesh (triangles)")
    ap.add_argument("--train-max", type=int, default=2000, help="largest training mesh (triangles)")
    ap.add_argument("--train-steps", type=int, default=3000, help="training steps of the learned workload")
    ap.add_argument("--max-iter", type=int, default=3000, help="GMRES iteration cap of the learned workload")
    ap.add_argument("--shared-edges", type=int, choices=[0, 1], default=1,
                    help="half-space free-surface corrections once per mesh edge (1, the library default) or per "
                         "triangle side (0, the reference's order of work); cad_set_shared_edges")
    args = ap.parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    if args.shared_edges != 1:
        from cutanddisplacejulia_b200 import _lib
        ctx = _lib.context(local_rank)
        _lib.check(_lib.load().cad_set_shared_edges(ctx, args.shared_edges), ctx)
    try:
        if args.workload == "batch":
            run_batch(args, rank, world, local_rank)
        elif args.workload == "learned":
            run_learned(args, rank, world, local_rank)
        elif args.workload == "friction":
            run_friction(args, rank, world, local_rank)
        elif args.workload == "gemm":
            run_gemm(args, rank, world, local_rank)
        elif args.workload == "tdsum":
            run_tdsum(args, rank, world, local_rank)
        elif args.workload == "dipping":
            run_c3(args, rank, world, local_rank)
        else:
            run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
