"""ctypes binding of libcad_td.so (the C ABI declared in include/cad_td.h).

The library must be built (cutanddisplacejulia_b200.build.build()); there is
no CPU fallback: every call goes to the CUDA library or raises.
"""
from __future__ import annotations

import ctypes
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcad_td.so")

CAD_OK = 0
CAD_ERR_DIMS = 1
CAD_ERR_HS_ABOVE_SURFACE = 2
CAD_ERR_UNSUPPORTED = 3
CAD_ERR_CUDA = 4
CAD_ERR_OOM = 5
CAD_ERR_TIMEOUT = 6
CAD_ERR_NOT_CONVERGED = 7
CAD_ERR_SINGULAR = 8
CAD_ERR_ARG = 9
CAD_ERR_TOO_LARGE = 10
CAD_SOLVER_LU64 = 0
CAD_SOLVER_MIXED = 1
CAD_SOLVER_GMRES_SPAI = 2
CAD_SOLVER_GMRES_LEARNED = 3
CAD_SOLVER_GMRES_BLOCK_JACOBI = 4
CAD_SOLVER_GMRES = 5
CAD_ASSEMBLY_FP64 = 0
CAD_ASSEMBLY_MIXED = 1

# Every symbol include/cad_td.h declares (checked by the tests).
EXPORTS = [
    "cad_init", "cad_destroy", "cad_last_error", "cad_set_stream", "cad_get_stream", "cad_last_time_ms",
    "cad_version", "cad_kernel_launches", "cad_set_assembly", "cad_set_solver", "cad_last_solve_stats", "cad_fp64_fma_probe", "cad_td_inf", "cad_td_sum_eval", "cad_td_sum", "cad_influence_traction",
    "cad_slip_calculator", "cad_slip_calculator_fixed", "cad_solve", "cad_td_inf_dev", "cad_td_sum_eval_dev", "cad_assemble_dev", "cad_assemble_update_dev",
    "cad_solve_dev", "cad_set_preconditioner", "cad_block_jacobi_dev", "cad_lpc_param_count", "cad_lpc_step",
    "cad_slip_calculator_batched", "cad_slip_calculator_batched_dev", "cad_td_sum_eval_noalloc",
    "cad_slip_calculator_friction", "cad_fischer_newton", "cad_friction_prepare", "cad_friction_solve",
    "cad_assemble_columns_dev", "cad_gemm_sub_dev", "cad_lpc_features_dev", "cad_lpc_set_network",
    "cad_lpc_get_network", "cad_lpc_dataset_add", "cad_lpc_dataset_rows", "cad_lpc_dataset_clear",
    "cad_lpc_dataset_get", "cad_lpc_dataset_set", "cad_lpc_forward_backward", "cad_lpc_train", "cad_lpc_install_dev",
    "cad_lpc_install", "cad_set_wait_limit", "cad_wait_timeout_probe", "cad_set_gmres_matvec", "cad_set_batch_solve",
    "cad_set_lu_block", "cad_set_gmres_restart", "cad_set_shared_edges",
    "cad_set_autotune", "cad_autotune_entries",
]


class CadError(RuntimeError):
    """Error raised by the library (message text follows the reference's `error(...)`)."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


_lib = None
_lock = threading.Lock()
_ctx = {}

P = ctypes.c_void_p
I64 = ctypes.c_int64
D = ctypes.c_double
INT = ctypes.c_int


def load():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CadError(CAD_ERR_CUDA, f"libcad_td.so is not built ({LIB_PATH}); run cutanddisplacejulia_b200.build.build()")
    L = ctypes.CDLL(LIB_PATH)
    L.cad_init.argtypes = [INT, ctypes.POINTER(P)]
    L.cad_destroy.argtypes = [P]
    L.cad_last_error.argtypes = [P]
    L.cad_last_error.restype = ctypes.c_char_p
    L.cad_set_stream.argtypes = [P, P]
    L.cad_get_stream.argtypes = [P]
    L.cad_get_stream.restype = P
    L.cad_last_time_ms.argtypes = [P, INT]
    L.cad_last_time_ms.restype = D
    L.cad_version.restype = ctypes.c_char_p
    L.cad_kernel_launches.argtypes = [P]
    L.cad_kernel_launches.restype = I64
    L.cad_set_solver.argtypes = [P, INT, D, INT]
    L.cad_set_assembly.argtypes = [P, INT, D]
    L.cad_last_solve_stats.argtypes = [P, ctypes.POINTER(INT), ctypes.POINTER(D)]
    L.cad_fp64_fma_probe.argtypes = [P, I64, ctypes.POINTER(D)]
    td = [P, P, P, P, I64, P, P, P, I64, P, P, P, D, D, INT, INT, INT, P, P]
    L.cad_td_inf.argtypes = td
    L.cad_td_sum_eval.argtypes = td
    L.cad_td_sum.argtypes = [P, I64, I64, P, P, P, P]
    L.cad_influence_traction.argtypes = [P, P, P, P, P, P, I64, D, D, D, P, INT, P]
    L.cad_slip_calculator.argtypes = [P, P, P, P, I64, D, D, D, P, P, INT, P, P, P, P, P, P, P, P]
    L.cad_solve.argtypes = [P, I64, P, P, I64, P]
    L.cad_slip_calculator_fixed.argtypes = [P, P, P, P, I64, D, D, D, P, P, INT, P, P, P, P, P, P, P, P, P]
    tdd = [P, P, P, P, I64, P, P, P, I64, P, P, P, D, INT, INT, INT, P, P]
    L.cad_td_inf_dev.argtypes = tdd
    L.cad_td_sum_eval_dev.argtypes = tdd
    L.cad_assemble_dev.argtypes = [P, P, P, P, P, P, I64, D, D, D, INT, P, I64]
    L.cad_assemble_update_dev.argtypes = [P, P, P, P, P, P, I64, D, D, D, INT, P, I64, P, I64]
    L.cad_solve_dev.argtypes = [P, I64, P, I64, P, I64, I64]
    L.cad_slip_calculator_batched_dev.argtypes = [P, I64, P, P, P, P, P, P, D, D, D, INT, P, P, P]
    L.cad_slip_calculator_batched.argtypes = [P, I64, P, P, P, P, P, P, D, D, D, INT, P, P, P]
    L.cad_set_preconditioner.argtypes = [P, I64, INT, P, P]
    L.cad_block_jacobi_dev.argtypes = [P, I64, P, I64, P, P]
    L.cad_lpc_param_count.restype = I64
    L.cad_lpc_step.argtypes = [P, P, P, P, I64, P, P, P, P, P, I64, ctypes.c_float]
    L.cad_td_sum_eval_noalloc.argtypes = [P, P, P, P, I64, P, P, P, I64, P, P, P, D, INT, INT, INT, P, P]
    L.cad_slip_calculator_friction.argtypes = [P, P, P, P, I64, D, D, D, P, P, INT, P, P, P, P, P, D, INT, P, P, P]
    L.cad_fischer_newton.argtypes = [P, I64, P, P, D, INT, P]
    L.cad_assemble_columns_dev.argtypes = [P, P, P, P, P, P, I64, D, D, D, INT, I64, I64, P, I64]
    L.cad_gemm_sub_dev.argtypes = [P, INT, I64, I64, I64, P, I64, P, I64, P, I64]
    L.cad_lpc_features_dev.argtypes = [P, P, P, P, I64, P, P, P]
    L.cad_lpc_set_network.argtypes = [P, P]
    L.cad_lpc_get_network.argtypes = [P, P]
    L.cad_lpc_dataset_add.argtypes = [P, P, P, P, I64, D, D, D, P, P, INT]
    L.cad_lpc_dataset_rows.argtypes = [P]
    L.cad_lpc_dataset_rows.restype = I64
    L.cad_lpc_dataset_clear.argtypes = [P]
    L.cad_lpc_dataset_get.argtypes = [P, I64, I64, P, P]
    L.cad_lpc_dataset_set.argtypes = [P, P, P, I64]
    L.cad_lpc_forward_backward.argtypes = [P, P, P, I64, P, P, P]
    L.cad_lpc_train.argtypes = [P, I64, I64, ctypes.c_float, ctypes.c_uint64, P]
    L.cad_lpc_install_dev.argtypes = [P, P, P, P, I64, D]
    L.cad_lpc_install.argtypes = [P, P, P, P, I64, D]
    L.cad_set_wait_limit.argtypes = [P, I64]
    L.cad_set_gmres_matvec.argtypes = [P, INT]
    L.cad_set_batch_solve.argtypes = [P, INT]
    L.cad_set_lu_block.argtypes = [P, INT]
    L.cad_set_gmres_restart.argtypes = [P, INT]
    L.cad_set_shared_edges.argtypes = [P, INT]
    L.cad_set_autotune.argtypes = [P, INT, ctypes.c_char_p]
    L.cad_autotune_entries.argtypes = [P, ctypes.POINTER(I64)]
    L.cad_autotune_entries.restype = I64
    L.cad_wait_timeout_probe.argtypes = [P, I64]
    L.cad_friction_prepare.argtypes = [P, P, P, P, I64, D, D, D, P, P, INT]
    L.cad_friction_solve.argtypes = [P, I64, P, P, P, P, P, D, INT, P, P, P]
    _lib = L
    return L


def context(device: int = 0):
    """Process-wide context for `device` (created on first use)."""
    with _lock:
        if device not in _ctx:
            L = load()
            h = P()
            rc = L.cad_init(device, ctypes.byref(h))
            if rc != CAD_OK:
                raise CadError(rc, f"cad_init failed on device {device} (status {rc}); a CUDA device is required")
            _ctx[device] = h
        return _ctx[device]


def check(rc, ctx):
    if rc != CAD_OK:
        msg = load().cad_last_error(ctx)
        raise CadError(rc, msg.decode() if msg else f"status {rc}")


def ptr_array(arrays):
    """double* const* from a list of numpy arrays (None -> NULL)."""
    arr = (P * len(arrays))()
    for k, a in enumerate(arrays):
        arr[k] = None if a is None else a.ctypes.data
    return arr


class solver_mode:
    """Context manager selecting the dense solver of `ctx` for the calls inside it
    ("lu64": FP64 LU as the reference's A\\b; "mixed": FP32/TF32 LU preconditioning
    FP64 GMRES to relative residual `tol`; "gmres_spai": FP64 GMRES with the
    installed block-sparse preconditioner; "gmres_learned": the same, the
    network's preconditioner installed by cad_slip_calculator for its mesh;
    "gmres_block_jacobi" / "gmres": element-block Jacobi / no preconditioner),
    restoring the FP64 LU afterwards."""

    def __init__(self, ctx, solver="lu64", tol=1e-10, max_iter=200):
        modes = {"lu64": CAD_SOLVER_LU64, "mixed": CAD_SOLVER_MIXED, "gmres_spai": CAD_SOLVER_GMRES_SPAI,
                 "gmres_learned": CAD_SOLVER_GMRES_LEARNED, "gmres_block_jacobi": CAD_SOLVER_GMRES_BLOCK_JACOBI,
                 "gmres": CAD_SOLVER_GMRES}
        if solver not in modes:
            raise ValueError("solver must be one of " + ", ".join(sorted(modes)))
        self.ctx, self.mode, self.tol, self.max_iter = ctx, modes[solver], float(tol), int(max_iter)

    def __enter__(self):
        check(load().cad_set_solver(self.ctx, self.mode, self.tol, self.max_iter), self.ctx)
        return self

    def __exit__(self, *exc):
        load().cad_set_solver(self.ctx, CAD_SOLVER_LU64, 1e-10, 200)
        return False


class assembly_mode:
    """Context manager selecting the system-matrix assembly precision of `ctx`
    ("fp64": every pair in FP64; "mixed": far-field pairs in FP32, pairs within
    `near_factor` mean edge lengths in FP64), restoring FP64 afterwards."""

    def __init__(self, ctx, assembly="fp64", near_factor=3.0):
        modes = {"fp64": CAD_ASSEMBLY_FP64, "mixed": CAD_ASSEMBLY_MIXED}
        if assembly not in modes:
            raise ValueError("assembly must be 'fp64' or 'mixed'")
        self.ctx, self.mode, self.near_factor = ctx, modes[assembly], float(near_factor)

    def __enter__(self):
        check(load().cad_set_assembly(self.ctx, self.mode, self.near_factor), self.ctx)
        return self

    def __exit__(self, *exc):
        load().cad_set_assembly(self.ctx, CAD_ASSEMBLY_FP64, 3.0)
        return False


def last_solve_stats(ctx):
    """(GMRES iterations, final relative residual) of the last mixed solve on `ctx`."""
    it, rr = ctypes.c_int(0), ctypes.c_double(0.0)
    check(load().cad_last_solve_stats(ctx, ctypes.byref(it), ctypes.byref(rr)), ctx)
    return it.value, rr.value
