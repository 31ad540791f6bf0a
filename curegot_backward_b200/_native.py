"""ctypes binding of the C ABI in ``include/curegot_b200.h``.

The shared library is the product: there is no CPU fallback.  Loading fails
loudly when the library is missing, and every call that needs a GPU raises
when CUDA is unavailable.
"""

from __future__ import annotations

import ctypes
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libcuregot_b200.so")

CG_OK = 0
CG_ERR_INVALID_ARG = 1
CG_ERR_CUDA = 2
CG_ERR_NOT_SPD = 3
CG_ERR_OOM = 4
CG_ERR_TIMEOUT = 5
CG_ERR_NONFINITE = 6
CG_ERR_INVALID_CONTEXT = 7
CG_ERR_SOLVER = 8
CG_ERR_ADMISSION = 9
CG_ERR_CANCELLED = 10
CG_INJECT_DIRECTION_SOLVE = 1
CG_POINTS_FP64 = 0
CG_POINTS_MIXED = 1

_STATUS_NAMES = {
    CG_ERR_INVALID_ARG: "invalid argument",
    CG_ERR_CUDA: "CUDA error",
    CG_ERR_NOT_SPD: "direction-solve factorization failed (matrix not SPD)",
    CG_ERR_OOM: "out of device memory",
    CG_ERR_TIMEOUT: "bounded device wait expired",
    CG_ERR_NONFINITE: "non-finite state",
    CG_ERR_INVALID_CONTEXT: "invalid backward context",
    CG_ERR_SOLVER: "linear solver error",
    CG_ERR_ADMISSION: "request exceeds the engine's HBM budget",
    CG_ERR_CANCELLED: "request cancelled",
}

_lib = None
_lock = threading.Lock()

c_int, c_double, c_void_p, c_long = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_long
c_size_t = ctypes.c_size_t
c_int_p = ctypes.POINTER(ctypes.c_int)
c_ll_p = ctypes.POINTER(ctypes.c_longlong)
c_void_pp = ctypes.POINTER(ctypes.c_void_p)


class CtxInfo(ctypes.Structure):
    """cg_ctx_info_t of include/curegot_b200.h."""
    _fields_ = [("n", ctypes.c_int), ("m", ctypes.c_int), ("dim", ctypes.c_int),
                ("nnz", ctypes.c_longlong), ("reg", ctypes.c_double), ("ys", ctypes.c_double),
                ("low_rank", ctypes.c_int), ("fallback", ctypes.c_int), ("valid", ctypes.c_int),
                ("has_diag", ctypes.c_int), ("has_point", ctypes.c_int),
                ("adopted", ctypes.c_int)]


class Request(ctypes.Structure):
    """cg_request_t."""
    _fields_ = [("algo", ctypes.c_int), ("n", ctypes.c_int), ("m", ctypes.c_int),
                ("m_f32", ctypes.c_int), ("host_inputs", ctypes.c_int),
                ("max_iter", ctypes.c_int), ("eta", ctypes.c_double), ("tol", ctypes.c_double),
                ("M", ctypes.c_void_p), ("a", ctypes.c_void_p), ("b", ctypes.c_void_p),
                ("dual_out", ctypes.c_void_p), ("tag", ctypes.c_uint64)]


class Result(ctypes.Structure):
    """cg_result_t."""
    _fields_ = [("id", ctypes.c_uint64), ("tag", ctypes.c_uint64), ("status", ctypes.c_int),
                ("niter", ctypes.c_int), ("converged", ctypes.c_int),
                ("fast_iters", ctypes.c_int), ("last_err", ctypes.c_double),
                ("t_submit", ctypes.c_double), ("t_admit", ctypes.c_double),
                ("t_done", ctypes.c_double)]


class EngineStats(ctypes.Structure):
    """cg_engine_stats_t."""
    _fields_ = [("in_use_bytes", ctypes.c_size_t), ("budget_bytes", ctypes.c_size_t),
                ("queued", ctypes.c_longlong), ("active_bcd", ctypes.c_longlong),
                ("active_splr", ctypes.c_longlong), ("completed", ctypes.c_longlong),
                ("bcd_bytes", ctypes.c_double), ("bcd_gpu_ms", ctypes.c_double),
                ("chunks", ctypes.c_longlong), ("graph_builds", ctypes.c_longlong)]


CG_ALGO_BCD, CG_ALGO_SPLR = 0, 1
CG_PRECOND_NONE, CG_PRECOND_DIAG, CG_PRECOND_SPLR = 0, 1, 2
(CG_CTX_CSR_VALUES, CG_CTX_CSR_COLIND, CG_CTX_CSR_ROWPTR, CG_CTX_SECANT_S, CG_CTX_SECANT_Y,
 CG_CTX_INV_DIAG, CG_CTX_POINT, CG_CTX_INVA_Y) = range(8)
_SPLR_ARGS = [c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_int, c_double, c_int, c_int,
              c_int_p, c_double, c_double, c_int, c_int, c_int, c_void_p, c_void_p, c_void_pp,
              c_int_p, c_void_p, c_void_p]

# name -> argtypes (every exported entry point of include/curegot_b200.h)
SIGNATURES = {
    "cg_last_error": [],
    "cg_version": [],
    "cg_launch_count": [],
    "cg_launch_count_reset": [],
    "cg_memory_pool": [c_int, c_void_pp],
    "cg_memory_pool_trim": [c_int, c_size_t],
    "cg_bcd_f64": [c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_int, c_double, c_int,
                   c_int, c_int_p, c_void_p, c_void_p, c_void_p],
    "cg_bcd_f64_noalloc": [c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_int, c_double,
                           c_int, c_int, c_int_p, c_void_p, c_void_p, c_void_p],
    "cg_bcd_set_cluster_path": [c_int],
    "cg_bcd_set_staging": [c_int],
    "cg_bcd_set_l2_prefetch": [c_int],
    "cg_bcd_set_shifted_lse": [c_int],
    "cg_points_cost_bf16": [c_void_p, c_void_p, c_int, c_int, c_int, c_double, c_void_p, c_void_p],
    "cg_bcd_points_bf16": [c_void_p, c_void_p, c_int, c_int, c_int, c_double, c_void_p, c_void_p,
                           c_double, c_int, c_double, c_int, c_int_p, c_void_p, c_int_p,
                           c_void_p],
    "cg_points_set_wait_limit": [ctypes.c_longlong],
    "cg_points_cost_stats_bf16": [c_void_p, c_void_p, c_int, c_int, c_int, c_void_p, c_void_p,
                                  c_void_p],
    "cg_bcd_mixed": [c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_int, c_double, c_int,
                     c_int, c_int_p, c_void_p, c_void_p, c_void_p],
    "cg_transport_plan_f64": [c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_int, c_int,
                              c_void_p],
    "cg_transport_plan_mixed": [c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_int, c_int,
                                c_void_p],
    "cg_diag_exp2": [c_void_p, c_void_p, c_int, c_int, c_void_p],
    "cg_splr_f64": _SPLR_ARGS,
    "cg_splr_mixed": _SPLR_ARGS,
    "cg_splr_set_direction_solver": [c_int],
    "cg_splr_last_direction_solver": [],
    "cg_ctx_info": [c_void_p, ctypes.POINTER(CtxInfo)],
    "cg_ctx_setup_diag": [c_void_p, c_void_p],
    "cg_ctx_apply": [c_void_p, c_void_p, c_void_p, c_int, c_void_p],
    "cg_ctx_copy": [c_void_p, c_int, c_void_p, c_void_p],
    "cg_ctx_destroy": [c_void_p],
    "cg_backward_f64": [c_void_p, c_void_p, c_void_p, c_double, c_int, c_double, c_int, c_int,
                        c_int, c_void_p, c_void_p, c_int_p, c_int_p, c_void_p],
    "cg_backward_batch_f64": [c_void_p, c_void_p, c_void_p, c_double, c_int, c_double, c_int,
                              c_int, c_int, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                              c_void_p],
    "cg_t_values_f64": [c_void_p, c_void_p, c_void_p, c_int, c_int, c_double, c_void_p,
                        c_void_p, c_void_p],
    "cg_test_t_sparsify_f64": [c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_double,
                               c_double, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p,
                               c_void_p, c_void_p, c_void_p, c_void_p, c_ll_p, c_void_p],
    "cg_test_spd_solve_f64": [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p,
                              c_void_p],
    "cg_engine_create": [c_size_t, c_int, c_int, c_int, c_void_pp],
    "cg_engine_submit": [c_void_p, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)],
    "cg_engine_poll": [c_void_p, ctypes.POINTER(Result), c_int, c_int, c_int_p],
    "cg_engine_stats": [c_void_p, ctypes.POINTER(EngineStats)],
    "cg_engine_cancel": [c_void_p, ctypes.c_uint64],
    "cg_test_inject_failure": [c_int, c_int],
    "cg_engine_clock": [],
    "cg_engine_destroy": [c_void_p],
}
RESTYPES = {"cg_last_error": ctypes.c_char_p, "cg_version": ctypes.c_char_p,
            "cg_engine_clock": ctypes.c_double, "cg_launch_count": ctypes.c_longlong,
            "cg_launch_count_reset": None}


class CuregotError(RuntimeError):
    """A native entry point returned a non-zero status."""

    def __init__(self, fn: str, status: int, detail: str):
        self.status = status
        super().__init__(f"{fn}: {_STATUS_NAMES.get(status, 'error')} (status {status})"
                         + (f": {detail}" if detail else ""))


def lib():
    """Load the native library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise ImportError(
                    f"curegot_backward_b200: native library not found at {LIB_PATH}; "
                    "build it with `python -m curegot_backward_b200.build`")
            L = ctypes.CDLL(LIB_PATH)
            for name, args in SIGNATURES.items():
                f = getattr(L, name)
                f.argtypes = args
                f.restype = RESTYPES.get(name, ctypes.c_int)
            _lib = L
    return _lib


def check(fn: str, status: int) -> None:
    if status != CG_OK:
        detail = lib().cg_last_error()
        raise CuregotError(fn, status, detail.decode() if detail else "")


def call(fn: str, *args) -> None:
    check(fn, getattr(lib(), fn)(*args))
