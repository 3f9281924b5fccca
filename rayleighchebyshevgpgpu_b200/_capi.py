"""ctypes binding of librcb200.so (include/rc_b200.h).

The shared library is built in-tree (``python -m rayleighchebyshevgpgpu_b200.build``). Loading
fails loudly when it is missing: there is no CPU fallback for any entry point.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "librcb200.so")

RC_OK = 0
STATUS_NAMES = {
    0: "RC_OK", 1: "RC_ERR_INVALID", 2: "RC_ERR_CUDA", 3: "RC_ERR_NOMEM", 4: "RC_ERR_NOT_HERMITIAN",
    5: "RC_ERR_BREAKDOWN", 6: "RC_ERR_TIMEOUT", 7: "RC_ERR_CANCELLED", 8: "RC_ERR_UNSUPPORTED",
    9: "RC_ERR_CALLBACK", 10: "RC_ERR_NOT_READY",
}
RC_REAL64, RC_COMPLEX128 = 0, 1
RC_PREC_FP64, RC_PREC_MIXED = 0, 1
RC_STOP_DEFAULT, RC_STOP_COMBINATION, RC_STOP_EIGENVALUE_ONLY, RC_STOP_RESIDUAL_ONLY = 0, 1, 2, 3
RC_STENCIL_5PT_2D, RC_STENCIL_7PT_3D, RC_STENCIL_27PT_3D = 5, 7, 27

c_i64 = C.c_int64
c_dp = C.POINTER(C.c_double)
c_vp = C.c_void_p

RANDOMIZE_FN = C.CFUNCTYPE(None, c_vp, c_vp, c_i64, c_i64)
BLOCK_APPLY_FN = C.CFUNCTYPE(C.c_int, c_vp, c_vp, c_vp, c_i64, c_i64, c_i64, c_dp, c_dp, c_vp)


class SolveParams(C.Structure):
    _fields_ = [
        ("struct_size", C.c_size_t),
        ("eig_count", c_i64),
        ("tol", C.c_double),
        ("subspace_increment", c_i64),
        ("buffer_size", c_i64),
        ("stop_condition", C.c_int),
        ("precision", C.c_int),
        ("poly_degree_max", c_i64),
        ("filter_repetition", c_i64),
        ("max_inner_loop", c_i64),
        ("max_min_tol", C.c_double),
        ("lanczos_max_iter", c_i64),
        ("mode", C.c_int),
        ("min_eig_est", C.c_double),
        ("max_eig_bound", C.c_double),
        ("lambda_max", C.c_double),
        ("host_buffers", C.c_int),
        ("non_random_start", C.c_int),
        ("v0_cols", c_i64),
        ("seed", C.c_uint64),
        ("randomize_fn", RANDOMIZE_FN),
        ("randomize_user", c_vp),
        ("lanczos_v0", c_vp),
        ("mixed_switch_tol", C.c_double),
        ("verbose", C.c_int),
        ("phase_timing", C.c_int),
        ("orth_mode", C.c_int),
        ("mixed_refine", C.c_int),
    ]


class SolveInfo(C.Structure):
    _fields_ = [
        ("struct_size", C.c_size_t),
        ("found", c_i64),
        ("inner_iterations", c_i64),
        ("outer_passes", c_i64),
        ("degree_steps", c_i64),
        ("fp64_degree_steps", c_i64),
        ("mixed_iterations", c_i64),
        ("lanczos_iterations", c_i64),
        ("cholqr_passes", c_i64),
        ("min_eig_est", C.c_double),
        ("max_eig_est", C.c_double),
        ("max_residual", C.c_double),
        ("max_eig_diff", C.c_double),
        ("max_rel_gap", C.c_double),
        ("count_ortho", c_i64),
        ("count_opapply", c_i64),
        ("count_eigenvalue", c_i64),
        ("time_total_ms", C.c_double),
        ("time_lanczos_ms", C.c_double),
        ("time_filter_ms", C.c_double),
        ("time_ortho_ms", C.c_double),
        ("time_eigenvalue_ms", C.c_double),
        ("kernel_launches", c_i64),
        ("guard_value", C.c_double),
        ("fused_rr", c_i64),
        ("fused_rr_fallbacks", c_i64),
        ("time_filter_steps_ms", C.c_double),
        ("correction_iterations", c_i64),
        ("correction_degree_steps", c_i64),
        ("correction_element_bytes", c_i64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "struct_size"}


class ServerParams(C.Structure):
    _fields_ = [
        ("struct_size", C.c_size_t),
        ("device", C.c_int),
        ("hbm_budget_bytes", c_i64),
        ("max_active", C.c_int),
        ("batch_window_us", C.c_double),
        ("use_graphs", C.c_int),
        ("starvation_ms", C.c_double),
    ]


class CorrectionJob(C.Structure):
    _fields_ = [
        ("struct_size", C.c_size_t),
        ("op", c_vp),
        ("V", c_vp),
        ("ld", c_i64),
        ("s", c_i64),
        ("lam", c_vp),
        ("degree", c_i64),
        ("gamma1", C.c_double),
        ("gamma2", C.c_double),
    ]


RC_REQ_QUEUED, RC_REQ_RUNNING, RC_REQ_DONE, RC_REQ_FAILED, RC_REQ_CANCELLED = 0, 1, 2, 3, 4
REQ_STATE_NAMES = {0: "queued", 1: "running", 2: "done", 3: "failed", 4: "cancelled"}


class RequestInfo(C.Structure):
    _fields_ = [
        ("struct_size", C.c_size_t),
        ("state", C.c_int),
        ("status", C.c_int),
        ("queue_ms", C.c_double),
        ("run_ms", C.c_double),
        ("latency_ms", C.c_double),
        ("batches", c_i64),
        ("reserved_bytes", c_i64),
        ("device_bytes", c_i64),
    ]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "struct_size"}


class ServerStats(C.Structure):
    _fields_ = [("struct_size", C.c_size_t)] + [(name, c_i64) for name in (
        "submitted", "completed", "failed", "cancelled", "queued", "running", "batches", "batched_jobs",
        "max_jobs_in_batch", "graph_launches", "graphs_built", "kernel_launches", "bytes_in_use", "bytes_peak",
        "budget")]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "struct_size"}


# Every symbol the header declares, with (restype, argtypes).
SIGNATURES = {
    "rc_abi_version": (C.c_int, []),
    "rc_ctx_create": (C.c_int, [C.c_int, C.POINTER(c_vp)]),
    "rc_ctx_destroy": (C.c_int, [c_vp]),
    "rc_ctx_last_error": (C.c_char_p, [c_vp]),
    "rc_ctx_set_stream": (C.c_int, [c_vp, c_vp]),
    "rc_ctx_synchronize": (C.c_int, [c_vp]),
    "rc_ctx_launch_count": (C.c_int, [c_vp, C.POINTER(c_i64), C.c_int]),
    "rc_ctx_device_bytes": (C.c_int, [c_vp, C.POINTER(c_i64)]),
    "rc_ctx_counter": (C.c_int, [c_vp, C.c_char_p, C.POINTER(c_i64)]),
    "rc_op_csr_create": (C.c_int, [c_vp, C.c_int, c_i64, c_i64, c_vp, c_vp, c_vp, C.POINTER(c_vp)]),
    "rc_op_stencil_create": (C.c_int, [c_vp, C.c_int, C.c_int, c_i64, c_i64, c_i64, c_vp, C.c_double,
                                       C.c_double, C.POINTER(c_vp)]),
    "rc_op_callback_create": (C.c_int, [c_vp, C.c_int, c_i64, BLOCK_APPLY_FN, c_vp, C.POINTER(c_vp)]),
    "rc_op_destroy": (C.c_int, [c_vp]),
    "rc_op_dim": (C.c_int, [c_vp, C.POINTER(c_i64), C.POINTER(C.c_int)]),
    "rc_cpoly_xstar": (C.c_int, [c_i64, c_dp, c_dp]),
    "rc_cpoly_star_degree": (C.c_int, [C.c_double, C.c_double, C.c_double, c_i64, C.POINTER(c_i64), c_dp]),
    "rc_cpoly_gammas": (C.c_int, [c_i64, C.c_double, C.c_double, c_dp, c_dp]),
    "rc_cpoly_pm": (C.c_double, [c_i64, C.c_double]),
    "rc_spmm": (C.c_int, [c_vp, c_vp, c_vp, c_i64, c_vp, c_i64, c_i64, c_dp, c_dp]),
    "rc_filter": (C.c_int, [c_vp, c_vp, c_vp, c_i64, c_i64, c_i64, c_i64, C.c_double, C.c_double, C.c_int]),
    "rc_rm_leading_dim": (c_i64, [C.c_int, C.c_int, c_i64]),
    "rc_filter_step_rm": (C.c_int, [c_vp, c_vp, c_vp, c_vp, c_vp, c_i64, c_i64, c_dp, c_dp, c_dp, C.c_int]),
    "rc_filter_correction": (C.c_int, [c_vp, c_vp, c_vp, c_i64, c_i64, c_dp, c_i64, C.c_double, C.c_double]),
    "rc_filter_correction_batch": (C.c_int, [c_vp, C.c_int, C.POINTER(CorrectionJob), C.POINTER(C.c_int)]),
    "rc_lanczos_bounds": (C.c_int, [c_vp, c_vp, c_vp, C.c_uint64, C.c_double, C.c_int, c_i64, c_dp, c_dp,
                                    C.POINTER(c_i64)]),
    "rc_cholqr": (C.c_int, [c_vp, C.c_int, c_vp, c_i64, c_i64, c_i64, C.POINTER(C.c_int)]),
    "rc_rayleigh_ritz": (C.c_int, [c_vp, c_vp, c_vp, c_vp, c_i64, c_i64, c_i64, c_dp, c_dp, c_vp]),
    "rc_small_eigh": (C.c_int, [c_vp, C.c_int, c_i64, c_vp, c_dp, c_vp]),
    "rc_small_eigh_noalloc": (C.c_int, [c_vp, C.c_int, c_i64, c_vp, c_dp, c_vp]),
    "rc_solve_params_default": (None, [C.POINTER(SolveParams)]),
    "rc_solve": (C.c_int, [c_vp, c_vp, C.POINTER(SolveParams), c_vp, c_dp, c_vp, c_dp, C.POINTER(SolveInfo)]),
    "rc_server_params_default": (None, [C.POINTER(ServerParams)]),
    "rc_server_create": (C.c_int, [C.POINTER(ServerParams), C.POINTER(c_vp)]),
    "rc_server_destroy": (C.c_int, [c_vp]),
    "rc_server_last_error": (C.c_char_p, [c_vp]),
    "rc_serve_submit": (C.c_int, [c_vp, c_vp, C.POINTER(SolveParams), c_vp, c_dp, c_vp, c_dp, C.POINTER(c_i64)]),
    "rc_serve_poll": (C.c_int, [c_vp, c_i64, C.POINTER(C.c_int)]),
    "rc_serve_wait": (C.c_int, [c_vp, c_i64, C.c_double, C.POINTER(C.c_int)]),
    "rc_serve_result": (C.c_int, [c_vp, c_i64, C.POINTER(SolveInfo), C.POINTER(RequestInfo), C.c_char_p,
                                  C.c_size_t]),
    "rc_serve_cancel": (C.c_int, [c_vp, c_i64]),
    "rc_serve_release": (C.c_int, [c_vp, c_i64]),
    "rc_server_stats_get": (C.c_int, [c_vp, C.POINTER(ServerStats)]),
}

_lib = None


class RCError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


def lib() -> C.CDLL:
    """Load librcb200.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        path = os.environ.get("RCB200_LIB", LIB_PATH)  # an alternative build of the same library
        if not os.path.exists(path):
            raise RuntimeError(
                f"{path} is missing: build it with `python -m rayleighchebyshevgpgpu_b200.build`; "
                "this package has no CPU fallback")
        L = C.CDLL(path)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int, ctx=None, what: str = "") -> None:
    if status != RC_OK:
        msg = ""
        if ctx:
            raw = lib().rc_ctx_last_error(ctx)
            msg = raw.decode() if raw else ""
        raise RCError(status, f"{what}: {msg}" if what else msg)


def default_params() -> SolveParams:
    p = SolveParams()
    lib().rc_solve_params_default(C.byref(p))
    return p
