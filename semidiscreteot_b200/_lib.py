"""ctypes binding of ``libsdot_cuda.so`` (declared in ``include/sdot.h``).

The shared library is built in-tree (``python -m semidiscreteot_b200.build``)
and is required: there is no CPU fallback.  Loading it needs no GPU (CUDA is
linked statically); creating a context does.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsdot_cuda.so")

SDOT_OK = 0
SDOT_ENOMEM = 2
SDOT_ELINESEARCH = 4
SDOT_ETIMEOUT = 7
SDOT_ESTATE = 9
STATUS_NAMES = {
    0: "SDOT_OK", 1: "SDOT_EINVAL", 2: "SDOT_ENOMEM", 3: "SDOT_ENONFINITE", 4: "SDOT_ELINESEARCH",
    5: "SDOT_EMAXITER", 6: "SDOT_EBUDGET", 7: "SDOT_ETIMEOUT", 8: "SDOT_ECUDA", 9: "SDOT_ESTATE",
}
PRECISION = {"fp64": 0, "hybrid": 1, "mixed": 2}
THRESHOLD = {"pointwise": 0, "integral": 1, "geometric": 2}
CONTROL = {"l1norm": 0, "componentwise": 1, "linf": 2}
LINE_SEARCH = {"upstream": 0, "vendored": 1}
HESSIAN_METHOD = {"auto": 0, "fp64": 1, "tensor": 2}
METHOD = {"auto": 0, "newton": 1, "lbfgs": 2}

# Every symbol include/sdot.h declares (checked by tests).
EXPORTED = [
    "sdot_abi_version", "sdot_build_info", "sdot_last_error", "sdot_create", "sdot_destroy",
    "sdot_set_source", "sdot_set_target", "sdot_configure", "sdot_default_params", "sdot_evaluate",
    "sdot_evaluate_device", "sdot_solve", "sdot_hessian", "sdot_get_last_functional_value",
    "sdot_get_last_iteration_count", "sdot_get_convergence_status", "sdot_get_last_distance_threshold",
    "sdot_get_C_global", "sdot_set_distance_threshold", "sdot_compute_covering_radius",
    "sdot_compute_geometric_radius_bound", "sdot_set_distance_function", "sdot_evaluate_partial_device",
    "sdot_set_state", "sdot_get_stream", "sdot_set_profiling", "sdot_get_kernel_times", "sdot_measure_peaks",
    "sdot_evaluate_device_noalloc", "sdot_hessian_device", "sdot_set_hessian_chunk", "sdot_set_hessian_wait_limit",
    "sdot_set_hessian_generation", "sdot_set_hessian_pairs",
    "sdot_solve_newton", "sdot_set_newton_hessian_reuse", "sdot_hessian_tile_count", "sdot_hessian_tiles_device",
    "sdot_hessian_matvec_device", "sdot_softmax_refinement", "sdot_weighted_barycenters", "sdot_conditioned_densities",
    "sdot_batch_create", "sdot_batch_destroy", "sdot_batch_last_error", "sdot_batch_size", "sdot_batch_set_verbose",
    "sdot_batch_add", "sdot_batch_evaluate", "sdot_batch_solve", "sdot_batch_problem_info",
    "sdot_batch_set_shape", "sdot_batch_get_shape", "sdot_batch_last_eval_ms", "sdot_batch_autotune",
    "sdot_debug_fail_allocation", "sdot_debug_allocation_count", "sdot_weighted_barycenters_spherical",
    "sdot_server_create", "sdot_server_destroy", "sdot_server_last_error", "sdot_server_submit", "sdot_server_poll",
    "sdot_server_wait", "sdot_server_get_stats", "sdot_server_reset_stats",
]

NOALLOC_SCRATCH_BYTES = 8 << 20  # SDOT_NOALLOC_SCRATCH_BYTES


class Options(C.Structure):
    _fields_ = [("device", C.c_int), ("precision", C.c_int), ("memory_budget", C.c_size_t),
                ("verbose", C.c_int)]


class SolverParams(C.Structure):
    _fields_ = [("max_iterations", C.c_uint), ("tolerance", C.c_double), ("control_type", C.c_int),
                ("epsilon", C.c_double), ("tau", C.c_double), ("threshold_type", C.c_int),
                ("use_log_sum_exp", C.c_int), ("line_search", C.c_int)]


class EvalInfo(C.Structure):
    _fields_ = [("value", C.c_double), ("C_global", C.c_double), ("threshold", C.c_double),
                ("n_pairs", C.c_int64), ("device_ms", C.c_double)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_uint), ("converged", C.c_int), ("n_evaluations", C.c_int64),
                ("last_value", C.c_double), ("last_check_value", C.c_double), ("total_pairs", C.c_int64),
                ("device_ms", C.c_double)]


class HessianInfo(C.Structure):
    _fields_ = [("method", C.c_int), ("eval_ms", C.c_double), ("hessian_ms", C.c_double),
                ("kernel_ms", C.c_double), ("tiles", C.c_int64)]


class NewtonInfo(C.Structure):
    _fields_ = [("iterations", C.c_uint), ("converged", C.c_int), ("n_evaluations", C.c_int64),
                ("cg_iterations", C.c_int64), ("last_value", C.c_double), ("last_check_value", C.c_double),
                ("total_pairs", C.c_int64), ("eval_ms", C.c_double), ("hessian_ms", C.c_double),
                ("cg_ms", C.c_double), ("hessian_method", C.c_int), ("n_hessians", C.c_int64)]


class BatchOptions(C.Structure):
    _fields_ = [("epsilon_scaling_factor", C.c_double), ("epsilon_scaling_steps", C.c_int),
                ("intermediate_tolerance", C.c_double), ("mixed_precision", C.c_int)]


class BatchInfo(C.Structure):
    _fields_ = [("n_problems", C.c_int), ("converged", C.c_int), ("rounds", C.c_int64),
                ("evaluations", C.c_int64), ("total_pairs", C.c_int64), ("eval_ms", C.c_double),
                ("solve_ms", C.c_double)]


class Request(C.Structure):
    _fields_ = [("dim", C.c_int), ("n_q", C.c_int64), ("x", C.c_void_p), ("jxw", C.c_void_p),
                ("density", C.c_void_p), ("n_cells", C.c_int64), ("cell_offsets", C.c_void_p),
                ("cell_centers", C.c_void_p), ("n_t", C.c_int64), ("y", C.c_void_p), ("nu", C.c_void_p),
                ("psi0", C.c_void_p), ("params", SolverParams), ("method", C.c_int), ("precision", C.c_int),
                ("hessian_method", C.c_int), ("epsilon_scaling_factor", C.c_double),
                ("epsilon_scaling_steps", C.c_int), ("intermediate_tolerance", C.c_double)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int), ("converged", C.c_int), ("method", C.c_int), ("iterations", C.c_uint),
                ("n_evaluations", C.c_int64), ("last_value", C.c_double), ("last_check_value", C.c_double),
                ("queue_ms", C.c_double), ("run_ms", C.c_double), ("latency_ms", C.c_double), ("slot", C.c_int),
                ("message", C.c_char * 160)]


class ServerStats(C.Structure):
    _fields_ = [("completed", C.c_int64), ("failed", C.c_int64), ("queued", C.c_int64), ("running", C.c_int),
                ("peak_running", C.c_int), ("in_use_bytes", C.c_size_t), ("peak_bytes", C.c_size_t),
                ("p50_ms", C.c_double), ("p99_ms", C.c_double), ("mean_ms", C.c_double)]


_lib = None


def load():
    """Load the library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA library first "
            "(python -m semidiscreteot_b200.build); there is no CPU fallback")
    lib = C.CDLL(LIB_PATH)
    vp, i64, d, ip = C.c_void_p, C.c_int64, C.c_double, C.c_int
    lib.sdot_abi_version.restype = ip
    lib.sdot_build_info.restype = C.c_char_p
    lib.sdot_last_error.argtypes = [vp]
    lib.sdot_last_error.restype = C.c_char_p
    lib.sdot_create.argtypes = [C.POINTER(vp), C.POINTER(Options)]
    lib.sdot_destroy.argtypes = [vp]
    lib.sdot_destroy.restype = None
    lib.sdot_set_source.argtypes = [vp, ip, i64, vp, vp, vp, i64, vp, vp]
    lib.sdot_set_target.argtypes = [vp, i64, vp, vp]
    lib.sdot_configure.argtypes = [vp, C.POINTER(SolverParams)]
    lib.sdot_default_params.argtypes = [C.POINTER(SolverParams)]
    lib.sdot_default_params.restype = None
    lib.sdot_evaluate.argtypes = [vp, vp, vp, C.POINTER(d), C.POINTER(EvalInfo)]
    lib.sdot_evaluate_device.argtypes = [vp, vp, vp, C.POINTER(d), C.POINTER(EvalInfo)]
    lib.sdot_solve.argtypes = [vp, vp, C.POINTER(SolverParams), C.POINTER(SolveInfo)]
    lib.sdot_hessian.argtypes = [vp, vp, vp]
    for name in ("sdot_get_last_functional_value", "sdot_get_last_distance_threshold", "sdot_get_C_global"):
        getattr(lib, name).argtypes = [vp]
        getattr(lib, name).restype = d
    lib.sdot_get_last_iteration_count.argtypes = [vp]
    lib.sdot_get_last_iteration_count.restype = C.c_uint
    lib.sdot_get_convergence_status.argtypes = [vp]
    lib.sdot_get_convergence_status.restype = ip
    lib.sdot_set_distance_threshold.argtypes = [vp, d]
    lib.sdot_compute_covering_radius.argtypes = [vp, C.POINTER(d)]
    lib.sdot_compute_geometric_radius_bound.argtypes = [vp, vp, d, d, C.POINTER(d)]
    lib.sdot_set_distance_function.argtypes = [vp, C.c_char_p]
    lib.sdot_evaluate_partial_device.argtypes = [vp, vp, vp, C.POINTER(EvalInfo)]
    lib.sdot_set_state.argtypes = [vp, d, d]
    lib.sdot_get_stream.argtypes = [vp]
    lib.sdot_get_stream.restype = vp
    lib.sdot_set_profiling.argtypes = [vp, ip]
    lib.sdot_get_kernel_times.argtypes = [vp, vp, vp, ip, ip]
    lib.sdot_measure_peaks.argtypes = [ip, vp]
    lib.sdot_evaluate_device_noalloc.argtypes = [vp, vp, vp, C.POINTER(d)]
    lib.sdot_evaluate_device_noalloc.restype = ip
    lib.sdot_hessian_device.argtypes = [vp, vp, vp, ip, ip, C.POINTER(HessianInfo)]
    lib.sdot_hessian_device.restype = ip
    lib.sdot_set_hessian_chunk.argtypes = [vp, ip]
    lib.sdot_set_hessian_chunk.restype = ip
    lib.sdot_set_hessian_wait_limit.argtypes = [vp, C.c_int64]
    lib.sdot_set_hessian_wait_limit.restype = ip
    lib.sdot_set_hessian_generation.argtypes = [vp, ip, vp]
    lib.sdot_set_hessian_generation.restype = ip
    lib.sdot_set_hessian_pairs.argtypes = [vp, ip, vp]
    lib.sdot_set_hessian_pairs.restype = ip
    lib.sdot_solve_newton.argtypes = [vp, vp, C.POINTER(SolverParams), ip, C.POINTER(NewtonInfo)]
    lib.sdot_solve_newton.restype = ip
    lib.sdot_set_newton_hessian_reuse.argtypes = [vp, d]
    lib.sdot_hessian_tile_count.argtypes = [vp, C.POINTER(i64)]
    lib.sdot_hessian_tile_count.restype = ip
    lib.sdot_hessian_tiles_device.argtypes = [vp, vp, vp, ip, i64, i64, C.POINTER(HessianInfo)]
    lib.sdot_hessian_tiles_device.restype = ip
    lib.sdot_hessian_matvec_device.argtypes = [vp, vp, ip, vp, vp]
    lib.sdot_hessian_matvec_device.restype = ip
    lib.sdot_set_newton_hessian_reuse.restype = ip
    lib.sdot_softmax_refinement.argtypes = [vp, vp, d, d, ip, i64, vp, vp, vp, vp]
    lib.sdot_softmax_refinement.restype = ip
    lib.sdot_weighted_barycenters.argtypes = [vp, vp, vp]
    lib.sdot_weighted_barycenters.restype = ip
    lib.sdot_conditioned_densities.argtypes = [vp, vp, d, d, i64, vp, vp, i64, vp, vp]
    lib.sdot_conditioned_densities.restype = ip
    lib.sdot_batch_create.argtypes = [C.POINTER(vp), ip, ip]
    lib.sdot_batch_create.restype = ip
    lib.sdot_batch_destroy.argtypes = [vp]
    lib.sdot_batch_destroy.restype = None
    lib.sdot_batch_last_error.argtypes = [vp]
    lib.sdot_batch_last_error.restype = C.c_char_p
    lib.sdot_batch_size.argtypes = [vp]
    lib.sdot_batch_size.restype = ip
    lib.sdot_batch_set_verbose.argtypes = [vp, ip]
    lib.sdot_batch_set_verbose.restype = ip
    lib.sdot_batch_add.argtypes = [vp, i64, vp, vp, vp, i64, vp, vp, C.POINTER(SolverParams), C.POINTER(ip)]
    lib.sdot_batch_add.restype = ip
    lib.sdot_batch_evaluate.argtypes = [vp, vp, vp, vp, ip]
    lib.sdot_batch_evaluate.restype = ip
    lib.sdot_batch_solve.argtypes = [vp, vp, C.POINTER(BatchOptions), C.POINTER(BatchInfo)]
    lib.sdot_batch_solve.restype = ip
    lib.sdot_batch_problem_info.argtypes = [vp, ip, C.POINTER(SolveInfo)]
    lib.sdot_batch_problem_info.restype = ip
    lib.sdot_batch_set_shape.argtypes = [vp, vp]
    lib.sdot_batch_set_shape.restype = ip
    lib.sdot_batch_get_shape.argtypes = [vp, vp]
    lib.sdot_batch_get_shape.restype = ip
    lib.sdot_batch_last_eval_ms.argtypes = [vp]
    lib.sdot_batch_last_eval_ms.restype = C.c_double
    lib.sdot_batch_autotune.argtypes = [vp, vp, ip, ip, vp, vp]
    lib.sdot_batch_autotune.restype = ip
    lib.sdot_debug_fail_allocation.argtypes = [C.c_int64]
    lib.sdot_debug_fail_allocation.restype = C.c_int64
    lib.sdot_debug_allocation_count.argtypes = []
    lib.sdot_debug_allocation_count.restype = C.c_int64
    lib.sdot_weighted_barycenters_spherical.argtypes = [vp, vp, vp, C.c_uint, C.c_double, vp, vp]
    lib.sdot_weighted_barycenters_spherical.restype = ip
    lib.sdot_server_create.argtypes = [C.POINTER(vp), ip, ip, C.c_size_t]
    lib.sdot_server_create.restype = ip
    lib.sdot_server_destroy.argtypes = [vp]
    lib.sdot_server_destroy.restype = None
    lib.sdot_server_last_error.argtypes = [vp]
    lib.sdot_server_last_error.restype = C.c_char_p
    lib.sdot_server_submit.argtypes = [vp, C.POINTER(Request), C.POINTER(i64)]
    lib.sdot_server_submit.restype = ip
    lib.sdot_server_poll.argtypes = [vp, i64]
    lib.sdot_server_poll.restype = ip
    lib.sdot_server_wait.argtypes = [vp, i64, d, vp, C.POINTER(Result)]
    lib.sdot_server_wait.restype = ip
    lib.sdot_server_get_stats.argtypes = [vp, C.POINTER(ServerStats)]
    lib.sdot_server_get_stats.restype = ip
    lib.sdot_server_reset_stats.argtypes = [vp]
    lib.sdot_server_reset_stats.restype = ip
    for fn in ("sdot_evaluate_partial_device", "sdot_set_state", "sdot_set_profiling", "sdot_get_kernel_times",
               "sdot_measure_peaks"):
        getattr(lib, fn).restype = ip
    for fn in ("sdot_create", "sdot_set_source", "sdot_set_target", "sdot_configure", "sdot_evaluate",
               "sdot_evaluate_device", "sdot_solve", "sdot_hessian", "sdot_set_distance_threshold",
               "sdot_compute_covering_radius", "sdot_compute_geometric_radius_bound",
               "sdot_set_distance_function"):
        getattr(lib, fn).restype = ip
    _lib = lib
    return lib


class SdotError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
