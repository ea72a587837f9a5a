"""ctypes binding of the C-ABI in ``include/uaamg.h`` (libuaamg_b200.so).

The library is the product: every solve runs on the GPU through it.  There is no
CPU fallback -- if the library is missing or no CUDA device is present, the calls
raise.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libuaamg_b200.so")

# uaamg_status
OK, NOT_CONVERGED, BREAKDOWN, NAN, OOM, INVALID_ARG, CUDA_ERROR, TIMEOUT, NO_PROBLEM = range(9)
STATUS_NAMES = {
    OK: "ok", NOT_CONVERGED: "not converged", BREAKDOWN: "breakdown", NAN: "nan",
    OOM: "out of device memory", INVALID_ARG: "invalid argument", CUDA_ERROR: "cuda error",
    TIMEOUT: "timeout", NO_PROBLEM: "no problem set",
}
# uaamg_precision
FP64, FP32, MIXED = 0, 1, 2
PRECISIONS = {"fp64": FP64, "fp32": FP32, "mixed": MIXED}
# uaamg_tol_mode
TOL_ABS, TOL_REL = 0, 1

# Every exported entry point of include/uaamg.h.
EXPORTS = [
    "uaamg_default_options", "uaamg_create", "uaamg_destroy", "uaamg_set_stream",
    "uaamg_set_problem_2d", "uaamg_set_problem_3d", "uaamg_set_problem_device",
    "uaamg_set_dirichlet_walls", "uaamg_set_variable_laplacian", "uaamg_solve",
    "uaamg_solve_device", "uaamg_precond_apply",
    "uaamg_residual_history", "uaamg_num_levels", "uaamg_level_dims", "uaamg_copy_level",
    "uaamg_level_trim",
    "uaamg_device_bytes", "uaamg_last_error", "uaamg_status_string", "uaamg_profile_solve",
    "uaamg_set_vcycle_kernels", "uaamg_residual_noalloc", "uaamg_solve_batch",
    "uaamg_set_autotune", "uaamg_server_default_config", "uaamg_server_start",
    "uaamg_server_submit", "uaamg_server_poll", "uaamg_server_drain", "uaamg_server_info",
    "uaamg_server_stop", "uaamg_project", "uaamg_project_device", "uaamg_static_pressure",
    "uaamg_static_pressure_device", "uaamg_set_smoothing", "uaamg_set_tune_cache",
    "uaamg_set_batch_group",
]


class KernelTime(C.Structure):
    _fields_ = [
        ("name", C.c_char * 32),
        ("level", C.c_int),
        ("launches", C.c_int),
        ("total_ms", C.c_double),
        ("bytes_per_launch", C.c_double),
    ]


class Options(C.Structure):
    _fields_ = [
        ("precision", C.c_int),
        ("tol_mode", C.c_int),
        ("max_iter", C.c_int),
        ("tol", C.c_double),
        ("warm_start", C.c_int),
        ("replace_every", C.c_int),
        ("project_mean", C.c_int),
        ("preconditioner", C.c_int),
    ]


class Stats(C.Structure):
    _fields_ = [
        ("status", C.c_int),
        ("iterations", C.c_int),
        ("replacements", C.c_int),
        ("levels", C.c_int),
        ("residual", C.c_double),
        ("rel_residual", C.c_double),
        ("recursive_residual", C.c_double),
        ("rhs_norm", C.c_double),
        ("solve_ms", C.c_double),
        ("kernel_launches", C.c_longlong),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class Problem(C.Structure):
    """uaamg_problem: one problem of uaamg_solve_batch (host arrays)."""
    _fields_ = [
        ("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("solid", C.c_void_p), ("rhs", C.c_void_p), ("p", C.c_void_p),
    ]


class ServerConfig(C.Structure):
    _fields_ = [
        ("device", C.c_int), ("precision", C.c_int), ("tol", C.c_double),
        ("max_iter", C.c_int), ("replace_every", C.c_int), ("warm_start", C.c_int),
        ("max_active", C.c_int), ("hbm_budget_bytes", C.c_size_t),
    ]


class Request(C.Structure):
    _fields_ = [
        ("sim_id", C.c_longlong),
        ("dim", C.c_int), ("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
        ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double),
        ("solid", C.c_void_p), ("rhs", C.c_void_p), ("p_out", C.c_void_p),
        ("flags", C.c_int),
    ]


REQUEST_BORROW = 1


class Result(C.Structure):
    _fields_ = [
        ("ticket", C.c_longlong), ("sim_id", C.c_longlong), ("status", C.c_int),
        ("iterations", C.c_int), ("rel_residual", C.c_double), ("wait_ms", C.c_double),
        ("latency_ms", C.c_double), ("warm", C.c_int),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class UaamgError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


_lib = None


def load(path: str | None = None):
    """Loads libuaamg_b200.so (raises if it is missing: there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise RuntimeError(f"{path} is missing: build it with `python -c 'import "
                           "__graft_entry__ as g; g.build()'` (needs nvcc)")
    L = C.CDLL(path)
    p, i, d = C.c_void_p, C.c_int, C.c_double
    L.uaamg_default_options.argtypes = [C.POINTER(Options)]
    L.uaamg_default_options.restype = None
    L.uaamg_create.argtypes = [C.POINTER(p), i]
    L.uaamg_destroy.argtypes = [p]
    L.uaamg_set_stream.argtypes = [p, p]
    L.uaamg_set_problem_2d.argtypes = [p, i, i, d, d, p]
    L.uaamg_set_problem_3d.argtypes = [p, i, i, i, d, d, d, p]
    L.uaamg_set_problem_device.argtypes = [p, i, i, i, i, d, d, d, p]
    L.uaamg_set_dirichlet_walls.argtypes = [p, i]
    L.uaamg_set_variable_laplacian.argtypes = [p, p, p, p]
    L.uaamg_set_vcycle_kernels.argtypes = [p, i]
    L.uaamg_set_smoothing.argtypes = [p, i, i]
    L.uaamg_set_tune_cache.argtypes = [C.c_char_p]
    L.uaamg_set_batch_group.argtypes = [p, C.c_longlong]
    L.uaamg_residual_noalloc.argtypes = [i, i, i, i, d, d, d, p, p, p, p, p]
    L.uaamg_solve.argtypes = [p, p, p, C.POINTER(Options), C.POINTER(Stats)]
    L.uaamg_solve_device.argtypes = [p, p, p, C.POINTER(Options), C.POINTER(Stats)]
    L.uaamg_project.argtypes = [p, d, p, p, p, p, C.POINTER(Options), C.POINTER(Stats)]
    L.uaamg_project_device.argtypes = [p, d, p, p, p, p, C.POINTER(Options), C.POINTER(Stats)]
    L.uaamg_static_pressure.argtypes = [p, p, p, p, C.POINTER(Options), C.POINTER(Stats)]
    L.uaamg_static_pressure_device.argtypes = [p, p, p, p, C.POINTER(Options), C.POINTER(Stats)]
    L.uaamg_precond_apply.argtypes = [p, i, p, p]
    L.uaamg_residual_history.argtypes = [p, p, i]
    L.uaamg_num_levels.argtypes = [p, C.POINTER(i)]
    L.uaamg_level_dims.argtypes = [p, i, C.POINTER(i), C.POINTER(i), C.POINTER(i)]
    L.uaamg_copy_level.argtypes = [p, i, i, p, p, p, p]
    L.uaamg_level_trim.argtypes = [p, i, i, C.POINTER(i), C.POINTER(i)]
    L.uaamg_device_bytes.argtypes = [p, C.POINTER(C.c_size_t)]
    L.uaamg_profile_solve.argtypes = [p, p, p, C.POINTER(Options), C.POINTER(Stats),
                                      C.POINTER(KernelTime), i, C.POINTER(i)]
    L.uaamg_solve_batch.argtypes = [p, i, C.POINTER(Problem), C.POINTER(Options), C.POINTER(Stats)]
    L.uaamg_set_autotune.argtypes = [p, i]
    L.uaamg_server_default_config.argtypes = [C.POINTER(ServerConfig)]
    L.uaamg_server_start.argtypes = [C.POINTER(p), C.POINTER(ServerConfig)]
    L.uaamg_server_submit.argtypes = [p, C.POINTER(Request), C.POINTER(C.c_longlong)]
    L.uaamg_server_poll.argtypes = [p, C.c_longlong, C.POINTER(Result), C.POINTER(i)]
    L.uaamg_server_drain.argtypes = [p]
    L.uaamg_server_info.argtypes = [p, C.POINTER(C.c_size_t), C.POINTER(i), C.POINTER(C.c_longlong)]
    L.uaamg_server_stop.argtypes = [p]
    L.uaamg_last_error.argtypes = [p]
    L.uaamg_last_error.restype = C.c_char_p
    L.uaamg_status_string.argtypes = [i]
    L.uaamg_status_string.restype = C.c_char_p
    for name in EXPORTS:
        if name not in ("uaamg_default_options", "uaamg_last_error", "uaamg_status_string",
                        "uaamg_server_default_config"):
            getattr(L, name).restype = i
    _lib = L
    return L


def default_options() -> Options:
    o = Options()
    load().uaamg_default_options(C.byref(o))
    return o
