"""ctypes binding of the C ABI declared in include/sparsesolv_b200.h.

The shared library ``libsparsesolv_b200.so`` sits next to this file (built
in-tree by ``ngsolve-sparsesolv_b200/build.py``). There is no CPU path: if the
library is missing, or no CUDA device is present, the first call raises.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

LIB_NAME = "libsparsesolv_b200.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

SSV_OK = 0
SSV_ERR_INVALID_ARG = 1
SSV_ERR_RUNTIME = 2
SSV_ERR_CUDA = 3
SSV_ERR_NO_DEVICE = 4
SSV_ERR_TYPE = 5
SSV_ERR_TIMEOUT = 6
SSV_ERR_ALLOC = 7

SSV_F64 = 0
SSV_C128 = 1

SSV_PREC_FP64 = 0
SSV_PREC_FP32 = 1
SSV_PREC_FP32_NODAL = 2

SSV_PROFILE_COLD = 1


class ssv_config(ctypes.Structure):
    """Mirror of sparsesolv::SolverConfig (core/solver_config.hpp:33-159)."""

    _fields_ = [
        ("tolerance", ctypes.c_double),
        ("max_iterations", ctypes.c_int32),
        ("abs_tolerance", ctypes.c_double),
        ("norm_type", ctypes.c_int32),
        ("custom_norm", ctypes.c_double),
        ("shift_parameter", ctypes.c_double),
        ("diagonal_scaling", ctypes.c_int32),
        ("auto_shift", ctypes.c_int32),
        ("shift_increment", ctypes.c_double),
        ("max_shift_value", ctypes.c_double),
        ("min_diagonal_threshold", ctypes.c_double),
        ("zero_diagonal_replacement", ctypes.c_double),
        ("max_shift_trials", ctypes.c_int32),
        ("divergence_check", ctypes.c_int32),
        ("divergence_threshold", ctypes.c_double),
        ("divergence_count", ctypes.c_int32),
        ("save_best_result", ctypes.c_int32),
        ("save_residual_history", ctypes.c_int32),
        ("conjugate", ctypes.c_int32),
        ("use_abmc", ctypes.c_int32),
        ("abmc_block_size", ctypes.c_int32),
        ("abmc_num_colors", ctypes.c_int32),
        ("abmc_reorder_spmv", ctypes.c_int32),
        ("abmc_use_rcm", ctypes.c_int32),
        ("precision", ctypes.c_int32),
    ]


class ssv_result(ctypes.Structure):
    """Mirror of sparsesolv::SolverResult (core/types.hpp:29-37) + timings."""

    _fields_ = [
        ("converged", ctypes.c_int32),
        ("iterations", ctypes.c_int32),
        ("final_residual", ctypes.c_double),
        ("history_len", ctypes.c_int32),
        ("history_total", ctypes.c_int32),
        ("actual_shift", ctypes.c_double),
        ("setup_seconds", ctypes.c_double),
        ("solve_seconds", ctypes.c_double),
        ("kernel_launches", ctypes.c_int64),
    ]


class ssv_batch_tune_entry(ctypes.Structure):
    _fields_ = [
        ("freq_tile", ctypes.c_int32),
        ("lanes", ctypes.c_int32),
        ("grid_x", ctypes.c_int32),
        ("microseconds", ctypes.c_double),
    ]


class ssv_refine_info(ctypes.Structure):
    _fields_ = [
        ("iterations", ctypes.c_int32),
        ("cycles", ctypes.c_int32),
        ("converged", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
        ("true_residual", ctypes.c_double),
    ]


SSV_MAX_PHASES = 8


class ssv_phase_profile(ctypes.Structure):
    _fields_ = [
        ("num_phases", ctypes.c_int32),
        ("names", (ctypes.c_char * 24) * SSV_MAX_PHASES),
        ("ms", ctypes.c_double * SSV_MAX_PHASES),
        ("bytes", ctypes.c_double * SSV_MAX_PHASES),
        ("kernels", ctypes.c_int32 * SSV_MAX_PHASES),
    ]

    def as_list(self):
        return [{"name": self.names[i].value.decode(), "ms": self.ms[i], "bytes": self.bytes[i],
                 "kernels": self.kernels[i]} for i in range(self.num_phases)]


def default_config(**overrides) -> ssv_config:
    """SolverConfig defaults (core/solver_config.hpp:39-157) with overrides."""
    c = ssv_config()
    c.tolerance = 1e-10
    c.max_iterations = 1000
    c.abs_tolerance = 1e-12
    c.norm_type = 0
    c.custom_norm = 1.0
    c.shift_parameter = 1.05
    c.diagonal_scaling = 0
    c.auto_shift = 0
    c.shift_increment = 0.05
    c.max_shift_value = 5.0
    c.min_diagonal_threshold = 1e-6
    c.zero_diagonal_replacement = 1e-10
    c.max_shift_trials = 100
    c.divergence_check = 0
    c.divergence_threshold = 1000.0
    c.divergence_count = 100
    c.save_best_result = 1
    c.save_residual_history = 0
    c.conjugate = 0
    c.use_abmc = 0
    c.abmc_block_size = 4
    c.abmc_num_colors = 4
    c.abmc_reorder_spmv = 0
    c.abmc_use_rcm = 0
    c.precision = SSV_PREC_FP64
    for k, v in overrides.items():
        if isinstance(v, bool):
            v = int(v)
        setattr(c, k, v)
    return c


# ---------------------------------------------------------------------------
# library loading
# ---------------------------------------------------------------------------

_lib = None

P = ctypes.c_void_p
I32 = ctypes.c_int32
PI32 = ctypes.POINTER(ctypes.c_int32)
PU8 = ctypes.POINTER(ctypes.c_uint8)
PD = ctypes.POINTER(ctypes.c_double)
PF = ctypes.POINTER(ctypes.c_float)
PP = ctypes.POINTER(ctypes.c_void_p)

# (name, restype, argtypes) of every exported entry point
SIGNATURES = [
    ("ssv_version", None, [PI32, PI32, PI32]),
    ("ssv_last_error", ctypes.c_char_p, []),
    ("ssv_device_info", I32, [PI32, ctypes.c_char_p, I32]),
    ("ssv_config_default", None, [ctypes.POINTER(ssv_config)]),
    ("ssv_matrix_create", I32, [I32, I32, PI32, PI32, P, I32, PP]),
    ("ssv_matrix_update_values", I32, [P, P]),
    ("ssv_matrix_destroy", I32, [P]),
    ("ssv_matrix_info", I32, [P, PI32, PI32, ctypes.POINTER(ctypes.c_int64), PI32]),
    ("ssv_matrix_spmv", I32, [P, P, P]),
    ("ssv_matrix_spmv_dev", I32, [P, P, P]),
    ("ssv_solver_create", I32, [P, PU8, PP]),
    ("ssv_solver_destroy", I32, [P]),
    ("ssv_solver_solve", I32, [P, ctypes.c_char_p, ctypes.POINTER(ssv_config), P, P,
                               ctypes.POINTER(ssv_result), PD, I32]),
    ("ssv_solver_solve_dev", I32, [P, ctypes.c_char_p, ctypes.POINTER(ssv_config), P, P,
                                   ctypes.POINTER(ssv_result), PD, I32]),
    ("ssv_solver_profile", I32, [P, ctypes.c_char_p, ctypes.POINTER(ssv_config), I32,
                                 ctypes.POINTER(ssv_phase_profile)]),
    ("ssv_ic_create", I32, [P, PU8, ctypes.c_double, PP]),
    ("ssv_ic_set_config", I32, [P, ctypes.POINTER(ssv_config)]),
    ("ssv_sgs_create", I32, [P, PU8, PP]),
    ("ssv_amg_create", I32, [P, PU8, ctypes.c_double, I32, I32, I32, PP]),
    ("ssv_amg_levels", I32, [P, PI32, I32, PI32]),
    ("ssv_precond_update", I32, [P]),
    ("ssv_precond_apply", I32, [P, P, P]),
    ("ssv_precond_apply_block", I32, [P, I32, P, P]),
    ("ssv_matrix_export", I32, [P, P, P, P]),
    ("ssv_hcurl_assemble", I32, [I32, P, I32, P, P, P, I32, P, P, P, P, P, P]),
    ("ssv_ams_subspace_apply", I32, [P, I32, P, P, P, P]),
    ("ssv_ams_profile_levels", I32, [P, I32, I32, P, P, P, P, I32, P, P]),
    ("ssv_precond_apply_dev", I32, [P, P, P]),
    ("ssv_ic_actual_shift", I32, [P, PD]),
    ("ssv_precond_destroy", I32, [P]),
    ("ssv_cocr_solve", I32, [P, P, PU8, I32, ctypes.c_double, I32, P, P, PI32]),
    ("ssv_cocr_solve_dev", I32, [P, P, PU8, I32, ctypes.c_double, I32, P, P, PI32]),
    ("ssv_cocr_refined_solve", I32, [P, P, PU8, I32, ctypes.c_double, ctypes.c_double, I32, P, P,
                                     ctypes.POINTER(ssv_refine_info)]),
    ("ssv_cocr_refined_solve_dev", I32, [P, P, PU8, I32, ctypes.c_double, ctypes.c_double, I32, P, P,
                                         ctypes.POINTER(ssv_refine_info)]),
    ("ssv_set_loop_guard", None, [I32]),
    ("ssv_set_alloc_budget", None, [ctypes.c_int64]),
    ("ssv_cocr_last_launches", I32, [ctypes.POINTER(ctypes.c_int64)]),
    ("ssv_gmres_solve", I32, [P, P, PU8, I32, ctypes.c_double, I32, P, P, PI32]),
    ("ssv_gmres_solve_dev", I32, [P, P, PU8, I32, ctypes.c_double, I32, P, P, PI32]),
    ("ssv_abmc_build", I32, [I32, PI32, PI32, I32, I32, PI32, PI32, PI32, PI32, PI32, PI32]),
    ("ssv_level_schedule", I32, [I32, PI32, PI32, I32, PI32, PI32]),
    ("ssv_rcm_order", I32, [I32, PI32, PI32, PI32, PI32]),
    ("ssv_spmv_dot_noalloc", I32, [I32, P, P, P, P, P, P]),
    ("ssv_ams_create", I32, [P, P, PU8, PD, PD, PD, I32, I32, ctypes.c_double, ctypes.c_double, I32, I32, PP]),
    ("ssv_ams_update", I32, [P, P]),
    ("ssv_ams_levels", I32, [P, I32, PI32, I32, PI32]),
    ("ssv_ams_set_precision", I32, [P, I32]),
    ("ssv_batch_create", I32, [P, P, I32, PD, PP, I32, PU8, PP]),
    ("ssv_batch_destroy", I32, [P]),
    ("ssv_batch_cocr_solve", I32, [P, I32, ctypes.c_double, P, P, PI32, PI32, PD]),
    ("ssv_batch_cocr_solve_dev", I32, [P, I32, ctypes.c_double, P, P, PI32, PI32, PD]),
    ("ssv_batch_tuning", I32, [P, ctypes.POINTER(ssv_batch_tune_entry), I32, PI32, PI32]),
    ("ssv_batch_set_replacement", I32, [P, I32]),
    ("ssv_batch_set_refinement", I32, [P, ctypes.c_double]),
    ("ssv_batch_last_cycles", I32, [P, PI32]),
    ("ssv_batch_last_timing", I32, [P, PD, PD, PI32, ctypes.POINTER(ctypes.c_int64)]),
    ("ssv_ams_get_precision", I32, [P, PI32]),
    ("ssv_ams_setup_times", I32, [P, PD]),
    ("ssv_ams_level_matrix", I32, [P, I32, I32, I32, PI32, PI32, PD, I32, PI32, PI32]),
    ("ssv_ams_profile", I32, [P, I32, I32, I32, ctypes.POINTER(ssv_phase_profile)]),
    ("ssv_mlp_create", I32, [I32, I32, ctypes.c_uint64, PP]),
    ("ssv_mlp_destroy", I32, [P]),
    ("ssv_mlp_num_params", I32, [P, PI32]),
    ("ssv_mlp_get_params", I32, [P, PF]),
    ("ssv_mlp_set_params", I32, [P, PF]),
    ("ssv_mlp_gradients", I32, [P, PF, PF, ctypes.c_int64, PF, PF]),
    ("ssv_mlp_train_dev", I32, [P, P, P, ctypes.c_int64, I32, I32, ctypes.c_float, ctypes.c_uint64, PF]),
    ("ssv_mlp_predict_dev", I32, [P, P, ctypes.c_int64, P]),
    ("ssv_pcg_solve", I32, [P, P, PU8, ctypes.POINTER(ssv_config), P, P, ctypes.POINTER(ssv_result), PD, I32]),
    ("ssv_pcg_solve_dev", I32, [P, P, PU8, ctypes.POINTER(ssv_config), P, P, ctypes.POINTER(ssv_result), PD, I32]),
]


def load(path: str | None = None):
    """Load the C-ABI library (once) and bind every declared symbol."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"sparsesolv_ngsolve: CUDA library {p} is not built; run "
            "`python ngsolve-sparsesolv_b200/build.py` (there is no CPU fallback)")
    lib = ctypes.CDLL(p)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


class SparseSolvError(RuntimeError):
    pass


def check(rc: int):
    """Map a status code to the Python exception the reference raises."""
    if rc == SSV_OK:
        return
    msg = (load().ssv_last_error() or b"").decode(errors="replace")
    if rc == SSV_ERR_INVALID_ARG:
        raise ValueError(msg)
    if rc == SSV_ERR_TYPE:
        raise TypeError(msg)
    if rc == SSV_ERR_ALLOC:  # pybind11's translation of std::bad_alloc
        raise MemoryError(msg)
    raise RuntimeError(msg or f"sparsesolv_b200 error {rc}")


def i32ptr(a: np.ndarray):
    return a.ctypes.data_as(PI32)


def u8ptr(a):
    if a is None:
        return None
    return a.ctypes.data_as(PU8)


def vptr(a: np.ndarray):
    return ctypes.c_void_p(a.ctypes.data)
