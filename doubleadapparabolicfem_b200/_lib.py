"""ctypes binding of libapf_b200.so (the C ABI declared in include/apf_b200.h).

The shared library is built in-tree by ``doubleadapparabolicfem_b200.build``.
Loading fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libapf_b200.so")

APF_OK = 0
APF_PATCH_FP64 = 0
APF_PATCH_FP32_REFINED = 1
APF_ERR_INVALID = -1
APF_ERR_CUDA = -2
APF_ERR_CAPACITY = -3
APF_ERR_NUMERIC = -4
APF_ERR_NOT_CONVERGED = -5
APF_ERR_NO_DEVICE = -6
APF_ERR_INTERNAL = -7

APF_U0_SIN_SIN = 0
APF_U0_ONE = 1
APF_U0_ZERO = 2

BLOCKS = {"A_y": 0, "B": 1, "BT": 2, "C_signed": 3, "K": 4, "Hhat": 5, "B_dt": 6, "A_x": 7}
APF_VEC_F = 0
APF_VEC_G = 1


class ApfError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"apf error {code}: {message}")
        self.code = code


class ProblemDesc(C.Structure):
    _fields_ = [
        ("p", C.c_int),
        ("n_y_cells", C.c_int),
        ("n_x_cells", C.c_int),
        ("n_lambda", C.c_int),
        ("n_u", C.c_int),
        ("y_geometry", C.c_void_p),
        ("x_geometry", C.c_void_p),
        ("y_to_x", C.c_void_p),
        ("y_restr_offsets", C.c_void_p),
        ("y_restr_dofs", C.c_void_p),
        ("y_restr_weights", C.c_void_p),
        ("y_restr_nnz", C.c_int32),
        ("x_restr_offsets", C.c_void_p),
        ("x_restr_dofs", C.c_void_p),
        ("x_restr_weights", C.c_void_p),
        ("x_restr_nnz", C.c_int32),
        ("m_cells", C.c_void_p),
        ("ell_cells", C.c_void_p),
        ("u0_kind", C.c_int),
        ("zero_tol", C.c_double),
        ("g_scale", C.c_double),
        ("dim_space", C.c_int),
    ]


class SolverOptions(C.Structure):
    _fields_ = [
        ("tolerance", C.c_double),
        ("max_iterations", C.c_int),
        ("use_true_residual_batching", C.c_int),
        ("true_residual_check_interval", C.c_int),
        ("preconditioner", C.c_int),
        ("amg_smooth_steps", C.c_int),
        ("amg_strength", C.c_double),
        ("amg_coarse_size", C.c_int),
        ("amg_aggressive_levels", C.c_int),
        ("amg_vcycles", C.c_int),
    ]


class SolverDiagnostics(C.Structure):
    _fields_ = [
        ("iterations", C.c_int),
        ("residual_check_batches", C.c_int),
        ("converged", C.c_int),
        ("backend_converged", C.c_int),
        ("backend_reported_error", C.c_double),
        ("final_true_residual", C.c_double),
        ("setup_seconds", C.c_double),
        ("solve_seconds", C.c_double),
        ("amg_levels_lambda", C.c_int),
        ("amg_levels_u", C.c_int),
        ("amg_nnz_lambda", C.c_int64),
        ("amg_nnz_u", C.c_int64),
        ("preconditioner_used", C.c_int),
        ("learned_fallback", C.c_int),
    ]


APF_PRECOND_AMG_BLOCK = 0
APF_PRECOND_LEARNED = 1

_lib = None

# exported symbols and their signatures (argtypes, restype)
SIGNATURES = {
    "apf_ctx_create": ([C.c_int, C.c_void_p, C.POINTER(C.c_void_p)], C.c_int),
    "apf_ctx_destroy": ([C.c_void_p], None),
    "apf_ctx_last_error": ([C.c_void_p], C.c_char_p),
    "apf_ctx_synchronize": ([C.c_void_p], C.c_int),
    "apf_ctx_kernel_launches": ([C.c_void_p], C.c_int64),
    "apf_ctx_set_timing": ([C.c_void_p, C.c_int], C.c_int),
    "apf_ctx_set_patch_precision": ([C.c_void_p, C.c_int], C.c_int),
    "apf_ctx_set_autotune": ([C.c_void_p, C.c_int], C.c_int),
    "apf_ctx_autotune_report": ([C.c_void_p], C.c_char_p),
    "apf_system_set_partition": ([C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p], C.c_int),
    "apf_system_part_residuals": ([C.c_void_p, C.c_void_p, C.c_void_p], C.c_int),
    "apf_ctx_timing_report": ([C.c_void_p], C.c_char_p),
    "apf_assemble_main_system": ([C.c_void_p, C.POINTER(ProblemDesc), C.c_int, C.POINTER(C.c_void_p)], C.c_int),
    "apf_assemble_graph_norm": ([C.c_void_p, C.c_void_p, C.c_double], C.c_int),
    "apf_write_cellwise_error_binary": ([C.c_void_p, C.c_char_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_int, C.c_int],
                                        C.c_int),
    "apf_write_cellwise_error_components_binary": ([C.c_void_p, C.c_char_p, C.c_int32, C.c_void_p, C.c_void_p,
                                                    C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_int], C.c_int),
    "apf_write_x_indicator_components_binary": ([C.c_void_p, C.c_char_p, C.c_int32, C.c_void_p, C.c_void_p,
                                                 C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "apf_two_pass_cache_create": ([C.c_void_p, C.POINTER(C.c_void_p)], C.c_int),
    "apf_two_pass_cache_destroy": ([C.c_void_p], None),
    "apf_two_pass_cache_stats": ([C.c_void_p, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64)],
                                 C.c_int),
    "apf_assemble_full_saddle_two_pass": ([C.c_void_p, C.POINTER(ProblemDesc), C.c_int, C.c_void_p,
                                           C.POINTER(C.c_void_p)], C.c_int),
    "apf_system_block_info": ([C.c_void_p, C.c_int, C.POINTER(C.c_int32), C.POINTER(C.c_int32),
                               C.POINTER(C.c_int64)], C.c_int),
    "apf_system_block_copy": ([C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "apf_system_block_device_ptrs": ([C.c_void_p, C.c_int, C.POINTER(C.c_void_p), C.POINTER(C.c_void_p),
                                      C.POINTER(C.c_void_p)], C.c_int),
    "apf_system_vector_copy": ([C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int], C.c_int),
    "apf_system_destroy": ([C.c_void_p], None),
    "apf_solver_options_default": ([C.POINTER(SolverOptions)], None),
    "apf_setup_preconditioner": ([C.c_void_p, C.c_void_p, C.POINTER(SolverOptions)], C.c_int),
    "apf_solve_minres": ([C.c_void_p, C.c_void_p, C.POINTER(SolverOptions), C.c_void_p, C.c_void_p, C.c_int,
                          C.POINTER(SolverDiagnostics)], C.c_int),
    "apf_solve_minres_with_rhs": ([C.c_void_p, C.c_void_p, C.POINTER(SolverOptions), C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_int, C.POINTER(SolverDiagnostics)], C.c_int),
    "apf_solve_minres_correction": ([C.c_void_p, C.c_void_p, C.POINTER(SolverOptions), C.c_void_p, C.c_void_p,
                                     C.c_int, C.POINTER(SolverDiagnostics)], C.c_int),
    "apf_system_residual_norms": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.POINTER(C.c_double),
                                   C.POINTER(C.c_double)], C.c_int),
    "apf_system_set_solution": ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "apf_preconditioner_apply": ([C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int], C.c_int),
    "apf_system_solution_device_ptr": ([C.c_void_p, C.POINTER(C.c_void_p)], C.c_int),
}


def load():
    """Load libapf_b200.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m doubleadapparabolicfem_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def check(ctx, rc: int):
    if rc != APF_OK:
        lib = load()
        msg = lib.apf_ctx_last_error(ctx).decode() if ctx else ""
        raise ApfError(rc, msg)


class EstimatorResult(C.Structure):
    _fields_ = [
        ("flux_squared", C.c_double),
        ("divergence_squared", C.c_double),
        ("reconstruction_squared", C.c_double),
        ("eta_squared", C.c_double),
        ("n_slabs", C.c_int),
        ("n_patches", C.c_int),
        ("max_patch_cells", C.c_int),
        ("reconstruction_iterations", C.c_int),
        ("reconstruction_residual", C.c_double),
    ]


SIGNATURES["apf_estimate"] = ([C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                               C.c_void_p, C.POINTER(EstimatorResult)], C.c_int)

SIGNATURES["apf_system_keep_flux"] = ([C.c_void_p, C.c_void_p, C.c_int], C.c_int)
SIGNATURES["apf_flux_cells"] = ([C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.c_void_p, C.c_void_p], C.c_int)
SIGNATURES["apf_flux_sample"] = ([C.c_void_p, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int],
                                 C.c_int)

SIGNATURES["apf_true_residual_noalloc"] = ([C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                            C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int)

APF_LEARNED_NUM_PARAMS = 1442
_P = C.c_void_p
SIGNATURES.update({
    "apf_learned_model_create": ([C.POINTER(_P)], C.c_int),
    "apf_learned_model_destroy": ([_P], C.c_int),
    "apf_learned_model_set_params": ([_P, _P, C.c_int], C.c_int),
    "apf_learned_model_get_params": ([_P, _P, C.c_int], C.c_int),
    "apf_ctx_set_learned_model": ([_P, _P], C.c_int),
    "apf_learned_loss_and_grad": ([_P, _P, _P, C.c_int, C.c_int, C.c_int, C.c_uint64, _P, C.c_int,
                                   C.POINTER(C.c_double), _P], C.c_int),
    "apf_learned_forward": ([_P, _P, C.c_int, _P, _P, C.c_int, C.c_int], C.c_int),
    "apf_amg_info": ([_P, _P, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int),
                      C.POINTER(C.c_int)], C.c_int),
    "apf_amg_level_info": ([_P, _P, C.c_int, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                            C.POINTER(C.c_double), C.POINTER(C.c_double)], C.c_int),
    "apf_amg_level_copy": ([_P, _P, C.c_int, C.c_int, C.c_int, _P, _P, _P], C.c_int),
    "apf_amg_level_weights": ([_P, _P, C.c_int, C.c_int, C.c_int, _P], C.c_int),
    "apf_amg_level_features": ([_P, _P, C.c_int, C.c_int, _P], C.c_int),
})


class XIndicatorTotals(C.Structure):
    _fields_ = [("lambda_y_squared", C.c_double), ("initial_trace_squared", C.c_double), ("eta_squared", C.c_double)]


SIGNATURES["apf_x_indicators"] = ([_P, _P, C.c_int, _P, _P, _P, _P, C.POINTER(XIndicatorTotals)], C.c_int)
SIGNATURES["apf_y_estimator_threshold_squared"] = ([C.c_double, C.c_double, C.c_double, C.POINTER(C.c_double)], C.c_int)


class GEstimatorResult(C.Structure):
    _fields_ = [("lambda_difference_squared", C.c_double), ("solve_relative_residual", C.c_double),
                ("solve_iterations", C.c_int), ("n_g", C.c_int)]


SIGNATURES["apf_g_estimator"] = ([_P, _P, C.c_int32, _P, _P, _P, C.c_int32, C.c_double,
                                  C.POINTER(GEstimatorResult)], C.c_int)

SIGNATURES["apf_ctx_reserve_pool"] = ([_P, C.c_int64], C.c_int)
SIGNATURES["apf_ctx_pool_stats"] = ([_P, C.POINTER(C.c_int64), C.POINTER(C.c_int64), C.POINTER(C.c_int64),
                                     C.POINTER(C.c_int64)], C.c_int)
