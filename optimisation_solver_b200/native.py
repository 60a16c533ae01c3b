"""ctypes binding of libpdlpgpu (include/pdlpgpu*.h).

The library is the product: there is no Python or CPU fallback. If it is not
built, loading raises ``NativeLibraryMissing`` naming the build command.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libpdlpgpu.so")


class NativeLibraryMissing(ImportError):
    pass


_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)


class Lp(C.Structure):
    _fields_ = [("num_rows", C.c_int32), ("num_cols", C.c_int32), ("row_start", _i64p),
                ("col_index", _i32p), ("values", _dp), ("objective", _dp),
                ("objective_offset", C.c_double), ("row_lower", _dp), ("row_upper", _dp),
                ("var_lower", _dp), ("var_upper", _dp)]


_i8p = C.POINTER(C.c_int8)


class PresolveModel(C.Structure):
    """pdlpgpu_presolve_model (include/pdlpgpu_presolve.h)."""
    _fields_ = [("num_variables", C.c_int64), ("num_constraints", C.c_int64),
                ("var_lower", _dp), ("var_upper", _dp), ("var_type", _i8p),
                ("row_lower", _dp), ("row_upper", _dp), ("row_start", _i64p),
                ("row_index", _i32p), ("row_value", _dp), ("objective_offset", C.c_double),
                ("num_objective_terms", C.c_int64), ("objective_index", _i32p),
                ("objective_value", _dp), ("num_quadratic_terms", C.c_int64),
                ("quadratic_index1", _i32p), ("quadratic_index2", _i32p),
                ("quadratic_value", _dp)]


class PresolveResult(C.Structure):
    """pdlpgpu_presolve_result (include/pdlpgpu_presolve.h)."""
    _fields_ = [("infeasible", C.c_int32), ("converged", C.c_int32), ("has_maps", C.c_int32),
                ("original_variables", C.c_int64), ("original_constraints", C.c_int64),
                ("presolved_variables", C.c_int64), ("presolved_constraints", C.c_int64),
                ("initial_objective_offset", C.c_double),
                ("presolved_objective_offset", C.c_double),
                ("variable_origin", _i64p), ("var_lower", _dp), ("var_upper", _dp),
                ("constraint_origin", _i64p), ("row_lower", _dp), ("row_upper", _dp),
                ("row_start", _i64p), ("row_index", _i32p), ("row_value", _dp),
                ("num_objective_terms", C.c_int64), ("objective_index", _i32p),
                ("objective_value", _dp), ("num_quadratic_terms", C.c_int64),
                ("quadratic_index1", _i32p), ("quadratic_index2", _i32p),
                ("quadratic_value", _dp),
                ("num_transformations", C.c_int64), ("tr_type", _i32p), ("tr_reason", _i32p),
                ("tr_index", _i64p), ("tr_variable", _i64p), ("tr_constraint", _i64p),
                ("tr_old_value", _dp), ("tr_new_value", _dp), ("tr_offset_change", _dp),
                ("num_fixed", C.c_int64), ("fixed_origin", _i64p), ("fixed_value", _dp),
                ("fixed_linear", _dp), ("fixed_quadratic_diagonal", _dp),
                ("fixed_cross_start", _i64p), ("fixed_cross_variable", _i64p),
                ("fixed_cross_value", _dp),
                ("num_removed", C.c_int64), ("removed_origin", _i64p), ("removed_lower", _dp),
                ("removed_upper", _dp), ("removed_reason", _i32p), ("removed_singleton", _i8p),
                ("removed_singleton_variable", _i64p), ("removed_singleton_coefficient", _dp),
                ("removed_duplicate", _i8p), ("removed_duplicate_of", _i64p),
                ("removed_scale", _dp)]


class Options(C.Structure):
    _fields_ = [("iteration_limit", C.c_int64), ("time_limit_seconds", C.c_double),
                ("primal_tolerance", C.c_double), ("dual_tolerance", C.c_double),
                ("gap_tolerance", C.c_double), ("termination_check_frequency", C.c_int32),
                ("power_iteration_count", C.c_int32), ("thread_count", C.c_int32),
                ("parallel_nonzero_threshold", C.c_int64), ("initial_step_safety", C.c_double),
                ("minimum_step_scale", C.c_double), ("maximum_primal_weight", C.c_double),
                ("minimum_primal_weight", C.c_double), ("use_ruiz_scaling", C.c_int32),
                ("ruiz_iterations", C.c_int32), ("detect_infeasibility", C.c_int32),
                ("infeasibility_tolerance", C.c_double),
                ("use_diagonal_preconditioning", C.c_int32),
                ("use_adaptive_linesearch", C.c_int32), ("maximum_step_trials", C.c_int32),
                ("use_averaging", C.c_int32), ("use_restarts", C.c_int32),
                ("use_feasibility_polishing", C.c_int32),
                ("minimum_restart_iterations", C.c_int32),
                ("maximum_restart_iterations", C.c_int32),
                ("restart_sufficient_decay", C.c_double), ("restart_necessary_decay", C.c_double),
                ("restart_artificial_fraction", C.c_double),
                ("initial_primal_weight", C.c_double), ("primal_weight_smoothing", C.c_double),
                ("polishing_iterations", C.c_int32)]


class ExtOptions(C.Structure):
    _fields_ = [("precision", C.c_int32), ("device", C.c_int32), ("lane_elements", C.c_int32),
                ("vector_width", C.c_int32), ("chunk_slack", C.c_int32),
                ("fp32_stall_checks", C.c_int32), ("fp32_switch_factor", C.c_int32),
                ("disable_graphs", C.c_int32), ("cta_slots", C.c_int32),
                ("layout", C.c_int32), ("lane_instances", C.c_int32),
                ("two_kernel_trials", C.c_int32), ("restart_metric", C.c_int32),
                ("reserved", C.c_int32 * 3)]


class WarmStart(C.Structure):
    _fields_ = [("primal", _dp), ("row_dual", _dp), ("primal_weight", C.c_double)]


class Result(C.Structure):
    _fields_ = [("status", C.c_int32), ("status_message", C.c_char * 160),
                ("num_rows", C.c_int32), ("num_cols", C.c_int32), ("primal", _dp),
                ("row_dual", _dp), ("dual_ray", _dp), ("primal_ray", _dp),
                ("primal_objective", C.c_double), ("dual_objective", C.c_double),
                ("primal_residual", C.c_double), ("dual_residual", C.c_double),
                ("relative_gap", C.c_double), ("iterations", C.c_int64),
                ("step_trials", C.c_int64), ("restart_count", C.c_int32),
                ("solve_time_seconds", C.c_double), ("final_step_size", C.c_double),
                ("static_step_bound", C.c_double), ("final_primal_weight", C.c_double),
                ("precision_used", C.c_int32), ("fp64_iterations", C.c_int64),
                ("device_seconds", C.c_double)]


# Every symbol the public headers declare, with its signature.
SIGNATURES = {
    "pdlpgpu_default_options": (None, [C.POINTER(Options)]),
    "pdlpgpu_default_ext_options": (None, [C.POINTER(ExtOptions)]),
    "pdlpgpu_solve": (C.c_int32, [C.POINTER(Lp), C.POINTER(Options), C.POINTER(WarmStart),
                                  C.POINTER(C.POINTER(Result))]),
    "pdlpgpu_solve_ex": (C.c_int32, [C.POINTER(Lp), C.POINTER(Options), C.POINTER(ExtOptions),
                                     C.POINTER(WarmStart), C.POINTER(C.POINTER(Result))]),
    "pdlpgpu_solve_batch": (C.c_int32, [C.POINTER(C.POINTER(Lp)), C.c_int32, C.POINTER(Options),
                                        C.POINTER(ExtOptions), C.POINTER(C.POINTER(WarmStart)),
                                        C.POINTER(C.POINTER(Result))]),
    "pdlpgpu_result_free": (None, [C.POINTER(Result)]),
    "pdlpgpu_status_string": (C.c_char_p, [C.c_int32]),
    "pdlpgpu_last_error": (C.c_char_p, []),
    "pdlpgpu_device_count": (C.c_int32, []),
    "pdlpgpu_spmv": (C.c_int32, [C.POINTER(Lp), C.c_int32, C.c_int32, _dp, _dp]),
    "pdlpgpu_ruiz": (C.c_int32, [C.POINTER(Lp), C.c_int32, _dp, _dp, _dp]),
    "pdlpgpu_precondition": (C.c_int32, [C.POINTER(Lp), _dp, _dp, _dp, _dp]),
    "pdlpgpu_trial": (C.c_int32, [C.POINTER(Lp), C.c_int32] + [_dp] * 7 +
                      [C.c_double, C.c_double] + [_dp] * 4),
    "pdlpgpu_evaluate": (C.c_int32, [C.POINTER(Lp), C.c_double] + [_dp] * 6),
    "pdlpgpu_normalized_gap": (C.c_int32, [C.c_int32, C.c_int32, C.c_double] + [_dp] * 10 + [_dp]),
    "pdlpgpu_trial_noalloc": (C.c_int32, [C.c_int32, C.c_int32] + [C.c_void_p] * 18 +
                              [C.c_double, C.c_double] + [C.c_void_p] * 5),
    "pdlpgpu_layout_stats": (C.c_int32, [C.POINTER(Lp), C.POINTER(ExtOptions), _i64p]),
    "pdlpgpu_layout_multiply": (C.c_int32, [C.POINTER(Lp), C.POINTER(ExtOptions), _dp, _dp]),
    "pdlpgpu_session_create": (C.c_int32, [C.POINTER(Lp), C.c_int32, C.POINTER(Options),
                                           C.POINTER(ExtOptions), C.POINTER(C.c_void_p)]),
    "pdlpgpu_session_destroy": (None, [C.c_void_p]),
    "pdlpgpu_session_load": (C.c_int32, [C.c_void_p, C.c_int32] + [C.c_void_p] * 8),
    "pdlpgpu_session_solve": (C.c_int32, [C.c_void_p]),
    "pdlpgpu_session_read": (C.c_int32, [C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                         _i32p, _i64p, _dp]),
    "pdlpgpu_session_last_timing": (C.c_int32, [C.c_void_p, _dp, _i64p]),
    "pdlpgpu_session_stream": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int64] + [C.c_void_p] * 10 +
                               [_i32p, _i64p, _dp]),
    "pdlpgpu_session_time_kernels": (C.c_int32, [C.c_void_p, C.c_int32, _dp]),
    "pdlpgpu_session_loop_timing": (C.c_int32, [C.c_void_p, _dp]),
    "pdlpgpu_batch_time_kernels": (C.c_int32, [C.POINTER(C.POINTER(Lp)), C.c_int32, C.POINTER(Options),
                                               C.POINTER(ExtOptions), C.c_int32, _dp]),
    "pdlpgpu_mlp_create": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_uint64,
                                       C.c_int32, C.POINTER(C.c_void_p)]),
    "pdlpgpu_mlp_destroy": (None, [C.c_void_p]),
    "pdlpgpu_mlp_forward": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p]),
    "pdlpgpu_mlp_train_step": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                           C.c_float, C.POINTER(C.c_float)]),
    "pdlpgpu_mlp_gradients": (C.c_int32, [C.c_void_p] + [C.c_void_p] * 9 + [C.POINTER(C.c_float)]),
    "pdlpgpu_mlp_get_params": (C.c_int32, [C.c_void_p] + [C.c_void_p] * 6),
    "pdlpgpu_mlp_set_params": (C.c_int32, [C.c_void_p] + [C.c_void_p] * 6),
    "pdlpgpu_gemm_bf16": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_int32]),
    "pdlpgpu_gemm_time": (C.c_int32, [C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_int32, C.c_int32, _dp]),
    "pdlpgpu_mlp_launches": (C.c_int64, [C.c_void_p]),
    "pdlpgpu_encode_features": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                            C.c_void_p, C.c_void_p, C.c_void_p]),
    "pdlpgpu_encode_targets": (C.c_int32, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                           C.c_int32, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                           C.c_void_p, C.c_float, C.c_float, C.c_void_p]),
    "pdlpgpu_decode_warmstart": (C.c_int32, [C.c_void_p, C.c_int32, C.c_int32, C.c_int32,
                                             C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_float, C.c_float, C.c_void_p, C.c_void_p,
                                             C.c_void_p]),
    # MPS files (include/pdlpgpu_mps.h)
    "pdlpgpu_mps_read": (C.c_int32, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "pdlpgpu_mps_free": (None, [C.c_void_p]),
    "pdlpgpu_mps_sizes": (None, [C.c_void_p, _i64p]),
    "pdlpgpu_mps_name": (C.c_char_p, [C.c_void_p, C.c_int32, C.c_int64]),
    "pdlpgpu_mps_model": (None, [C.c_void_p, _dp, _i32p, _dp, _i32p, _dp, _dp, _dp, _dp, _i64p,
                                 _i32p, _dp, _i32p, _i32p, _dp]),
    "pdlpgpu_mps_lp": (C.c_int32, [C.c_void_p, C.POINTER(Lp), _i32p]),
    "pdlpgpu_mps_write": (C.c_int32, [C.c_char_p, C.POINTER(Lp), C.c_char_p]),
    # presolve (include/pdlpgpu_presolve.h)
    "pdlpgpu_presolve": (C.c_int32, [C.POINTER(PresolveModel),
                                     C.POINTER(C.POINTER(PresolveResult))]),
    "pdlpgpu_presolve_free": (None, [C.POINTER(PresolveResult)]),
    "pdlpgpu_presolve_reason_string": (C.c_char_p, [C.c_int32]),
}

_LIB = None


def lib():
    """Loads libpdlpgpu.so once; raises NativeLibraryMissing if it is not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise NativeLibraryMissing(
                f"{LIB_PATH} is not built; run `python -m optimisation_solver_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def ptr(a, ctype=C.c_double):
    return None if a is None else a.ctypes.data_as(C.POINTER(ctype))


class LpHandle:
    """Holds the contiguous arrays of one LP alive while the C struct is used.

    The C ABI receives bare pointers, so lengths are checked here: a vector
    whose length does not match A is passed as NULL, which the library
    rejects with the reference's dimension message, and an inconsistent CSR
    (row_start not of length rows + 1, or fewer entries than it claims) is
    passed with a NULL row_start ("CompiledLp contains an invalid sparse
    matrix") -- never an array the library would read past its end."""

    def __init__(self, lp):
        m, n = int(lp.num_rows), int(lp.num_cols)
        self.row_start = np.ascontiguousarray(lp.row_start, dtype=np.int64)
        self.col_index = np.ascontiguousarray(lp.col_index, dtype=np.int32)
        self.values = np.ascontiguousarray(lp.values, dtype=np.float64)

        def vec(a, k):
            v = np.ascontiguousarray(a, dtype=np.float64)
            return v if v.ndim == 1 and v.shape[0] == k else None

        self.objective = vec(lp.objective, n)
        self.row_lower = vec(lp.row_lower, m)
        self.row_upper = vec(lp.row_upper, m)
        self.var_lower = vec(lp.var_lower, n)
        self.var_upper = vec(lp.var_upper, n)
        csr_ok = (m >= 0 and self.row_start.ndim == 1 and self.row_start.shape[0] == m + 1 and
                  self.col_index.shape[0] == self.values.shape[0] and
                  0 <= int(self.row_start[-1]) <= self.values.shape[0])
        starts = ptr(self.row_start, C.c_int64) if csr_ok else None
        self.struct = Lp(m, n, starts, ptr(self.col_index, C.c_int32), ptr(self.values),
                         ptr(self.objective), float(lp.objective_offset), ptr(self.row_lower),
                         ptr(self.row_upper), ptr(self.var_lower), ptr(self.var_upper))


def options_struct(options) -> Options:
    o = Options()
    lib().pdlpgpu_default_options(C.byref(o))
    if options is not None:
        for name, _ in Options._fields_:
            setattr(o, name, type(getattr(o, name))(getattr(options, name)))
    return o


def ext_struct(**kw) -> ExtOptions:
    e = ExtOptions()
    lib().pdlpgpu_default_ext_options(C.byref(e))
    for k, v in kw.items():
        setattr(e, k, int(v))
    return e


def last_error() -> str:
    return lib().pdlpgpu_last_error().decode()
