"""ctypes binding for the CPU oracles (TEST INFRASTRUCTURE ONLY).

Two shared libraries export the interface of ``oracle_abi.h``:

* ``oracle/_ref/libpdlp_ref.so`` -- the reference pdlp_engine compiled from its
  own sources by ``oracle/Makefile`` (parity flags), and
  ``oracle/_ref/libpdlp_ref_fast.so`` -- the same sources at the reference's
  Release flags, used only as the timed CPU baseline;
* ``oracle/_port/libpdlp_port.so`` -- the plain-C restatement ``pdlp_port.c``.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg
import this module, and only as the checker; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_LIB = os.path.join(HERE, "_ref", "libpdlp_ref.so")
REF_FAST_LIB = os.path.join(HERE, "_ref", "libpdlp_ref_fast.so")
PORT_LIB = os.path.join(HERE, "_port", "libpdlp_port.so")

STATUS_NAMES = ["optimal", "infeasible", "unbounded", "iteration_limit", "time_limit",
                "numerical_failure", "invalid_problem"]

_dp = C.POINTER(C.c_double)
_i64p = C.POINTER(C.c_int64)
_i32p = C.POINTER(C.c_int32)


class OrcLp(C.Structure):
    _fields_ = [("rows", C.c_int32), ("cols", C.c_int32), ("nnz", C.c_int64),
                ("row_start", _i64p), ("col_index", _i32p), ("values", _dp),
                ("objective", _dp), ("objective_offset", C.c_double),
                ("row_lower", _dp), ("row_upper", _dp), ("var_lower", _dp), ("var_upper", _dp)]


class OrcOptions(C.Structure):
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


class OrcResult(C.Structure):
    _fields_ = [("status", C.c_int32), ("has_dual_ray", C.c_int32),
                ("has_primal_ray", C.c_int32), ("restart_count", C.c_int32),
                ("iterations", C.c_int64), ("step_trials", C.c_int64),
                ("primal_objective", C.c_double), ("dual_objective", C.c_double),
                ("primal_residual", C.c_double), ("dual_residual", C.c_double),
                ("relative_gap", C.c_double), ("solve_time_seconds", C.c_double),
                ("final_step_size", C.c_double), ("static_step_bound", C.c_double),
                ("final_primal_weight", C.c_double), ("primal_size", C.c_int32),
                ("dual_size", C.c_int32), ("message", C.c_char * 160)]


# Option names in snake_case, matching the product's PdlpOptions mirror.
OPTION_FIELDS = [f for f, _ in OrcOptions._fields_]


@dataclass
class OracleResult:
    status: str
    message: str
    primal: np.ndarray
    row_dual: np.ndarray
    dual_ray: np.ndarray
    primal_ray: np.ndarray
    primal_objective: float
    dual_objective: float
    primal_residual: float
    dual_residual: float
    relative_gap: float
    iterations: int
    step_trials: int
    restart_count: int
    solve_time_seconds: float
    final_step_size: float
    static_step_bound: float
    final_primal_weight: float
    extra: dict = field(default_factory=dict)


def _ptr(a, ctype):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None


def build_port():
    """Compiles the C restatement with gcc if it is not built yet (no reference needed)."""
    if not os.path.exists(PORT_LIB):
        subprocess.run(["make", "-s", "-C", HERE, "port"], check=True)
    return PORT_LIB


def available(kind: str) -> bool:
    return os.path.exists({"ref": REF_LIB, "ref_fast": REF_FAST_LIB, "port": PORT_LIB}[kind])


class Oracle:
    """One loaded oracle library. ``kind`` is "ref", "ref_fast" or "port"."""

    def __init__(self, kind: str = "port"):
        if kind == "port":
            build_port()
        path = {"ref": REF_LIB, "ref_fast": REF_FAST_LIB, "port": PORT_LIB}[kind]
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library {path} is not built (make -C oracle)")
        self.kind = kind
        self.lib = C.CDLL(path)
        L = self.lib
        L.orc_default_options.argtypes = [C.POINTER(OrcOptions)]
        L.orc_solve.argtypes = [C.POINTER(OrcLp), C.POINTER(OrcOptions), _dp, _dp, _dp, _dp,
                                C.POINTER(OrcResult)]
        L.orc_solve.restype = C.c_int
        L.orc_from_triplets.argtypes = [C.c_int32, C.c_int32, C.c_int64, _i32p, _i32p, _dp,
                                        _i64p, _i32p, _dp, _i64p, _i32p, _dp, _i64p]
        L.orc_from_triplets.restype = C.c_int
        L.orc_multiply.argtypes = [C.POINTER(OrcLp), _dp, _dp]
        L.orc_transpose_multiply.argtypes = [C.POINTER(OrcLp), _dp, _dp]
        L.orc_ruiz.argtypes = [C.POINTER(OrcLp), C.c_int32] + [_dp] * 8
        L.orc_condition_spread.argtypes = [C.POINTER(OrcLp)]
        L.orc_condition_spread.restype = C.c_double
        L.orc_precondition.argtypes = [C.POINTER(OrcLp), C.c_int32, _dp, _dp, _dp, _dp]
        L.orc_spectral_norm.argtypes = [C.POINTER(OrcLp), C.c_int32, _i32p]
        L.orc_spectral_norm.restype = C.c_double
        L.orc_trial.argtypes = [C.POINTER(OrcLp), _dp, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double,
                                C.c_double, _dp, _dp, _dp, _dp]
        L.orc_trial.restype = C.c_int
        L.orc_evaluate.argtypes = [C.POINTER(OrcLp), _dp, _dp, _dp]
        L.orc_test_dual_ray.argtypes = [C.POINTER(OrcLp), C.c_double, _dp, _dp]
        L.orc_test_primal_ray.argtypes = [C.POINTER(OrcLp), C.c_double, _dp, _dp]

    # -- conversion --------------------------------------------------------
    @staticmethod
    def _lp(lp):
        """``lp`` is any object with the CompiledLp-like fields used in the
        product's mirror (num_rows, num_cols, row_start, col_index, values,
        objective, objective_offset, row_lower, row_upper, var_lower, var_upper)."""
        keep = dict(
            row_start=np.ascontiguousarray(lp.row_start, dtype=np.int64),
            col_index=np.ascontiguousarray(lp.col_index, dtype=np.int32),
            values=np.ascontiguousarray(lp.values, dtype=np.float64),
            objective=np.ascontiguousarray(lp.objective, dtype=np.float64),
            row_lower=np.ascontiguousarray(lp.row_lower, dtype=np.float64),
            row_upper=np.ascontiguousarray(lp.row_upper, dtype=np.float64),
            var_lower=np.ascontiguousarray(lp.var_lower, dtype=np.float64),
            var_upper=np.ascontiguousarray(lp.var_upper, dtype=np.float64),
        )
        s = OrcLp(int(lp.num_rows), int(lp.num_cols), int(keep["values"].size),
                  _ptr(keep["row_start"], C.c_int64), _ptr(keep["col_index"], C.c_int32),
                  _ptr(keep["values"], C.c_double), _ptr(keep["objective"], C.c_double),
                  float(lp.objective_offset), _ptr(keep["row_lower"], C.c_double),
                  _ptr(keep["row_upper"], C.c_double), _ptr(keep["var_lower"], C.c_double),
                  _ptr(keep["var_upper"], C.c_double))
        return s, keep

    def default_options(self) -> dict:
        o = OrcOptions()
        self.lib.orc_default_options(C.byref(o))
        return {f: getattr(o, f) for f in OPTION_FIELDS}

    def _options(self, overrides):
        o = OrcOptions()
        self.lib.orc_default_options(C.byref(o))
        for k, v in (overrides or {}).items():
            if k not in OPTION_FIELDS:
                raise KeyError(k)
            setattr(o, k, v)
        return o

    # -- entry points ------------------------------------------------------
    def solve(self, lp, options: dict | None = None) -> OracleResult:
        s, keep = self._lp(lp)
        o = self._options(options)
        n, m = int(lp.num_cols), int(lp.num_rows)
        primal = np.zeros(n)
        dual = np.zeros(m)
        dray = np.zeros(m)
        pray = np.zeros(n)
        r = OrcResult()
        self.lib.orc_solve(C.byref(s), C.byref(o), _ptr(primal, C.c_double),
                           _ptr(dual, C.c_double), _ptr(dray, C.c_double),
                           _ptr(pray, C.c_double), C.byref(r))
        del keep
        return OracleResult(
            status=STATUS_NAMES[r.status], message=r.message.decode(),
            primal=primal if r.primal_size else np.zeros(0),
            row_dual=dual if r.dual_size else np.zeros(0),
            dual_ray=dray if r.has_dual_ray else np.zeros(0),
            primal_ray=pray if r.has_primal_ray else np.zeros(0),
            primal_objective=r.primal_objective, dual_objective=r.dual_objective,
            primal_residual=r.primal_residual, dual_residual=r.dual_residual,
            relative_gap=r.relative_gap, iterations=r.iterations, step_trials=r.step_trials,
            restart_count=r.restart_count, solve_time_seconds=r.solve_time_seconds,
            final_step_size=r.final_step_size, static_step_bound=r.static_step_bound,
            final_primal_weight=r.final_primal_weight)

    def from_triplets(self, rows, cols, ti, tj, tv):
        ti = np.ascontiguousarray(ti, dtype=np.int32)
        tj = np.ascontiguousarray(tj, dtype=np.int32)
        tv = np.ascontiguousarray(tv, dtype=np.float64)
        cnt = ti.size
        rs = np.zeros(rows + 1, np.int64)
        ci = np.zeros(max(cnt, 1), np.int32)
        va = np.zeros(max(cnt, 1))
        cs = np.zeros(cols + 1, np.int64)
        ri = np.zeros(max(cnt, 1), np.int32)
        cv = np.zeros(max(cnt, 1))
        nnz = C.c_int64(0)
        rc = self.lib.orc_from_triplets(rows, cols, cnt, _ptr(ti, C.c_int32), _ptr(tj, C.c_int32),
                                        _ptr(tv, C.c_double), _ptr(rs, C.c_int64),
                                        _ptr(ci, C.c_int32), _ptr(va, C.c_double),
                                        _ptr(cs, C.c_int64), _ptr(ri, C.c_int32),
                                        _ptr(cv, C.c_double), C.byref(nnz))
        if rc != 0:
            raise ValueError("invalid triplets")
        k = nnz.value
        return rs, ci[:k].copy(), va[:k].copy(), cs, ri[:k].copy(), cv[:k].copy()

    def multiply(self, lp, x):
        s, keep = self._lp(lp)
        x = np.ascontiguousarray(x, dtype=np.float64)
        out = np.zeros(int(lp.num_rows))
        self.lib.orc_multiply(C.byref(s), _ptr(x, C.c_double), _ptr(out, C.c_double))
        return out

    def transpose_multiply(self, lp, y):
        s, keep = self._lp(lp)
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros(int(lp.num_cols))
        self.lib.orc_transpose_multiply(C.byref(s), _ptr(y, C.c_double), _ptr(out, C.c_double))
        return out

    def ruiz(self, lp, iterations=10):
        s, keep = self._lp(lp)
        n, m, k = int(lp.num_cols), int(lp.num_rows), int(np.asarray(lp.values).size)
        out = dict(row_scale=np.zeros(m), col_scale=np.zeros(n), values=np.zeros(max(k, 1)),
                   objective=np.zeros(n), row_lower=np.zeros(m), row_upper=np.zeros(m),
                   var_lower=np.zeros(n), var_upper=np.zeros(n))
        self.lib.orc_ruiz(C.byref(s), iterations, *[_ptr(out[f], C.c_double) for f in
                          ["row_scale", "col_scale", "values", "objective", "row_lower",
                           "row_upper", "var_lower", "var_upper"]])
        out["values"] = out["values"][:k]
        return out

    def condition_spread(self, lp):
        s, keep = self._lp(lp)
        return self.lib.orc_condition_spread(C.byref(s))

    def precondition(self, lp, enabled=True):
        s, keep = self._lp(lp)
        n, m = int(lp.num_cols), int(lp.num_rows)
        tau, tinv, sig, sinv = np.zeros(n), np.zeros(n), np.zeros(m), np.zeros(m)
        self.lib.orc_precondition(C.byref(s), int(enabled), _ptr(tau, C.c_double),
                                  _ptr(tinv, C.c_double), _ptr(sig, C.c_double),
                                  _ptr(sinv, C.c_double))
        return tau, tinv, sig, sinv

    def spectral_norm(self, lp, iterations=100):
        s, keep = self._lp(lp)
        conv = C.c_int32(0)
        v = self.lib.orc_spectral_norm(C.byref(s), iterations, C.byref(conv))
        return v, bool(conv.value)

    def trial(self, lp, tau, tinv, sig, sinv, x, y, ax, step, weight):
        s, keep = self._lp(lp)
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (tau, tinv, sig, sinv, x, y, ax)]
        n, m = int(lp.num_cols), int(lp.num_rows)
        xo, yo, axo, red = np.zeros(n), np.zeros(m), np.zeros(m), np.zeros(3)
        fin = self.lib.orc_trial(C.byref(s), *[_ptr(a, C.c_double) for a in arrs], step, weight,
                                 _ptr(xo, C.c_double), _ptr(yo, C.c_double),
                                 _ptr(axo, C.c_double), _ptr(red, C.c_double))
        return xo, yo, axo, red, bool(fin)

    def evaluate(self, lp, x, y):
        s, keep = self._lp(lp)
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64)
        out = np.zeros(8)
        self.lib.orc_evaluate(C.byref(s), _ptr(x, C.c_double), _ptr(y, C.c_double),
                              _ptr(out, C.c_double))
        return dict(primal_objective=out[0], dual_objective=out[1], primal_residual=out[2],
                    dual_residual=out[3], relative_gap=out[4], kkt=out[5],
                    finite=bool(out[6]), dual_valid=bool(out[7]))

    def test_dual_ray(self, lp, direction, tolerance=1e-8):
        s, keep = self._lp(lp)
        d = np.ascontiguousarray(direction, dtype=np.float64)
        v = np.zeros(3)
        self.lib.orc_test_dual_ray(C.byref(s), tolerance, _ptr(d, C.c_double), _ptr(v, C.c_double))
        return bool(v[0]), v[1], v[2]

    def test_primal_ray(self, lp, direction, tolerance=1e-8):
        s, keep = self._lp(lp)
        d = np.ascontiguousarray(direction, dtype=np.float64)
        v = np.zeros(3)
        self.lib.orc_test_primal_ray(C.byref(s), tolerance, _ptr(d, C.c_double),
                                     _ptr(v, C.c_double))
        return bool(v[0]), v[1], v[2]


def best_available() -> Oracle:
    """The reference library when it is built, else the restatement."""
    return Oracle("ref") if available("ref") else Oracle("port")
