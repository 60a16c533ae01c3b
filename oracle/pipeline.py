"""ctypes wrapper of oracle/pipeline_shim.cpp -- TEST INFRASTRUCTURE ONLY.

Builds of the reference's own pipeline (oracle/Makefile):

* ``Pipeline("ref")`` -- oracle/_ref/libpipeline_ref.so, the reference as it is;
* ``Pipeline("gpu")`` -- oracle/_ref/libpipeline_gpu.so, the same sources with
  the GPU engine's ``pdlp::PdlpSolver::solve`` (include/pdlpgpu_override.hpp)
  linked in place of pdlp_engine/src/pdlp_solver.cpp, so ``solver::solve``
  reaches the GPU through ``solver::runPdlp`` (src/solver/orchestrator.cpp:337);
* ``Pipeline("fastpre")`` -- oracle/_ref/libpipeline_fastpre.so (`make presolve`),
  the reference with the library's fast presolve
  (include/pdlpgpu_presolve_override.hpp) linked in place of
  src/presolve/presolver.cpp and the reference's own PDLP;
* ``Pipeline("gpufast")`` -- oracle/_ref/libpipeline_gpufast.so, both: the fast
  presolve and the GPU engine behind ``solver::runPdlp``.

Models come from an MPS file read by the reference ``MpsReader`` or from the
flat Model IR arrays that ``export`` writes (fixtures travel that way).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBS = {"ref": os.path.join(HERE, "_ref", "libpipeline_ref.so"),
        "gpu": os.path.join(HERE, "_ref", "libpipeline_gpu.so"),
        "fastpre": os.path.join(HERE, "_ref", "libpipeline_fastpre.so"),
        "gpufast": os.path.join(HERE, "_ref", "libpipeline_gpufast.so")}
POSTSOLVE_TEST = {"ref": os.path.join(HERE, "_ref", "test_postsolve_integration_ref"),
                  "gpu": os.path.join(HERE, "_ref", "test_postsolve_integration_gpu")}

# solver::Engine (include/solver/dispatcher.h:14-30) and solver::SolveStatus
# (include/solver/solve_result.h:19-38), in declaration order.
ENGINE_PDLP, ENGINE_DUAL_SIMPLEX = 0, 1
STATUSES = ["optimal", "infeasible", "unbounded", "limit_reached", "numerical_failure",
            "invalid_model", "unsupported"]

_i32p, _i64p, _dp = C.POINTER(C.c_int32), C.POINTER(C.c_int64), C.POINTER(C.c_double)


class SolveOut(C.Structure):
    _fields_ = [("status", C.c_int32), ("executed_engine", C.c_int32),
                ("has_primal", C.c_int32), ("has_duals", C.c_int32), ("objective", C.c_double),
                ("max_dual_residual", C.c_double), ("iterations", C.c_int64),
                ("reduced_variables", C.c_int64), ("reduced_constraints", C.c_int64),
                ("status_name", C.c_char * 32), ("message", C.c_char * 256)]


@dataclass
class PipelineResult:
    status: str
    executed_engine: int
    has_primal: bool
    has_duals: bool
    objective: float
    max_dual_residual: float
    iterations: int
    message: str
    x: np.ndarray
    duals: np.ndarray
    reduced_costs: np.ndarray


MODEL_FIELDS = ("sense", "offset", "objective_index", "objective_value", "var_type", "var_lower",
                "var_upper", "row_lower", "row_upper", "row_start", "row_index", "row_value")


def available(kind: str) -> bool:
    return os.path.exists(LIBS[kind])


def _p(a, t):
    return a.ctypes.data_as(t)


class Pipeline:
    def __init__(self, kind: str = "ref"):
        if not available(kind):
            raise FileNotFoundError(f"{LIBS[kind]} is not built (make -C oracle pipeline)")
        self.kind = kind
        L = self.lib = C.CDLL(LIBS[kind])
        L.pl_read_mps.argtypes = [C.c_char_p, C.POINTER(C.c_void_p), C.c_char_p, C.c_int]
        L.pl_model_free.argtypes = [C.c_void_p]
        L.pl_model_dims.argtypes = [C.c_void_p, _i64p, _i64p]
        L.pl_compile.argtypes = [C.c_void_p, _i32p, _i32p, _i64p, C.c_char_p, C.c_int]
        L.pl_compiled_copy.argtypes = [C.c_void_p, _i64p, _i32p, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.pl_solve.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.c_double, C.c_int32,
                               C.POINTER(SolveOut), _dp, _dp, _dp]
        L.pl_model_sizes.argtypes = [C.c_void_p, _i64p, _i64p, _i64p]
        L.pl_model_export.argtypes = [C.c_void_p, _i32p, _dp, _i32p, _dp, _i32p, _dp, _dp, _dp,
                                      _dp, _i64p, _i32p, _dp]
        L.pl_model_import.argtypes = [C.c_int64, C.c_int64, C.c_int32, C.c_double, C.c_int64,
                                      _i32p, _dp, _i32p, _dp, _dp, _dp, _dp, _i64p, _i32p, _dp]
        L.pl_model_import.restype = C.c_void_p
        L.pl_name.argtypes = [C.c_void_p, C.c_int32, C.c_int64]
        L.pl_name.restype = C.c_char_p
        L.pl_warning_count.argtypes = [C.c_void_p]
        L.pl_warning_count.restype = C.c_int64
        L.pl_model_quadratic.argtypes = [C.c_void_p, _i32p, _i32p, _dp]

    # -- models --------------------------------------------------------------
    def read_mps(self, path: str) -> "Model":
        h, msg = C.c_void_p(), C.create_string_buffer(512)
        if self.lib.pl_read_mps(path.encode(), C.byref(h), msg, 512) != 0:
            raise ValueError(msg.value.decode())
        return Model(self, h)

    def import_model(self, arrays: dict) -> "Model":
        a = {k: np.ascontiguousarray(arrays[k]) for k in MODEL_FIELDS}
        nv, nc = a["var_lower"].size, a["row_lower"].size
        h = self.lib.pl_model_import(
            nv, nc, int(a["sense"].reshape(-1)[0]), float(a["offset"].reshape(-1)[0]),
            a["objective_index"].size,
            _p(a["objective_index"].astype(np.int32), _i32p),
            _p(a["objective_value"].astype(np.float64), _dp),
            _p(a["var_type"].astype(np.int32), _i32p), _p(a["var_lower"].astype(np.float64), _dp),
            _p(a["var_upper"].astype(np.float64), _dp), _p(a["row_lower"].astype(np.float64), _dp),
            _p(a["row_upper"].astype(np.float64), _dp), _p(a["row_start"].astype(np.int64), _i64p),
            _p(a["row_index"].astype(np.int32), _i32p), _p(a["row_value"].astype(np.float64), _dp))
        return Model(self, C.c_void_p(h))


class Model:
    def __init__(self, pipeline: Pipeline, handle: C.c_void_p):
        self.pl, self.h = pipeline, handle
        v, c = C.c_int64(), C.c_int64()
        pipeline.lib.pl_model_dims(handle, C.byref(v), C.byref(c))
        self.variables, self.constraints = v.value, c.value

    def __del__(self):
        try:
            self.pl.lib.pl_model_free(self.h)
        except Exception:
            pass

    def names(self) -> dict:
        """Model name, variable and row names, and the reader's warnings."""
        L = self.pl.lib
        get = lambda kind, i: L.pl_name(self.h, kind, i).decode()   # noqa: E731
        return dict(name=get(0, 0), variables=[get(1, j) for j in range(self.variables)],
                    rows=[get(2, i) for i in range(self.constraints)],
                    warnings=[get(3, k) for k in range(L.pl_warning_count(self.h))])

    def quadratic(self):
        """(i, j, value) arrays of the quadratic objective terms."""
        L = self.pl.lib
        no, nr, nq = C.c_int64(), C.c_int64(), C.c_int64()
        L.pl_model_sizes(self.h, C.byref(no), C.byref(nr), C.byref(nq))
        i, j, v = np.zeros(nq.value, np.int32), np.zeros(nq.value, np.int32), np.zeros(nq.value)
        if nq.value:
            L.pl_model_quadratic(self.h, _p(i, _i32p), _p(j, _i32p), _p(v, _dp))
        return i, j, v

    def export(self, allow_quadratic: bool = False) -> dict:
        """The Model IR as flat arrays (MODEL_FIELDS); quadratic terms are not
        carried (refused unless `allow_quadratic`)."""
        L = self.pl.lib
        no, nr, nq = C.c_int64(), C.c_int64(), C.c_int64()
        L.pl_model_sizes(self.h, C.byref(no), C.byref(nr), C.byref(nq))
        if nq.value and not allow_quadratic:
            raise ValueError("quadratic objective terms are not carried")
        sense, offset = np.zeros(1, np.int32), np.zeros(1)
        out = dict(objective_index=np.zeros(no.value, np.int32),
                   objective_value=np.zeros(no.value), var_type=np.zeros(self.variables, np.int32),
                   var_lower=np.zeros(self.variables), var_upper=np.zeros(self.variables),
                   row_lower=np.zeros(self.constraints), row_upper=np.zeros(self.constraints),
                   row_start=np.zeros(self.constraints + 1, np.int64),
                   row_index=np.zeros(nr.value, np.int32), row_value=np.zeros(nr.value))
        L.pl_model_export(self.h, _p(sense, _i32p), _p(offset, _dp),
                          _p(out["objective_index"], _i32p), _p(out["objective_value"], _dp),
                          _p(out["var_type"], _i32p), _p(out["var_lower"], _dp),
                          _p(out["var_upper"], _dp), _p(out["row_lower"], _dp),
                          _p(out["row_upper"], _dp), _p(out["row_start"], _i64p),
                          _p(out["row_index"], _i32p), _p(out["row_value"], _dp))
        out["sense"], out["offset"] = int(sense[0]), float(offset[0])
        return out

    def compile(self):
        """adapter::toCompiledLp -> the product's CompiledLp mirror."""
        from optimisation_solver_b200.lp import CompiledLp, SparseMatrix
        L = self.pl.lib
        rows, cols, nnz, msg = C.c_int32(), C.c_int32(), C.c_int64(), C.create_string_buffer(512)
        if L.pl_compile(self.h, C.byref(rows), C.byref(cols), C.byref(nnz), msg, 512) != 0:
            raise ValueError(msg.value.decode())
        m, n, k = rows.value, cols.value, nnz.value
        rs, ci, va = np.zeros(m + 1, np.int64), np.zeros(k, np.int32), np.zeros(k)
        c, off = np.zeros(n), np.zeros(1)
        rl, ru, xl, xu = np.zeros(m), np.zeros(m), np.zeros(n), np.zeros(n)
        L.pl_compiled_copy(self.h, _p(rs, _i64p), _p(ci, _i32p), _p(va, _dp), _p(c, _dp),
                           _p(off, _dp), _p(rl, _dp), _p(ru, _dp), _p(xl, _dp), _p(xu, _dp))
        return CompiledLp(SparseMatrix(m, n, rs, ci, va), c, rl, ru, xl, xu, float(off[0]))

    def solve(self, engine: int | None = ENGINE_PDLP, tolerance: float = 1e-8,
              time_limit: float = 0.0, threads: int = 1) -> PipelineResult:
        """solver::solve (presolve, dispatch, engine, postsolve)."""
        out = SolveOut()
        x, y, rc = np.zeros(self.variables), np.zeros(self.constraints), np.zeros(self.variables)
        st = self.pl.lib.pl_solve(self.h, -1 if engine is None else engine, tolerance, time_limit,
                                  threads, C.byref(out), _p(x, _dp), _p(y, _dp), _p(rc, _dp))
        if st != 0:
            raise RuntimeError(out.message.decode())
        return PipelineResult(status=STATUSES[out.status], executed_engine=out.executed_engine,
                              has_primal=bool(out.has_primal), has_duals=bool(out.has_duals),
                              objective=out.objective, max_dual_residual=out.max_dual_residual,
                              iterations=out.iterations, message=out.message.decode(),
                              x=x if out.has_primal else np.zeros(0),
                              duals=y if out.has_duals else np.zeros(0),
                              reduced_costs=rc if out.has_duals else np.zeros(0))
