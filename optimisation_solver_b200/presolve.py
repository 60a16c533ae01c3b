"""Presolve: presolve::Presolver::run (src/presolve/presolver.cpp:1045-1155)
through the library's pdlpgpu_presolve (include/pdlpgpu_presolve.h).

``Presolver().run(model)`` takes a ``PresolveModel`` (a model::Model as
arrays) and returns a ``PresolveResult`` holding the reference's result
fields as numpy arrays: the reduced model, the flags and counts, the
transformation log with reason codes (``reason_text`` maps each code to the
reference's string; a per-entry list would cost a string per log entry, 15M
of them on the 500k-row configuration), the fixed-variable
and removed-constraint records and the index maps (empty when the first
infeasibility test refused the input, as in the reference). Host code only.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import native

CONTINUOUS, INTEGER, BINARY = 0, 1, 2


@dataclass
class PresolveModel:
    """A model::Model (include/model/model.h) as arrays: variables (bounds,
    type), rows (bounds, CSR terms in the row's order), the objective's
    linear and quadratic term lists and its constant."""
    var_lower: np.ndarray
    var_upper: np.ndarray
    row_lower: np.ndarray
    row_upper: np.ndarray
    row_start: np.ndarray
    row_index: np.ndarray
    row_value: np.ndarray
    objective_index: np.ndarray
    objective_value: np.ndarray
    var_type: np.ndarray | None = None
    objective_offset: float = 0.0
    quadratic_index1: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    quadratic_index2: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    quadratic_value: np.ndarray = field(default_factory=lambda: np.zeros(0))

    @staticmethod
    def from_lp(lp) -> "PresolveModel":
        """The model of a CompiledLp-shaped LP (CSR rows, row and variable
        bounds, dense objective; zero objective entries left out)."""
        nz = np.flatnonzero(lp.objective)
        return PresolveModel(
            var_lower=lp.var_lower, var_upper=lp.var_upper, row_lower=lp.row_lower,
            row_upper=lp.row_upper, row_start=lp.row_start, row_index=lp.col_index,
            row_value=lp.values, objective_index=nz.astype(np.int32),
            objective_value=lp.objective[nz], objective_offset=float(lp.objective_offset))

    def buffers(self) -> "_Buffers":
        return _Buffers(self)


class _Buffers:
    """Contiguous, correctly typed copies of a model's arrays and the C struct
    that points at them (alive as long as this object)."""

    def __init__(self, m: PresolveModel):
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)  # noqa: E731
        n = int(np.asarray(m.var_lower).size)
        rows = int(np.asarray(m.row_lower).size)
        self.keep = dict(
            vlo=f64(m.var_lower), vhi=f64(m.var_upper),
            vt=np.ascontiguousarray(np.zeros(n, np.int8) if m.var_type is None else m.var_type,
                                    dtype=np.int8),
            rlo=f64(m.row_lower), rhi=f64(m.row_upper),
            rs=np.ascontiguousarray(m.row_start, dtype=np.int64), ri=i32(m.row_index),
            rv=f64(m.row_value), oi=i32(m.objective_index), ov=f64(m.objective_value),
            q1=i32(m.quadratic_index1), q2=i32(m.quadratic_index2), qv=f64(m.quadratic_value))
        k = self.keep
        if k["vhi"].size != n or k["vt"].size != n or k["rhi"].size != rows or \
                k["rs"].size != rows + 1 or k["ov"].size != k["oi"].size or \
                not (k["q1"].size == k["q2"].size == k["qv"].size):
            raise ValueError("presolve model arrays have inconsistent lengths")
        nnz = int(k["rs"][-1]) if rows + 1 == k["rs"].size else 0
        if k["ri"].size < nnz or k["rv"].size < nnz:
            raise ValueError("presolve model: row_start names more terms than given")
        p = native.ptr
        self.struct = native.PresolveModel(
            n, rows, p(k["vlo"]), p(k["vhi"]), p(k["vt"], C.c_int8), p(k["rlo"]), p(k["rhi"]),
            p(k["rs"], C.c_int64), p(k["ri"], C.c_int32), p(k["rv"]), float(m.objective_offset),
            k["oi"].size, p(k["oi"], C.c_int32), p(k["ov"]), k["qv"].size, p(k["q1"], C.c_int32),
            p(k["q2"], C.c_int32), p(k["qv"]))


@dataclass
class PresolveResult:
    """presolve::PresolveResult (include/presolve/presolve_result.h) as arrays."""
    infeasible: bool
    converged: bool
    has_maps: bool
    original_variables: int
    original_constraints: int
    presolved_variables: int
    presolved_constraints: int
    initial_objective_offset: float
    presolved_objective_offset: float
    model: PresolveModel
    variable_origin: np.ndarray
    constraint_origin: np.ndarray
    transformations: dict
    fixed_variables: dict
    removed_constraints: dict
    reason_text: dict   # reason code (PDLPGPU_PR_*) -> the reference's text


def _arr(ptr, count, dtype):
    count = int(count)
    if count == 0 or not ptr:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dtype, copy=True)


class Presolver:
    """presolve::Presolver (include/presolve/presolver.h:9-60)."""

    def run(self, model: PresolveModel) -> PresolveResult:
        L = native.lib()
        buf = model.buffers()
        out = C.POINTER(native.PresolveResult)()
        if L.pdlpgpu_presolve(C.byref(buf.struct), C.byref(out)) != 0:
            raise ValueError(L.pdlpgpu_last_error().decode())
        try:
            r = out.contents
            nv, nc = r.presolved_variables, r.presolved_constraints
            rs = _arr(r.row_start, nc + 1, np.int64)
            nnz = int(rs[-1]) if rs.size else 0
            reduced = PresolveModel(
                var_lower=_arr(r.var_lower, nv, np.float64),
                var_upper=_arr(r.var_upper, nv, np.float64),
                row_lower=_arr(r.row_lower, nc, np.float64),
                row_upper=_arr(r.row_upper, nc, np.float64),
                row_start=rs, row_index=_arr(r.row_index, nnz, np.int32),
                row_value=_arr(r.row_value, nnz, np.float64),
                objective_index=_arr(r.objective_index, r.num_objective_terms, np.int32),
                objective_value=_arr(r.objective_value, r.num_objective_terms, np.float64),
                objective_offset=r.presolved_objective_offset,
                quadratic_index1=_arr(r.quadratic_index1, r.num_quadratic_terms, np.int32),
                quadratic_index2=_arr(r.quadratic_index2, r.num_quadratic_terms, np.int32),
                quadratic_value=_arr(r.quadratic_value, r.num_quadratic_terms, np.float64))
            vo = _arr(r.variable_origin, nv, np.int64)
            reduced.var_type = buf.keep["vt"][vo]
            nt, nf, nr = r.num_transformations, r.num_fixed, r.num_removed
            reasons = _arr(r.tr_reason, nt, np.int32)
            removed_reasons = _arr(r.removed_reason, nr, np.int32)
            text = {int(c): L.pdlpgpu_presolve_reason_string(int(c)).decode()
                    for c in np.unique(np.concatenate([reasons, removed_reasons]))}
            cs = _arr(r.fixed_cross_start, nf + 1, np.int64)
            return PresolveResult(
                infeasible=bool(r.infeasible), converged=bool(r.converged),
                has_maps=bool(r.has_maps), original_variables=r.original_variables,
                original_constraints=r.original_constraints, presolved_variables=nv,
                presolved_constraints=nc, initial_objective_offset=r.initial_objective_offset,
                presolved_objective_offset=r.presolved_objective_offset, model=reduced,
                variable_origin=vo, constraint_origin=_arr(r.constraint_origin, nc, np.int64),
                reason_text=text,
                transformations=dict(
                    type=_arr(r.tr_type, nt, np.int32), reason=reasons,
                    index=_arr(r.tr_index, nt, np.int64),
                    variable=_arr(r.tr_variable, nt, np.int64),
                    constraint=_arr(r.tr_constraint, nt, np.int64),
                    old_value=_arr(r.tr_old_value, nt, np.float64),
                    new_value=_arr(r.tr_new_value, nt, np.float64),
                    offset_change=_arr(r.tr_offset_change, nt, np.float64)),
                fixed_variables=dict(
                    origin=_arr(r.fixed_origin, nf, np.int64),
                    value=_arr(r.fixed_value, nf, np.float64),
                    linear=_arr(r.fixed_linear, nf, np.float64),
                    quadratic_diagonal=_arr(r.fixed_quadratic_diagonal, nf, np.float64),
                    cross_start=cs,
                    cross_variable=_arr(r.fixed_cross_variable, cs[-1] if cs.size else 0,
                                        np.int64),
                    cross_value=_arr(r.fixed_cross_value, cs[-1] if cs.size else 0,
                                     np.float64)),
                removed_constraints=dict(
                    origin=_arr(r.removed_origin, nr, np.int64),
                    lower=_arr(r.removed_lower, nr, np.float64),
                    upper=_arr(r.removed_upper, nr, np.float64),
                    reason=removed_reasons,
                    singleton=_arr(r.removed_singleton, nr, np.int8),
                    singleton_variable=_arr(r.removed_singleton_variable, nr, np.int64),
                    singleton_coefficient=_arr(r.removed_singleton_coefficient, nr,
                                               np.float64),
                    duplicate=_arr(r.removed_duplicate, nr, np.int8),
                    duplicate_of=_arr(r.removed_duplicate_of, nr, np.int64),
                    scale=_arr(r.removed_scale, nr, np.float64)))
        finally:
            L.pdlpgpu_presolve_free(out)
