"""Host-side LP data types, mirroring the reference's PDLP engine interface.

``CompiledLp`` mirrors ``pdlp::CompiledLp`` (pdlp_engine/include/pdlp/compiled_lp.h:17-63):

    minimize  objective' x + objective_offset
    s.t.      row_lower <= A x <= row_upper,   var_lower <= x <= var_upper

with A in canonical CSR (int64 row starts, int32 column indices, float64
values), and IEEE infinities for absent bounds. ``from_triplets`` restates
``SparseMatrix::fromTriplets`` (pdlp_engine/src/sparse_matrix.cpp:76-201):
entries are ordered by row then column, duplicates are summed and exact zeros
are dropped.

``PdlpOptions`` is ``pdlp::PdlpOptions`` field for field
(pdlp_engine/include/pdlp/pdlp_options.h:7-75) in snake_case, and ``PdlpStatus``
the seven-value status enum with the reference's ``toString`` spellings
(pdlp_engine/src/pdlp_solver.cpp:103-114).
"""
from __future__ import annotations

import enum
from dataclasses import dataclass, field, fields

import numpy as np

INF = float("inf")


class PdlpStatus(enum.IntEnum):
    OPTIMAL = 0
    INFEASIBLE = 1
    UNBOUNDED = 2
    ITERATION_LIMIT = 3
    TIME_LIMIT = 4
    NUMERICAL_FAILURE = 5
    INVALID_PROBLEM = 6

    def __str__(self) -> str:  # toString, pdlp_solver.cpp:103-114
        return self.name.lower()


@dataclass
class SparseMatrix:
    """Canonical CSR. ``from_triplets`` is the only builder, as in the reference."""

    rows: int
    columns: int
    row_start: np.ndarray   # int64 [rows+1]
    col_index: np.ndarray   # int32 [nnz]
    values: np.ndarray      # float64 [nnz]

    @property
    def nonzeros(self) -> int:
        return int(self.values.size)

    @staticmethod
    def from_triplets(rows: int, columns: int, row, col, value) -> "SparseMatrix":
        if rows < 0 or columns < 0:
            raise ValueError("Sparse matrix dimensions must be nonnegative")
        row = np.asarray(row, dtype=np.int64).ravel()
        col = np.asarray(col, dtype=np.int64).ravel()
        value = np.asarray(value, dtype=np.float64).ravel()
        if not (row.size == col.size == value.size):
            raise ValueError("triplet arrays differ in length")
        if row.size and (row.min() < 0 or row.max() >= rows or col.min() < 0 or col.max() >= columns):
            raise ValueError("Sparse matrix triplet index is out of range")
        if not np.all(np.isfinite(value)):
            raise ValueError("Sparse matrix coefficient must be finite")
        # Order by (row, column, input position); sum each (row, column) run in
        # input order, then drop exact zeros.
        order = np.lexsort((np.arange(row.size), col, row))
        r, c, v = row[order], col[order], value[order]
        if r.size:
            first = np.ones(r.size, dtype=bool)
            first[1:] = (r[1:] != r[:-1]) | (c[1:] != c[:-1])
            starts = np.flatnonzero(first)
            summed = v[starts].copy()
            run_len = np.diff(np.append(starts, r.size))
            for extra in range(1, int(run_len.max())):
                has = run_len > extra
                summed[has] += v[starts[has] + extra]
            r, c, v = r[starts], c[starts], summed
            keep = v != 0.0
            r, c, v = r[keep], c[keep], v[keep]
        counts = np.bincount(r, minlength=rows) if rows else np.zeros(0, np.int64)
        row_start = np.zeros(rows + 1, dtype=np.int64)
        np.cumsum(counts, out=row_start[1:])
        return SparseMatrix(rows, columns, row_start, c.astype(np.int32), v.astype(np.float64))

    def multiply(self, x: np.ndarray) -> np.ndarray:
        """y = A x in float64 (host helper for generators and tests)."""
        rows_of = np.repeat(np.arange(self.rows), np.diff(self.row_start))
        return np.bincount(rows_of, weights=self.values * np.asarray(x)[self.col_index],
                           minlength=self.rows)

    def transpose_multiply(self, y: np.ndarray) -> np.ndarray:
        rows_of = np.repeat(np.arange(self.rows), np.diff(self.row_start))
        return np.bincount(self.col_index, weights=self.values * np.asarray(y)[rows_of],
                           minlength=self.columns)


@dataclass
class CompiledLp:
    matrix: SparseMatrix
    objective: np.ndarray
    row_lower: np.ndarray
    row_upper: np.ndarray
    var_lower: np.ndarray
    var_upper: np.ndarray
    objective_offset: float = 0.0

    # Flat accessors used by the C-ABI marshalling and the oracles.
    @property
    def num_rows(self) -> int:
        return self.matrix.rows

    @property
    def num_cols(self) -> int:
        return self.matrix.columns

    @property
    def row_start(self) -> np.ndarray:
        return self.matrix.row_start

    @property
    def col_index(self) -> np.ndarray:
        return self.matrix.col_index

    @property
    def values(self) -> np.ndarray:
        return self.matrix.values

    @property
    def nnz(self) -> int:
        return self.matrix.nonzeros

    @staticmethod
    def build(rows, columns, triplets, objective, row_lower, row_upper, var_lower, var_upper,
              objective_offset=0.0) -> "CompiledLp":
        """Convenience constructor from a list of (row, column, value) triplets."""
        if len(triplets):
            t = np.asarray(triplets, dtype=np.float64).reshape(-1, 3)
            ti, tj, tv = t[:, 0].astype(np.int64), t[:, 1].astype(np.int64), t[:, 2]
        else:
            ti = tj = np.zeros(0, np.int64)
            tv = np.zeros(0)
        return CompiledLp(SparseMatrix.from_triplets(rows, columns, ti, tj, tv),
                          np.asarray(objective, np.float64), np.asarray(row_lower, np.float64),
                          np.asarray(row_upper, np.float64), np.asarray(var_lower, np.float64),
                          np.asarray(var_upper, np.float64), float(objective_offset))


@dataclass
class PdlpOptions:
    """pdlp::PdlpOptions, same defaults (pdlp_options.h:7-75)."""

    iteration_limit: int = 200000
    time_limit_seconds: float = 0.0
    primal_tolerance: float = 1e-6
    dual_tolerance: float = 1e-6
    gap_tolerance: float = 1e-6
    termination_check_frequency: int = 100
    power_iteration_count: int = 100
    thread_count: int = 0
    parallel_nonzero_threshold: int = 20000
    initial_step_safety: float = 0.90
    minimum_step_scale: float = 1e-6
    maximum_primal_weight: float = 1e6
    minimum_primal_weight: float = 1e-6
    use_ruiz_scaling: bool = True
    ruiz_iterations: int = 10
    detect_infeasibility: bool = True
    infeasibility_tolerance: float = 1e-8
    use_diagonal_preconditioning: bool = True
    use_adaptive_linesearch: bool = True
    maximum_step_trials: int = 60
    use_averaging: bool = True
    use_restarts: bool = True
    use_feasibility_polishing: bool = True
    minimum_restart_iterations: int = 64
    maximum_restart_iterations: int = 100000
    restart_sufficient_decay: float = 0.20
    restart_necessary_decay: float = 0.80
    restart_artificial_fraction: float = 0.36
    initial_primal_weight: float = 1.0
    primal_weight_smoothing: float = 0.50
    polishing_iterations: int = 5000

    def as_dict(self) -> dict:
        return {f.name: getattr(self, f.name) for f in fields(self)}

    def with_tolerance(self, tol: float) -> "PdlpOptions":
        """All three tolerances at once, as the reference's runPdlp sets them
        from SolverOptions.tolerance (src/solver/orchestrator.cpp:330-335)."""
        d = self.as_dict()
        d.update(primal_tolerance=tol, dual_tolerance=tol, gap_tolerance=tol)
        return PdlpOptions(**d)


@dataclass
class PdlpResult:
    """pdlp::PdlpResult (pdlp_result.h:26-62) plus this engine's extensions."""

    status: PdlpStatus = PdlpStatus.INVALID_PROBLEM
    status_message: str = ""
    primal: np.ndarray = field(default_factory=lambda: np.zeros(0))
    row_dual: np.ndarray = field(default_factory=lambda: np.zeros(0))
    dual_ray: np.ndarray = field(default_factory=lambda: np.zeros(0))
    primal_ray: np.ndarray = field(default_factory=lambda: np.zeros(0))
    primal_objective: float = float("nan")
    dual_objective: float = -INF
    primal_residual: float = INF
    dual_residual: float = INF
    relative_gap: float = INF
    iterations: int = 0
    step_trials: int = 0
    restart_count: int = 0
    solve_time_seconds: float = 0.0
    final_step_size: float = 0.0
    static_step_bound: float = 0.0
    final_primal_weight: float = 1.0
    # Extensions: precision that produced the point ("fp64", "fp32", "fp32+fp64"),
    # iterations spent in the FP64 stage, and the device time of the solve.
    precision: str = "fp64"
    fp64_iterations: int = 0
    device_seconds: float = 0.0
