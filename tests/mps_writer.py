"""Free-format MPS writer for CompiledLp (test infrastructure).

Used to write the 1000 x 2000 planted LP as an MPS file and read it back with
the reference MpsReader (src/mps/mps_reader.cpp). Numbers are written with 17
significant digits, so the round trip is exact. Row senses: equal bounds ->
E; only an upper bound -> L; only a lower bound -> G; both finite -> G with a
RANGES entry of (upper - lower), which the MPS convention maps back to
[rhs, rhs + |R|]. Rows with neither bound are not representable (an N row is
dropped by readers) and are refused.
"""
from __future__ import annotations

import numpy as np


def _num(v: float) -> str:
    return repr(float(v))


def write_free_mps(lp, path: str, name: str = "LP") -> None:
    m, n = lp.num_rows, lp.num_cols
    rl, ru = np.asarray(lp.row_lower), np.asarray(lp.row_upper)
    xl, xu = np.asarray(lp.var_lower), np.asarray(lp.var_upper)
    lines = [f"NAME {name}", "ROWS", " N obj"]
    rhs, ranges = [], []
    for i in range(m):
        lo, hi = rl[i], ru[i]
        if np.isfinite(lo) and np.isfinite(hi) and lo == hi:
            lines.append(f" E r{i}")
            rhs.append((i, lo))
        elif np.isfinite(hi) and not np.isfinite(lo):
            lines.append(f" L r{i}")
            rhs.append((i, hi))
        elif np.isfinite(lo) and not np.isfinite(hi):
            lines.append(f" G r{i}")
            rhs.append((i, lo))
        elif np.isfinite(lo) and np.isfinite(hi):
            lines.append(f" G r{i}")
            rhs.append((i, lo))
            ranges.append((i, hi - lo))
        else:
            raise ValueError(f"row {i} has no finite bound")
    lines.append("COLUMNS")
    # Column-wise entries: the transpose of the CSR.
    rows_of = np.repeat(np.arange(m), np.diff(lp.row_start))
    order = np.lexsort((rows_of, lp.col_index))
    cols_sorted = np.asarray(lp.col_index)[order]
    rows_sorted = rows_of[order]
    vals_sorted = np.asarray(lp.values)[order]
    starts = np.searchsorted(cols_sorted, np.arange(n + 1))
    c = np.asarray(lp.objective)
    for j in range(n):
        # The objective entry first, even when zero, so that every column is
        # declared in order.
        lines.append(f" x{j} obj {_num(c[j])}")
        for k in range(starts[j], starts[j + 1]):
            lines.append(f" x{j} r{rows_sorted[k]} {_num(vals_sorted[k])}")
    lines.append("RHS")
    if lp.objective_offset != 0.0:
        # MPS stores the negated objective constant on the objective row.
        lines.append(f" rhs obj {_num(-lp.objective_offset)}")
    for i, v in rhs:
        if v != 0.0:
            lines.append(f" rhs r{i} {_num(v)}")
    if ranges:
        lines.append("RANGES")
        for i, v in ranges:
            lines.append(f" rng r{i} {_num(v)}")
    lines.append("BOUNDS")
    for j in range(n):
        lo, hi = xl[j], xu[j]
        if np.isfinite(lo) and np.isfinite(hi) and lo == hi:
            lines.append(f" FX bnd x{j} {_num(lo)}")
            continue
        if not np.isfinite(lo) and not np.isfinite(hi):
            lines.append(f" FR bnd x{j}")
            continue
        if not np.isfinite(lo):
            lines.append(f" MI bnd x{j}")
        elif lo != 0.0:
            lines.append(f" LO bnd x{j} {_num(lo)}")
        if np.isfinite(hi):
            lines.append(f" UP bnd x{j} {_num(hi)}")
    lines.append("ENDATA")
    with open(path, "w") as f:
        f.write("\n".join(lines) + "\n")
