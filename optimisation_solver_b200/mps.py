"""MPS files in and out (include/pdlpgpu_mps.h), the fast replacement of the
reference reader mps::MpsReader (src/mps/mps_reader.cpp).

    model = read_mps("lp.mps")        # the reference reader's model, as arrays
    lp = model.compiled_lp()           # adapter::toCompiledLp, ready for PdlpSolver
    write_mps(lp, "out.mps")           # free format, exact round trip
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import native
from .lp import CompiledLp, SparseMatrix

VARIABLE_TYPES = ("continuous", "integer", "binary")   # model::VariableType


@dataclass
class MpsModel:
    """model::Model (include/model/model.h) as flat arrays. Row terms are CSR
    (`row_start`, `row_index`, `row_value`), one entry per (row, column)
    pair, columns increasing."""

    name: str
    sense: int                     # 0 minimize, 1 maximize
    offset: float
    variable_names: list
    row_names: list
    var_type: np.ndarray
    var_lower: np.ndarray
    var_upper: np.ndarray
    row_lower: np.ndarray
    row_upper: np.ndarray
    objective_index: np.ndarray
    objective_value: np.ndarray
    row_start: np.ndarray
    row_index: np.ndarray
    row_value: np.ndarray
    quadratic_i: np.ndarray
    quadratic_j: np.ndarray
    quadratic_value: np.ndarray
    warnings: list = field(default_factory=list)
    _handle: object = None

    def compiled_lp(self) -> tuple[CompiledLp, bool]:
        """adapter::toCompiledLp: (the LP to minimise, whether the objective was
        negated because the model maximises). Raises ValueError with the
        adapter's message for integer or quadratic models and bad bounds."""
        lp = native.Lp()
        neg = C.c_int32()
        if native.lib().pdlpgpu_mps_lp(self._handle.ptr, C.byref(lp), C.byref(neg)) != 0:
            raise ValueError(native.last_error())
        m, n = lp.num_rows, lp.num_cols
        nnz = int(lp.row_start[m]) if m > 0 else 0

        def arr(p, k, dtype):
            return np.ctypeslib.as_array(p, shape=(k,)).astype(dtype, copy=True) if k else np.zeros(0, dtype)
        rs = arr(lp.row_start, m + 1, np.int64) if m >= 0 else np.zeros(1, np.int64)
        A = SparseMatrix(m, n, rs, arr(lp.col_index, nnz, np.int32), arr(lp.values, nnz, np.float64))
        out = CompiledLp(A, arr(lp.objective, n, np.float64), arr(lp.row_lower, m, np.float64),
                         arr(lp.row_upper, m, np.float64), arr(lp.var_lower, n, np.float64),
                         arr(lp.var_upper, n, np.float64), float(lp.objective_offset))
        return out, bool(neg.value)


class _Handle:
    def __init__(self, ptr):
        self.ptr = ptr

    def __del__(self):
        try:
            native.lib().pdlpgpu_mps_free(self.ptr)
        except Exception:
            pass


def read_mps(path: str) -> MpsModel:
    """Reads an MPS file; raises ValueError with the reference reader's message
    ("MpsReader Error (line N): ...") for a file it refuses."""
    L = native.lib()
    h = C.c_void_p()
    if L.pdlpgpu_mps_read(str(path).encode(), C.byref(h)) != 0:
        raise ValueError(native.last_error())
    handle = _Handle(h)
    sizes = np.zeros(8, np.int64)
    L.pdlpgpu_mps_sizes(h, native.ptr(sizes, C.c_int64))
    nv, nc, no, nr, nq, nw = (int(x) for x in sizes[:6])
    a = dict(var_type=np.zeros(nv, np.int32), var_lower=np.zeros(nv), var_upper=np.zeros(nv),
             row_lower=np.zeros(nc), row_upper=np.zeros(nc),
             objective_index=np.zeros(no, np.int32), objective_value=np.zeros(no),
             row_start=np.zeros(nc + 1, np.int64), row_index=np.zeros(nr, np.int32),
             row_value=np.zeros(nr), quadratic_i=np.zeros(nq, np.int32),
             quadratic_j=np.zeros(nq, np.int32), quadratic_value=np.zeros(nq))
    off = np.zeros(1)
    P = lambda k, t=C.c_double: native.ptr(a[k], t)   # noqa: E731
    L.pdlpgpu_mps_model(h, native.ptr(off), P("objective_index", C.c_int32), P("objective_value"),
                        P("var_type", C.c_int32), P("var_lower"), P("var_upper"), P("row_lower"),
                        P("row_upper"), P("row_start", C.c_int64), P("row_index", C.c_int32),
                        P("row_value"), P("quadratic_i", C.c_int32), P("quadratic_j", C.c_int32),
                        P("quadratic_value"))
    name = lambda kind, i: L.pdlpgpu_mps_name(h, kind, i).decode()   # noqa: E731
    return MpsModel(name=name(0, 0), sense=int(sizes[6]), offset=float(off[0]),
                    variable_names=[name(1, j) for j in range(nv)],
                    row_names=[name(2, i) for i in range(nc)],
                    warnings=[name(3, k) for k in range(nw)], _handle=handle, **a)


def write_mps(lp: CompiledLp, path: str, name: str = "LP") -> None:
    """Free-format MPS that reads back to the same LP bit for bit."""
    h = native.LpHandle(lp)
    if native.lib().pdlpgpu_mps_write(str(path).encode(), C.byref(h.struct), name.encode()) != 0:
        raise ValueError(native.last_error())
