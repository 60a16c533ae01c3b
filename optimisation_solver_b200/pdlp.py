"""``PdlpSolver`` -- the reference's PDLP entry point, on the device.

Mirrors ``pdlp::PdlpSolver::solve(const CompiledLp&, const PdlpOptions&) const
-> PdlpResult`` (pdlp_engine/include/pdlp/pdlp_solver.h:9-15): same options,
same statuses and messages, same sign conventions (row duals satisfy
stationarity c + A'y), and it never raises for bad input -- an invalid LP or
invalid options come back as ``PdlpStatus.INVALID_PROBLEM`` with the
reference's message. Every call goes through libpdlpgpu's C ABI.

Extensions, all optional: ``precision`` ("fp64" as the reference, or "mixed":
FP32 iterations with FP64 checks), a warm start, and ``solve_batch`` for many
independent LPs in one device solve.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import native
from .lp import CompiledLp, PdlpOptions, PdlpResult, PdlpStatus

_PRECISIONS = {"fp64": 0, "mixed": 1}
_PRECISION_NAMES = {0: "fp64", 1: "fp32", 2: "fp32+fp64"}


def _to_result(r: native.Result) -> PdlpResult:
    n, m = r.num_cols, r.num_rows

    def arr(p, k):
        if not p or k <= 0:
            return np.zeros(0)
        a = np.empty(k)
        C.memmove(a.ctypes.data, p, a.nbytes)
        return a

    return PdlpResult(
        status=PdlpStatus(r.status), status_message=r.status_message.decode(),
        primal=arr(r.primal, n), row_dual=arr(r.row_dual, m),
        dual_ray=arr(r.dual_ray, m), primal_ray=arr(r.primal_ray, n),
        primal_objective=r.primal_objective, dual_objective=r.dual_objective,
        primal_residual=r.primal_residual, dual_residual=r.dual_residual,
        relative_gap=r.relative_gap, iterations=r.iterations, step_trials=r.step_trials,
        restart_count=r.restart_count, solve_time_seconds=r.solve_time_seconds,
        final_step_size=r.final_step_size, static_step_bound=r.static_step_bound,
        final_primal_weight=r.final_primal_weight,
        precision=_PRECISION_NAMES.get(r.precision_used, "fp64"),
        fp64_iterations=r.fp64_iterations, device_seconds=r.device_seconds)


def _warm_struct(warm, keep):
    if warm is None:
        return None
    primal = warm.get("primal")
    dual = warm.get("row_dual")
    p = None if primal is None else np.ascontiguousarray(primal, dtype=np.float64)
    d = None if dual is None else np.ascontiguousarray(dual, dtype=np.float64)
    keep.extend([p, d])
    return native.WarmStart(native.ptr(p), native.ptr(d), float(warm.get("primal_weight", 0.0)))


class PdlpSolver:
    """Device PDLP solver. ``precision`` is "fp64" (the reference's
    arithmetic) or "mixed"; ``device`` is the CUDA ordinal. Further keywords
    are fields of ``pdlpgpu_ext_options`` (include/pdlpgpu.h), e.g.
    ``lane_elements``, ``vector_width``, ``two_kernel_trials=1`` or
    ``restart_metric=1`` (restarts on the normalised duality gap)."""

    def __init__(self, precision: str = "fp64", device: int = 0, **tuning):
        if precision not in _PRECISIONS:
            raise ValueError(f"precision must be one of {sorted(_PRECISIONS)}")
        self.precision = precision
        self.device = device
        self.tuning = tuning

    def _ext(self):
        return native.ext_struct(precision=_PRECISIONS[self.precision], device=self.device,
                                 **self.tuning)

    def solve(self, problem: CompiledLp, options: PdlpOptions | None = None,
              warm_start: dict | None = None) -> PdlpResult:
        L = native.lib()
        h = native.LpHandle(problem)
        o = native.options_struct(options or PdlpOptions())
        e = self._ext()
        keep: list = []
        w = _warm_struct(warm_start, keep)
        out = C.POINTER(native.Result)()
        L.pdlpgpu_solve_ex(C.byref(h.struct), C.byref(o), C.byref(e),
                           C.byref(w) if w is not None else None, C.byref(out))
        try:
            return _to_result(out.contents)
        finally:
            L.pdlpgpu_result_free(out)

    def solve_batch(self, problems, options: PdlpOptions | None = None,
                    warm_starts=None) -> list[PdlpResult]:
        L = native.lib()
        hs = [native.LpHandle(p) for p in problems]
        count = len(hs)
        arr = (C.POINTER(native.Lp) * count)(*[C.pointer(h.struct) for h in hs])
        o = native.options_struct(options or PdlpOptions())
        e = self._ext()
        keep: list = []
        warr = None
        if warm_starts is not None:
            ws = [_warm_struct(w, keep) for w in warm_starts]
            keep.append(ws)
            warr = (C.POINTER(native.WarmStart) * count)(
                *[C.pointer(w) if w is not None else C.POINTER(native.WarmStart)() for w in ws])
        outs = (C.POINTER(native.Result) * count)()
        L.pdlpgpu_solve_batch(arr, count, C.byref(o), C.byref(e), warr, outs)
        try:
            return [_to_result(outs[i].contents) for i in range(count)]
        finally:
            for i in range(count):
                L.pdlpgpu_result_free(outs[i])


    def time_kernels_batch(self, problems, options: PdlpOptions | None = None, reps: int = 10) -> dict:
        """The two trial kernels of a batch laid out as solve_batch lays it out,
        timed with every instance active (no solve)."""
        hs = [native.LpHandle(p) for p in problems]
        arr = (C.POINTER(native.Lp) * len(hs))(*[C.pointer(h.struct) for h in hs])
        o = native.options_struct(options or PdlpOptions())
        e = self._ext()
        out = np.zeros(6)
        rc = native.lib().pdlpgpu_batch_time_kernels(arr, len(hs), C.byref(o), C.byref(e), reps,
                                                     native.ptr(out))
        _check(rc, "batch_time_kernels")
        return dict(primal_ms=out[0], dual_ms=out[1], primal_bytes=out[2], dual_bytes=out[3],
                    at_padding=out[4], a_padding=out[5])


# ---------------------------------------------------------------------------
# Components (include/pdlpgpu_components.h)
# ---------------------------------------------------------------------------

def _check(rc: int, what: str):
    if rc != 0:
        raise RuntimeError(f"{what} failed: {native.last_error()}")


def spmv(problem: CompiledLp, v: np.ndarray, transpose: bool = False, precision: str = "fp64"):
    """A v (or A^T v) on the device (SparseMatrix::multiply / transposeMultiply)."""
    h = native.LpHandle(problem)
    v = np.ascontiguousarray(v, dtype=np.float64)
    out = np.zeros(problem.num_cols if transpose else problem.num_rows)
    _check(native.lib().pdlpgpu_spmv(C.byref(h.struct), int(transpose), _PRECISIONS[precision],
                                     native.ptr(v), native.ptr(out)), "spmv")
    return out


def ruiz(problem: CompiledLp, iterations: int = 10):
    """RuizScaler::equilibrate on the device: (row_scale, col_scale, scaled CSR values)."""
    h = native.LpHandle(problem)
    rs, cs = np.zeros(problem.num_rows), np.zeros(problem.num_cols)
    vals = np.zeros(max(problem.nnz, 1))
    _check(native.lib().pdlpgpu_ruiz(C.byref(h.struct), iterations, native.ptr(rs),
                                     native.ptr(cs), native.ptr(vals)), "ruiz")
    return rs, cs, vals[:problem.nnz]


def precondition(problem: CompiledLp):
    """Preconditioner::compute on the device: (tau, tau_inv, sigma, sigma_inv)."""
    h = native.LpHandle(problem)
    n, m = problem.num_cols, problem.num_rows
    t, ti, s, si = np.zeros(n), np.zeros(n), np.zeros(m), np.zeros(m)
    _check(native.lib().pdlpgpu_precondition(C.byref(h.struct), native.ptr(t), native.ptr(ti),
                                             native.ptr(s), native.ptr(si)), "precondition")
    return t, ti, s, si


def trial(problem: CompiledLp, tau, tau_inv, sigma, sigma_inv, x, y, ax, step, weight,
          precision: str = "fp64"):
    """One fused PDHG trial on the device (CpuPdhgKernel::trial)."""
    h = native.LpHandle(problem)
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (tau, tau_inv, sigma, sigma_inv, x, y, ax)]
    n, m = problem.num_cols, problem.num_rows
    xo, yo, axo, red = np.zeros(n), np.zeros(m), np.zeros(m), np.zeros(3)
    _check(native.lib().pdlpgpu_trial(C.byref(h.struct), _PRECISIONS[precision],
                                      *[native.ptr(a) for a in arrs], float(step), float(weight),
                                      native.ptr(xo), native.ptr(yo), native.ptr(axo),
                                      native.ptr(red)), "trial")
    return xo, yo, axo, red


def evaluate(problem: CompiledLp, x, y, rx=None, ry=None, infeasibility_tolerance=1e-8):
    """KKT metrics of (x, y) and ray verdicts of (x - rx, y - ry), on the device."""
    h = native.LpHandle(problem)
    n, m = problem.num_cols, problem.num_rows
    x = np.ascontiguousarray(x, dtype=np.float64)
    y = np.ascontiguousarray(y, dtype=np.float64)
    rx = np.zeros(n) if rx is None else np.ascontiguousarray(rx, dtype=np.float64)
    ry = np.zeros(m) if ry is None else np.ascontiguousarray(ry, dtype=np.float64)
    met, ver = np.zeros(8), np.zeros(6)
    _check(native.lib().pdlpgpu_evaluate(C.byref(h.struct), infeasibility_tolerance,
                                         native.ptr(x), native.ptr(y), native.ptr(rx),
                                         native.ptr(ry), native.ptr(met), native.ptr(ver)),
           "evaluate")
    metrics = dict(primal_objective=met[0], dual_objective=met[1], primal_residual=met[2],
                   dual_residual=met[3], relative_gap=met[4], kkt=met[5],
                   finite=bool(met[6]), dual_valid=bool(met[7]))
    verdicts = dict(dual_proves=bool(ver[0]), dual_value=ver[1], dual_relative=ver[2],
                    primal_proves=bool(ver[3]), primal_value=ver[4], primal_relative=ver[5])
    return metrics, verdicts


def normalized_gap(weight, x, g, x_lower, x_upper, x_ref, y, a, r_lower, r_upper, y_ref):
    """The normalised duality gap of (x, y) on the device (pdlpgpu_normalized_gap):
    g = c + A'y, a = A x, radius = the weighted distance to (x_ref, y_ref).
    Returns (gap, radius)."""
    arr = [np.ascontiguousarray(v, dtype=np.float64)
           for v in (x, g, x_lower, x_upper, x_ref, y, a, r_lower, r_upper, y_ref)]
    n, m = arr[0].size, arr[5].size
    out = np.zeros(2)
    _check(native.lib().pdlpgpu_normalized_gap(n, m, float(weight), *[native.ptr(v) for v in arr],
                                               native.ptr(out)), "normalized_gap")
    return float(out[0]), float(out[1])


def layout_stats(problem: CompiledLp, lane_elements: int = 0, vector_width: int = 0,
                 precision: str = "fp64") -> dict:
    """Host-only statistics of the SELL-G layout (no device needed)."""
    h = native.LpHandle(problem)
    e = native.ext_struct(precision=_PRECISIONS[precision], lane_elements=lane_elements,
                          vector_width=vector_width)
    st = np.zeros(8, dtype=np.int64)
    _check(native.lib().pdlpgpu_layout_stats(C.byref(h.struct), C.byref(e),
                                             native.ptr(st, C.c_int64)), "layout_stats")
    return dict(a_slices=int(st[0]), a_slots=int(st[1]), a_entries=int(st[2]),
                at_slices=int(st[3]), at_slots=int(st[4]), at_entries=int(st[5]),
                lane_elements=int(st[6]), vector_width=int(st[7]))


def layout_multiply(problem: CompiledLp, x, lane_elements: int = 0, vector_width: int = 0):
    """A x computed on the host by walking the SELL-G layout (no device)."""
    h = native.LpHandle(problem)
    e = native.ext_struct(lane_elements=lane_elements, vector_width=vector_width)
    x = np.ascontiguousarray(x, dtype=np.float64)
    out = np.zeros(problem.num_rows)
    _check(native.lib().pdlpgpu_layout_multiply(C.byref(h.struct), C.byref(e), native.ptr(x),
                                                native.ptr(out)), "layout_multiply")
    return out
