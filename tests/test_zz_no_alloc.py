"""pdlpgpu_trial_noalloc: the fused PDHG trial for callers that cannot let the
library allocate device memory (a process that owns all device memory through
its own pool and budget, or a loop that must not take cudaMalloc's
device-wide synchronisation). Every buffer here is allocated by the caller
(torch), and the library's only scratch is its fixed static device array.

Each call's result is compared with the CPU oracle's trial (the reference's
CpuPdhgKernel::trial) and, where both halves are non-empty, with the
allocating entry point pdlpgpu_trial (reached through `pdlp.trial`), on two
calls in a row: the second starts
from the first one's output, so the shared scratch is reused. Tolerance as in
the trial parity tests: 1e-10 relative. The cases cover a problem with many
CTAs per half, and problems with no rows or no columns, where only one of the
two halves launches and the skipped half's sums must come back as zero.

This file is collected last, so a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from optimisation_solver_b200 import native
from optimisation_solver_b200 import pdlp
from optimisation_solver_b200.lp import CompiledLp
from oracle.oracle import best_available
from tests import cases

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _transpose_csr(lp):
    rows_of = np.repeat(np.arange(lp.num_rows, dtype=np.int64), np.diff(lp.row_start))
    order = np.lexsort((rows_of, lp.col_index))
    counts = np.bincount(lp.col_index, minlength=lp.num_cols)
    start = np.zeros(lp.num_cols + 1, dtype=np.int64)
    np.cumsum(counts, out=start[1:])
    return start, rows_of[order].astype(np.int32), lp.values[order]


def _close(a, b):
    a, b = np.asarray(a), np.asarray(b)
    if a.size == 0 and b.size == 0:
        return True
    return np.abs(a - b).max() <= TOL * max(1.0, np.abs(b).max())


def _columns_only(n):
    """No rows: every column is a free-standing box-constrained variable."""
    rng = np.random.default_rng(3)
    return CompiledLp.build(0, n, ([], [], []), rng.standard_normal(n), [], [],
                            np.zeros(n), np.full(n, 4.0))


def _rows_only(m):
    """No columns: only the dual half runs (every row is empty)."""
    rng = np.random.default_rng(4)
    lo = -rng.random(m)
    return CompiledLp.build(m, 0, ([], [], []), [], lo, lo + 1.0, [], [])


CASES = [
    ("random_feasible", lambda: cases.random_feasible(300, 420, 21)),
    ("feasible_box", lambda: cases.feasible_box(2500, 3000, 5, per_row=10)),
    # 24 primal CTAs and 12 dual CTAs of 1024 lines each.
    ("many_ctas", lambda: cases.feasible_box(12000, 24000, 9, per_row=6)),
    ("no_rows", lambda: _columns_only(3000)),
    ("no_columns", lambda: _rows_only(2100)),
]


@pytest.mark.parametrize("name,build", CASES, ids=[c[0] for c in CASES])
def test_noalloc_trial_matches_allocating_trial_and_oracle_twice(name, build):
    import torch

    lp = build()
    dev = torch.device("cuda", 0)
    oracle = best_available()
    tau, tinv, sig, sinv = oracle.precondition(lp)
    at_start, at_index, at_values = _transpose_csr(lp)

    def d(a, dtype=torch.float64):
        # One element at least, so that an empty vector still has a device address.
        a = np.ascontiguousarray(a)
        if a.size == 0:
            a = np.zeros(1, dtype=a.dtype)
        return torch.as_tensor(a).to(device=dev, dtype=dtype)

    buffers = dict(
        a_start=d(lp.row_start, torch.int64), a_index=d(lp.col_index, torch.int32),
        a_values=d(lp.values), at_start=d(at_start, torch.int64),
        at_index=d(at_index, torch.int32), at_values=d(at_values), c=d(lp.objective),
        xl=d(lp.var_lower), xu=d(lp.var_upper), tau=d(tau), tinv=d(tinv),
        rl=d(lp.row_lower), ru=d(lp.row_upper), sig=d(sig), sinv=d(sinv))
    rng = np.random.default_rng(7)
    lo = np.where(np.isfinite(lp.var_lower), lp.var_lower, -5.0)
    hi = np.where(np.isfinite(lp.var_upper), lp.var_upper, 5.0)
    x = lo + (hi - lo) * rng.random(lp.num_cols)
    y = rng.standard_normal(lp.num_rows)
    ax = oracle.multiply(lp, x)

    lib = native.lib()
    for step, weight in ((0.7, 1.3), (0.45, 0.8)):
        want = oracle.trial(lp, tau, tinv, sig, sinv, x, y, ax, step, weight)[:4]
        references = [want]
        if lp.num_rows > 0 and lp.num_cols > 0:
            references.append(pdlp.trial(lp, tau, tinv, sig, sinv, x, y, ax, step, weight))
        dx, dy, dax = d(x), d(y), d(ax)
        ox = torch.empty(max(lp.num_cols, 1), dtype=torch.float64, device=dev)
        oy = torch.empty(max(lp.num_rows, 1), dtype=torch.float64, device=dev)
        oax = torch.empty(max(lp.num_rows, 1), dtype=torch.float64, device=dev)
        red = torch.full((3,), float("nan"), dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        b = buffers
        args = [b["a_start"], b["a_index"], b["a_values"], b["at_start"], b["at_index"],
                b["at_values"], b["c"], b["xl"], b["xu"], b["tau"], b["tinv"], b["rl"], b["ru"],
                b["sig"], b["sinv"], dx, dy, dax]
        rc = lib.pdlpgpu_trial_noalloc(lp.num_rows, lp.num_cols,
                                       *[C.c_void_p(t.data_ptr()) for t in args],
                                       step, weight, C.c_void_p(ox.data_ptr()),
                                       C.c_void_p(oy.data_ptr()), C.c_void_p(oax.data_ptr()),
                                       C.c_void_p(red.data_ptr()), None)
        assert rc == 0, native.last_error()
        torch.cuda.synchronize()
        got_x = ox.cpu().numpy()[:lp.num_cols]
        got_y = oy.cpu().numpy()[:lp.num_rows]
        got_ax = oax.cpu().numpy()[:lp.num_rows]
        got_red = red.cpu().numpy()
        for reference in references:
            ref_x, ref_y, ref_ax, ref_red = reference
            assert _close(got_x, ref_x)
            assert _close(got_y, ref_y)
            assert _close(got_ax, ref_ax)
            for g_, w_ in zip(got_red, ref_red):
                assert abs(g_ - w_) <= TOL * max(1.0, abs(w_))
        if lp.num_rows == 0:
            assert got_red[1] == 0.0 and got_red[2] == 0.0
        if lp.num_cols == 0:
            assert got_red[0] == 0.0
        # The next call starts from this call's output.
        x, y, ax = got_x, got_y, got_ax


def test_noalloc_rejects_oversized_problems():
    rc = native.lib().pdlpgpu_trial_noalloc(9_000_000, 10, *([None] * 18), 1.0, 1.0,
                                            None, None, None, None, None)
    assert rc == -1
    assert "at most 8388608" in native.last_error()
