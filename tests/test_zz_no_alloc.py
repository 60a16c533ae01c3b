"""pdlpgpu_trial_noalloc: the fused PDHG trial for callers that cannot let the
library allocate device memory (a process that owns all device memory through
its own pool and budget, or a loop that must not take cudaMalloc's
device-wide synchronisation). Every buffer here is allocated by the caller
(torch), the library's only scratch is its fixed static device array, and the
result must equal the allocating entry point pdlpgpu_trial's on two calls in
a row (the second starting from the first one's output, so the shared
scratch is reused). Tolerance as in the trial parity tests: 1e-10 relative.

This file is collected last, so a run that stops at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from optimisation_solver_b200 import native
from optimisation_solver_b200 import pdlp
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
    return np.abs(a - b).max() <= TOL * max(1.0, np.abs(b).max())


@pytest.mark.parametrize("name,build", [
    ("random_feasible", lambda: cases.random_feasible(300, 420, 21)),
    ("feasible_box", lambda: cases.feasible_box(2500, 3000, 5, per_row=10)),
])
def test_noalloc_trial_matches_allocating_trial_twice(name, build):
    import torch

    lp = build()
    dev = torch.device("cuda", 0)
    tau, tinv, sig, sinv = pdlp.precondition(lp)
    at_start, at_index, at_values = _transpose_csr(lp)

    def d(a, dtype=torch.float64):
        return torch.as_tensor(np.ascontiguousarray(a)).to(device=dev, dtype=dtype)

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
    ax = lp.matrix.multiply(x)

    lib = native.lib()
    for step, weight in ((0.7, 1.3), (0.45, 0.8)):
        want_x, want_y, want_ax, want_red = pdlp.trial(lp, tau, tinv, sig, sinv, x, y, ax, step, weight)
        dx, dy, dax = d(x), d(y), d(ax)
        ox = torch.empty(lp.num_cols, dtype=torch.float64, device=dev)
        oy = torch.empty(lp.num_rows, dtype=torch.float64, device=dev)
        oax = torch.empty(lp.num_rows, dtype=torch.float64, device=dev)
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
        got_x, got_y, got_ax, got_red = (t.cpu().numpy() for t in (ox, oy, oax, red))
        assert _close(got_x, want_x)
        assert _close(got_y, want_y)
        assert _close(got_ax, want_ax)
        for g_, w_ in zip(got_red, want_red):
            assert abs(g_ - w_) <= TOL * max(1.0, abs(w_))
        # The next call starts from this call's output.
        x, y, ax = got_x, got_y, got_ax


def test_noalloc_rejects_oversized_problems():
    rc = native.lib().pdlpgpu_trial_noalloc(9_000_000, 10, *([None] * 18), 1.0, 1.0,
                                            None, None, None, None, None)
    assert rc == -1
    assert "at most 8388608" in native.last_error()
