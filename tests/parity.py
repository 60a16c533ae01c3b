"""Helpers that compare device results with the CPU oracle (the reference
pdlp_engine built from its sources, else the C restatement). Test
infrastructure only.

The acceptance rules follow the reference's own definitions:

* status equality with the reference's solve of the same input;
* the returned point, scored again by the oracle's TerminationChecker
  (pdlp_engine/src/termination.cpp:211-333), meets the requested tolerance on
  the primal residual, the dual residual and the relative gap;
* the device's own FP64 scores of that point agree with the oracle's;
* objectives: within `objective_rel` of the oracle's when both ran to a tight
  tolerance (the FP64-mode bar is 1e-6 relative), otherwise within
  4 x tol x (1 + |p| + |d|) -- two points that each pass the relative gap
  test at `tol` lie within about twice that bound of the optimum.
"""
from __future__ import annotations

import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np

# Slack on the oracle's rescoring of a point the device already accepted at
# `tol`: the two FP64 scores differ only in summation order.
SCORE_SLACK = 1e-9


def oracle_options(tol: float, **extra) -> dict:
    return dict(primal_tolerance=tol, dual_tolerance=tol, gap_tolerance=tol, thread_count=1,
                **extra)


def solve_many(oracle, lps, tol: float, **extra):
    """Oracle solves of `lps`, one host thread each (the library call releases
    the interpreter lock; the reference's solve keeps no global state)."""
    opts = oracle_options(tol, **extra)
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        return list(ex.map(lambda lp: oracle.solve(lp, opts), lps))


def status_name(status) -> str:
    return str(status)


def check_point(oracle, lp, x, y, tol: float, device_scores: dict | None = None):
    """The oracle's scores of (x, y); asserts they meet `tol` and, when given,
    agree with the device's own FP64 scores of the same point."""
    ev = oracle.evaluate(lp, x, y)
    assert ev["finite"]
    bound = tol * (1.0 + SCORE_SLACK)
    assert ev["primal_residual"] <= bound, ev
    assert ev["dual_residual"] <= bound, ev
    assert ev["relative_gap"] <= bound, ev
    if device_scores is not None:
        # The scores are ratios of FP64 sums; a tiny gap is a difference of two
        # objectives of ordinary size, so its summation-order error is absolute
        # (about 1e-15 of the objectives), hence the 1e-12 floor.
        for key in ("primal_residual", "dual_residual", "relative_gap"):
            got, want = device_scores[key], ev[key]
            assert abs(got - want) <= 1e-8 * max(abs(want), tol) + 1e-12, (key, got, want)
        for key in ("primal_objective", "dual_objective"):
            got, want = device_scores[key], ev[key]
            assert abs(got - want) <= 1e-10 * (1.0 + abs(want)), (key, got, want)
    return ev


def check_objective(device_obj: float, ref, tol: float, objective_rel: float | None = None):
    """Device objective against the oracle result `ref`."""
    p, d = ref.primal_objective, ref.dual_objective
    if objective_rel is not None:
        assert abs(device_obj - p) <= objective_rel * max(1.0, abs(p)), (device_obj, p)
    else:
        assert abs(device_obj - p) <= 4.0 * tol * (1.0 + abs(p) + abs(d)), (device_obj, p, d)


def max_relative(a: np.ndarray, b: np.ndarray) -> float:
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(1.0, np.abs(b)))) if a.size else 0.0
