"""Fused trials (k_fused): one thread-block cluster per small LP runs the
trials of a check interval in one launch. Its arithmetic and reduction order
are the two-kernel path's (k_primal, k_dual and the decision in the last dual
CTA), so a solve must give the same statuses, counters and points bit for bit
with either; `two_kernel_trials=1` forces the two-kernel path. Cases: the
1000 x 2000 planted LP (FP64 and mixed through its FP64 stage), the
reference's KATs (infeasible, unbounded, polishing after an iteration limit),
a 10000 x 20000 LP too large to stage its slices in shared memory, a batch of
different LPs, and the per-iteration time of both paths.
"""
import time

import numpy as np
import pytest

from optimisation_solver_b200 import generators as g
from optimisation_solver_b200.lp import PdlpOptions
from optimisation_solver_b200.pdlp import PdlpSolver
from tests import cases

pytestmark = pytest.mark.gpu


def _same(a, b):
    assert a.status == b.status
    assert a.iterations == b.iterations and a.step_trials == b.step_trials
    assert a.restart_count == b.restart_count
    assert np.array_equal(a.primal, b.primal) and np.array_equal(a.row_dual, b.row_dual)
    assert np.array_equal(a.dual_ray, b.dual_ray) and np.array_equal(a.primal_ray, b.primal_ray)
    assert a.primal_objective == b.primal_objective


def _opts(tol=1e-6, **kw):
    o = PdlpOptions().with_tolerance(tol)
    for k, v in kw.items():
        setattr(o, k, v)
    return o


CASES = [
    ("planted_fp64", lambda: g.reference_lp(0).lp, "fp64", _opts()),
    ("planted_seed1_fp64", lambda: g.reference_lp(1).lp, "fp64", _opts(1e-8)),
    ("planted_mixed_fp64_stage", lambda: g.reference_lp(0).lp, "mixed", _opts(1e-8)),
    ("infeasible_rows", cases.infeasible_rows, "fp64", cases.strict_options(iteration_limit=20000)),
    ("unbounded_ray", cases.unbounded_ray, "fp64", cases.strict_options(iteration_limit=20000)),
    ("limit_then_polish", lambda: cases.random_feasible(300, 420, 21), "fp64",
     cases.convergence_options(iteration_limit=150, use_feasibility_polishing=True,
                               polishing_iterations=300)),
    # 625 column slices: more than a 16-CTA cluster has warps, so the slices
    # are read from global memory in every trial instead of being staged.
    ("planted_10k_unstaged", lambda: g.planted_lp(10000, 20000, seed=4).lp, "mixed", _opts(1e-5)),
]


@pytest.mark.parametrize("name,build,precision,options", CASES, ids=[c[0] for c in CASES])
def test_fused_trials_match_two_kernel_trials(name, build, precision, options):
    lp = build()
    fused = PdlpSolver(precision).solve(lp, options)
    plain = PdlpSolver(precision, two_kernel_trials=1).solve(lp, options)
    _same(fused, plain)


def test_fused_batch_matches_two_kernel_batch():
    lps = [g.planted_lp(m, 2 * m, seed=60 + m).lp for m in (150, 400, 900, 1300)]
    opts = _opts(1e-7)
    fused = PdlpSolver("fp64").solve_batch(lps, opts)
    plain = PdlpSolver("fp64", two_kernel_trials=1).solve_batch(lps, opts)
    for a, b in zip(fused, plain):
        _same(a, b)


def test_fused_trials_time_per_iteration():
    """The 1000 x 2000 planted LP at 1e-6, FP64: device time per iteration of
    both paths (printed), fused no slower."""
    lp = g.reference_lp(0).lp
    out = {}
    for label, kw in (("fused", {}), ("two_kernel", {"two_kernel_trials": 1})):
        solver = PdlpSolver("fp64", **kw)
        solver.solve(lp, _opts())   # warm-up (module load, graph capture)
        best = None
        for _ in range(3):
            t0 = time.perf_counter()
            r = solver.solve(lp, _opts())
            wall = time.perf_counter() - t0
            us = 1e6 * r.device_seconds / max(1, r.iterations)
            best = us if best is None else min(best, us)
        out[label] = best
        print(f"{label}: {best:.2f} us per iteration ({r.iterations} iterations, wall {wall * 1e3:.1f} ms)")
    assert out["fused"] <= out["two_kernel"] * 1.05
