"""Batched solves of different LPs (`solve_batch`, the config-2 path): one
device layout for every instance, per-instance control, results scattered
back per LP. Checked against one-LP solves of the same instances, against
the planted optima, and for run-to-run identity, including a batch large
enough that its matrices cross the host's pinned staging buffers in several
chunks and its solutions come back through them.
"""
import numpy as np
import pytest

from optimisation_solver_b200 import generators as g
from optimisation_solver_b200.lp import PdlpOptions, PdlpStatus
from optimisation_solver_b200.pdlp import PdlpSolver
from tests import cases

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return abs(a - b) / (1.0 + abs(b))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_matches_single_solves(precision):
    """Six LPs of different shapes at 1e-7: every batched result has the
    status of its one-LP solve and the same objective to the tolerance."""
    lps = [g.planted_lp(m, 2 * m, degree=d, seed=s).lp
           for m, d, s in ((200, 4, 0), (1000, 4, 1), (350, 6, 2), (1500, 3, 3), (600, 8, 4), (900, 5, 5))]
    opts = PdlpOptions().with_tolerance(1e-7)
    solver = PdlpSolver(precision)
    batch = solver.solve_batch(lps, opts)
    assert len(batch) == len(lps)
    for lp, r in zip(lps, batch):
        one = solver.solve(lp, opts)
        assert r.status == one.status == PdlpStatus.OPTIMAL
        assert r.primal.shape == (lp.num_cols,) and r.row_dual.shape == (lp.num_rows,)
        assert _rel(r.primal_objective, one.primal_objective) <= 1e-6
        assert max(r.primal_residual, r.dual_residual, r.relative_gap) <= 1e-7


def test_invalid_instance_does_not_stop_the_batch():
    """An invalid LP in the middle of a batch gets the reference's message;
    the others are solved as if it were absent."""
    good = [g.reference_lp(s).lp for s in (0, 1)]
    bad = cases.crossed_row_bounds()
    opts = PdlpOptions().with_tolerance(1e-6)
    out = PdlpSolver().solve_batch([good[0], bad, good[1]], opts)
    assert out[1].status == PdlpStatus.INVALID_PROBLEM and out[1].status_message
    alone = PdlpSolver().solve_batch(good, opts)
    for r, a in zip((out[0], out[2]), alone):
        assert r.status == a.status == PdlpStatus.OPTIMAL
        assert r.iterations == a.iterations and np.array_equal(r.primal, a.primal)


def test_large_batch_through_staging_buffers():
    """Fourteen LPs of 20,000 x 40,000 (about 4.5M nonzeros, well over one
    64 MiB staging buffer of matrix slots; 560,000 columns of results, more
    than a direct download): all optimal near their planted optima, and a
    second run returns the same bits."""
    planted = []
    for i in range(14):
        rng = np.random.default_rng(40_000 + i)
        planted.append(g.planted_lp(20_000, 40_000, seed=i, degrees=rng.integers(4, 13, size=40_000)))
    lps = [p.lp for p in planted]
    opts = PdlpOptions().with_tolerance(1e-4)
    solver = PdlpSolver("mixed")
    a = solver.solve_batch(lps, opts)
    b = solver.solve_batch(lps, opts)
    for p, ra, rb in zip(planted, a, b):
        assert ra.status == PdlpStatus.OPTIMAL
        assert _rel(ra.primal_objective, p.objective) <= 1e-2
        assert ra.iterations == rb.iterations
        assert np.array_equal(ra.primal, rb.primal) and np.array_equal(ra.row_dual, rb.row_dual)
