"""HiGHS (scipy.optimize.linprog, method="highs") as a second, independent
oracle: a simplex/interior-point solver that shares no code with the
reference, run on the planted configuration-0 LPs and on instances of the
min-cost flow family. It must reach the planted optimum (the known answer
the generator builds in) and agree with the reference oracle solved tightly,
which pins the oracle itself, and with it every parity test that compares
this engine against it.
"""
import numpy as np
import pytest
import scipy.sparse as sp
from scipy.optimize import linprog

from optimisation_solver_b200 import generators as g


def highs(lp):
    """min c'x + offset s.t. row_lower <= Ax <= row_upper, var bounds, by HiGHS."""
    A = sp.csr_matrix((lp.values, lp.col_index, lp.row_start), shape=(lp.num_rows, lp.num_cols))
    eq = np.isfinite(lp.row_lower) & np.isfinite(lp.row_upper) & (lp.row_lower == lp.row_upper)
    up = np.isfinite(lp.row_upper) & ~eq
    lo = np.isfinite(lp.row_lower) & ~eq
    res = linprog(lp.objective, A_ub=sp.vstack([A[up], -A[lo]]),
                  b_ub=np.concatenate([lp.row_upper[up], -lp.row_lower[lo]]),
                  A_eq=A[eq] if eq.any() else None, b_eq=lp.row_upper[eq] if eq.any() else None,
                  bounds=np.column_stack([lp.var_lower, lp.var_upper]), method="highs")
    assert res.status == 0, res.message
    return res.fun + lp.objective_offset


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_highs_reaches_the_planted_optimum_and_agrees_with_the_oracle(seed, oracle):
    planted = g.reference_lp(seed)
    h = highs(planted.lp)
    assert abs(h - planted.objective) <= 1e-9 * max(1.0, abs(planted.objective))
    r = oracle.solve(planted.lp, dict(thread_count=1, primal_tolerance=1e-8,
                                      dual_tolerance=1e-8, gap_tolerance=1e-8))
    assert r.status == "optimal"
    assert abs(r.primal_objective - h) <= 1e-6 * max(1.0, abs(h)), (r.primal_objective, h)


def test_highs_agrees_with_the_oracle_on_flow_instances(oracle):
    graph = g.flow_graph()
    supplies, costs = g.flow_parameters(graph, 3, seed=11)
    for k in range(3):
        lp = g.flow_lp(graph, supplies[k], costs[k])
        h = highs(lp)
        r = oracle.solve(lp, dict(thread_count=4, primal_tolerance=1e-8,
                                  dual_tolerance=1e-8, gap_tolerance=1e-8))
        assert r.status == "optimal", r.status
        assert abs(r.primal_objective - h) <= 1e-6 * max(1.0, abs(h)), (k, r.primal_objective, h)
