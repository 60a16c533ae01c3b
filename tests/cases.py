"""The reference's PDLP test problems and their known answers, restated as
``CompiledLp`` builders (pdlp_engine/tests/test_pdlp.cpp, cited per case).

These are the golden values the oracle is pinned against and the GPU engine
is checked against: exact optima of tiny LPs, statuses of infeasible and
unbounded ones, and the option sets the reference's tests use.
"""
from __future__ import annotations

import numpy as np

from optimisation_solver_b200.lp import INF, CompiledLp, PdlpOptions, SparseMatrix


def strict_options(**kw) -> PdlpOptions:
    """strictOptions() (test_pdlp.cpp:49-58)."""
    d = dict(iteration_limit=100000, primal_tolerance=2e-6, dual_tolerance=2e-6,
             gap_tolerance=2e-6, termination_check_frequency=50, polishing_iterations=2000)
    d.update(kw)
    return PdlpOptions(**d)


def convergence_options(**kw) -> PdlpOptions:
    """convergenceOptions() (test_pdlp.cpp:552-561)."""
    d = dict(iteration_limit=60000, primal_tolerance=1e-8, dual_tolerance=1e-8,
             gap_tolerance=1e-8, termination_check_frequency=40, use_feasibility_polishing=False)
    d.update(kw)
    return PdlpOptions(**d)


def equality_row():          # :209-223  x = (1, 0), objective 1
    return CompiledLp.build(1, 2, [(0, 0, 1.0), (0, 1, 1.0)], [1.0, 2.0], [1.0], [1.0],
                            [0.0, 0.0], [INF, INF])


def upper_bound_row():       # :225-238  x = 3, objective -3
    return CompiledLp.build(1, 1, [(0, 0, 1.0)], [-1.0], [-INF], [3.0], [0.0], [10.0])


def lower_bound_row():       # :240-253  x = 2, objective 2
    return CompiledLp.build(1, 1, [(0, 0, 1.0)], [1.0], [2.0], [INF], [-10.0], [10.0])


def ranged_row():            # :255-268  x = 3, objective -3
    return CompiledLp.build(1, 1, [(0, 0, 2.0)], [-1.0], [2.0], [6.0], [0.0], [10.0])


def inactive_row():          # :273-288  the slack row's dual is exactly 0.0
    return CompiledLp.build(2, 1, [(0, 0, 1.0), (1, 0, 1.0)], [1.0], [2.0, -INF], [INF, 1000.0],
                            [0.0], [10.0])


def ill_conditioned():       # :293-323  objective -3 at 1e-8, absolute feasibility
    return CompiledLp.build(2, 2, [(0, 0, 1e-4), (0, 1, 1e-4), (1, 0, 1e4)], [-1.0, -1.0],
                            [-INF, -INF], [3e-4, 2e4], [0.0, 0.0], [10.0, 10.0])


def badly_scaled():          # :325-345  Ruiz spread > 1e6 before, < 10 after
    return CompiledLp.build(3, 3, [(0, 0, 1e-5), (0, 1, 2e-5), (1, 1, 1e3), (1, 2, 5e2),
                                   (2, 0, 7.0), (2, 2, 3.0)],
                            [1.0, 1.0, 1.0], [0.0] * 3, [1.0] * 3, [0.0] * 3, [1.0] * 3)


def degenerate(n=12):        # :349-375  objective -6
    t = []
    row = 0
    for i in range(n - 1):
        for _ in range(2):
            t += [(row, i, 1.0), (row, i + 1, 1.0)]
            row += 1
    return CompiledLp.build(row, n, t, [-1.0] * n, [-INF] * row, [1.0] * row, [0.0] * n, [1.0] * n)


def unbounded_simple():      # :379-393  never reported optimal
    return CompiledLp.build(1, 1, [(0, 0, 1.0)], [-1.0], [-INF], [INF], [0.0], [INF])


def crossed_row_bounds():    # :395-406  invalid_problem
    return CompiledLp.build(1, 1, [(0, 0, 1.0)], [1.0], [5.0], [1.0], [0.0], [1.0])


def crossed_var_bounds():    # :408-413  invalid_problem
    return CompiledLp.build(1, 1, [(0, 0, 1.0)], [1.0], [0.0], [1.0], [2.0], [1.0])


def infeasible_rows():       # :608-640  infeasible, Farkas ray
    return CompiledLp.build(2, 2, [(0, 0, 1.0), (0, 1, 1.0), (1, 0, 1.0), (1, 1, 1.0)],
                            [1.0, 1.0], [2.0, -INF], [INF, 1.0], [0.0, 0.0], [10.0, 10.0])


def infeasible_equalities():  # :643-659  infeasible
    return CompiledLp.build(2, 2, [(0, 0, 1.0), (0, 1, 1.0), (1, 0, 1.0), (1, 1, 1.0)],
                            [0.0, 0.0], [1.0, 2.0], [1.0, 2.0], [-INF, -INF], [INF, INF])


def unbounded_ray():         # :662-680  unbounded, ray[0] > 0
    return CompiledLp.build(1, 2, [(0, 1, 1.0)], [-1.0, 0.0], [-INF], [5.0], [0.0, 0.0],
                            [INF, 10.0])


def farkas_value(y):
    """The independent certificate check of test_pdlp.cpp:629-639."""
    r0 = y[0] + y[1]
    r1 = y[0] + y[1]
    box = (0.0 if r0 > 0 else r0 * 10.0) + (0.0 if r1 > 0 else r1 * 10.0)
    support = (0.0 if y[0] > 0 else y[0] * 2.0) + (y[1] * 1.0 if y[1] > 0 else 0.0)
    return box - support


def random_feasible(rows, cols, seed, per_row=6):
    """randomFeasibleProblem (test_pdlp.cpp:510-550), with numpy's generator:
    random rows of `per_row` U(-1,1) entries, U(-1,1) costs, bounds [0,10],
    a reference point in the box, every third row an equality through it and
    the rest <= its activity + 1."""
    rng = np.random.default_rng(seed)
    ti = np.repeat(np.arange(rows), per_row)
    tj = rng.integers(0, cols, rows * per_row)
    tv = rng.uniform(-1.0, 1.0, rows * per_row)
    A = SparseMatrix.from_triplets(rows, cols, ti, tj, tv)
    c = rng.uniform(-1.0, 1.0, cols)
    ref = 10.0 * rng.random(cols)
    act = A.multiply(ref)
    rl = np.where(np.arange(rows) % 3 == 0, act, -INF)
    ru = np.where(np.arange(rows) % 3 == 0, act, act + 1.0)
    return CompiledLp(A, c, rl, ru, np.zeros(cols), np.full(cols, 10.0))


def feasible_box(rows, cols, seed, per_row=8, width=0.5, upper=4.0):
    """The feasibleProblemsAreNotFlagged family (test_pdlp.cpp:684-728):
    two-sided rows around the activity of an interior point."""
    rng = np.random.default_rng(seed)
    ti = np.repeat(np.arange(rows), per_row)
    tj = rng.integers(0, cols, rows * per_row)
    tv = rng.uniform(-1.0, 1.0, rows * per_row)
    A = SparseMatrix.from_triplets(rows, cols, ti, tj, tv)
    c = rng.uniform(-1.0, 1.0, cols)
    ref = upper * rng.random(cols)
    act = A.multiply(ref)
    return CompiledLp(A, c, act - width, act + width, np.zeros(cols), np.full(cols, upper))


# (name, builder, options, expected) for the solver-behaviour KATs.
SOLVER_KATS = [
    ("equality_row", equality_row, strict_options(), dict(status="optimal", x=[1.0, 0.0], obj=1.0, tol=2e-4)),
    ("upper_bound_row", upper_bound_row, strict_options(), dict(status="optimal", x=[3.0], obj=-3.0, tol=2e-4)),
    ("lower_bound_row", lower_bound_row, strict_options(), dict(status="optimal", x=[2.0], obj=2.0, tol=2e-4)),
    ("ranged_row", ranged_row, strict_options(), dict(status="optimal", x=[3.0], obj=-3.0, tol=2e-4)),
    ("degenerate", degenerate, strict_options(), dict(status="optimal", obj=-6.0, tol=1e-3)),
    ("ill_conditioned", ill_conditioned,
     strict_options(primal_tolerance=1e-8, dual_tolerance=1e-8, gap_tolerance=1e-8),
     dict(status="optimal", obj=-3.0, tol=1e-5)),
]
