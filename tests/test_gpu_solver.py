"""Whole solves through the C ABI against the reference's own expected
values (pdlp_engine/tests/test_pdlp.cpp) and against the CPU oracle on the
same inputs: same status, objective within 1e-6 relative in FP64 mode.
"""
import numpy as np
import pytest

from optimisation_solver_b200 import generators as g
from optimisation_solver_b200.lp import PdlpOptions, PdlpStatus
from optimisation_solver_b200.pdlp import PdlpSolver
from tests import cases

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    return PdlpSolver()


@pytest.mark.parametrize("name,build,options,expected", cases.SOLVER_KATS,
                         ids=[k[0] for k in cases.SOLVER_KATS])
def test_reference_kats(name, build, options, expected, solver):
    r = solver.solve(build(), options)
    assert str(r.status) == expected["status"], r.status_message
    assert abs(r.primal_objective - expected["obj"]) <= expected["tol"]
    if "x" in expected:
        assert np.allclose(r.primal, expected["x"], atol=expected["tol"])


def test_ill_conditioned_absolute_feasibility(solver):
    opts = cases.strict_options(primal_tolerance=1e-8, dual_tolerance=1e-8, gap_tolerance=1e-8)
    r = solver.solve(cases.ill_conditioned(), opts)
    assert r.status == PdlpStatus.OPTIMAL
    a0 = 1e-4 * (r.primal[0] + r.primal[1])
    a1 = 1e4 * r.primal[0]
    assert a0 <= 3e-4 + 1e-9
    assert a1 <= 2e4 + 1e-3


def test_inactive_row_dual_is_exactly_zero(solver):
    r = solver.solve(cases.inactive_row(), cases.strict_options())
    assert r.status == PdlpStatus.OPTIMAL
    assert r.row_dual[1] == 0.0


def test_unbounded_never_optimal(solver):
    r = solver.solve(cases.unbounded_simple(), cases.strict_options(iteration_limit=2000))
    assert r.status != PdlpStatus.OPTIMAL


def test_invalid_problems_rejected(solver):
    for lp in (cases.crossed_row_bounds(), cases.crossed_var_bounds()):
        r = solver.solve(lp, cases.strict_options())
        assert r.status == PdlpStatus.INVALID_PROBLEM
        assert r.status_message
    r = solver.solve(cases.equality_row(), PdlpOptions(termination_check_frequency=0))
    assert r.status == PdlpStatus.INVALID_PROBLEM
    assert r.status_message == "Invalid PDLP options"


def test_infeasible_rows_with_farkas_ray(solver):
    r = solver.solve(cases.infeasible_rows(), cases.strict_options(iteration_limit=20000))
    assert r.status == PdlpStatus.INFEASIBLE, r.status_message
    assert r.dual_ray.size == 2
    assert cases.farkas_value(r.dual_ray) > 1e-9


def test_infeasible_equalities(solver):
    r = solver.solve(cases.infeasible_equalities(), cases.strict_options(iteration_limit=20000))
    assert r.status == PdlpStatus.INFEASIBLE, r.status_message


def test_unbounded_with_ray(solver):
    r = solver.solve(cases.unbounded_ray(), cases.strict_options(iteration_limit=20000))
    assert r.status == PdlpStatus.UNBOUNDED, r.status_message
    assert r.primal_ray.size == 2 and r.primal_ray[0] > 0.0


def test_feasible_never_flagged(solver):
    for k in range(6):
        lp = cases.feasible_box(300 + 40 * k, 600, 17 + k)
        r = solver.solve(lp, cases.strict_options(iteration_limit=6000))
        assert r.status not in (PdlpStatus.INFEASIBLE, PdlpStatus.UNBOUNDED)


def test_linesearch_exceeds_static_bound(solver):
    r = solver.solve(cases.random_feasible(300, 420, 21), cases.convergence_options())
    assert r.static_step_bound > 0.0
    assert r.final_step_size > r.static_step_bound
    assert r.step_trials >= r.iterations


def test_step_policies_agree(solver):
    lp = cases.random_feasible(260, 360, 33)
    a = solver.solve(lp, cases.convergence_options(use_adaptive_linesearch=True))
    b = solver.solve(lp, cases.convergence_options(use_adaptive_linesearch=False))
    assert a.status == PdlpStatus.OPTIMAL and b.status == PdlpStatus.OPTIMAL
    assert abs(a.primal_objective - b.primal_objective) <= 1e-6 * (1 + abs(a.primal_objective))


def test_time_limit_honoured(solver):
    lp = cases.feasible_box(3000, 4000, 3, per_row=12, width=1.0, upper=1.0)
    opts = PdlpOptions(iteration_limit=100_000_000, primal_tolerance=0.0, dual_tolerance=0.0,
                       gap_tolerance=0.0, time_limit_seconds=0.25)
    r = solver.solve(lp, opts)
    assert r.status == PdlpStatus.TIME_LIMIT
    assert r.solve_time_seconds < 3.0


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_reference_lp_matches_oracle(seed, solver, oracle):
    """The 1000 x 2000 planted LP at tolerance 1e-6: same status as the
    reference, objective within 1e-6 relative of it and of the planted one."""
    p = g.reference_lp(seed)
    ref = oracle.solve(p.lp, dict(thread_count=1))
    r = solver.solve(p.lp, PdlpOptions())
    assert str(r.status) == ref.status == "optimal"
    assert abs(r.primal_objective - ref.primal_objective) <= 1e-6 * abs(ref.primal_objective)
    assert abs(r.primal_objective - p.objective) <= 1e-6 * abs(p.objective)
    assert r.relative_gap <= 1e-6 and r.primal_residual <= 1e-6


def test_iteration_limit_and_polishing(solver, oracle):
    lp = cases.random_feasible(300, 420, 21)
    opts = cases.convergence_options(iteration_limit=150, use_feasibility_polishing=True,
                                     polishing_iterations=300)
    r = solver.solve(lp, opts)
    ref = oracle.solve(lp, opts.as_dict())
    assert str(r.status) == ref.status
    assert r.iterations >= 150


def test_deterministic(solver):
    lp = g.reference_lp(3).lp
    a = solver.solve(lp)
    b = solver.solve(lp)
    assert a.iterations == b.iterations and np.array_equal(a.primal, b.primal)
