"""The reference's own test expectations (pdlp_engine/tests/test_pdlp.cpp),
checked on the CPU oracle -- the values every device test is held to."""
import numpy as np
import pytest

from tests import cases


@pytest.mark.parametrize("name,build,options,expected", cases.SOLVER_KATS,
                         ids=[k[0] for k in cases.SOLVER_KATS])
def test_oracle_meets_reference_kats(name, build, options, expected, oracle):
    r = oracle.solve(build(), options.as_dict())
    assert r.status == expected["status"]
    assert abs(r.primal_objective - expected["obj"]) <= expected["tol"]
    if "x" in expected:
        assert np.allclose(r.primal, expected["x"], atol=expected["tol"])


def test_oracle_inactive_row_dual_zero(oracle):
    r = oracle.solve(cases.inactive_row(), cases.strict_options().as_dict())
    assert r.status == "optimal" and r.row_dual[1] == 0.0


def test_oracle_certificates(oracle):
    r = oracle.solve(cases.infeasible_rows(), cases.strict_options(iteration_limit=20000).as_dict())
    assert r.status == "infeasible" and cases.farkas_value(r.dual_ray) > 1e-9
    r = oracle.solve(cases.unbounded_ray(), cases.strict_options(iteration_limit=20000).as_dict())
    assert r.status == "unbounded" and r.primal_ray[0] > 0.0
    r = oracle.solve(cases.infeasible_equalities(), cases.strict_options(iteration_limit=20000).as_dict())
    assert r.status == "infeasible"


def test_oracle_ruiz_spread(oracle):
    lp = cases.badly_scaled()
    from optimisation_solver_b200.lp import CompiledLp, SparseMatrix
    s = oracle.ruiz(lp, 10)
    m = lp.matrix
    scaled = CompiledLp(SparseMatrix(m.rows, m.columns, m.row_start, m.col_index, s["values"]),
                        lp.objective, lp.row_lower, lp.row_upper, lp.var_lower, lp.var_upper)
    assert oracle.condition_spread(lp) > 1e6 and oracle.condition_spread(scaled) < 10.0


def test_oracle_invalid_problems(oracle):
    for lp in (cases.crossed_row_bounds(), cases.crossed_var_bounds()):
        assert oracle.solve(lp, cases.strict_options().as_dict()).status == "invalid_problem"
