"""Pins the C restatement (oracle/pdlp_port.c) to the reference pdlp_engine.

Against the reference library built from its sources (skipped where the
reference is absent): bit-for-bit equality of every output on the serial path.
Against the committed fixtures of the reference's outputs
(tests/golden/reference_solves.npz, made by tests/golden/make_golden.py): the
same equality, so the restatement stays pinned on a machine without the
reference.
"""
import os

import numpy as np
import pytest

from optimisation_solver_b200 import generators as g
from tests import cases
from tests.golden.make_golden import golden_cases

GOLDEN = os.path.join(os.path.dirname(__file__), "golden", "reference_solves.npz")

SCALARS = ["iterations", "step_trials", "restart_count", "primal_objective", "dual_objective",
           "primal_residual", "dual_residual", "relative_gap", "final_step_size",
           "static_step_bound", "final_primal_weight"]


def _same(a, b):
    a, b = np.asarray(a, dtype=float), np.asarray(b, dtype=float)
    return a.shape == b.shape and np.array_equal(a, b, equal_nan=True)


@pytest.mark.parametrize("name,lp,opts", golden_cases(), ids=[c[0] for c in golden_cases()])
def test_port_matches_golden_fixtures(name, lp, opts, port_oracle):
    d = np.load(GOLDEN)
    r = port_oracle.solve(lp, opts)
    assert r.status == str(d[f"{name}/status"])
    got = [getattr(r, k) for k in SCALARS]
    assert _same(got, d[f"{name}/scalars"]), list(zip(SCALARS, got, d[f"{name}/scalars"]))
    for k in ("primal", "row_dual", "dual_ray", "primal_ray"):
        assert _same(getattr(r, k), d[f"{name}/{k}"]), k


PIN_CASES = [
    ("reference_lp_2", lambda: g.reference_lp(2).lp, dict(thread_count=1)),
    ("equality", cases.equality_row, cases.strict_options().as_dict()),
    ("inactive_row", cases.inactive_row, cases.strict_options().as_dict()),
    ("ill_conditioned", cases.ill_conditioned,
     cases.strict_options(primal_tolerance=1e-8, dual_tolerance=1e-8, gap_tolerance=1e-8).as_dict()),
    ("infeasible_equalities", cases.infeasible_equalities, cases.strict_options(iteration_limit=20000).as_dict()),
    ("fixed_step", lambda: cases.random_feasible(260, 360, 33), cases.convergence_options(use_adaptive_linesearch=False).as_dict()),
    ("no_averaging_no_restarts", lambda: cases.random_feasible(200, 300, 4),
     cases.convergence_options(use_averaging=False, use_restarts=False, iteration_limit=2000).as_dict()),
    ("no_ruiz", lambda: cases.random_feasible(200, 300, 5), cases.convergence_options(use_ruiz_scaling=False).as_dict()),
    ("invalid_options", cases.equality_row, dict(termination_check_frequency=0)),
    ("invalid_bounds", cases.crossed_var_bounds, {}),
    ("stress_small", lambda: g.planted_lp(300, 600, 5, seed=9, magnitudes="loguniform",
                                          free_fraction=0.2, ranged_fraction=0.1,
                                          rescale=(-2.0, 2.0)).lp, dict(thread_count=1, iteration_limit=5000)),
]


@pytest.mark.parametrize("name,build,opts", PIN_CASES, ids=[c[0] for c in PIN_CASES])
def test_port_bitwise_equals_reference(name, build, opts, port_oracle, ref_oracle):
    lp = build()
    a = ref_oracle.solve(lp, opts)
    b = port_oracle.solve(lp, opts)
    assert a.status == b.status and a.message == b.message
    for k in SCALARS:
        assert _same(getattr(a, k), getattr(b, k)), k
    for k in ("primal", "row_dual", "dual_ray", "primal_ray"):
        assert _same(getattr(a, k), getattr(b, k)), k


def test_components_bitwise_equal_reference(port_oracle, ref_oracle):
    lp = cases.random_feasible(300, 420, 21)
    rng = np.random.default_rng(0)
    x = rng.standard_normal(lp.num_cols)
    y = rng.standard_normal(lp.num_rows)
    assert _same(port_oracle.multiply(lp, x), ref_oracle.multiply(lp, x))
    assert _same(port_oracle.transpose_multiply(lp, y), ref_oracle.transpose_multiply(lp, y))
    ra, rb = port_oracle.ruiz(lp, 10), ref_oracle.ruiz(lp, 10)
    for k in ra:
        assert _same(ra[k], rb[k]), k
    for a, b in zip(port_oracle.precondition(lp), ref_oracle.precondition(lp)):
        assert _same(a, b)
    assert port_oracle.spectral_norm(lp) == ref_oracle.spectral_norm(lp)
    tau, tinv, sig, sinv = ref_oracle.precondition(lp)
    ax = ref_oracle.multiply(lp, x)
    out_a = port_oracle.trial(lp, tau, tinv, sig, sinv, x, y, ax, 0.7, 1.3)
    out_b = ref_oracle.trial(lp, tau, tinv, sig, sinv, x, y, ax, 0.7, 1.3)
    for a, b in zip(out_a[:4], out_b[:4]):
        assert _same(a, b)
    ea, eb = port_oracle.evaluate(lp, x, y), ref_oracle.evaluate(lp, x, y)
    assert ea == eb
    assert port_oracle.test_dual_ray(lp, y) == ref_oracle.test_dual_ray(lp, y)
    assert port_oracle.test_primal_ray(lp, x) == ref_oracle.test_primal_ray(lp, x)


def test_from_triplets_bitwise_equal_reference(port_oracle, ref_oracle):
    rng = np.random.default_rng(1)
    ti = rng.integers(0, 40, 600)
    tj = rng.integers(0, 50, 600)
    tv = rng.uniform(-2, 2, 600)
    tv[::17] = 0.0
    a = port_oracle.from_triplets(40, 50, ti, tj, tv)
    b = ref_oracle.from_triplets(40, 50, ti, tj, tv)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
