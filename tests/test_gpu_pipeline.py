"""The GPU engine behind the reference's own pipeline (end to end).

`oracle/Makefile` links the reference's presolve, dispatch, engines and
postsolve with the GPU engine's pdlp::PdlpSolver::solve
(include/pdlpgpu_override.hpp) in place of pdlp_engine/src/pdlp_solver.cpp,
so solver::runPdlp (src/solver/orchestrator.cpp:315-352) calls the GPU with no
reference line changed. Checked here:

* the reference's own pipeline test, tests/pipeline/test_postsolve_integration.cpp,
  every case (forced PDLP: x = {2, 0, 5.6}, objective 39.4, duals {0, 0.8, 0},
  reduced costs {5, -0.2, 0}; limit semantics; failure statuses);
* the reference's LP fixture files (benchmarks/instances/known/*.mps and
  netlib/afiro.mps, carried as Model IR arrays in tests/golden/) through
  solver::solve with PDLP forced: their published objectives to 1e-6
  relative, the statuses of the infeasible and unbounded files, and the
  reference pipeline's own primal values, shadow prices and reduced costs;
* the same fixtures compiled by adapter::toCompiledLp and solved by the engine
  directly, against the reference oracle on the same CompiledLp;
* the 1000 x 2000 planted LP written as free-format MPS, read back by the
  reference MpsReader and solved through the pipeline.
"""
import os
import subprocess

import numpy as np
import pytest

from optimisation_solver_b200 import generators as g
from optimisation_solver_b200.lp import PdlpOptions
from optimisation_solver_b200.pdlp import PdlpSolver
from oracle.pipeline import ENGINE_PDLP, POSTSOLVE_TEST, Pipeline, available
from tests.mps_writer import write_free_mps
from tests.parity import check_objective, solve_many
from tests.test_pipeline import fixture_models

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not available("gpu"),
                                 reason="GPU pipeline not built (make -C oracle pipeline)")]

CASES = ["lp_engines", "qp_signs", "all_eliminated", "bound_only", "integer_models",
         "unavailable_duals", "failure_statuses", "limit_no_solution", "limit_feasible_solution",
         "reduced_api"]


@pytest.fixture(scope="module")
def gpu_pipeline():
    return Pipeline("gpu")


@pytest.mark.parametrize("case", CASES)
def test_reference_postsolve_integration_with_gpu_engine(case):
    r = subprocess.run([POSTSOLVE_TEST["gpu"], case], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0 and f"[PASSED] {case}" in r.stdout, r.stdout + r.stderr


def test_fixture_files_through_gpu_pipeline(gpu_pipeline):
    """Statuses and published objectives; which vectors postsolve publishes
    (primal, shadow prices) as the reference pipeline's own PDLP run does,
    with validated multipliers. The points themselves are not compared: the
    optima of these files are not unique (afiro's primal differs in a
    degenerate direction at the same objective)."""
    for name, d in fixture_models().items():
        r = gpu_pipeline.import_model(d).solve(engine=ENGINE_PDLP, tolerance=1e-8)
        assert r.status == str(d["pdlp_status"]), (name, r.status, r.message)
        if r.status != "optimal":
            continue
        assert r.executed_engine == ENGINE_PDLP, name
        want = float(d["expected_objective"])
        assert abs(r.objective - want) <= 1e-6 * max(1.0, abs(want)), (name, r.objective, want)
        assert r.has_primal and r.x.shape == d["pdlp_x"].shape, name
        assert r.has_duals == (d["pdlp_duals"].size > 0 or d["pdlp_reduced_costs"].size > 0), name
        if r.has_duals:
            assert r.max_dual_residual < 1e-5, (name, r.max_dual_residual)


def test_compiled_fixtures_engine_matches_oracle(oracle, gpu_pipeline):
    lps, names = [], []
    for name, d in fixture_models().items():
        lps.append(gpu_pipeline.import_model(d).compile())
        names.append(name)
    refs = solve_many(oracle, lps, 1e-8)
    solver = PdlpSolver("fp64")
    for name, lp, ref in zip(names, lps, refs):
        r = solver.solve(lp, PdlpOptions().with_tolerance(1e-8))
        assert str(r.status) == ref.status, (name, r.status, ref.status)
        if ref.status == "optimal":
            check_objective(r.primal_objective, ref, 1e-8, objective_rel=1e-6)


def test_planted_lp_mps_file_through_gpu_pipeline(tmp_path, gpu_pipeline):
    """The planted LP's MPS file through both pipelines. Both engines converge
    (the same engine message). Postsolve then validates the point with an
    absolute bound check that relative PDLP tolerances do not promise: the
    reference pipeline's own point fails it on this file ("Constraint upper
    bound violation", status numerical_failure); the GPU engine's point may
    pass or fail it, and when it passes the objective is the planted one."""
    planted = g.reference_lp(0)
    path = str(tmp_path / "planted_0.mps")
    write_free_mps(planted.lp, path, "planted_0")
    r = gpu_pipeline.read_mps(path).solve(engine=ENGINE_PDLP, tolerance=1e-8)
    ref = Pipeline("ref").read_mps(path).solve(engine=ENGINE_PDLP, tolerance=1e-8)
    assert r.executed_engine == ENGINE_PDLP
    assert r.message.split(";")[0] == ref.message.split(";")[0], (r.message, ref.message)
    assert r.status in ("optimal", "numerical_failure"), r.status
    if r.status == "optimal":
        assert abs(r.objective - planted.objective) <= 1e-6 * abs(planted.objective)
    else:
        assert "violation" in r.message


@pytest.mark.skipif(not available("gpufast"), reason="make -C oracle presolve not run")
def test_fast_presolve_and_gpu_engine_together_match_gpu_pipeline(gpu_pipeline):
    """Both drop-ins linked at once (the fast presolve in place of
    presolver.cpp, the engine behind solver::runPdlp): on the reference's
    fixture LPs every answer is the one of the pipeline with the reference's
    presolve, bit for bit (same reduced model, same deterministic engine)."""
    fast = Pipeline("gpufast")
    for name, d in fixture_models().items():
        for engine in (ENGINE_PDLP, None):
            a = gpu_pipeline.import_model(d).solve(engine=engine, tolerance=1e-8)
            b = fast.import_model(d).solve(engine=engine, tolerance=1e-8)
            assert (a.status, a.executed_engine, a.iterations) == \
                (b.status, b.executed_engine, b.iterations), (name, engine)
            assert np.array_equal(np.float64(a.objective), np.float64(b.objective),
                                  equal_nan=True), name
            for f in ("x", "duals", "reduced_costs"):
                assert np.array_equal(getattr(a, f), getattr(b, f)), (name, engine, f)


@pytest.mark.skipif(not available("gpufast"), reason="make -C oracle presolve not run")
def test_config3_through_solver_solve_with_fast_presolve():
    """Configuration 3 (100,000 x 200,000, 1.6M nonzeros, rescaled rows and
    columns, free variables, ranged rows) through the reference's whole
    solver::solve -- model validation, presolve, dispatch, adapter, the GPU
    engine, postsolve -- which the reference's own presolve does not finish
    in practical time (its pairwise row pass). Records the wall time and the
    outcome."""
    import time
    from optimisation_solver_b200.presolve import PresolveModel, Presolver
    lp = g.stress_lp(0).lp
    nz = np.flatnonzero(lp.objective)
    arrays = dict(sense=np.array([0]), offset=np.array([lp.objective_offset]),
                  objective_index=nz.astype(np.int32), objective_value=lp.objective[nz],
                  var_type=np.zeros(lp.num_cols, np.int32), var_lower=lp.var_lower,
                  var_upper=lp.var_upper, row_lower=lp.row_lower, row_upper=lp.row_upper,
                  row_start=lp.row_start, row_index=lp.col_index, row_value=lp.values)
    pre = Presolver().run(PresolveModel.from_lp(lp))
    model = Pipeline("gpufast").import_model(arrays)
    t0 = time.perf_counter()
    r = model.solve(engine=ENGINE_PDLP, tolerance=1e-4, threads=os.cpu_count() or 1)
    wall = time.perf_counter() - t0
    print(f"config 3 through solver::solve: {r.status} in {wall:.1f} s, {r.iterations} "
          f"iterations, objective {r.objective:.10g}; {r.message[:120]}")
    assert r.status not in ("invalid_model", "unsupported"), r.message
    assert r.executed_engine == ENGINE_PDLP
    assert not pre.infeasible and pre.presolved_constraints == lp.num_rows
    assert wall < 600.0
