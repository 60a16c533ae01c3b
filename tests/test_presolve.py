"""The fast presolve against the reference's presolve::Presolver::run
(src/presolve/presolver.cpp), on the CPU (the presolve is host code).

* Committed results (tests/golden/presolve_results.npz, made by
  tests/golden/make_presolve_golden.py after a field-by-field comparison with
  the reference): the library reproduces every array bit for bit, with no
  reference build needed.
* Where the reference is built (`make -C oracle presolve`): both presolvers
  on the same model::Model, every field of PresolveResult compared, doubles
  by their bits -- generated models reaching every step (tests/presolve_cases.py),
  every MPS file the reference ships that its reader accepts, planted LPs of
  configuration 0; and solver::solve end to end with the fast presolve linked
  in place of the reference's, against the reference pipeline.
* The reference's own presolve and postsolve test programs, built with its
  presolver and with this one in its place: both pass, with the same output.
* Refused inputs, and models far beyond what the reference's O(m^2) passes
  reach in the time the tests allow.
"""
import glob
import os
import time

import numpy as np
import pytest

import __graft_entry__
from optimisation_solver_b200 import generators as g
from optimisation_solver_b200.presolve import PresolveModel, Presolver
from oracle import presolve_cmp
from tests import presolve_cases

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "presolve_results.npz")
MODEL_KEYS = ("var_lower", "var_upper", "var_type", "row_lower", "row_upper", "row_start",
              "row_index", "row_value", "objective_index", "objective_value",
              "quadratic_index1", "quadratic_index2", "quadratic_value")

needs_reference = pytest.mark.skipif(
    not presolve_cmp.available(), reason="reference presolver not built (make -C oracle presolve)")


@pytest.fixture(scope="module")
def cmp():
    return presolve_cmp.PresolveCompare()


def bits_equal(a, b) -> bool:
    a, b = np.asarray(a), np.asarray(b)
    if a.shape != b.shape:
        return False
    if a.dtype.kind == "f" or b.dtype.kind == "f":
        return np.array_equal(a.astype(np.float64).view(np.int64),
                              b.astype(np.float64).view(np.int64))
    return np.array_equal(a, b)


def test_golden_results_reproduce_bit_for_bit():
    from tests.golden.make_presolve_golden import flatten
    data = np.load(GOLDEN)
    P = Presolver()
    for name in data["names"]:
        name = str(name)
        m = PresolveModel(**{k: data[f"{name}/model_{k}"] for k in MODEL_KEYS},
                          objective_offset=float(data[f"{name}/model_objective_offset"]))
        got = flatten(P.run(m))
        keys = [k.split("/", 1)[1][len("result_"):] for k in data.files
                if k.startswith(f"{name}/result_")]
        assert sorted(keys) == sorted(got), name
        for k in keys:
            assert bits_equal(got[k], data[f"{name}/result_{k}"]), (name, k)


@needs_reference
def test_generated_models_match_reference(cmp):
    seen_infeasible = seen_feasible = 0
    for k, m in enumerate(presolve_cases.flavours(240)):
        rc, msg, summary = cmp.compare(m)
        assert rc == 0, (k, msg)
        seen_infeasible += summary["infeasible"]
        seen_feasible += not summary["infeasible"]
    assert seen_infeasible > 20 and seen_feasible > 20


@needs_reference
def test_larger_feasible_models_match_reference(cmp):
    """Models of a few hundred to 1500 variables with rows up to 40 terms and
    many copies, feasible by construction, so that the passes run to their
    fixed point over many passes."""
    rng = np.random.default_rng(7)
    feasible = 0
    for k in range(12):
        n, m = int(rng.integers(300, 1500)), int(rng.integers(200, 1000))
        model = presolve_cases.random_model(
            60000 + k, n=n, m=m, integers=k % 3 == 1, quadratic=k % 4 == 2,
            copies=float(rng.choice([0.1, 0.3, 0.6])), max_row=int(rng.choice([6, 12, 40])),
            exact=True)
        rc, msg, summary = cmp.compare(model)
        assert rc == 0, (k, msg)
        feasible += not summary["infeasible"]
    assert feasible >= 10


@needs_reference
def test_long_rows_match_reference(cmp):
    """Rows of 64 terms and more take the bracketed sums of bound tightening;
    budget rows make most of their targets tighten (the exact sums), the
    others stay within their brackets."""
    feasible = tightened = 0
    for seed in range(60):
        rc, msg, summary = cmp.compare(presolve_cases.long_row_model(seed))
        assert rc == 0, (seed, msg)
        feasible += not summary["infeasible"]
        tightened += summary["transformations"]
    assert feasible >= 20 and tightened > 1000


def test_dense_row_presolves_in_linear_time():
    """One budget row over all 200,000 variables of a planted LP: the
    reference sums the row's other terms afresh for each of its 200,000
    terms (4 x 10^10 additions a pass); with the bracketed sums the whole
    presolve takes well under a second (the bound below is loose on purpose)."""
    lp = g.planted_lp(m=20_000, n=200_000, seed=3).lp
    n = lp.num_cols
    m = PresolveModel(var_lower=lp.var_lower, var_upper=lp.var_upper,
                      row_lower=np.append(lp.row_lower, -np.inf),
                      row_upper=np.append(lp.row_upper, 0.9 * lp.var_upper.sum()),
                      row_start=np.append(lp.row_start, lp.row_start[-1] + n),
                      row_index=np.concatenate([lp.col_index, np.arange(n, dtype=np.int32)]),
                      row_value=np.concatenate([lp.values, np.ones(n)]),
                      objective_index=np.arange(n, dtype=np.int32), objective_value=lp.objective)
    t0 = time.perf_counter()
    r = Presolver().run(m)
    assert not r.infeasible and r.converged
    assert time.perf_counter() - t0 < 20.0


@needs_reference
def test_threshold_models_match_reference(cmp):
    """Candidate bounds within a few ulps of the reference's decision
    threshold (the bound plus or minus 1e-9): the brackets cannot settle these
    targets and the exact sums decide them as the reference does."""
    for seed in range(100):
        rc, msg, _ = cmp.compare(presolve_cases.threshold_model(seed))
        assert rc == 0, (seed, msg)


@needs_reference
@pytest.mark.parametrize("name", sorted(presolve_cases.edge_models()))
def test_edge_models_match_reference(cmp, name):
    rc, msg, _ = cmp.compare(presolve_cases.edge_models()[name])
    assert rc == 0, msg


@needs_reference
def test_reference_mps_files_match_reference(cmp):
    root = __graft_entry__.REFERENCE_ROOT
    files = sorted(glob.glob(os.path.join(root, "**", "*.mps"), recursive=True))
    if not files:
        pytest.skip("reference MPS files not present")
    compared = 0
    for f in files:
        rc, msg, _ = cmp.compare_mps(f)
        if rc == -1 and msg.startswith("MpsReader Error"):
            continue  # files the reference reader itself refuses
        assert rc == 0, (f, msg)
        compared += 1
    assert compared >= 20


@needs_reference
@pytest.mark.parametrize("seed", [1, 2])
def test_planted_config0_lps_match_reference(cmp, seed):
    rc, msg, summary = cmp.compare(PresolveModel.from_lp(g.reference_lp(seed).lp))
    assert rc == 0, msg
    assert summary["transformations"] > 100 and not summary["infeasible"]


@pytest.mark.skipif(not (presolve_cmp.available() and
                         os.path.exists(os.path.join(os.path.dirname(presolve_cmp.LIB),
                                                     "libpipeline_fastpre.so"))),
                    reason="pipelines not built (make -C oracle pipeline presolve)")
def test_pipeline_with_fast_presolve_matches_reference_pipeline():
    """solver::solve on the reference's fixture LPs, PDLP forced and the
    dispatcher's own choice: with the fast presolve linked in place of
    presolver.cpp every answer is the reference pipeline's, bit for bit."""
    from oracle.pipeline import Pipeline
    from tests.test_pipeline import fixture_models
    ref, fast = Pipeline("ref"), Pipeline("fastpre")
    for name, d in fixture_models().items():
        for engine in (0, None):
            a = ref.import_model(d).solve(engine=engine, tolerance=1e-8)
            b = fast.import_model(d).solve(engine=engine, tolerance=1e-8)
            assert (a.status, a.executed_engine, a.iterations) == \
                (b.status, b.executed_engine, b.iterations), (name, engine)
            assert bits_equal(a.objective, b.objective), (name, engine)
            for f in ("x", "duals", "reduced_costs"):
                assert bits_equal(getattr(a, f), getattr(b, f)), (name, engine, f)


def test_repeated_variable_tightening_is_the_reference_s():
    """x + x + y >= 2, x + y <= 1.6, y in [0, 1]: the reference's
    tightenBounds leaves both x terms out of the other terms' activity and
    divides by one coefficient, so it sets x >= 1 (0.5 is implied) and then
    y <= 0.6; the drop-in returns the reference's result, this included."""
    m = PresolveModel(var_lower=np.array([0.0, 0.0]), var_upper=np.array([10.0, 1.0]),
                      row_lower=np.array([2.0, -np.inf]), row_upper=np.array([np.inf, 1.6]),
                      row_start=np.array([0, 3, 5]), row_index=np.array([0, 0, 1, 0, 1], np.int32),
                      row_value=np.ones(5), objective_index=np.array([0], np.int32),
                      objective_value=np.array([1.0]))
    r = Presolver().run(m)
    t = r.transformations
    assert [r.reason_text[int(c)] for c in t["reason"][:3]] == [
        "Constraint tightened variable lower bound", "Constraint tightened variable upper bound",
        "Constraint tightened variable upper bound"]
    assert list(t["variable"][:3]) == [0, 0, 1] and list(t["constraint"][:3]) == [0, 1, 1]
    assert list(t["new_value"][:3]) == [1.0, 1.6, 1.6 - 1.0]
    assert list(r.model.var_lower) == [1.0, 0.0]


PRESOLVE_TESTS = os.path.join(os.path.dirname(presolve_cmp.LIB), "presolve_tests")
REFERENCE_TEST_PROGRAMS = [
    ("test_batch2", None), ("test_presolve_correctness", None),
    ("test_transformation_metadata", None), ("test_pipeline_cascades", None),
    ("test_adversarial", None), ("test_postsolver", None), ("test_presolve_metadata", None),
] + [("test_dual_reconstruction", case) for case in (
    "known_shadow_price derived_bound singleton_lower singleton_upper singleton_equality "
    "singleton_ranged inactive_singleton reduced_costs equality_dual lower_dual upper_dual "
    "fixed_variable empty_duals wrong_dual_size invalid_constraint_mapping residual_gate "
    "nonfinite_duals nonfinite_reconstruction quadratic_gradient quadratic_reconstruction "
    "primal_only missing_bound_provenance invalid_bound_indices invalid_bound_direction "
    "invalid_source_coefficient invalid_singleton_provenance provenance_after_elimination "
    "provenance_bound_history derived_bound_directions").split()] + [
    ("test_classifier_dispatcher", None), ("test_end_to_end", None),
    ("test_qp_convention", None), ("test_milp_enumeration", None),
] + [("test_postsolve_integration", case) for case in (
    "lp_engines qp_signs all_eliminated bound_only integer_models unavailable_duals "
    "failure_statuses limit_no_solution limit_feasible_solution reduced_api").split()]


@pytest.mark.skipif(not os.path.isdir(PRESOLVE_TESTS),
                    reason="reference test programs not built (make -C oracle presolve)")
@pytest.mark.parametrize("program,case", REFERENCE_TEST_PROGRAMS)
def test_reference_presolve_test_programs_pass_with_fast_presolve(program, case):
    """The reference's own presolve and postsolve tests (tests/presolve/*.cpp,
    tests/postsolve/*.cpp) and its tests of the whole pipeline
    (tests/solver, tests/pipeline, tests/qp, tests/milp: classifier and
    dispatcher, end to end, postsolve integration, the QP convention, 200
    MILPs against enumeration), with the cases its CMakeLists.txt registers,
    built with its presolver and with the fast presolve linked in its place:
    both pass, and print the same output."""
    import subprocess
    args = [case] if case else []
    ref = subprocess.run([os.path.join(PRESOLVE_TESTS, program + "_ref"), *args],
                         capture_output=True, text=True, timeout=300)
    fast = subprocess.run([os.path.join(PRESOLVE_TESTS, program + "_fast"), *args],
                          capture_output=True, text=True, timeout=300)
    assert ref.returncode == 0, ref.stdout + ref.stderr
    assert fast.returncode == 0, fast.stdout + fast.stderr
    assert fast.stdout == ref.stdout


@pytest.mark.skipif(not os.path.exists(os.path.join(PRESOLVE_TESTS, "test_cli_fast")),
                    reason="reference CLI not built (make -C oracle presolve)")
def test_reference_cli_tests_pass_with_fast_reader_and_presolve():
    """The reference's command-line program and its own test
    (tests/cli/test_cli.cpp), built with its MPS reader and presolve and with
    the fast ones linked in their place: every test passes in both, the same
    tests in the same order."""
    import subprocess
    runs = {k: subprocess.run([os.path.join(PRESOLVE_TESTS, f"test_cli_{k}")],
                              capture_output=True, text=True, timeout=600)
            for k in ("ref", "fast")}
    for k, r in runs.items():
        assert r.returncode == 0, (k, r.stdout[-2000:] + r.stderr[-2000:])
    passed = {k: [ln for ln in r.stdout.splitlines() if ln.startswith("[PASSED]")]
              for k, r in runs.items()}
    assert passed["fast"] == passed["ref"] and len(passed["ref"]) > 5


def _small_model(**change):
    m = dict(var_lower=np.zeros(2), var_upper=np.ones(2), row_lower=np.array([0.0]),
             row_upper=np.array([1.0]), row_start=np.array([0, 2]),
             row_index=np.array([0, 1], np.int32), row_value=np.array([1.0, 1.0]),
             objective_index=np.array([0], np.int32), objective_value=np.array([1.0]))
    m.update(change)
    return PresolveModel(**m)


@pytest.mark.parametrize("change,message", [
    (dict(row_index=np.array([0, 2], np.int32)), "names no variable"),
    (dict(row_value=np.array([1.0, np.nan])), "non-finite"),
    (dict(objective_index=np.array([5], np.int32)), "names no variable"),
    (dict(var_type=np.array([0, 3], np.int8)), "unknown variable type"),
    (dict(row_start=np.array([1, 2])), "row_start"),
])
def test_refused_inputs(change, message):
    with pytest.raises(ValueError, match=message):
        Presolver().run(_small_model(**change))


def test_result_does_not_depend_on_host_threads(tmp_path):
    """The read-only steps of a 20,000-row model split across threads: one
    thread (PDLPGPU_PRESOLVE_THREADS=1) and eight give the same result, bit
    for bit (separate processes: the variable is read at each call)."""
    import subprocess
    import sys
    code = (
        "import sys, numpy as np\n"
        "from optimisation_solver_b200 import generators as g\n"
        "from optimisation_solver_b200.presolve import PresolveModel, Presolver\n"
        "from tests.golden.make_presolve_golden import flatten\n"
        "r = flatten(Presolver().run(PresolveModel.from_lp("
        "g.planted_lp(m=20000, n=40000, seed=3).lp)))\n"
        "np.savez(sys.argv[1], **{k: np.asarray(v) for k, v in r.items()})\n")
    root = os.path.dirname(HERE)
    out = {}
    for threads in ("1", "8"):
        path = str(tmp_path / f"threads_{threads}.npz")
        subprocess.run([sys.executable, "-c", code, path], check=True, cwd=root,
                       env={**os.environ, "PDLPGPU_PRESOLVE_THREADS": threads,
                            "PYTHONPATH": root}, timeout=600)
        out[threads] = np.load(path)
    assert all(bits_equal(out["1"][k], out["8"][k]) for k in out["1"].files)


def test_large_model_presolves_in_linear_time():
    """A planted 20,000 x 40,000 LP: the reference's pairwise row pass alone
    builds about 2 x 10^8 coefficient maps here; the fast presolve needs well
    under a second (the bound below is loose on purpose)."""
    m = PresolveModel.from_lp(g.planted_lp(m=20_000, n=40_000, seed=3).lp)
    t0 = time.perf_counter()
    r = Presolver().run(m)
    elapsed = time.perf_counter() - t0
    assert not r.infeasible and r.converged
    assert r.presolved_constraints > 19_000
    assert elapsed < 20.0, elapsed
