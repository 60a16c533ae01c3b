"""The reference pipeline as the oracle of the end-to-end path (CPU part).

`oracle/Makefile` (`make pipeline`) compiles the reference's presolve,
dispatch, engines, postsolve and MPS reader from its sources; these tests
check the committed fixtures against it and the MPS round trip of the
1000 x 2000 planted LP through the reference MpsReader. The GPU engine behind
the same pipeline is tested in test_gpu_pipeline.py.
"""
import os

import numpy as np
import pytest

from optimisation_solver_b200 import generators as g
from oracle.pipeline import MODEL_FIELDS, Pipeline, available
from tests.mps_writer import write_free_mps

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = os.path.join(HERE, "golden", "pipeline_models.npz")

pytestmark = pytest.mark.skipif(not available("ref"),
                                reason="reference pipeline not built (make -C oracle pipeline)")


def fixture_models():
    data = np.load(FIXTURES)
    out = {}
    for name in data["names"]:
        out[str(name)] = {k.split("/", 1)[1]: data[k] for k in data.files
                          if k.startswith(f"{name}/")}
    return out


@pytest.fixture(scope="module")
def ref_pipeline():
    return Pipeline("ref")


def test_fixture_models_rebuild_exactly(ref_pipeline):
    for name, d in fixture_models().items():
        model = ref_pipeline.import_model(d)
        back = model.export()
        for f in MODEL_FIELDS:
            assert np.array_equal(np.asarray(back[f]), np.asarray(d[f])), (name, f)


def test_reference_pipeline_reproduces_published_answers(ref_pipeline):
    """PDLP forced through solver::solve, on the rebuilt models: the
    reference's own statuses and objectives, and its published answers
    (benchmarks/instances/known_answers.json, netlib/best_known.json)."""
    for name, d in fixture_models().items():
        r = ref_pipeline.import_model(d).solve(engine=0, tolerance=1e-8)
        assert r.status == str(d["pdlp_status"]), name
        if r.status == "optimal":
            assert r.objective == float(d["pdlp_objective"]), name
            want = float(d["expected_objective"])
            assert abs(r.objective - want) <= 1e-6 * max(1.0, abs(want)), (name, r.objective, want)


def test_planted_lp_mps_round_trip_is_exact(tmp_path, ref_pipeline):
    """The 1000 x 2000 planted LP written as free-format MPS and read back by
    the reference MpsReader, then adapter::toCompiledLp: the same LP, bit for
    bit."""
    lp = g.reference_lp(0).lp
    path = str(tmp_path / "planted_0.mps")
    write_free_mps(lp, path, "planted_0")
    back = ref_pipeline.read_mps(path).compile()
    assert back.num_rows == lp.num_rows and back.num_cols == lp.num_cols
    for f in ("row_start", "col_index", "values", "objective", "row_lower", "row_upper",
              "var_lower", "var_upper"):
        assert np.array_equal(getattr(back, f), getattr(lp, f)), f
    assert back.objective_offset == lp.objective_offset
