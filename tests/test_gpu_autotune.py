"""The measured autotuner: it returns parameters from its grid whose trial
kernels are no slower than the heuristic's, and a solve with them gives the
same result as the default layout (layout parameters change only the order of
additions inside a line)."""
import numpy as np
import pytest

from optimisation_solver_b200 import generators as g
from optimisation_solver_b200.autotune import SELL_GRID, tune, tune_session
from optimisation_solver_b200.lp import PdlpOptions, PdlpStatus
from optimisation_solver_b200.pdlp import PdlpSolver

pytestmark = pytest.mark.gpu


def test_tune_single_lp():
    p = g.planted_lp(3000, 6000, 6, seed=4)
    opts = PdlpOptions()
    out = tune([p.lp], opts, precision="mixed", reps=3)
    assert out["trial_ms"] <= out["default_trial_ms"]
    for k, v in out["params"].items():
        assert v in SELL_GRID[k]
    a = PdlpSolver("fp64").solve(p.lp, opts)
    b = PdlpSolver("fp64", **out["params"]).solve(p.lp, opts)
    assert a.status == b.status == PdlpStatus.OPTIMAL
    assert abs(a.primal_objective - b.primal_objective) <= 1e-6 * (1 + abs(a.primal_objective))


def test_tune_session_picks_a_layout():
    G = g.flow_graph()
    s, c = g.flow_parameters(G, 64, seed=2)
    out = tune_session(g.flow_lp(G, s[0], c[0]), 64, PdlpOptions(), precision="mixed",
                       objective=c, row_lower=s, row_upper=s, reps=3)
    assert out["params"]["layout"] in ("interleaved", "sell")
    assert len(out["tried"]) == 4 and np.isfinite(out["trial_ms"])
