"""Mixed precision: FP32 iterations with FP64 checks, and the FP64 stage an
instance enters when its FP32 iterations stop improving the KKT score. The
FP64 stage starts from the instance's last FP32 restart point, so a mixed
solve reaches tolerances that FP32 iterates cannot represent, with the
result of an FP64 solve.
"""
import numpy as np
import pytest

from optimisation_solver_b200 import generators as g
from optimisation_solver_b200.lp import PdlpOptions, PdlpStatus
from optimisation_solver_b200.pdlp import PdlpSolver
from optimisation_solver_b200.session import Session

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("seed", [0, 1])
def test_mixed_reaches_tight_tolerance_through_fp64_stage(seed, oracle):
    """1000 x 2000 planted LP at 1e-8: FP32 iterates stall above that, the
    instance moves to FP64 and ends optimal with the reference's objective."""
    p = g.reference_lp(seed)
    opts = PdlpOptions().with_tolerance(1e-8)
    ref = oracle.solve(p.lp, dict(opts.as_dict(), thread_count=1))
    r = PdlpSolver("mixed").solve(p.lp, opts)
    assert r.status == PdlpStatus.OPTIMAL and ref.status == "optimal"
    assert r.precision == "fp32+fp64"
    assert 0 < r.fp64_iterations < r.iterations
    assert r.relative_gap <= 1e-8 and r.primal_residual <= 1e-8 and r.dual_residual <= 1e-8
    assert abs(r.primal_objective - ref.primal_objective) <= 1e-7 * (1 + abs(ref.primal_objective))


def test_mixed_loose_tolerance_stays_fp32():
    """At 1e-4 the FP32 iterations reach the tolerance on their own."""
    p = g.reference_lp(2)
    r = PdlpSolver("mixed").solve(p.lp, PdlpOptions().with_tolerance(1e-4))
    assert r.status == PdlpStatus.OPTIMAL
    assert r.precision == "fp32" and r.fp64_iterations == 0


@pytest.mark.parametrize("layout", ["sell", "interleaved"])
def test_mixed_session_matches_fp64_session_at_tight_tolerance(layout):
    """A mixed session at 1e-7 (FP64 stage on stall) and an FP64 session give
    the same statuses and objectives to the tolerance."""
    G = g.flow_graph()
    s, c = g.flow_parameters(G, 32, seed=5)
    fam = g.flow_lp(G, s[0], c[0])
    opts = PdlpOptions().with_tolerance(1e-7)
    out = {}
    for prec in ("mixed", "fp64"):
        S = Session(fam, 32, opts, precision=prec, layout=layout)
        S.load(objective=c, row_lower=s, row_upper=s)
        S.solve()
        out[prec] = S.read()
        S.close()
    a, b = out["mixed"], out["fp64"]
    # A hard instance may need more than the default 200,000 iterations at
    # this tolerance in either precision; the others must agree.
    both = [i for i in range(32) if a["status"][i] == b["status"][i] == PdlpStatus.OPTIMAL]
    assert len(both) >= 30
    rel = np.abs(a["primal_objective"][both] - b["primal_objective"][both]) / (1 + np.abs(b["primal_objective"][both]))
    assert rel.max() <= 1e-6
    assert np.max(np.maximum(a["primal_residual"][both], a["relative_gap"][both])) <= 1e-7


def test_stream_reproduces_batches_with_fp64_stage():
    """Per-instance arithmetic is independent of the batch even when some
    instances run their FP64 stage next to others still in FP32."""
    G = g.flow_graph()
    s, c = g.flow_parameters(G, 48, seed=9)
    fam = g.flow_lp(G, s[0], c[0])
    S = Session(fam, 16, PdlpOptions().with_tolerance(1e-7), precision="mixed", layout="interleaved")
    out = S.stream(48, objective=c, row_lower=s, row_upper=s)
    assert out["optimal"] >= 46   # a hard instance may need more than 200,000 iterations
    S.load(objective=c[16:32], row_lower=s[16:32], row_upper=s[16:32])
    S.solve()
    r = S.read()
    for k in range(16):
        assert r["iterations"][k] == out["iterations"][16 + k]
        assert np.array_equal(r["primal"][k], out["primal"][16 + k])
