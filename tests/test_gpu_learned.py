"""The learned warm start on the min-cost flow family: what the trained
network gains over the cold start, and the warm-started mixed-precision
stream (the headline path) pinned to the CPU oracle.

The network is trained as the benchmark trains it, on fewer labels: 4096
instances solved by the engine itself (cold start, 1e-4, mixed precision),
3-layer BF16 MLP of width 512 fitted with the library's tensor-core kernels.
It is then evaluated on 256 held-out instances of other seeds.
"""
import numpy as np
import pytest

from optimisation_solver_b200 import generators as g
from optimisation_solver_b200.lp import PdlpOptions
from optimisation_solver_b200.session import Session
from tests.parity import check_objective, check_point, solve_many

pytestmark = pytest.mark.gpu

TOL = 1e-4
HELD_OUT = 256


@pytest.fixture(scope="module")
def trained():
    import torch

    from optimisation_solver_b200.learned import train_flow_model
    G = g.flow_graph()
    model, info = train_flow_model(G, 4096, tol=TOL, precision="mixed", slots=1024, seed=7,
                                   epochs=40)
    s, c = g.flow_parameters(G, HELD_OUT, seed=4242)
    dev = torch.device("cuda", 0)
    sd = torch.as_tensor(s, device=dev)
    cd = torch.as_tensor(c, device=dev)
    family = g.flow_lp(G, s[0], c[0])
    S = Session(family, HELD_OUT, PdlpOptions().with_tolerance(TOL), precision="mixed",
                layout="interleaved")
    cold = S.stream(HELD_OUT, objective=cd.data_ptr(), row_lower=sd.data_ptr(),
                    row_upper=sd.data_ptr(), on_device=True)
    wx, wy, ww = model.predict(sd, cd)
    px = torch.empty((HELD_OUT, G.arcs), dtype=torch.float64, device=dev)
    py = torch.empty((HELD_OUT, G.nodes), dtype=torch.float64, device=dev)
    warm = S.stream(HELD_OUT, objective=cd.data_ptr(), row_lower=sd.data_ptr(),
                    row_upper=sd.data_ptr(), warm_primal=wx.data_ptr(), warm_dual=wy.data_ptr(),
                    warm_weight=ww.data_ptr(), primal=px.data_ptr(), dual=py.data_ptr(),
                    on_device=True)
    torch.cuda.synchronize()
    warm["primal"], warm["dual"] = px.cpu().numpy(), py.cpu().numpy()
    S.close()
    return dict(graph=G, supply=s, cost=c, info=info, cold=cold, warm=warm)


def test_training_fits_the_labels(trained):
    """The final loss against the constant predictor's (the weighted sum of
    the targets' variances): the network must explain a clear share."""
    info = trained["info"]
    assert info["solved"] == info["instances"]
    print(f"final loss {info['final_loss']:.4f}, constant predictor {info['baseline_loss']:.4f}, "
          f"explained {info['explained_fraction']:.3f}")
    assert info["explained_fraction"] > 0.3, info


def test_warm_start_needs_fewer_iterations_than_cold(trained):
    cold, warm = trained["cold"], trained["warm"]
    assert cold["optimal"] == warm["optimal"] == HELD_OUT
    cold_mean = float(np.mean(cold["iterations"]))
    warm_mean = float(np.mean(warm["iterations"]))
    print(f"held-out mean iterations to {TOL:g}: cold {cold_mean:.0f}, learned {warm_mean:.0f} "
          f"({warm_mean / cold_mean:.3f}x)")
    assert warm_mean < 0.95 * cold_mean, (warm_mean, cold_mean)


def test_warm_started_stream_matches_oracle(oracle, trained):
    """The first 64 held-out instances: the warm-started mixed results against
    the reference's cold FP64 solves of the same LPs."""
    G, s, c, warm = trained["graph"], trained["supply"], trained["cost"], trained["warm"]
    count = 64
    lps = [g.flow_lp(G, s[i], c[i]) for i in range(count)]
    refs = solve_many(oracle, lps, TOL)
    for i, (lp, ref) in enumerate(zip(lps, refs)):
        assert str(warm["status"][i]) == ref.status == "optimal"
        scores = {k: warm[k][i] for k in ("primal_residual", "dual_residual", "relative_gap",
                                          "primal_objective", "dual_objective")}
        check_point(oracle, lp, warm["primal"][i], warm["dual"][i], TOL, scores)
        check_objective(warm["primal_objective"][i], ref, TOL)
