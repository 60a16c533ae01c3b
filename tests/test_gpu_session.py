"""Sessions (one shared matrix, repeated batched solves) and streams (slots
refilled as instances finish) against one-LP-per-call solves.

An instance's arithmetic never depends on the other instances of its batch
(every reduction is per instance, in a fixed order), so a stream reproduces a
batch solve bit for bit, whichever slot an instance lands in.
"""
import numpy as np
import pytest

from optimisation_solver_b200 import generators as g
from optimisation_solver_b200.lp import PdlpOptions, PdlpStatus
from optimisation_solver_b200.pdlp import PdlpSolver
from optimisation_solver_b200.session import Session

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def family():
    G = g.flow_graph()
    s, c = g.flow_parameters(G, 40, seed=11)
    return G, g.flow_lp(G, s[0], c[0]), s, c


def test_session_matches_single_solves(family):
    G, fam, s, c = family
    opts = PdlpOptions().with_tolerance(1e-5)
    S = Session(fam, 8, opts, precision="fp64")
    S.load(objective=c[:8], row_lower=s[:8], row_upper=s[:8])
    S.solve()
    res = S.read()
    solver = PdlpSolver("fp64")
    for i in range(3):
        r = solver.solve(g.flow_lp(G, s[i], c[i]), opts)
        assert res["status"][i] == r.status == PdlpStatus.OPTIMAL
        assert abs(res["primal_objective"][i] - r.primal_objective) <= 1e-5 * abs(r.primal_objective)
        assert res["primal_residual"][i] <= 1e-5 and res["relative_gap"][i] <= 1e-5


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_stream_reproduces_batches_bitwise(family, precision):
    G, fam, s, c = family
    opts = PdlpOptions().with_tolerance(1e-4)
    S = Session(fam, 16, opts, precision=precision)
    out = S.stream(40, objective=c, row_lower=s, row_upper=s)
    assert out["optimal"] == 40
    for b0 in (0, 16, 24):
        S.load(objective=c[b0:b0 + 16], row_lower=s[b0:b0 + 16], row_upper=s[b0:b0 + 16])
        S.solve()
        r = S.read()
        for k in range(16):
            i = b0 + k
            assert r["iterations"][k] == out["iterations"][i]
            assert r["primal_objective"][k] == out["primal_objective"][i]
            assert np.array_equal(r["primal"][k], out["primal"][i])
            assert np.array_equal(r["dual"][k], out["dual"][i])


def test_device_pointers_match_host_arrays(family):
    import torch
    G, fam, s, c = family
    opts = PdlpOptions().with_tolerance(1e-4)
    S = Session(fam, 8, opts, precision="mixed")
    S.load(objective=c[:8], row_lower=s[:8], row_upper=s[:8])
    S.solve()
    host = S.read()
    sd = torch.as_tensor(s[:8], device="cuda")
    cd = torch.as_tensor(c[:8], device="cuda")
    S.load(objective=cd, row_lower=sd, row_upper=sd, on_device=True)
    S.solve()
    px = torch.empty((8, fam.num_cols), dtype=torch.float64, device="cuda")
    py = torch.empty((8, fam.num_rows), dtype=torch.float64, device="cuda")
    dev = S.read(primal=px, dual=py, on_device=True)
    torch.cuda.synchronize()
    assert np.array_equal(dev["iterations"], host["iterations"])
    assert np.array_equal(px.cpu().numpy(), host["primal"])
    assert np.array_equal(py.cpu().numpy(), host["dual"])


def test_warm_start_from_solution_converges_fast(family):
    G, fam, s, c = family
    opts = PdlpOptions().with_tolerance(1e-4)
    S = Session(fam, 8, opts, precision="fp64")
    S.load(objective=c[:8], row_lower=s[:8], row_upper=s[:8])
    S.solve()
    cold = S.read()
    S.load(objective=c[:8], row_lower=s[:8], row_upper=s[:8], warm_primal=cold["primal"],
           warm_dual=cold["dual"], warm_weight=cold["final_primal_weight"])
    S.solve()
    warm = S.read()
    assert all(st == PdlpStatus.OPTIMAL for st in warm["status"])
    assert warm["iterations"].max() <= 100
    assert cold["iterations"].min() > 500
