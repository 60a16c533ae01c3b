"""Sessions (one shared matrix, repeated batched solves) and streams (slots
refilled as instances finish) against one-LP-per-call solves, in both device
layouts of the trial kernels (per-instance SELL-G walks and the
batch-interleaved layout).

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


LAYOUTS = ["sell", "interleaved"]


@pytest.mark.parametrize("layout", LAYOUTS)
def test_session_matches_single_solves(family, layout):
    G, fam, s, c = family
    opts = PdlpOptions().with_tolerance(1e-5)
    S = Session(fam, 8, opts, precision="fp64", layout=layout)
    S.load(objective=c[:8], row_lower=s[:8], row_upper=s[:8])
    S.solve()
    res = S.read()
    solver = PdlpSolver("fp64")
    for i in range(3):
        r = solver.solve(g.flow_lp(G, s[i], c[i]), opts)
        assert res["status"][i] == r.status == PdlpStatus.OPTIMAL
        # Both points are within the 1e-5 relative gap of the optimum, so
        # their objectives may differ by up to twice that bound.
        assert abs(res["primal_objective"][i] - r.primal_objective) <= 4e-5 * (1 + abs(r.primal_objective))
        assert res["primal_residual"][i] <= 1e-5 and res["relative_gap"][i] <= 1e-5


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_stream_reproduces_batches_bitwise(family, precision, layout):
    G, fam, s, c = family
    opts = PdlpOptions().with_tolerance(1e-4)
    S = Session(fam, 16, opts, precision=precision, layout=layout)
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


@pytest.mark.parametrize("layout", LAYOUTS)
def test_device_pointers_match_host_arrays(family, layout):
    import torch
    G, fam, s, c = family
    opts = PdlpOptions().with_tolerance(1e-4)
    S = Session(fam, 8, opts, precision="mixed", layout=layout)
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


def test_device_inputs_written_just_before_the_call(family):
    """Device inputs whose values are still being written by the caller's
    kernels on the default stream when the stream call is made (behind a
    long chain of matrix products): the session waits for them, so the
    results are those of the same instances passed as host arrays."""
    import torch
    G, fam, s, c = family
    opts = PdlpOptions().with_tolerance(1e-4)
    S = Session(fam, 16, opts, precision="mixed")
    host = S.stream(24, objective=c[:24], row_lower=s[:24], row_upper=s[:24])
    sd = torch.full((24, fam.num_rows), float("nan"), dtype=torch.float64, device="cuda")
    cd = torch.full((24, fam.num_cols), float("nan"), dtype=torch.float64, device="cuda")
    px = torch.empty((24, fam.num_cols), dtype=torch.float64, device="cuda")
    py = torch.empty((24, fam.num_rows), dtype=torch.float64, device="cuda")
    s_h = torch.as_tensor(s[:24]).pin_memory()
    c_h = torch.as_tensor(c[:24]).pin_memory()
    torch.cuda.synchronize()
    busy = torch.randn((4096, 4096), device="cuda")
    for _ in range(40):          # tens of milliseconds of default-stream work
        busy = torch.tanh(busy @ busy)
    sd.copy_(s_h, non_blocking=True)
    cd.copy_(c_h, non_blocking=True)
    dev = S.stream(24, objective=cd, row_lower=sd, row_upper=sd, primal=px, dual=py, on_device=True)
    torch.cuda.synchronize()
    assert dev["optimal"] == host["optimal"] == 24
    assert np.array_equal(dev["iterations"], host["iterations"])
    assert np.array_equal(px.cpu().numpy(), host["primal"])
    assert np.array_equal(py.cpu().numpy(), host["dual"])


@pytest.mark.parametrize("layout", LAYOUTS)
def test_warm_start_from_solution_converges_fast(family, layout):
    G, fam, s, c = family
    opts = PdlpOptions().with_tolerance(1e-4)
    S = Session(fam, 8, opts, precision="fp64", layout=layout)
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


@pytest.mark.parametrize("batch,precision", [(40, "fp64"), (96, "fp64"), (160, "mixed")])
def test_interleaved_matches_sell_layout(batch, precision):
    """Same instances, same tolerance: the two layouts differ only in the
    rounding of their sums, so statuses agree and objectives agree to the
    tolerance; iteration counts stay close. The batch sizes give 1, 2 and 4
    instances per lane (the last with a partly filled group)."""
    G = g.flow_graph()
    s, c = g.flow_parameters(G, batch, seed=21)
    fam = g.flow_lp(G, s[0], c[0])
    tol = 1e-6 if precision == "fp64" else 1e-4
    opts = PdlpOptions().with_tolerance(tol)
    out = {}
    for layout in LAYOUTS:
        S = Session(fam, batch, opts, precision=precision, layout=layout)
        S.load(objective=c, row_lower=s, row_upper=s)
        S.solve()
        out[layout] = S.read()
        S.close()
    a, b = out["sell"], out["interleaved"]
    assert list(a["status"]) == list(b["status"])
    assert all(st == PdlpStatus.OPTIMAL for st in b["status"])
    rel = np.abs(a["primal_objective"] - b["primal_objective"]) / (1 + np.abs(a["primal_objective"]))
    assert rel.max() <= 10 * tol
    ratio = b["iterations"].mean() / a["iterations"].mean()
    assert 0.8 <= ratio <= 1.25


def test_interleaved_own_vectors_equal_family_vectors(family):
    """Loading the family's variable bounds per instance (own interleaved
    vectors) gives bit for bit the solve that reads the broadcast family
    vectors, and the captured loop is rebuilt when that choice changes."""
    G, fam, s, c = family
    opts = PdlpOptions().with_tolerance(1e-4)
    S = Session(fam, 32, opts, precision="mixed", layout="interleaved")
    S.load(objective=c[:32], row_lower=s[:32], row_upper=s[:32])
    S.solve()
    shared = S.read()
    xl = np.repeat(fam.var_lower[None, :], 32, axis=0)
    xu = np.repeat(fam.var_upper[None, :], 32, axis=0)
    S.load(objective=c[:32], row_lower=s[:32], row_upper=s[:32], var_lower=xl, var_upper=xu)
    S.solve()
    own = S.read()
    assert np.array_equal(shared["iterations"], own["iterations"])
    assert np.array_equal(shared["primal"], own["primal"])
    assert np.array_equal(shared["dual"], own["dual"])


def test_interleaved_infeasible_and_iteration_limit(family):
    """Certificates and the iteration limit inside an interleaved batch: an
    unbalanced supply vector is primal infeasible (every incidence row sums to
    zero); a tiny iteration limit ends the others through polishing, with
    the same outcome as the per-instance layout."""
    G, fam, s, c = family
    sup = s[:32].copy()
    sup[3, 0] += 50.0
    sup[17, 5] -= 40.0
    opts = PdlpOptions().with_tolerance(1e-4)
    res = {}
    for layout in LAYOUTS:
        S = Session(fam, 32, opts, precision="fp64", layout=layout)
        S.load(objective=c[:32], row_lower=sup, row_upper=sup)
        S.solve()
        res[layout] = S.read()
        S.close()
    for r in res.values():
        assert r["status"][3] == PdlpStatus.INFEASIBLE
        assert r["status"][17] == PdlpStatus.INFEASIBLE
        assert sum(st == PdlpStatus.OPTIMAL for st in r["status"]) == 30
    limited = PdlpOptions().with_tolerance(1e-8)
    limited.iteration_limit = 300
    out = {}
    for layout in LAYOUTS:
        S = Session(fam, 32, limited, precision="fp64", layout=layout)
        S.load(objective=c[:32], row_lower=s[:32], row_upper=s[:32])
        S.solve()
        out[layout] = S.read()
        S.close()
    assert list(out["sell"]["status"]) == list(out["interleaved"]["status"])
    assert all(st == PdlpStatus.ITERATION_LIMIT for st in out["interleaved"]["status"])
    assert np.all(np.isfinite(out["interleaved"]["primal_objective"]))


def test_interleaved_kernel_timing():
    """The interleaved trial kernels in timing mode report positive times and
    their algorithmic bytes; a solve after the timing is unaffected."""
    G = g.flow_graph()
    s, c = g.flow_parameters(G, 64, seed=3)
    fam = g.flow_lp(G, s[0], c[0])
    opts = PdlpOptions().with_tolerance(1e-4)
    S = Session(fam, 64, opts, precision="mixed", layout="interleaved")
    S.load(objective=c, row_lower=s, row_upper=s)
    S.solve()
    before = S.read()
    tk = S.time_kernels(5)
    assert tk["primal_ms"] > 0 and tk["dual_ms"] > 0
    n, m = G.arcs, G.nodes
    # x, x', c and the gathered y per instance; tau, itau and the bounds once.
    assert tk["primal_bytes"] >= 64 * (3 * n + m) * 4
    S.load(objective=c, row_lower=s, row_upper=s)
    S.solve()
    after = S.read()
    assert np.array_equal(before["primal"], after["primal"])
