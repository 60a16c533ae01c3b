"""Device components against the CPU oracle, one reference routine each.

Tolerances: FP64 kernels sum in a different order than the reference's four
interleaved accumulators, so they agree to round-off (relative 1e-12 on
products, 1e-13 on scale vectors). The Ruiz scale vectors are computed from
maxima, which are exact, and must match bit for bit. FP32 kernels are checked
against the FP64 oracle at relative 2e-5.
"""
import numpy as np
import pytest

from optimisation_solver_b200 import generators as g
from optimisation_solver_b200 import pdlp
from tests import cases

pytestmark = pytest.mark.gpu

RTOL64 = 1e-12


def _problems():
    out = [("reference_lp", g.reference_lp(0).lp),
           ("random_feasible", cases.random_feasible(300, 420, 21)),
           ("badly_scaled", cases.badly_scaled()),
           ("degenerate", cases.degenerate())]
    zipf = np.clip(np.random.default_rng(5).zipf(1.6, 3000), 1, 1200)
    out.append(("zipf", g.planted_lp(2000, 3000, degrees=zipf, seed=3, magnitudes="loguniform").lp))
    return out


PROBLEMS = _problems()


def _close(a, b, rtol, scale=None):
    a, b = np.asarray(a), np.asarray(b)
    s = np.abs(b).max() if scale is None else scale
    return np.abs(a - b).max() <= rtol * max(1.0, s)


@pytest.mark.parametrize("name,lp", PROBLEMS, ids=[p[0] for p in PROBLEMS])
def test_spmv_matches_oracle(name, lp, oracle):
    rng = np.random.default_rng(1)
    x = rng.standard_normal(lp.num_cols)
    y = rng.standard_normal(lp.num_rows)
    ax_ref = oracle.multiply(lp, x)
    aty_ref = oracle.transpose_multiply(lp, y)
    scale_ax = (np.abs(lp.values) * np.abs(x[lp.col_index])).sum()
    assert _close(pdlp.spmv(lp, x), ax_ref, RTOL64, scale_ax)
    assert _close(pdlp.spmv(lp, y, transpose=True), aty_ref, RTOL64, scale_ax + 1)
    # FP32 kernels against the FP64 oracle
    assert _close(pdlp.spmv(lp, x, precision="mixed"), ax_ref, 2e-5, scale_ax)


@pytest.mark.parametrize("name,lp", PROBLEMS, ids=[p[0] for p in PROBLEMS])
def test_spmv_deterministic(name, lp):
    x = np.random.default_rng(2).standard_normal(lp.num_cols)
    a = pdlp.spmv(lp, x)
    b = pdlp.spmv(lp, x)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("name,lp", PROBLEMS, ids=[p[0] for p in PROBLEMS])
def test_ruiz_scales_bitwise(name, lp, oracle):
    rs, cs, vals = pdlp.ruiz(lp, 10)
    ref = oracle.ruiz(lp, 10)
    assert np.array_equal(rs, ref["row_scale"])
    assert np.array_equal(cs, ref["col_scale"])
    assert np.array_equal(vals, ref["values"])


def test_ruiz_reduces_spread(oracle):
    lp = cases.badly_scaled()
    _, _, vals = pdlp.ruiz(lp, 10)
    from optimisation_solver_b200.lp import CompiledLp, SparseMatrix
    m = lp.matrix
    scaled = CompiledLp(SparseMatrix(m.rows, m.columns, m.row_start, m.col_index, vals),
                        lp.objective, lp.row_lower, lp.row_upper, lp.var_lower, lp.var_upper)
    assert oracle.condition_spread(lp) > 1e6
    assert oracle.condition_spread(scaled) < 10.0


@pytest.mark.parametrize("name,lp", PROBLEMS, ids=[p[0] for p in PROBLEMS])
def test_precondition_matches_oracle(name, lp, oracle):
    got = pdlp.precondition(lp)
    ref = oracle.precondition(lp)
    for a, b in zip(got, ref):
        assert _close(a, b, 1e-13)


@pytest.mark.parametrize("name,lp", PROBLEMS, ids=[p[0] for p in PROBLEMS])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_trial_matches_oracle(name, lp, precision, oracle):
    rng = np.random.default_rng(3)
    tau, tinv, sig, sinv = oracle.precondition(lp)
    lo = np.where(np.isfinite(lp.var_lower), lp.var_lower, -5.0)
    hi = np.where(np.isfinite(lp.var_upper), lp.var_upper, 5.0)
    x = lo + (hi - lo) * rng.random(lp.num_cols)
    y = rng.standard_normal(lp.num_rows)
    ax = oracle.multiply(lp, x)
    xo, yo, axo, red, fin = oracle.trial(lp, tau, tinv, sig, sinv, x, y, ax, 0.7, 1.3)
    gx, gy, gax, gred = pdlp.trial(lp, tau, tinv, sig, sinv, x, y, ax, 0.7, 1.3, precision=precision)
    tol = RTOL64 * 100 if precision == "fp64" else 2e-4
    assert fin
    assert _close(gx, xo, tol)
    assert _close(gax, axo, tol)
    assert _close(gy, yo, tol)
    for a, b in zip(gred, red):
        assert abs(a - b) <= (1e-10 if precision == "fp64" else 1e-3) * max(1.0, abs(b))


def test_inactive_row_dual_exactly_zero_in_trial(oracle):
    lp = cases.inactive_row()
    tau, tinv, sig, sinv = oracle.precondition(lp)
    x, y, ax = np.array([3.0]), np.zeros(2), np.array([3.0, 3.0])
    for prec in ("fp64", "mixed"):
        _, gy, _, _ = pdlp.trial(lp, tau, tinv, sig, sinv, x, y, ax, 0.5, 1.0, precision=prec)
        assert gy[1] == 0.0


@pytest.mark.parametrize("name,lp", PROBLEMS, ids=[p[0] for p in PROBLEMS])
def test_evaluate_matches_oracle(name, lp, oracle):
    rng = np.random.default_rng(4)
    x = rng.standard_normal(lp.num_cols)
    y = rng.standard_normal(lp.num_rows)
    got, _ = pdlp.evaluate(lp, x, y)
    ref = oracle.evaluate(lp, x, y)
    for k in ("primal_objective", "dual_objective", "primal_residual", "dual_residual", "relative_gap", "kkt"):
        assert abs(got[k] - ref[k]) <= 1e-11 * max(1.0, abs(ref[k])), k
    assert got["finite"] == ref["finite"] and got["dual_valid"] == ref["dual_valid"]


def test_rays_match_oracle(oracle):
    lp = cases.infeasible_rows()
    d = np.array([1.0, -1.0])   # a Farkas direction
    _, v = pdlp.evaluate(lp, np.zeros(2), d)
    proves, value, rel = oracle.test_dual_ray(lp, d)
    assert v["dual_proves"] == proves
    assert abs(v["dual_value"] - value) <= 1e-12
    lp2 = cases.unbounded_ray()
    p = np.array([1.0, 0.0])
    _, v2 = pdlp.evaluate(lp2, p, np.zeros(1))
    proves2, value2, rel2 = oracle.test_primal_ray(lp2, p)
    assert v2["primal_proves"] == proves2 and proves2
    assert abs(v2["primal_value"] - value2) <= 1e-12
