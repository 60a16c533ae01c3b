"""Host-side layout (no device): the SELL-G slices encode A exactly, the
canonicalisation equals SparseMatrix::fromTriplets bit for bit, and padding
stays bounded on the workload shapes."""
import numpy as np
import pytest

from optimisation_solver_b200 import generators as g
from optimisation_solver_b200 import pdlp
from optimisation_solver_b200.lp import CompiledLp, SparseMatrix
from tests import cases


def _integer_copy(lp):
    """Same pattern, small-integer values: every sum is exact in FP64."""
    v = np.round(lp.values * 4)
    v[v == 0] = 1.0
    m = lp.matrix
    return CompiledLp(SparseMatrix(m.rows, m.columns, m.row_start, m.col_index, v),
                      lp.objective, lp.row_lower, lp.row_upper, lp.var_lower, lp.var_upper)


SHAPES = [
    ("reference_lp", lambda: g.reference_lp(0).lp),
    ("dense_rows", lambda: g.planted_lp(300, 500, 30, seed=1).lp),
    ("zipf", lambda: g.planted_lp(2000, 3000, degrees=np.clip(np.random.default_rng(3).zipf(1.6, 3000), 1, 1500), seed=2).lp),
    ("flow", lambda: g.flow_lp(g.flow_graph(), *[a[0] for a in g.flow_parameters(g.flow_graph(), 1, 0)])),
    ("empty_rows_and_cols", lambda: cases.inactive_row()),
    ("degenerate", cases.degenerate),
]


@pytest.mark.parametrize("name,build", SHAPES, ids=[s[0] for s in SHAPES])
@pytest.mark.parametrize("lane,vw", [(8, 1), (8, 2), (4, 4), (2, 1), (32, 4)])
def test_layout_encodes_matrix_exactly(name, build, lane, vw):
    lp = _integer_copy(build())
    x = np.random.default_rng(0).integers(-5, 6, lp.num_cols).astype(float)
    assert np.array_equal(pdlp.layout_multiply(lp, x, lane, vw), lp.matrix.multiply(x))
    st = pdlp.layout_stats(lp, lane, vw)
    assert st["a_entries"] == lp.nnz and st["at_entries"] == lp.nnz
    assert st["a_slots"] % 32 == 0 and st["a_slots"] >= lp.nnz


def test_padding_bounded_on_workloads():
    for build in (lambda: g.reference_lp(0).lp,
                  lambda: g.flow_lp(g.flow_graph(), *[a[0] for a in g.flow_parameters(g.flow_graph(), 1, 0)])):
        lp = build()
        st = pdlp.layout_stats(lp)
        assert st["a_slots"] <= 1.25 * lp.nnz + 64 * 32
        assert st["at_slots"] <= 1.25 * lp.nnz + 64 * 32


def test_canonicalisation_matches_from_triplets(port_oracle):
    rng = np.random.default_rng(5)
    ti = rng.integers(0, 30, 500)
    tj = rng.integers(0, 40, 500)
    tv = rng.uniform(-2, 2, 500)
    tv[::13] = 0.0
    ours = SparseMatrix.from_triplets(30, 40, ti, tj, tv)
    rs, ci, va, *_ = port_oracle.from_triplets(30, 40, ti, tj, tv)
    assert np.array_equal(ours.row_start, rs)
    assert np.array_equal(ours.col_index, ci)
    assert np.array_equal(ours.values, va)
    # The library's canonicalisation of a non-canonical CSR agrees too: feed
    # the unsorted triplets as CSR rows and multiply with integer values.
    order = np.argsort(ti, kind="stable")
    raw = SparseMatrix(30, 40, np.concatenate([[0], np.cumsum(np.bincount(ti, minlength=30))]),
                       tj[order].astype(np.int32), np.round(tv[order] * 8))
    canon = SparseMatrix.from_triplets(30, 40, ti[order], tj[order], np.round(tv[order] * 8))
    lp_raw = CompiledLp(raw, np.zeros(40), np.zeros(30), np.zeros(30), np.zeros(40), np.ones(40))
    x = rng.integers(-3, 4, 40).astype(float)
    assert np.array_equal(pdlp.layout_multiply(lp_raw, x), canon.multiply(x))


def test_invalid_matrix_rejected_on_host():
    bad = SparseMatrix(2, 2, np.array([0, 1, 2]), np.array([0, 5], dtype=np.int32), np.array([1.0, 1.0]))
    lp = CompiledLp(bad, np.zeros(2), np.zeros(2), np.zeros(2), np.zeros(2), np.ones(2))
    with pytest.raises(RuntimeError, match="out of range"):
        pdlp.layout_stats(lp)
