"""Seeded synthetic LP families (numpy PCG64), the workloads this engine is
measured and tested on. Every generator returns ``CompiledLp`` objects plus the
planted optimum where one exists, so the objective error of a solve can be
measured against an exact answer.

planted_lp          sparse LP with a planted primal-dual optimum: m rows (a
                    fraction equalities, the rest <=), n columns of fixed or
                    drawn degree, N(0,1) or log-uniform magnitudes, box bounds.
                    At its defaults (m=1000, n=2000, degree 4, N(0,1), bounds
                    [0,10]) it is the reference-solvable single LP.
large_lp            planted_lp at m=500k, n=1M with Zipf column degrees
                    (truncated at 1000) and log-uniform magnitudes in
                    [1e-2, 1e2]; 30% equality rows, bounds [0, U(1,100)].
stress_lp           large_lp's matrix at m=100k, n=200k, with 20% free
                    variables, 10% ranged rows, and rows/columns rescaled by
                    log-uniform factors in [1e-4, 1e4] after planting.
uneven_batch        1024 planted_lp instances, seed i for instance i, m
                    log-uniform in [200, 50000], n = 2m, degree U{4..12}.
network_flow_family min-cost flow on a fixed geometric graph (2000 nodes; for
                    every node and each of its 5 nearest neighbours one arc in
                    each direction, so 20,000 arcs with parallel arcs kept as
                    separate columns; capacities U(5,50)); per instance a random
                    feasible flow fixes the supplies and costs are length x
                    lognormal(0, 0.2).

Planting: with shadow prices y (c = A'y + z), a <= row that is tight has
y <= 0, a slack row has y = 0, an equality row has any y; z >= 0 where x sits
at its lower bound, z <= 0 at its upper bound, z = 0 strictly inside. The
engine's own dual (stationarity c + A'y_engine) is y_engine = -y.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .lp import INF, CompiledLp, SparseMatrix


@dataclass
class Planted:
    lp: CompiledLp
    x: np.ndarray          # planted primal optimum
    y: np.ndarray          # planted shadow prices (engine dual is -y)
    objective: float       # c'x* + offset, the exact optimal value


def _distinct_rows(rng, m, degrees):
    """For column j, degrees[j] distinct uniformly random rows. Returns the
    (row, col) arrays of the pattern."""
    n = degrees.size
    col = np.repeat(np.arange(n, dtype=np.int64), degrees)
    row = rng.integers(0, m, size=col.size, dtype=np.int64)
    # Re-draw collisions inside a column until none remain.
    for _ in range(64):
        key = col * m + row
        order = np.argsort(key, kind="stable")
        dup = np.zeros(key.size, dtype=bool)
        dup[order[1:]] = key[order[1:]] == key[order[:-1]]
        if not dup.any():
            break
        row[dup] = rng.integers(0, m, size=int(dup.sum()), dtype=np.int64)
    return row, col


def _zipf_degrees(rng, n, s, cap):
    k = np.arange(1, cap + 1, dtype=np.float64)
    p = k ** (-s)
    p /= p.sum()
    return rng.choice(np.arange(1, cap + 1), size=n, p=p).astype(np.int64)


def planted_lp(m=1000, n=2000, degree=4, seed=0, eq_fraction=0.5, slack_fraction=0.5,
               magnitudes="normal", upper=10.0, interior_fraction=0.7, degrees=None,
               free_fraction=0.0, ranged_fraction=0.0, rescale=None) -> Planted:
    rng = np.random.default_rng(seed)
    if degrees is None:
        degrees = np.full(n, degree, dtype=np.int64)
    degrees = np.minimum(degrees, m)
    row, col = _distinct_rows(rng, m, degrees)
    if magnitudes == "normal":
        val = rng.standard_normal(row.size)
        val[val == 0.0] = 1.0
    else:   # log-uniform magnitude in [1e-2, 1e2] with a random sign
        val = 10.0 ** rng.uniform(-2.0, 2.0, row.size)
        val *= np.where(rng.random(row.size) < 0.5, -1.0, 1.0)
    A = SparseMatrix.from_triplets(m, n, row, col, val)

    # Variable bounds and the planted primal point.
    if np.isscalar(upper):
        xu = np.full(n, float(upper))
    else:
        xu = np.asarray(upper, dtype=np.float64)
    xl = np.zeros(n)
    kind = rng.random(n)
    interior = kind < interior_fraction
    at_upper = (~interior) & (rng.random(n) < 0.5)
    at_lower = (~interior) & (~at_upper)
    x = np.where(interior, rng.uniform(0.0, 1.0, n) * xu, 0.0)
    x[at_upper] = xu[at_upper]
    free = np.zeros(n, dtype=bool)
    if free_fraction > 0.0:
        free = rng.random(n) < free_fraction
        xl[free] = -INF
        xu[free] = INF
        x[free] = rng.standard_normal(int(free.sum())) * 5.0
        interior |= free
        at_upper &= ~free
        at_lower &= ~free

    # Row bounds and planted shadow prices.
    b = A.multiply(x)
    n_eq = int(round(eq_fraction * m))
    rl = np.full(m, -INF)
    ru = b.copy()
    y = np.zeros(m)
    is_eq = np.zeros(m, dtype=bool)
    is_eq[:n_eq] = True
    rl[is_eq] = b[is_eq]
    y[is_eq] = rng.standard_normal(n_eq)
    ineq = np.flatnonzero(~is_eq)
    slack = rng.random(ineq.size) < slack_fraction
    ru[ineq[slack]] = b[ineq[slack]] + rng.uniform(0.0, 1.0, int(slack.sum()))
    tight = ineq[~slack]
    y[tight] = -np.abs(rng.standard_normal(tight.size))
    if ranged_fraction > 0.0:
        ranged = ineq[rng.random(ineq.size) < ranged_fraction / max(1e-12, 1.0 - eq_fraction)]
        width = rng.uniform(0.1, 10.0, ranged.size)
        side = rng.integers(0, 3, ranged.size)      # 0 tight upper, 1 tight lower, 2 slack
        up = side == 0
        lo = side == 1
        sl = side == 2
        ru[ranged[up]] = b[ranged[up]]
        rl[ranged[up]] = b[ranged[up]] - width[up]
        y[ranged[up]] = -np.abs(rng.standard_normal(int(up.sum())))
        rl[ranged[lo]] = b[ranged[lo]]
        ru[ranged[lo]] = b[ranged[lo]] + width[lo]
        y[ranged[lo]] = np.abs(rng.standard_normal(int(lo.sum())))
        off = rng.uniform(0.0, 1.0, int(sl.sum())) * width[sl]
        rl[ranged[sl]] = b[ranged[sl]] - off
        ru[ranged[sl]] = b[ranged[sl]] - off + width[sl]
        y[ranged[sl]] = 0.0

    # Reduced costs and the objective c = A'y + z.
    z = np.zeros(n)
    z[at_lower] = np.abs(rng.standard_normal(int(at_lower.sum())))
    z[at_upper] = -np.abs(rng.standard_normal(int(at_upper.sum())))
    c = A.transpose_multiply(y) + z

    if rescale is not None:   # rows and columns by log-uniform factors (optimum preserved)
        lo_exp, hi_exp = rescale
        dr = 10.0 ** rng.uniform(lo_exp, hi_exp, m)
        dc = 10.0 ** rng.uniform(lo_exp, hi_exp, n)
        rows_of = np.repeat(np.arange(m), np.diff(A.row_start))
        A = SparseMatrix(m, n, A.row_start, A.col_index,
                         A.values * dr[rows_of] * dc[A.col_index])
        # x = Dc x', so x' = x / dc; bounds likewise; rows scale by dr.
        x = x / dc
        xl = np.where(np.isfinite(xl), xl / dc, xl)
        xu = np.where(np.isfinite(xu), xu / dc, xu)
        rl = np.where(np.isfinite(rl), rl * dr, rl)
        ru = np.where(np.isfinite(ru), ru * dr, ru)
        c = c * dc
        y = y / dr
    lp = CompiledLp(A, c, rl, ru, xl, xu, 0.0)
    return Planted(lp, x, y, float(c @ x))


def reference_lp(seed=0) -> Planted:
    """The reference-solvable single LP: m=1000 (500 equality, 500 <=), n=2000,
    4 nonzeros per column, N(0,1) values, bounds [0, 10]."""
    return planted_lp(1000, 2000, 4, seed=seed)


def large_lp(seed=0, m=500_000, n=1_000_000, zipf_s=1.8, cap=1000) -> Planted:
    """Zipf column degrees truncated at ``cap``. s = 1.8 gives a mean degree
    of about 8.2 (nnz about 8M at n = 1M); see the module docstring."""
    rng = np.random.default_rng(10_000 + seed)
    degrees = _zipf_degrees(rng, n, zipf_s, cap)
    upper = rng.uniform(1.0, 100.0, n)
    return planted_lp(m, n, seed=seed, eq_fraction=0.3, magnitudes="loguniform", upper=upper,
                      degrees=degrees)


def stress_lp(seed=0, m=100_000, n=200_000, zipf_s=1.8, cap=1000) -> Planted:
    rng = np.random.default_rng(20_000 + seed)
    degrees = _zipf_degrees(rng, n, zipf_s, cap)
    upper = rng.uniform(1.0, 100.0, n)
    return planted_lp(m, n, seed=seed, eq_fraction=0.3, magnitudes="loguniform", upper=upper,
                      degrees=degrees, free_fraction=0.2, ranged_fraction=0.1,
                      rescale=(-4.0, 4.0))


def uneven_batch_sizes(count=1024, lo=200, hi=50_000, seed=0):
    rng = np.random.default_rng(30_000 + seed)
    return np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)


def uneven_batch(count=1024, lo=200, hi=50_000, seed=0, sizes=None):
    """Instance i: m_i log-uniform in [lo, hi], n_i = 2 m_i, column degree
    U{4..12}, seeded with i."""
    if sizes is None:
        sizes = uneven_batch_sizes(count, lo, hi, seed)
    out = []
    for i, m in enumerate(sizes):
        rng = np.random.default_rng(40_000 + i)
        deg = rng.integers(4, 13, size=2 * int(m))
        out.append(planted_lp(int(m), 2 * int(m), seed=i, degrees=deg))
    return out


# ---------------------------------------------------------------------------
# Min-cost network flow family
# ---------------------------------------------------------------------------

@dataclass
class FlowGraph:
    nodes: int
    tail: np.ndarray        # int64 [arcs]
    head: np.ndarray        # int64 [arcs]
    length: np.ndarray      # float64 [arcs]
    capacity: np.ndarray    # float64 [arcs]
    incidence: SparseMatrix  # nodes x arcs, +1 at the tail, -1 at the head

    @property
    def arcs(self) -> int:
        return int(self.tail.size)


def flow_graph(nodes=2000, neighbours=5, seed=0) -> FlowGraph:
    rng = np.random.default_rng(50_000 + seed)
    pts = rng.random((nodes, 2))
    d2 = ((pts[:, None, :] - pts[None, :, :]) ** 2).sum(-1)
    np.fill_diagonal(d2, np.inf)
    nn = np.argpartition(d2, neighbours, axis=1)[:, :neighbours]
    src = np.repeat(np.arange(nodes), neighbours)
    dst = nn.ravel()
    tail = np.concatenate([src, dst])
    head = np.concatenate([dst, src])
    order = np.argsort(tail * nodes + head, kind="stable")   # arcs grouped by (tail, head)
    tail, head = tail[order], head[order]
    length = np.sqrt(((pts[tail] - pts[head]) ** 2).sum(-1))
    capacity = rng.uniform(5.0, 50.0, tail.size)
    arcs = tail.size
    inc = SparseMatrix.from_triplets(
        nodes, arcs, np.concatenate([tail, head]), np.concatenate([np.arange(arcs)] * 2),
        np.concatenate([np.ones(arcs), -np.ones(arcs)]))
    return FlowGraph(nodes, tail, head, length, capacity, inc)


def flow_parameters(graph: FlowGraph, count: int, seed: int):
    """(supply [count, nodes], cost [count, arcs]) for ``count`` instances."""
    rng = np.random.default_rng(60_000 + seed)
    f = rng.random((count, graph.arcs)) * graph.capacity
    supply = np.zeros((count, graph.nodes))
    np.add.at(supply.T, graph.tail, f.T)
    np.add.at(supply.T, graph.head, -f.T)
    cost = graph.length * rng.lognormal(0.0, 0.2, (count, graph.arcs))
    return supply, cost


def flow_lp(graph: FlowGraph, supply: np.ndarray, cost: np.ndarray) -> CompiledLp:
    """min cost'f  s.t.  incidence f = supply,  0 <= f <= capacity."""
    return CompiledLp(graph.incidence, np.asarray(cost, np.float64),
                      np.asarray(supply, np.float64).copy(), np.asarray(supply, np.float64).copy(),
                      np.zeros(graph.arcs), graph.capacity.copy(), 0.0)
