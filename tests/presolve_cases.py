"""Seeded presolve models that reach every step of the reference's presolve
(src/presolve/presolver.cpp): exact and tiny zero coefficients, repeated
variables in a row and in the objective, fixed and nearly fixed variables,
empty rows (satisfied and not), singleton rows, rows that tighten bounds,
redundant rows, exact, scaled, negated and loosened copies of rows,
contradictory parallel rows, free, half-bounded, integer and binary
variables, quadratic objective terms. Most models are feasible by
construction (row bounds placed around the activity of a point inside the
variable bounds) so that the passes run to their fixed point; some carry a
planted contradiction.
"""
from __future__ import annotations

import numpy as np

from optimisation_solver_b200.presolve import BINARY, CONTINUOUS, INTEGER, PresolveModel

INF = np.inf


def random_model(seed: int, n: int = 40, m: int = 30, *, integers: bool = False,
                 quadratic: bool = False, contradiction: bool = False,
                 copies: float = 0.25, max_row: int = 6, exact: bool = False) -> PresolveModel:
    """exact=True plants no infeasibility: every empty row admits 0, fixed
    variables are fixed exactly and no row names a variable twice (the
    reference's bound tightening divides by one of a repeated variable's
    coefficients, which can cut off feasible points), so large models run to
    the fixed point."""
    rng = np.random.default_rng(seed)
    kind = rng.integers(0, 6, n)
    lo = np.zeros(n)
    hi = np.full(n, 10.0)
    vtype = np.zeros(n, np.int8)
    for j in range(n):
        k = kind[j]
        if k == 0:
            lo[j], hi[j] = 0.0, rng.uniform(1, 20)
        elif k == 1:
            lo[j], hi[j] = -INF, rng.uniform(-5, 5)
        elif k == 2:
            lo[j], hi[j] = rng.uniform(-5, 5), INF
        elif k == 3:
            lo[j], hi[j] = -INF, INF
        elif k == 4:  # fixed, or fixed to within the tolerance
            v = float(np.round(rng.uniform(-3, 3), 2))
            lo[j], hi[j] = v, v + (0.0 if exact or rng.random() < 0.6 else 5e-10)
        else:
            lo[j], hi[j] = rng.uniform(-4, 0), rng.uniform(0, 4)
    if integers:
        pick = rng.random(n)
        for j in range(n):
            if pick[j] < 0.2:
                vtype[j] = BINARY
                lo[j], hi[j] = 0.0, 1.0
            elif pick[j] < 0.4 and np.isfinite(lo[j]) and np.isfinite(hi[j]):
                vtype[j] = INTEGER
                lo[j], hi[j] = np.floor(lo[j]), np.ceil(hi[j]) + 1
    # a point inside the bounds
    x0 = np.where(np.isfinite(lo), lo, np.where(np.isfinite(hi), hi - 1.0, 0.0))
    span = np.where(np.isfinite(lo) & np.isfinite(hi), hi - lo, 2.0)
    x0 = x0 + rng.uniform(0, 1, n) * span * (np.isfinite(lo) & np.isfinite(hi))
    x0 = np.where(vtype == BINARY, rng.integers(0, 2, n), x0)
    x0 = np.where(vtype == INTEGER, np.clip(np.round(x0), lo, hi), x0)

    rows_idx, rows_val, rlo, rhi = [], [], [], []

    def add_row(idx, val, act=None, shape=None):
        idx = np.asarray(idx, np.int32)
        val = np.asarray(val, np.float64)
        a = float(val @ x0[idx]) if act is None else act
        s = rng.integers(0, 5) if shape is None else shape
        slack = rng.uniform(0.0, 3.0) * (rng.random() < 0.7)
        if s == 0:
            b = (a, a)
        elif s == 1:
            b = (-INF, a + slack)
        elif s == 2:
            b = (a - slack, INF)
        elif s == 3:
            b = (a - slack - 1.0, a + slack)
        else:
            b = (-INF, INF) if rng.random() < 0.3 else (a - 50.0, a + 50.0)
        rows_idx.append(idx)
        rows_val.append(val)
        rlo.append(b[0])
        rhi.append(b[1])

    for _ in range(m):
        r = rng.random()
        if r < 0.06:  # empty row, usually satisfied
            rows_idx.append(np.zeros(0, np.int32))
            rows_val.append(np.zeros(0))
            ok = rng.random() < 0.9 or contradiction or exact
            rlo.append(-1.0 if ok else 1.0)
            rhi.append(1.0 if ok else 2.0)
            continue
        length = 1 if r < 0.2 else int(rng.integers(2, max_row + 1))
        idx = rng.choice(n, size=length, replace=False)
        val = rng.normal(0, 2, length)
        if rng.random() < 0.2:
            val[rng.integers(0, length)] = 0.0 if rng.random() < 0.5 else 1e-12
        if rng.random() < 0.1 and length > 1 and not exact:  # a variable twice
            idx = np.append(idx, idx[0])
            val = np.append(val, rng.normal())
        if rng.random() < 0.3:
            val = np.round(val)
            val[val == 0] = 1.0
        add_row(idx, val)
    # copies of rows: exact, scaled, negated, loosened
    base = len(rows_idx)
    for _ in range(int(copies * base)):
        k = int(rng.integers(0, base))
        idx, val = rows_idx[k], rows_val[k]
        if idx.size == 0:
            continue
        r = rng.random()
        s = 1.0 if r < 0.3 else float(rng.choice([2.0, -1.0, 0.5, -3.0, 4.0]))
        lo_k, hi_k = rlo[k], rhi[k]
        nlo, nhi = (s * lo_k, s * hi_k) if s > 0 else (s * hi_k, s * lo_k)
        if r > 0.85:  # loosened: parallel, not a duplicate
            nlo = nlo - 1.0 if np.isfinite(nlo) else nlo
        perm = rng.permutation(idx.size)
        rows_idx.append(idx[perm])
        rows_val.append(s * val[perm])
        rlo.append(nlo)
        rhi.append(nhi)
    if contradiction:  # a parallel row whose range misses the original's
        cand = [k for k in range(base) if rows_idx[k].size >= 2 and np.isfinite(rhi[k])]
        if cand:
            k = cand[int(rng.integers(0, len(cand)))]
            rows_idx.append(rows_idx[k].copy())
            rows_val.append(rows_val[k].copy())
            rlo.append(rhi[k] + 10.0)
            rhi.append(rhi[k] + 20.0)
    order = rng.permutation(len(rows_idx))
    rows_idx = [rows_idx[k] for k in order]
    rows_val = [rows_val[k] for k in order]
    rlo = np.asarray(rlo)[order]
    rhi = np.asarray(rhi)[order]
    rs = np.zeros(len(rows_idx) + 1, np.int64)
    rs[1:] = np.cumsum([r.size for r in rows_idx])
    ri = np.concatenate(rows_idx) if rows_idx else np.zeros(0, np.int32)
    rv = np.concatenate(rows_val) if rows_val else np.zeros(0)

    nobj = int(rng.integers(n // 2, n + 1))
    oi = rng.choice(n, size=nobj, replace=True).astype(np.int32)
    ov = rng.normal(0, 3, nobj)
    ov[rng.random(nobj) < 0.1] = 0.0
    q1 = q2 = np.zeros(0, np.int32)
    qv = np.zeros(0)
    if quadratic:
        nq = int(rng.integers(3, 2 * n))
        a = rng.integers(0, n, nq).astype(np.int32)
        b = rng.integers(0, n, nq).astype(np.int32)
        diag = rng.random(nq) < 0.3
        b[diag] = a[diag]
        q1, q2 = np.minimum(a, b), np.maximum(a, b)
        qv = rng.normal(0, 1, nq)
        qv[rng.random(nq) < 0.05] = 1e-11
    return PresolveModel(var_lower=lo, var_upper=hi, var_type=vtype, row_lower=rlo,
                         row_upper=rhi, row_start=rs, row_index=ri.astype(np.int32),
                         row_value=rv, objective_index=oi, objective_value=ov,
                         objective_offset=float(rng.normal()), quadratic_index1=q1,
                         quadratic_index2=q2, quadratic_value=qv)


def flavours(count: int):
    """`count` models across the flavours, seeded by their position."""
    out = []
    for s in range(count):
        f = s % 6
        out.append(random_model(
            1000 + s, n=int(20 + (s * 7) % 90), m=int(10 + (s * 13) % 80),
            integers=f in (1, 4), quadratic=f in (2, 4), contradiction=f == 3,
            copies=0.5 if f == 5 else 0.25, max_row=3 if f == 5 else 6))
    return out


def long_row_model(seed: int) -> PresolveModel:
    """Rows of 64 to 400 terms (and some short ones) over a few hundred to
    2000 variables: equality, one-sided, ranged and loose rows around a point
    inside the bounds, some with quarter-step coefficients, and on even seeds
    budget rows over variables bounded at 0 whose right-hand sides are small
    enough that most of their terms tighten a bound; integer variables on
    every third seed."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(300, 2000))
    m = int(rng.integers(20, 120))
    lo = np.where(rng.random(n) < 0.8, 0.0, rng.uniform(-5, 0, n))
    hi = np.where(rng.random(n) < 0.9, rng.uniform(1, 20, n), INF)
    lo[rng.random(n) < 0.03] = -INF
    vt = np.zeros(n, np.int8)
    if seed % 3 == 1:
        ints = rng.random(n) < 0.3
        vt[ints] = INTEGER
        lo[ints & np.isfinite(lo)] = np.floor(lo[ints & np.isfinite(lo)])
        hi[ints & np.isfinite(hi)] = np.ceil(hi[ints & np.isfinite(hi)])
    box = np.isfinite(hi) & np.isfinite(lo)
    x0 = np.where(np.isfinite(lo), lo, 0.0) + rng.random(n) * np.where(box, hi - lo, 1.0)
    x0 = np.where(vt == INTEGER, np.clip(np.round(x0), lo, hi), x0)
    rows_idx, rows_val, rlo, rhi = [], [], [], []
    for _ in range(m):
        length = int(rng.choice([64, 65, 100, 200, 400, 8, 3]))
        kind = int(rng.integers(0, 5)) if seed % 2 == 0 else int(rng.choice([0, 1, 2, 4]))
        pool = np.flatnonzero((lo == 0) & np.isfinite(hi)) if kind == 3 else np.arange(n)
        idx = rng.choice(pool, size=min(length, pool.size), replace=False)
        val = rng.normal(0, 1, idx.size) if kind != 3 else np.abs(rng.normal(1, 0.2, idx.size))
        if rng.random() < 0.3:
            val = np.round(val * 4) / 4
            val[val == 0] = 0.5
        act = float(val @ x0[idx])
        if kind == 0:
            b = (act, act)
        elif kind == 1:
            b = (-INF, act + rng.uniform(0, 2))
        elif kind == 2:
            b = (act - rng.uniform(0, 2), INF)
        elif kind == 3:
            b = (-INF, rng.uniform(1, 15)) if rng.random() < 0.7 else \
                (float(np.sum(np.abs(val) * hi[idx])) - rng.uniform(0, 5), INF)
        else:
            b = (act - 100.0, act + 100.0)
        rows_idx.append(idx.astype(np.int32))
        rows_val.append(val)
        rlo.append(b[0])
        rhi.append(b[1])
    rs = np.zeros(m + 1, np.int64)
    rs[1:] = np.cumsum([r.size for r in rows_idx])
    return PresolveModel(var_lower=lo, var_upper=hi, var_type=vt, row_lower=np.array(rlo),
                         row_upper=np.array(rhi), row_start=rs,
                         row_index=np.concatenate(rows_idx), row_value=np.concatenate(rows_val),
                         objective_index=np.arange(n, dtype=np.int32),
                         objective_value=rng.normal(0, 1, n))


def _model(vl, vu, rl, ru, rows, obj=(), vt=None, q=()) -> PresolveModel:
    rs = np.zeros(len(rows) + 1, np.int64)
    rs[1:] = np.cumsum([len(r) for r in rows])
    return PresolveModel(
        var_lower=np.array(vl, float), var_upper=np.array(vu, float),
        row_lower=np.array(rl, float), row_upper=np.array(ru, float), row_start=rs,
        row_index=np.array([i for r in rows for i, _ in r], np.int32),
        row_value=np.array([v for r in rows for _, v in r], float),
        objective_index=np.array([i for i, _ in obj], np.int32),
        objective_value=np.array([v for _, v in obj], float),
        var_type=None if vt is None else np.array(vt, np.int8),
        quadratic_index1=np.array([a for a, _, _ in q], np.int32),
        quadratic_index2=np.array([b for _, b, _ in q], np.int32),
        quadratic_value=np.array([c for _, _, c in q], float))


def edge_models() -> dict:
    """Small models at the edges of the reference's presolve: nothing at all,
    no rows, no variables (with a satisfied and an unsatisfiable empty row),
    every variable fixed, a variable fixed at +inf, fixing with quadratic
    terms, integer and binary variables with fractional bounds, a NaN bound,
    coefficients near the top of the double range, a row of zeros, and
    scaled, negated and parallel copies of a row."""
    inf = INF
    return {
        "empty model": _model([], [], [], [], []),
        "no rows": _model([0, -inf], [1, inf], [], [], [], obj=[(0, 1.0), (1, -2.0)]),
        "no variables, empty rows": _model([], [], [-1, 0], [1, 0], [[], []]),
        "no variables, unsatisfiable empty row": _model([], [], [1], [2], [[]]),
        "all fixed": _model([1, 2, 3], [1, 2, 3], [0, -inf], [10, 5],
                            [[(0, 1), (1, 1)], [(1, 1), (2, 1)]], obj=[(0, 1), (2, 4)]),
        "fixed at +inf": _model([inf, 0], [inf, 1], [-inf], [5], [[(0, 1), (1, 1)]]),
        "fixed with quadratic terms": _model(
            [2, 0, -1], [2, 5, 3], [-inf], [4], [[(0, 1), (1, 2), (2, 1)]], obj=[(1, 1)],
            q=[(0, 0, 1.5), (0, 1, 2.0), (1, 2, -1.0), (0, 2, 3.0)]),
        "integer with fractional bounds": _model([0.5, 0], [2.5, 1], [1.2], [inf],
                                                 [[(0, 1), (1, 1)]], vt=[INTEGER, BINARY]),
        "binary singletons": _model([0, 0], [1, 1], [0.3, -inf], [inf, 0.7],
                                    [[(0, 1)], [(1, 2)]], vt=[BINARY, BINARY]),
        "NaN bound": _model([0, np.nan], [1, 1], [-inf], [1], [[(0, 1), (1, 1)]]),
        "huge coefficients": _model([0, 0], [1e300, 1e300], [-inf], [1e308],
                                    [[(0, 1e300), (1, 1e300)]]),
        "row of zeros": _model([0, 0], [1, 1], [-1], [1], [[(0, 0.0), (1, 1e-12)]]),
        "parallel, scaled, negated": _model(
            [0, 0], [5, 5], [1, -3, -inf], [2, -1, inf],
            [[(0, 1), (1, 2)], [(1, -4), (0, -2)], [(0, 3), (1, 6)]]),
    }


def threshold_model(seed: int, rows: int = 40, width: int = 24) -> PresolveModel:
    """Rows whose first term's candidate bound lands on the reference's
    decision threshold (its bound plus or minus 1e-9) to within a few units
    in the last place: x_t + sum a_k y_k >= lo with y_k in [0, u_k], the
    other activity summed in the reference's order, and x_t's bound placed
    at candidate - 1e-9 shifted by -3..3 ulps. Rows share no variables, so
    each row's outcome is decided on these values alone."""
    rng = np.random.default_rng(seed)
    n = rows * (width + 1)
    lo = np.zeros(n)
    hi = rng.uniform(0.5, 50.0, n)
    rlo, rhi, idx_all, val_all = [], [], [], []
    for r in range(rows):
        base = r * (width + 1)
        t = base
        others = np.arange(base + 1, base + width + 1)
        a = rng.choice([-1.0, 1.0]) * rng.uniform(0.5, 3.0)
        c = rng.uniform(0.1, 5.0, width) * rng.choice([-1.0, 1.0], width)
        lower_side = rng.random() < 0.5
        bound = float(rng.uniform(-100, 100))
        # the other terms' extreme activity, summed in row order as the reference does
        acc = 0.0
        for k in range(width):
            if lower_side:   # row >= bound: the others at their largest
                acc += c[k] * (hi[others[k]] if c[k] > 0 else lo[others[k]])
            else:            # row <= bound: the others at their smallest
                acc += c[k] * (lo[others[k]] if c[k] > 0 else hi[others[k]])
        cand = (bound - acc) / a
        shift = int(rng.integers(-3, 4))
        moves_lower = (a > 0) == lower_side
        if moves_lower:      # the test is cand > lower + 1e-9
            lo[t] = np.nextafter(cand - 1e-9, np.inf * np.sign(shift)) if shift else cand - 1e-9
            for _ in range(abs(shift) - 1):
                lo[t] = np.nextafter(lo[t], np.inf * np.sign(shift))
            hi[t] = lo[t] + 100.0
        else:                # the test is cand < upper - 1e-9
            hi[t] = np.nextafter(cand + 1e-9, np.inf * np.sign(shift)) if shift else cand + 1e-9
            for _ in range(abs(shift) - 1):
                hi[t] = np.nextafter(hi[t], np.inf * np.sign(shift))
            lo[t] = hi[t] - 100.0
        idx_all.append(np.concatenate([[t], others]).astype(np.int32))
        val_all.append(np.concatenate([[a], c]))
        rlo.append(bound if lower_side else -INF)
        rhi.append(INF if lower_side else bound)
    rs = np.zeros(rows + 1, np.int64)
    rs[1:] = np.cumsum([i.size for i in idx_all])
    return PresolveModel(var_lower=lo, var_upper=hi, row_lower=np.array(rlo),
                         row_upper=np.array(rhi), row_start=rs,
                         row_index=np.concatenate(idx_all), row_value=np.concatenate(val_all),
                         objective_index=np.arange(n, dtype=np.int32),
                         objective_value=np.ones(n))
