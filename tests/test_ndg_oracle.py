"""The normalised-gap oracle (oracle/ndg_oracle.py) against a generic
constrained optimiser (scipy SLSQP, several starts) on small random states:
the oracle's closed forms and bisection give the maximum of the gap problem."""
import numpy as np
import pytest
from scipy.optimize import minimize

from oracle.ndg_oracle import normalized_gap
from tests.ndg_cases import state


def _support(v, lo, hi):
    with np.errstate(invalid="ignore"):
        return np.where(v > 0, hi * v, np.where(v < 0, lo * v, 0.0))


def _brute(rng, w, x, g, xl, xu, xr, y, a, rl, ru, yr):
    n = x.size
    r = np.sqrt(w * np.sum((x - xr) ** 2) + np.sum((y - yr) ** 2) / w)

    def f(z):
        xh, yh = z[:n], z[n:]
        return -(np.sum(-g * (xh - x)) + np.sum((yh - y) * a - _support(yh, rl, ru) + _support(y, rl, ru)))

    ball = {"type": "ineq",
            "fun": lambda z: r * r - (w * np.sum((z[:n] - x) ** 2) + np.sum((z[n:] - y) ** 2) / w)}
    bnds = [(lo if np.isfinite(lo) else None, hi if np.isfinite(hi) else None) for lo, hi in zip(xl, xu)]
    bnds += [(None if np.isfinite(lo) else 0.0, None if np.isfinite(hi) else 0.0) for lo, hi in zip(rl, ru)]
    lo_b = np.array([b[0] if b[0] is not None else -np.inf for b in bnds])
    hi_b = np.array([b[1] if b[1] is not None else np.inf for b in bnds])
    best = np.inf
    for _ in range(20):
        z0 = np.clip(np.concatenate([x, y]) + rng.normal(0, r / 6, x.size + y.size), lo_b, hi_b)
        res = minimize(f, z0, method="SLSQP", bounds=bnds, constraints=[ball],
                       options={"maxiter": 500, "ftol": 1e-12})
        if res.success and ball["fun"](res.x) > -1e-9:
            best = min(best, res.fun)
    return -best / r


@pytest.mark.parametrize("seed", range(12))
def test_oracle_matches_generic_optimiser(seed):
    rng = np.random.default_rng(1000 + seed)
    case = state(rng, int(rng.integers(1, 5)), int(rng.integers(1, 4)))
    got, _ = normalized_gap(*case)
    want = _brute(rng, *case)
    assert abs(got - want) <= 1e-6 * max(1.0, abs(want)), (got, want)


def test_zero_radius_is_infinite_and_box_inside_ball():
    rng = np.random.default_rng(5)
    w, x, g, xl, xu, xr, y, a, rl, ru, yr = state(rng, 4, 3)
    gap, r = normalized_gap(w, x, g, xl, xu, x, y, a, rl, ru, y)
    assert r == 0.0 and gap == np.inf
    # A bounded box inside a large ball: the gap is the box maximum over r.
    # (|a| < 1 keeps each dual coordinate's maximum at y = 0.)
    xl, xu = x - 0.1, x + 0.1
    rl, ru = np.full(3, -1.0), np.full(3, 1.0)
    y = np.zeros(3)
    a = np.clip(a, -0.9, 0.9)
    gap, r = normalized_gap(w, x, g, xl, xu, x + 100.0, y, a, rl, ru, y)
    box = np.sum(np.abs(g) * 0.1)
    assert abs(gap * r - box) <= 1e-9 * max(1.0, box)
