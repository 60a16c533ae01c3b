"""Normalised duality gap in numpy, FP64 (TEST INFRASTRUCTURE ONLY).

The reference has no normalised-gap restart (pdlp_engine/README.md:226-233
names it as its main missing algorithmic item), so this oracle restates the
published definition and method instead: Applegate et al., "Practical
large-scale linear programming using primal-dual hybrid gradient" (NeurIPS
2021), section 3 and appendix. For

    L(x, y) = c'x + y'Ax - h*(y),   x in [l_x, u_x],

h* the support function of the row bounds [l_r, u_r] (the engine's dual sign:
stationarity c + A'y), the gap at radius r of z = (x, y) is

    rho(r; z) = max { L(x, yh) - L(xh, y) : zh feasible, ||zh - z||_w <= r } / r,
    ||(dx, dy)||_w^2 = w ||dx||^2 + ||dy||^2 / w.

The objective separates by coordinate; for a multiplier lam of the ball
constraint each coordinate's maximiser has a closed form, and the distance it
reaches falls with lam. This oracle finds lam by 200 bisection steps on
log(lam), independently of the device's bracketing passes. Only tests import
it, as the checker.
"""
from __future__ import annotations

import numpy as np


def _primal_step(x, g, lo, hi, lam, w):
    with np.errstate(divide="ignore", invalid="ignore"):
        if lam > 0:
            s = -g / (lam * w)
        else:
            s = np.where(g < 0, np.inf, np.where(g > 0, -np.inf, 0.0))
    return np.clip(s, lo - x, hi - x)


def _dual_point(y, a, lo, hi, lam, w):
    hi_f, lo_f = np.isfinite(hi), np.isfinite(lo)
    if lam > 0:
        with np.errstate(invalid="ignore"):
            up = y + (w / lam) * (a - hi)
            dn = y + (w / lam) * (a - lo)
        out = np.zeros_like(y)
        pos = hi_f & (up > 0)
        neg = ~pos & lo_f & (dn < 0)
        out[pos] = up[pos]
        out[neg] = dn[neg]
        return out
    out = np.zeros_like(y)
    out[hi_f & (a - hi > 0)] = np.inf
    out[lo_f & (a - lo < 0) & ~(hi_f & (a - hi > 0))] = -np.inf
    return out


def _support(v, lo, hi):
    out = np.zeros_like(v)
    pos, neg = v > 0, v < 0
    out[pos] = hi[pos] * v[pos]
    out[neg] = lo[neg] * v[neg]
    return out


def _dist2(x, g, xl, xu, y, a, rl, ru, lam, w):
    s = _primal_step(x, g, xl, xu, lam, w)
    e = _dual_point(y, a, rl, ru, lam, w) - y
    return w * float(np.sum(s * s)) + float(np.sum(e * e)) / w


def _objective(x, g, xl, xu, y, a, rl, ru, lam, w):
    s = _primal_step(x, g, xl, xu, lam, w)
    yh = _dual_point(y, a, rl, ru, lam, w)
    prim = -g * s
    prim[s == 0] = 0.0
    return float(np.sum(prim) + np.sum((yh - y) * a - _support(yh, rl, ru) + _support(y, rl, ru)))


def normalized_gap(weight, x, g, xl, xu, xr, y, a, rl, ru, yr):
    """(gap, radius) of z = (x, y) with g = c + A'y, a = A x, radius the
    weighted distance to (xr, yr)."""
    w = float(weight)
    arr = [np.asarray(v, dtype=np.float64) for v in (x, g, xl, xu, xr, y, a, rl, ru, yr)]
    x, g, xl, xu, xr, y, a, rl, ru, yr = arr
    r = np.sqrt(w * np.sum((x - xr) ** 2) + np.sum((y - yr) ** 2) / w)
    if not (r > 0) or not np.isfinite(r):
        return np.inf, float(r)
    # The whole box inside the ball: the box maximum.
    if _dist2(x, g, xl, xu, y, a, rl, ru, 0.0, w) <= r * r:
        return _objective(x, g, xl, xu, y, a, rl, ru, 0.0, w) / r, float(r)
    lo, hi = -60.0, 60.0          # log10(lam)
    while _dist2(x, g, xl, xu, y, a, rl, ru, 10.0 ** hi, w) > r * r:
        hi += 20.0
    while _dist2(x, g, xl, xu, y, a, rl, ru, 10.0 ** lo, w) <= r * r and lo > -300:
        lo -= 20.0
    for _ in range(200):
        mid = 0.5 * (lo + hi)
        if _dist2(x, g, xl, xu, y, a, rl, ru, 10.0 ** mid, w) > r * r:
            lo = mid
        else:
            hi = mid
    return _objective(x, g, xl, xu, y, a, rl, ru, 10.0 ** hi, w) / r, float(r)
