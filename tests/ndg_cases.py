"""Random primal-dual states for the normalised-gap tests: variable bounds
finite, one-sided or free, row bounds ranged, one-sided, equality or free,
duals in the dual domain (y_i <= 0 where the upper row bound is infinite,
y_i >= 0 where the lower one is), a random restart point."""
import numpy as np


def state(rng, n, m, radius_scale=0.5):
    xl = rng.uniform(-2, 0, n)
    xu = xl + rng.uniform(0.1, 3, n)
    kind = rng.integers(0, 5, n)
    xl[kind == 1] = -np.inf
    xu[kind == 2] = np.inf
    xl[kind == 3] = -np.inf
    xu[kind == 3] = np.inf
    x = np.clip(rng.normal(size=n), xl, xu)
    rl = rng.uniform(-2, 0, m)
    ru = rl + rng.uniform(0, 3, m)
    kind = rng.integers(0, 5, m)
    rl[kind == 1] = -np.inf
    ru[kind == 2] = np.inf
    ru[kind == 4] = rl[kind == 4]
    y = rng.normal(size=m)
    y = np.where(~np.isfinite(ru), np.minimum(y, 0), y)
    y = np.where(~np.isfinite(rl), np.maximum(y, 0), y)
    g = rng.normal(size=n)
    a = rng.normal(size=m)
    w = float(10 ** rng.uniform(-1, 1))
    xr = x + rng.normal(0, radius_scale, n)
    yr = y + rng.normal(0, radius_scale, m)
    return w, x, g, xl, xu, xr, y, a, rl, ru, yr
