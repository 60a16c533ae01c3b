"""Measured choice of the device layout parameters.

The kernels' speed on a given matrix depends on how rows map to lanes and
warps: entries per lane (`lane_elements`, which sets how many lanes share a
long line), the lane load width (`vector_width`), the slots per CTA
(`cta_slots`), and for sessions the layout itself and the instances per lane.
`tune` times the two PDHG trial kernels (CUDA events, every instance active,
no solve) for each candidate and returns the fastest as keyword arguments for
`PdlpSolver` / `Session`. The termination-check period is not tuned: it
decides when a solve may stop, so it stays the caller's
(`termination_check_frequency`, 100 by default as in the reference).
"""
from __future__ import annotations

import itertools

from .lp import PdlpOptions
from .pdlp import PdlpSolver

# lane_elements x vector_width x cta_slots (0: the heuristic's CTA size)
SELL_GRID = {
    "lane_elements": (8, 16, 32),
    "vector_width": (1, 2, 4),
    "cta_slots": (0,),
}


def tune(problems, options: PdlpOptions | None = None, precision: str = "mixed",
         grid: dict | None = None, reps: int = 5, device: int = 0) -> dict:
    """Fastest SELL-G parameters for a list of LPs solved together (one LP is
    a list of one). Returns {"params": kwargs, "primal_ms", "dual_ms",
    "trial_ms", "default_trial_ms", "tried": [...]}."""
    grid = grid or SELL_GRID
    options = options or PdlpOptions()
    if not isinstance(problems, (list, tuple)):
        problems = [problems]
    base = PdlpSolver(precision, device=device).time_kernels_batch(problems, options, reps=reps)
    default_ms = base["primal_ms"] + base["dual_ms"]
    best = (default_ms, {}, base)
    tried = [({}, default_ms)]
    keys = sorted(grid)
    for values in itertools.product(*(grid[k] for k in keys)):
        params = dict(zip(keys, values))
        if precision == "fp64" and params.get("vector_width") == 4:
            continue   # 4 doubles per lane load exceed one 16-byte access
        tk = PdlpSolver(precision, device=device, **params).time_kernels_batch(problems, options,
                                                                             reps=reps)
        ms = tk["primal_ms"] + tk["dual_ms"]
        tried.append((params, ms))
        if ms < best[0]:
            best = (ms, params, tk)
    ms, params, tk = best
    return {"params": params, "primal_ms": tk["primal_ms"], "dual_ms": tk["dual_ms"],
            "primal_bytes": tk["primal_bytes"], "dual_bytes": tk["dual_bytes"],
            "trial_ms": ms, "default_trial_ms": default_ms, "tried": tried}


def tune_session(family, batch: int, options: PdlpOptions | None = None,
                 precision: str = "mixed", objective=None, row_lower=None, row_upper=None,
                 reps: int = 5, device: int = 0) -> dict:
    """Fastest layout for a session: the interleaved layout at 1, 2 and 4
    instances per lane, and the SELL-G layout. The instance vectors (host
    arrays of `batch` rows, or None for the family's) are loaded so that the
    timed kernels read real data. Returns {"params": kwargs for Session,
    "trial_ms", "tried": [...]}."""
    from .session import Session
    options = options or PdlpOptions()
    cands = [dict(layout="interleaved", lane_instances=v) for v in (1, 2, 4)
             if not (precision == "fp64" and v == 4)]
    cands.append(dict(layout="sell"))
    tried = []
    for params in cands:
        S = Session(family, batch, options, precision=precision, device=device, **params)
        try:
            S.load(objective=objective, row_lower=row_lower, row_upper=row_upper)
            tk = S.time_kernels(reps)
        finally:
            S.close()
        tried.append((params, tk["primal_ms"] + tk["dual_ms"]))
    params, ms = min(tried, key=lambda t: t[1])
    return {"params": params, "trial_ms": ms, "tried": tried}
