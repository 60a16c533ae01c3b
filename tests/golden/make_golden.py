"""Writes tests/golden/reference_solves.npz: outputs of the reference pdlp_engine
(built from its own sources by oracle/Makefile, parity flags) on small seeded
problems, so the oracle restatement and the device engine can be checked
against the reference on a machine where the reference is not present.

    make -C oracle ref && python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Oracle  # noqa: E402
from optimisation_solver_b200 import generators as g  # noqa: E402
from tests import cases  # noqa: E402

OUT = os.path.join(HERE, "reference_solves.npz")


def golden_cases():
    """(name, lp, options dict) of the fixtures."""
    out = []
    for seed in (0, 1):
        out.append((f"reference_lp_{seed}", g.reference_lp(seed).lp, dict(thread_count=1)))
    out.append(("random_feasible_300x420", cases.random_feasible(300, 420, 21),
                cases.convergence_options().as_dict()))
    out.append(("iteration_limit_polish", cases.random_feasible(300, 420, 21),
                cases.convergence_options(iteration_limit=150, use_feasibility_polishing=True,
                                          polishing_iterations=300).as_dict()))
    out.append(("no_preconditioning", cases.random_feasible(120, 160, 3),
                cases.convergence_options(use_diagonal_preconditioning=False,
                                          iteration_limit=3000).as_dict()))
    out.append(("infeasible_rows", cases.infeasible_rows(), cases.strict_options(iteration_limit=20000).as_dict()))
    out.append(("unbounded_ray", cases.unbounded_ray(), cases.strict_options(iteration_limit=20000).as_dict()))
    out.append(("degenerate", cases.degenerate(), cases.strict_options().as_dict()))
    return out


def main():
    ref = Oracle("ref")
    arrays = {}
    for name, lp, opts in golden_cases():
        r = ref.solve(lp, opts)
        arrays[f"{name}/status"] = np.array(r.status)
        arrays[f"{name}/scalars"] = np.array([r.iterations, r.step_trials, r.restart_count,
                                              r.primal_objective, r.dual_objective,
                                              r.primal_residual, r.dual_residual, r.relative_gap,
                                              r.final_step_size, r.static_step_bound,
                                              r.final_primal_weight])
        arrays[f"{name}/primal"] = r.primal
        arrays[f"{name}/row_dual"] = r.row_dual
        arrays[f"{name}/dual_ray"] = r.dual_ray
        arrays[f"{name}/primal_ray"] = r.primal_ray
    np.savez_compressed(OUT, **arrays)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
