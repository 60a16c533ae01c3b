"""Writes tests/golden/presolve_results.npz: models and the reference
presolve's results for them, so the fast presolve is pinned where the
reference tree is absent.

Models: the first 12 generated presolve models (tests/presolve_cases.py,
every flavour twice) and the reference's own
LP fixture files (tests/golden/pipeline_models.npz: its known-answer LPs and
Netlib afiro, read by its MpsReader). For each, the reference's
presolve::Presolver::run and the library's presolve are run on the same
model::Model by oracle/_ref/libpresolve_cmp.so and must agree field by field,
bit for bit; the result stored is then the reference's (taken through the
library's arrays).

    make -C oracle presolve && python tests/golden/make_presolve_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from optimisation_solver_b200.presolve import PresolveModel, Presolver  # noqa: E402
from oracle.presolve_cmp import PresolveCompare  # noqa: E402
from tests import presolve_cases  # noqa: E402

MODEL_KEYS = ("var_lower", "var_upper", "var_type", "row_lower", "row_upper", "row_start",
              "row_index", "row_value", "objective_index", "objective_value",
              "quadratic_index1", "quadratic_index2", "quadratic_value")


def pipeline_fixture_models():
    data = np.load(os.path.join(HERE, "pipeline_models.npz"))
    out = []
    for name in data["names"]:
        d = {k.split("/", 1)[1]: data[k] for k in data.files if k.startswith(f"{name}/")}
        out.append((f"fixture_{name}", PresolveModel(
            var_lower=d["var_lower"], var_upper=d["var_upper"],
            var_type=d["var_type"].astype(np.int8), row_lower=d["row_lower"],
            row_upper=d["row_upper"], row_start=d["row_start"], row_index=d["row_index"],
            row_value=d["row_value"], objective_index=d["objective_index"],
            objective_value=d["objective_value"], objective_offset=float(d["offset"]))))
    return out


def models():
    out = [(f"generated_{k}", m) for k, m in enumerate(presolve_cases.flavours(12))]
    return out + pipeline_fixture_models()


def flatten(r) -> dict:
    d = {"infeasible": r.infeasible, "converged": r.converged, "has_maps": r.has_maps,
         "counts": np.array([r.original_variables, r.original_constraints,
                             r.presolved_variables, r.presolved_constraints]),
         "offsets": np.array([r.initial_objective_offset, r.presolved_objective_offset]),
         "variable_origin": r.variable_origin, "constraint_origin": r.constraint_origin}
    for k in MODEL_KEYS:
        d[f"reduced_{k}"] = getattr(r.model, k)
    for group in ("transformations", "fixed_variables", "removed_constraints"):
        for k, v in getattr(r, group).items():
            if k != "reason_text":
                d[f"{group}_{k}"] = np.asarray(v)
    return d


def main():
    cmp, P = PresolveCompare(), Presolver()
    arrays = {}
    names = []
    for name, m in models():
        rc, msg, _ = cmp.compare(m)
        assert rc == 0, (name, msg)
        names.append(name)
        for k in MODEL_KEYS:
            arrays[f"{name}/model_{k}"] = np.asarray(getattr(m, k) if getattr(m, k) is not None
                                                     else np.zeros(len(m.var_lower), np.int8))
        arrays[f"{name}/model_objective_offset"] = np.array(m.objective_offset)
        for k, v in flatten(P.run(m)).items():
            arrays[f"{name}/result_{k}"] = np.asarray(v)
    arrays["names"] = np.array(names)
    path = os.path.join(HERE, "presolve_results.npz")
    np.savez_compressed(path, **arrays)
    print(f"wrote {path}: {len(names)} models")


if __name__ == "__main__":
    main()
