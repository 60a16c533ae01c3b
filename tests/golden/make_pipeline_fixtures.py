"""Writes tests/golden/pipeline_models.npz: the reference's own LP fixture
files, read by the reference MpsReader (src/mps/mps_reader.cpp), as flat
Model IR arrays, together with

* the expected objectives the reference publishes for them
  (benchmarks/instances/known_answers.json, benchmarks/instances/netlib/best_known.json);
* the reference pipeline's own answers: solver::solve with PDLP forced at
  tolerance 1e-8, and with the dispatcher's choice (the dual simplex on these
  sizes) -- status, objective, primal values, shadow prices, reduced costs.

The fixture travels where the reference tree is absent; the GPU tests rebuild
each model from it and run the same pipeline with the GPU engine behind
solver::runPdlp.

    make -C oracle pipeline && python tests/golden/make_pipeline_fixtures.py

The reference checkout is OPTSOLVER_REFERENCE_ROOT (default /root/reference).
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.pipeline import MODEL_FIELDS, Pipeline  # noqa: E402

REFERENCE = os.environ.get("OPTSOLVER_REFERENCE_ROOT", "/root/reference")
INSTANCES = os.path.join(REFERENCE, "benchmarks", "instances")
OUT = os.path.join(HERE, "pipeline_models.npz")

# The LP files among the reference's known-answer fixtures (the MILP and QP
# ones belong to other engines), and the one Netlib file it ships.
KNOWN = ["opt_lp", "degenerate_lp", "ranged_lp", "max_offset_lp", "free_fixed", "infeasible_lp",
         "unbounded_lp"]
NETLIB = ["afiro"]


def main():
    pipe = Pipeline("ref")
    known = json.load(open(os.path.join(INSTANCES, "known_answers.json")))
    netlib = json.load(open(os.path.join(INSTANCES, "netlib", "best_known.json")))
    out = {}
    names = []
    for name in KNOWN + NETLIB:
        folder = "known" if name in KNOWN else "netlib"
        path = os.path.join(INSTANCES, folder, name + ".mps")
        model = pipe.read_mps(path)
        arrays = model.export()
        for f in MODEL_FIELDS:
            out[f"{name}/{f}"] = np.asarray(arrays[f])
        answers = known if name in KNOWN else netlib
        out[f"{name}/expected_objective"] = np.float64(answers.get(name + ".mps", np.nan))
        for tag, engine in (("pdlp", 0), ("dispatch", None)):
            r = model.solve(engine=engine, tolerance=1e-8, threads=1)
            out[f"{name}/{tag}_status"] = np.array(r.status)
            out[f"{name}/{tag}_objective"] = np.float64(r.objective)
            out[f"{name}/{tag}_x"] = r.x
            out[f"{name}/{tag}_duals"] = r.duals
            out[f"{name}/{tag}_reduced_costs"] = r.reduced_costs
            out[f"{name}/{tag}_engine"] = np.int32(r.executed_engine)
            print(f"{name:16s} {tag:8s} {r.status:14s} {r.objective:.10g} "
                  f"(expected {out[f'{name}/expected_objective']:.10g}) iterations {r.iterations}")
        names.append(name)
    out["names"] = np.array(names)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT)


if __name__ == "__main__":
    main()
