#!/usr/bin/env python
"""Headline benchmark: LPs solved per second at 1e-4 relative KKT on the
min-cost network-flow family (2000 nodes, 20,000 arcs, one shared incidence
matrix; per instance random supplies and costs), learned warm start plus
batched mixed-precision PDLP, 256 instances per step through 256 device
slots.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Before the timed region the learned warm start is trained: seeded training
instances of the family are solved by the engine itself (cold start) and the
3-layer BF16 MLP is fitted on their solutions with the library's tensor-core
kernels. One step = 256 fresh instances: their warm starts are predicted on
the device and they are solved to the tolerance. The timed region holds all
K steps -- K x 256 predictions, and one stream of K x 256 instances through
the session's slots (a slot is refilled as soon as its instance ends).
`value` has the step inputs resident in HBM; `e2e` is the same from pinned
host buffers, with the solutions copied back to the host. Under torchrun
every rank solves its own instances (weak scaling, no collective in the
loop); the timed region is bracketed by a barrier and a device synchronize,
and the time is the max over ranks. The reference arm times the reference's
own CPU PDLP (the library oracle/Makefile builds from the reference sources)
on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "LPs solved/s at 1e-4 rel. KKT (min-cost flow family, learned warm start + batched)"
FALLBACK_HBM_GBS = 6650.0
PROFILE_SUMMARY = os.path.join(ROOT, "profiles", "il_trial_kernels_flow_batch256.md")


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--batch", type=int, default=256, help="instances per step")
    p.add_argument("--slots", type=int, default=256, help="device slots of the session")
    p.add_argument("--tol", type=float, default=1e-4)
    p.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    p.add_argument("--cold", action="store_true", help="no learned warm start in the timed path")
    p.add_argument("--train", type=int, default=20000, help="training instances of the warm start")
    p.add_argument("--train-tol", type=float, default=1e-4, help="tolerance of the training labels")
    p.add_argument("--train-precision", choices=["mixed", "fp64"], default="mixed")
    p.add_argument("--epochs", type=int, default=30)
    p.add_argument("--cpu-sample", type=int, default=32, help="instances in the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extras", action="store_true",
                   help="skip the cold-start, plain-GPU and large-LP side measurements")
    p.add_argument("--profile", action="store_true",
                   help="a short cold stream only (for ncu captures of the trial kernels)")
    p.add_argument("--workload", choices=["flow", "large", "stress", "uneven", "presolve"],
                   default="flow",
                   help="flow: the headline (config 4); large, stress, uneven: configs 1, 3 and 2, "
                        "each reported on its own line")
    p.add_argument("--count", type=int, default=1024, help="uneven: instances in the batch")
    return p.parse_args()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", FALLBACK_HBM_GBS)), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, or None."""
    if not os.path.exists(PROFILE_SUMMARY):
        return None
    for line in open(PROFILE_SUMMARY):
        if line.startswith(f"traffic_bytes_per_launch[{kernel}]:"):
            return float(line.split(":", 1)[1].strip())
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, smax, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = max(smax, float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def workload(batch: int, steps: int, rank: int, graph):
    """Per-step (supply, cost) of fresh instances, seeded per rank and step
    (disjoint across ranks and from the training seeds)."""
    from optimisation_solver_b200 import generators as g
    from optimisation_solver_b200.sharding import rank_seeds
    return [g.flow_parameters(graph, batch, seed=sd) for sd in rank_seeds(rank, steps)]


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_solve_sequential(lib_kind: str, graph, supply, cost, tol: float, threads: int):
    """The instances one after another, each solve with `threads` solver
    threads (the reference parallelises one LP above 20,000 nonzeros). Returns
    (seconds, statuses)."""
    from oracle.oracle import Oracle
    from optimisation_solver_b200 import generators as g
    orc = Oracle(lib_kind)
    opts = dict(thread_count=threads, primal_tolerance=tol, dual_tolerance=tol, gap_tolerance=tol)
    lps = [g.flow_lp(graph, supply[i], cost[i]) for i in range(supply.shape[0])]
    t0 = time.perf_counter()
    res = [orc.solve(lp, opts) for lp in lps]
    return time.perf_counter() - t0, [r.status for r in res]


def cpu_solve_sample(lib_kind: str, graph, supply, cost, tol: float, threads: int):
    """Solves each (supply, cost) instance with the CPU library, instance
    parallel over `threads` host threads (one solver thread each). Returns
    (seconds, statuses, objectives)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle.oracle import Oracle
    from optimisation_solver_b200 import generators as g
    orc = Oracle(lib_kind)
    opts = dict(thread_count=1, primal_tolerance=tol, dual_tolerance=tol, gap_tolerance=tol)
    lps = [g.flow_lp(graph, supply[i], cost[i]) for i in range(supply.shape[0])]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        res = list(ex.map(lambda lp: orc.solve(lp, opts), lps))
    return time.perf_counter() - t0, [r.status for r in res], [r.primal_objective for r in res]


def trial_bytes(n, m, nnz, slots, s, family_bounds_x=True):
    """Algorithmic bytes of one launch of each interleaved trial kernel in the
    loop (every slot active, average update owed): per instance the line's
    own vectors once and the gathered vector once; once per launch the
    matrix (value, index, line pointer) and the broadcast vectors."""
    primal = (slots * n * s * 5            # x read, c read, average read+write, x' written
              + n * s * (2 + (2 if family_bounds_x else 0))   # tau, 1/tau, family bounds
              + nnz * (s + 4) + (n + 1) * 8 + slots * m * s)  # matrix, y gathered
    dual = (slots * m * s * 8              # Ax, y, row bounds (2), y', Ax', average read+write
            + m * s * 2 + nnz * (s + 4) + (m + 1) * 8 + slots * n * s)  # sigma, 1/sigma, matrix, x'
    return primal, dual


def launch_ranks(args) -> int:
    """`--gpus N` outside torchrun: start N ranks on this node with the same
    arguments (one process per GPU, rendezvous on 127.0.0.1) and return the
    launcher's exit status. Rank 0 prints the JSON line."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={args.gpus}", "--master-addr=127.0.0.1", f"--master-port={port}",
           os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.run(cmd).returncode


def main():
    args = parse_args()
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        sys.exit(launch_ranks(args))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world != args.gpus:
        raise SystemExit(f"--gpus {args.gpus} but WORLD_SIZE={world}: launch one rank per GPU")
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    assert args.warmup >= 3, "at least 3 warm-up steps"

    from optimisation_solver_b200 import generators as g
    graph = g.flow_graph()
    config = {"workload": "min-cost flow family: 2000 nodes, 20000 arcs, 40000 nnz; "
                          f"{args.batch} instances per step through {args.slots} device slots; "
                          f"tolerance {args.tol:g} relative KKT",
              "batch": args.batch, "slots": args.slots, "nodes": graph.nodes, "arcs": graph.arcs,
              "tolerance": args.tol, "warm_start": "cold" if args.cold else "learned",
              "l2": "working set > L2 (126 MB): 256 x 20000 x 4 B per vector, six vectors per trial"}

    if args.impl == "reference":
        return reference_arm(args, world, rank, graph, config)
    if args.workload == "presolve":
        # Host code: rank 0 measures it.
        if rank == 0:
            print(json.dumps(presolve_workload()))
        return
    if args.workload in ("large", "stress"):
        # One LP: replicas only, so rank 0 measures it.
        if rank == 0:
            print(json.dumps(side_workload(args, 0, 1, 0)))
        return
    if args.workload == "uneven":
        # Instances split across ranks, balanced by nonzeros.
        import torch.distributed as dist
        if world > 1:
            dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
        line = side_workload(args, rank, world, local_rank)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps(line))
        return

    import torch
    import torch.distributed as dist
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)

    from optimisation_solver_b200.lp import PdlpOptions
    from optimisation_solver_b200.session import Session

    family = g.flow_lp(graph, *[a[0] for a in g.flow_parameters(graph, 1, seed=7)])
    options = PdlpOptions().with_tolerance(args.tol)
    session = Session(family, args.slots, options, precision=args.precision, device=local_rank)
    n, m, nnz = graph.arcs, graph.nodes, family.nnz
    K, W, B = args.steps, args.warmup, args.batch
    steps_in = workload(B, W + K, rank, graph)
    sup_all = torch.from_numpy(np.concatenate([s for s, _ in steps_in])).to(dev)
    cost_all = torch.from_numpy(np.concatenate([c for _, c in steps_in])).to(dev)
    torch.cuda.synchronize()

    if args.profile:
        out = session.stream(B, objective=cost_all[:B].data_ptr(), row_lower=sup_all[:B].data_ptr(),
                             row_upper=sup_all[:B].data_ptr(), on_device=True)
        print(json.dumps({"profile": session.loop_timing(), "optimal": out["optimal"]}, default=float))
        session.close()
        return

    model, train_info = None, None
    if not args.cold:
        from optimisation_solver_b200.learned import train_flow_model
        model, train_info = train_flow_model(graph, args.train, tol=args.train_tol,
                                             precision=args.train_precision, device=local_rank,
                                             epochs=args.epochs)

    px = torch.empty((K * B, n), dtype=torch.float64, device=dev)
    py = torch.empty((K * B, m), dtype=torch.float64, device=dev)

    def predict(sup, cost):
        """Warm starts for the rows of sup/cost, 256 per network pass."""
        if model is None:
            return None, None, None, 0
        count = sup.shape[0]
        wx = torch.empty((count, n), dtype=torch.float64, device=dev)
        wy = torch.empty((count, m), dtype=torch.float64, device=dev)
        ww = torch.empty((count,), dtype=torch.float64, device=dev)
        launches = 0
        for b0 in range(0, count, model.batch):
            b1 = b0 + model.batch
            x, y, w = model.predict(sup[b0:b1], cost[b0:b1])
            wx[b0:b1], wy[b0:b1], ww[b0:b1] = x, y, w
            launches += 2 + model.mlp.launches()
        return wx, wy, ww, launches

    def solve(sup, cost, outx=None, outy=None, warm=True, sess=None):
        sess = session if sess is None else sess
        wx, wy, ww, launches = predict(sup, cost) if warm else (None, None, None, 0)
        ptr = lambda t: None if t is None else t.data_ptr()
        res = sess.stream(sup.shape[0], objective=ptr(cost), row_lower=ptr(sup), row_upper=ptr(sup),
                             warm_primal=ptr(wx), warm_dual=ptr(wy), warm_weight=ptr(ww),
                             primal=ptr(outx), dual=ptr(outy), on_device=True)
        return res, launches + sess.last_timing()[1]

    # Warm-up: the first W steps, each solved on its own.
    for k in range(W):
        solve(sup_all[k * B:(k + 1) * B], cost_all[k * B:(k + 1) * B])

    timed = slice(W * B, (W + K) * B)
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        start.record()
        res, launches = solve(sup_all[timed], cost_all[timed], px, py)
        end.record()
        torch.cuda.synchronize()
    loop = session.loop_timing()
    if world > 1:
        dist.barrier()
    from optimisation_solver_b200.sharding import max_over_ranks
    elapsed_max = max_over_ranks(start.elapsed_time(end) / 1e3, dev)
    value = world * K * B / elapsed_max
    optimal = res["optimal"]
    iters = res["iterations"]

    # End to end: pinned host inputs copied in, warm starts predicted, the
    # stream solved, the solutions copied back to pinned host memory.
    sup_h = torch.from_numpy(np.concatenate([s for s, _ in steps_in[W:]])).pin_memory()
    cost_h = torch.from_numpy(np.concatenate([c for _, c in steps_in[W:]])).pin_memory()
    out_xh = torch.empty((K * B, n), dtype=torch.float64).pin_memory()
    out_yh = torch.empty((K * B, m), dtype=torch.float64).pin_memory()
    h2d = sup_h.numel() * 8 + cost_h.numel() * 8
    d2h = out_xh.numel() * 8 + out_yh.numel() * 8
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    sup_d = sup_h.to(dev, non_blocking=True)
    cost_d = cost_h.to(dev, non_blocking=True)
    res_e2e, _ = solve(sup_d, cost_d, px, py)
    out_xh.copy_(px, non_blocking=True)
    out_yh.copy_(py, non_blocking=True)
    e1.record()
    torch.cuda.synchronize()
    e2e_value = world * K * B / max_over_ranks(e0.elapsed_time(e1) / 1e3, dev)

    # Roofline of the dominant trial kernel, live durations from the events
    # captured in the timed loop.
    s_bytes = 4 if args.precision == "mixed" else 8
    pb, db = trial_bytes(n, m, nnz, args.slots, s_bytes)
    kernel = "k_il_primal" if loop["primal_ms"] >= loop["dual_ms"] else "k_il_dual"
    ms = loop["primal_ms"] if kernel == "k_il_primal" else loop["dual_ms"]
    nbytes = pb if kernel == "k_il_primal" else db
    other = "k_il_dual" if kernel == "k_il_primal" else "k_il_primal"
    oms = loop["dual_ms"] if kernel == "k_il_primal" else loop["primal_ms"]
    obytes = db if kernel == "k_il_primal" else pb
    peak, peak_kind = peaks()
    achieved = nbytes / (ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": kernel, "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "frac_of_nominal_8000": round(achieved / 8000.0, 4),
                "traffic": ncu_traffic(kernel), "algorithmic_bytes_per_launch": nbytes,
                "launch_ms": round(ms, 5), "launch_samples": loop["samples"],
                "other_kernel": {"name": other, "launch_ms": round(oms, 5),
                                 "gbs": round(obytes / (oms * 1e-3) / 1e9, 1)},
                "chunk_ms": round(loop["chunk_ms"], 3), "check_stage_ms": round(loop["check_ms"], 3)}

    line = {"metric": METRIC, "value": round(value, 2), "unit": "LPs/s", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": round(1e3 * elapsed_max / K, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if args.precision == "mixed" else "f64",
            "data": "synthetic (seeded generators); random-init network trained in the run",
            "config": config, "optimal_fraction": optimal / (K * B),
            "mean_iterations": float(iters.mean()), "max_iterations": int(iters.max()),
            "max_relative_kkt": float(np.max(np.maximum(np.maximum(res["primal_residual"], res["dual_residual"]),
                                                         res["relative_gap"]))),
            "clocks": clocks.summary(), "gpu_launches": int(launches),
            "e2e": {"value": round(e2e_value, 2), "unit": "LPs/s", "h2d_bytes_per_step": h2d // K,
                    "d2h_bytes_per_step": d2h // K, "optimal_fraction": res_e2e["optimal"] / (K * B)},
            "roofline": roofline}
    if train_info is not None:
        line["training"] = train_info

    if rank == 0 and not args.no_extras:
        line["extras"] = extras(args, session, graph, sup_all[timed], cost_all[timed], steps_in[-1],
                                value, iters, solve, family, options, local_rank)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, graph, steps_in[-1], res)
    session.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def _kernel_roofline(tk):
    peak, kind = peaks()
    out = {}
    for name, ms, nbytes in (("primal", tk["primal_ms"], tk["primal_bytes"]),
                             ("dual", tk["dual_ms"], tk["dual_bytes"])):
        gbs = nbytes / (ms * 1e-3) / 1e9
        out[name] = {"launch_us": round(ms * 1e3, 1), "algorithmic_bytes": nbytes,
                     "gbs": round(gbs, 1), "frac": round(gbs / peak, 4)}
    out["peak_gbs"] = peak
    out["peak_source"] = kind
    return out


def _planted_instance(args):
    from optimisation_solver_b200 import generators as g
    i, m = args
    rng = np.random.default_rng(40_000 + i)
    deg = rng.integers(4, 13, size=2 * int(m))
    return g.planted_lp(int(m), 2 * int(m), seed=i, degrees=deg)


def presolve_workload() -> dict:
    """The presolve that solver::solve runs before any engine
    (src/solver/orchestrator.cpp:596-597): seconds per presolve of planted
    LPs, the library's (Presolver.run through pdlpgpu_presolve, marshalling
    included) beside the reference's presolve::Presolver::run (compiled from
    its sources, oracle/_ref/libpresolve_cmp.so) where the reference finishes
    in about a minute; the two results are compared field by field on those
    sizes. Configurations 3 and 1 are timed for the library alone."""
    from optimisation_solver_b200 import generators as g
    from optimisation_solver_b200.presolve import PresolveModel, Presolver
    from oracle import presolve_cmp
    P = Presolver()
    rows = []
    cases = [("planted", 1000, 2000), ("planted", 2000, 4000), ("planted", 4000, 8000),
             ("stress (config 3)", 100_000, 200_000), ("large (config 1)", 500_000, 1_000_000)]
    cmp = presolve_cmp.PresolveCompare() if presolve_cmp.available() else None
    P.run(PresolveModel.from_lp(g.planted_lp(m=200, n=400, seed=1).lp))  # first load untimed
    for kind, m, n in cases:
        if kind == "planted":
            lp = g.planted_lp(m=m, n=n, seed=0).lp
        else:
            lp = (g.stress_lp(0) if m == 100_000 else g.large_lp(0)).lp
        model = PresolveModel.from_lp(lp)
        t0 = time.perf_counter()
        r = P.run(model)
        fast = time.perf_counter() - t0
        row = {"model": kind, "rows": m, "cols": n, "nnz": int(lp.nnz), "fast_s": round(fast, 4),
               "presolved_rows": r.presolved_constraints, "presolved_cols": r.presolved_variables,
               "transformations": int(r.transformations["type"].size),
               "infeasible": r.infeasible, "converged": r.converged}
        if cmp is not None and kind == "planted":
            ref_s, _ = cmp.time(model, "reference")
            rc, diff, _ = cmp.compare(model)
            row.update(reference_s=round(ref_s, 3), speedup=round(ref_s / fast, 1),
                       identical=rc == 0)
        rows.append(row)
    return {"workload": "presolve", "metric": "seconds per presolve (presolve::Presolver::run)",
            "unit": "s", "higher_is_better": False, "data": "synthetic (seeded generators)",
            "cpu": cpu_model(), "host_threads": os.cpu_count(),
            "reference": "built from its sources" if cmp is not None else "unavailable",
            "cases": rows}


def side_workload(args, rank: int, world: int, local_rank: int):
    """Configs 1-3, one JSON line each: solve time, PDHG iterations/s, the
    trial kernels' algorithmic GB/s (CUDA events, every instance active) and
    each result's objective error against the planted FP64 optimum. Config 2
    splits its instances across the ranks (nonzero-balanced, strong
    scaling)."""
    import torch
    from optimisation_solver_b200 import generators as g
    from optimisation_solver_b200.lp import PdlpOptions
    from optimisation_solver_b200.pdlp import PdlpSolver
    from optimisation_solver_b200.sharding import balanced_shards, max_over_ranks, sum_over_ranks
    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    opts = PdlpOptions().with_tolerance(args.tol)
    line = {"workload": args.workload, "tolerance": args.tol, "data": "synthetic (seeded generators)"}
    if args.profile:
        return side_profile(args, opts, line)
    if args.workload in ("large", "stress"):
        p = g.large_lp(0) if args.workload == "large" else g.stress_lp(0)
        line["config"] = {"rows": p.lp.num_rows, "cols": p.lp.num_cols, "nnz": int(p.lp.nnz)}
        line["metric"] = "PDHG iterations/s, trial-kernel GB/s, objective error vs planted optimum"
        from optimisation_solver_b200.autotune import tune
        for prec in ("fp64", "mixed"):
            tuned = tune([p.lp], opts, precision=prec, reps=5)
            solver = PdlpSolver(prec, **tuned["params"])
            tk = solver.time_kernels_batch([p.lp], opts, reps=20)
            r = solver.solve(p.lp, opts)
            line[prec] = {"status": str(r.status), "iterations": r.iterations,
                          "precision": r.precision, "fp64_iterations": r.fp64_iterations,
                          "device_seconds": round(r.device_seconds, 3),
                          "iterations_per_s": round(r.iterations / max(r.device_seconds, 1e-9), 1),
                          "objective_rel_error": abs(r.primal_objective - p.objective) / (1 + abs(p.objective)),
                          "primal_residual": r.primal_residual, "dual_residual": r.dual_residual,
                          "relative_gap": r.relative_gap, "kernels": _kernel_roofline(tk),
                          "tuned": {"params": tuned["params"], "trial_ms": round(tuned["trial_ms"], 4),
                                    "default_trial_ms": round(tuned["default_trial_ms"], 4)}}
        return line
    # uneven: config 2, `count` LPs of uneven sizes in one batched solve
    import multiprocessing as mp
    from concurrent.futures import ProcessPoolExecutor
    sizes = g.uneven_batch_sizes(args.count)
    mine = balanced_shards(sizes * 16, world)[rank]   # about 16 nonzeros per row
    t0 = time.perf_counter()
    with ProcessPoolExecutor(max_workers=min(16, os.cpu_count() or 1),
                             mp_context=mp.get_context("spawn")) as ex:
        lps = list(ex.map(_planted_instance, [(int(i), sizes[i]) for i in mine], chunksize=8))
    gen = time.perf_counter() - t0
    nnz = int(sum_over_ranks(sum(q.lp.nnz for q in lps), dev))
    line["config"] = {"instances": args.count, "sum_rows": int(sizes.sum()), "sum_cols": int(2 * sizes.sum()),
                      "nnz": nnz, "generation_seconds": round(gen, 1), "n_gpus": world,
                      "scaling": "strong" if world > 1 else None}
    line["metric"] = "LPs solved/s at 1e-4 rel. KKT, one batched solve (config 2)"
    from optimisation_solver_b200.autotune import tune
    tuned = tune([q.lp for q in lps], opts, precision=args.precision, reps=3,
                 grid={"lane_elements": (8, 32), "vector_width": (1, 4), "cta_slots": (0,)})
    solver = PdlpSolver(args.precision, **tuned["params"])
    tk = solver.time_kernels_batch([q.lp for q in lps], opts, reps=10)
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    t0 = time.perf_counter()
    res = solver.solve_batch([q.lp for q in lps], opts)
    wall = max_over_ranks(time.perf_counter() - t0, dev)
    its = np.array([r.iterations for r in res])
    err = np.array([abs(r.primal_objective - q.objective) / (1 + abs(q.objective)) for r, q in zip(res, lps)])
    ok = np.array([r.status == 0 for r in res])
    line.update({"value": round(args.count / wall, 2), "unit": "LPs/s", "wall_seconds": round(wall, 2),
                 "device_seconds": round(max_over_ranks(max(r.device_seconds for r in res), dev), 2),
                 "optimal_fraction": sum_over_ranks(float(ok.sum()), dev) / args.count,
                 "mean_iterations": float(its.mean()),
                 "max_iterations": int(its.max()),
                 "objective_rel_error_max": float(err[ok].max()) if ok.any() else None,
                 "kernels": _kernel_roofline(tk), "precision": args.precision,
                 "tuned": {"params": tuned["params"], "trial_ms": round(tuned["trial_ms"], 4),
                           "default_trial_ms": round(tuned["default_trial_ms"], 4)}})
    return line


def side_profile(args, opts, line):
    """`--profile` with a side workload: the two SELL-G trial kernels only,
    timed with every instance active (no solve), for ncu captures. large /
    stress: the one LP in FP64 then FP32, V = 1 / 4; uneven: `--count` LPs of
    the uneven family as one batch in `--precision`, V = 4, 32 entries per
    lane."""
    from optimisation_solver_b200 import generators as g
    from optimisation_solver_b200.pdlp import PdlpSolver
    out = {}
    if args.workload in ("large", "stress"):
        p = g.large_lp(0) if args.workload == "large" else g.stress_lp(0)
        line["config"] = {"rows": p.lp.num_rows, "cols": p.lp.num_cols, "nnz": int(p.lp.nnz)}
        for prec, width in (("fp64", 1), ("mixed", 4)):
            tk = PdlpSolver(prec, vector_width=width).time_kernels_batch([p.lp], opts, reps=20)
            out[prec] = dict(_kernel_roofline(tk), padding={"at": tk["at_padding"], "a": tk["a_padding"]})
    else:
        sizes = g.uneven_batch_sizes(args.count)
        lps = [_planted_instance((i, sizes[i])).lp for i in range(args.count)]
        line["config"] = {"instances": args.count, "nnz": int(sum(q.nnz for q in lps))}
        tk = PdlpSolver(args.precision, vector_width=4, lane_elements=32).time_kernels_batch(lps, opts, reps=10)
        out[args.precision] = dict(_kernel_roofline(tk), padding={"at": tk["at_padding"], "a": tk["a_padding"]})
    line["profile"] = out
    return line


def extras(args, session, graph, sup, cost, inputs, value, iters, solve, family, options, device):
    """Side measurements: the same instances cold (the learned gain), the same
    instances with FP64 iterations (the share of the speed-up that FP32
    arithmetic brings), plain FP64 one-LP-per-call GPU PDLP (the comparison
    the target is quoted against), and the trial kernels on the single large
    LP."""
    import torch

    from optimisation_solver_b200.session import Session
    out = {}
    if args.precision == "mixed":
        s64 = Session(family, args.slots, options, precision="fp64", device=device)
        solve(sup[: args.batch], cost[: args.batch], warm=not args.cold, sess=s64)   # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r64, _ = solve(sup, cost, warm=not args.cold, sess=s64)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        s64.close()
        out["fp64_batched"] = {"lps_per_s": round(sup.shape[0] / dt, 2),
                               "mean_iterations": float(r64["iterations"].mean()),
                               "optimal_fraction": r64["optimal"] / sup.shape[0],
                               "warm_start": "cold" if args.cold else "learned",
                               "mixed_over_fp64": round(value / (sup.shape[0] / dt), 3)}
    # The same instances with restarts on the normalised duality gap instead
    # of the reference's KKT score (restart_metric=1; the statuses and the
    # tolerance stay the reference's).
    sg = Session(family, args.slots, options, precision=args.precision, device=device, restart_metric=1)
    solve(sup[: args.batch], cost[: args.batch], warm=not args.cold, sess=sg)   # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    rg, _ = solve(sup, cost, warm=not args.cold, sess=sg)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    sg.close()
    out["gap_restarts"] = {"lps_per_s": round(sup.shape[0] / dt, 2),
                           "mean_iterations": float(rg["iterations"].mean()),
                           "optimal_fraction": rg["optimal"] / sup.shape[0],
                           "max_relative_kkt": float(np.max(np.maximum.reduce(
                               [rg["primal_residual"], rg["dual_residual"], rg["relative_gap"]])))}
    if not args.cold:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        cold, _ = solve(sup, cost, warm=False)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        out["cold_batched"] = {"lps_per_s": round(sup.shape[0] / dt, 2),
                               "mean_iterations": float(cold["iterations"].mean()),
                               "max_iterations": int(cold["iterations"].max()),
                               "optimal_fraction": cold["optimal"] / sup.shape[0]}
        out["learned_gain"] = {"lps_ratio": round(value / out["cold_batched"]["lps_per_s"], 3),
                               "iteration_ratio": round(float(iters.mean()) / float(cold["iterations"].mean()), 3)}
    out["gemm"] = gemm_throughput()
    out["plain_gpu_fp64_single"] = plain_gpu(graph, inputs, args.tol)
    out["speedup_vs_plain_gpu_fp64"] = round(value / out["plain_gpu_fp64_single"]["lps_per_s"], 2)
    out["large_lp_trial_kernels"] = large_lp_kernels()
    return out


def gemm_throughput():
    """The network's tensor-core GEMM alone (CUDA events, 20 calls after a
    warm-up): an 8192^3 product and the first layer's forward shape of the
    flow model (256 instances x 512 hidden x 22,000 features, split-K 18),
    in TFLOP/s and as a fraction of the measured dense BF16 peak."""
    import ctypes as C

    import torch
    from optimisation_solver_b200 import native
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak = json.load(open(path)).get("bf16_tflops", 1590.0) if os.path.exists(path) else 1590.0
    out = {"peak_tflops": peak}
    g = torch.Generator(device="cuda").manual_seed(0)
    for name, (M, N, K, splits) in {"square_8192": (8192, 8192, 8192, 1),
                                    "flow_layer1_forward": (256, 512, 22000, 18)}.items():
        a = torch.randn((M, K), device="cuda", generator=g).to(torch.bfloat16)
        b = torch.randn((N, K), device="cuda", generator=g).to(torch.bfloat16)
        c = torch.empty((M, N), device="cuda", dtype=torch.float32)
        ms = C.c_double()
        rc = native.lib().pdlpgpu_gemm_time(M, N, K, C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
                                            C.c_void_p(c.data_ptr()), splits, 20, C.byref(ms))
        if rc != 0:
            out[name] = {"error": native.last_error()}
            continue
        tf = 2.0 * M * N * K / (ms.value * 1e-3) / 1e12
        out[name] = {"us": round(ms.value * 1e3, 2), "tflops": round(tf, 1), "frac": round(tf / peak, 4)}
        del a, b, c
    return out


def plain_gpu(graph, inputs, tol, count=32):
    """Plain FP64 single-instance GPU PDLP on the same instances, one LP per
    call; the device time of the solves and the host time around them are
    reported apart."""
    from optimisation_solver_b200 import generators as g
    from optimisation_solver_b200.lp import PdlpOptions
    from optimisation_solver_b200.pdlp import PdlpSolver
    solver = PdlpSolver("fp64")
    opts = PdlpOptions().with_tolerance(tol)
    supply, cost = inputs
    solver.solve(g.flow_lp(graph, supply[0], cost[0]), opts)
    # The LPs are built before the clock starts: only the solves are timed.
    lps = [g.flow_lp(graph, supply[i], cost[i]) for i in range(1, count + 1)]
    t0 = time.perf_counter()
    iters, device = [], 0.0
    for lp in lps:
        r = solver.solve(lp, opts)
        iters.append(r.iterations)
        device += r.device_seconds
    dt = time.perf_counter() - t0
    return {"lps_per_s": round(count / dt, 3), "instances": count,
            "mean_iterations": float(np.mean(iters)),
            "device_seconds_per_lp": round(device / count, 5),
            "host_seconds_per_lp": round((dt - device) / count, 5),
            "us_per_iteration": round(1e6 * device / max(1, sum(iters)), 2)}


def large_lp_kernels():
    """PDHG trial kernels (fused SpMV + projections) on the single large LP
    (500,000 x 1,000,000, 8.2M nonzeros), FP64 and FP32, timed with CUDA
    events: GB/s of algorithmic bytes."""
    from optimisation_solver_b200 import generators as g
    from optimisation_solver_b200.lp import PdlpOptions
    from optimisation_solver_b200.session import Session
    p = g.large_lp(0)
    out = {}
    for prec in ("fp64", "mixed"):
        S = Session(p.lp, 1, PdlpOptions(), precision=prec)
        S.load()
        tk = S.time_kernels(10)
        S.close()
        out[prec] = {"primal_us": round(tk["primal_ms"] * 1e3, 1), "dual_us": round(tk["dual_ms"] * 1e3, 1),
                     "primal_gbs": round(tk["primal_bytes"] / tk["primal_ms"] / 1e6, 1),
                     "dual_gbs": round(tk["dual_bytes"] / tk["dual_ms"] / 1e6, 1)}
    return out


def cpu_baseline(args, graph, inputs, res):
    """The reference's CPU PDLP (built from its sources) on a bounded sample of
    the same instances, with every host thread; also the objective error of
    the device results for those instances against it."""
    from oracle.oracle import available
    kind = "ref_fast" if available("ref_fast") else "port"
    threads = os.cpu_count() or 1
    supply, cost = inputs
    k = min(args.cpu_sample, supply.shape[0])
    seconds, statuses, objs = cpu_solve_sample(kind, graph, supply[:k], cost[:k], args.tol, threads)
    last = res["primal_objective"][-args.batch:][:k]
    rel = np.abs(last - np.array(objs)) / (1.0 + np.abs(np.array(objs)))
    ks = min(8, k)
    seq_seconds, seq_statuses = cpu_solve_sequential(kind, graph, supply[:ks], cost[:ks], args.tol,
                                                     threads)
    return {"value": round(k / seconds, 3), "unit": "LPs/s", "cores": threads,
            "cpu_model": cpu_model(),
            "kind": "reference" if kind == "ref_fast" else "port",
            "sample": f"{k} instances of the last step, instance-parallel, one solver thread each, "
                      f"{seconds:.1f} s",
            "optimal_fraction": statuses.count("optimal") / k,
            "sequential_all_cores": {"value": round(ks / seq_seconds, 3), "unit": "LPs/s",
                                     "sample": f"{ks} instances one after another, {threads} solver "
                                               f"threads each, {seq_seconds:.1f} s",
                                     "optimal_fraction": seq_statuses.count("optimal") / ks},
            "device_vs_cpu_objective_rel_max": float(rel.max())}


def reference_arm(args, world, rank, graph, config):
    """The reference's own CPU PDLP on the host cores (rank 0 only)."""
    if rank != 0:
        return
    from oracle.oracle import available
    kind = "ref_fast" if available("ref_fast") else "port"
    if not (available("ref_fast") or available("port")):
        print(json.dumps({"impl": "reference", "unavailable": "CPU oracle libraries not built"}))
        return
    threads = os.cpu_count() or 1
    per_step = max(threads, 16)
    inputs = workload(per_step, args.warmup + args.steps, 0, graph)
    for k in range(args.warmup):
        cpu_solve_sample(kind, graph, inputs[k][0], inputs[k][1], args.tol, threads)
    total = 0.0
    optimal = 0
    for k in range(args.warmup, args.warmup + args.steps):
        seconds, statuses, _ = cpu_solve_sample(kind, graph, inputs[k][0], inputs[k][1], args.tol, threads)
        total += seconds
        optimal += statuses.count("optimal")
    value = per_step * args.steps / total
    line = {"metric": METRIC, "value": round(value, 3), "unit": "LPs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generators)",
            "config": dict(config, batch=per_step, warm_start="cold (the reference has no warm start)"),
            "impl": "reference", "optimal_fraction": optimal / (per_step * args.steps),
            "cpu_baseline": {"value": round(value, 3), "unit": "LPs/s", "cores": threads,
                             "cpu_model": cpu_model(),
                             "kind": "reference" if kind == "ref_fast" else "port",
                             "sample": f"{per_step} instances per step, instance-parallel"},
            "e2e": {"value": round(value, 3), "unit": "LPs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
