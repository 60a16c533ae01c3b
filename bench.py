#!/usr/bin/env python
"""Headline benchmark: LPs solved per second at 1e-4 relative KKT on the
min-cost network-flow family (2000 nodes, 20,000 arcs, one shared incidence
matrix; per instance random supplies and costs), 256 instances per batched
device solve, mixed precision (FP32 iterations, FP64 checks).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one batch of `batch` LPs solved to the tolerance. `value` is the
whole-job throughput with the step inputs already resident in HBM; `e2e` is
the same through the C ABI from pinned host buffers with the solutions read
back to the host every step. Under torchrun every rank solves its own
batches (weak scaling, no collective in the loop); the timed region is
bracketed by a barrier and a device synchronize, and the time is the max over
ranks. The reference arm times the reference's own CPU PDLP (the library
oracle/Makefile builds from the reference sources) on the host cores.
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

METRIC = "LPs solved/s at 1e-4 rel. KKT (min-cost flow family, batched)"
FALLBACK_HBM_GBS = 6650.0


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--batch", type=int, default=256)
    p.add_argument("--tol", type=float, default=1e-4)
    p.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    p.add_argument("--cpu-sample", type=int, default=32, help="instances in the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-extras", action="store_true", help="skip the plain-GPU and large-LP side measurements")
    p.add_argument("--profile", action="store_true",
                   help="load one batch and launch only the timed trial kernels (for ncu captures)")
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
    path = os.path.join(ROOT, "profiles", "pdhg_kernels_flow_batch256.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
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
    from optimisation_solver_b200 import generators as g
    out = []
    for k in range(steps):
        supply, cost = g.flow_parameters(graph, batch, seed=100_000 * (rank + 1) + k)
        out.append((supply, cost))
    return out


def cpu_solve_sample(lib_kind: str, graph, supply, cost, tol: float, threads: int):
    """Solves each (supply, cost) instance with the CPU library, instance
    parallel over `threads` host threads (one solver thread each). Returns
    (seconds, statuses)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle.oracle import Oracle
    from optimisation_solver_b200 import generators as g
    orc = Oracle(lib_kind)
    opts = dict(thread_count=1, primal_tolerance=tol, dual_tolerance=tol, gap_tolerance=tol)
    lps = [g.flow_lp(graph, supply[i], cost[i]) for i in range(supply.shape[0])]
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        res = list(ex.map(lambda lp: orc.solve(lp, opts), lps))
    return time.perf_counter() - t0, [r.status for r in res]


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    assert args.warmup >= 3, "at least 3 warm-up steps"

    from optimisation_solver_b200 import generators as g
    graph = g.flow_graph()
    config = {"workload": "min-cost flow family: 2000 nodes, 20000 arcs, 40000 nnz; "
                          f"batch {args.batch} per step; tolerance {args.tol:g} relative KKT",
              "batch": args.batch, "nodes": graph.nodes, "arcs": graph.arcs,
              "tolerance": args.tol, "l2": "working set > L2 (126 MB) every step"}

    if args.impl == "reference":
        return reference_arm(args, world, rank, graph, config)

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
    session = Session(family, args.batch, options, precision=args.precision, device=local_rank)

    steps_in = workload(args.batch, args.warmup + args.steps, rank, graph)
    # Inputs resident in HBM before the timed region.
    dev_in = [(torch.from_numpy(s).to(dev), torch.from_numpy(c).to(dev)) for s, c in steps_in]
    torch.cuda.synchronize()

    def step(k):
        sup, cost = dev_in[k]
        session.load(objective=cost.data_ptr(), row_lower=sup.data_ptr(), row_upper=sup.data_ptr(),
                     on_device=True)
        return session.solve()

    if args.profile:
        sup, cost = dev_in[0]
        session.load(objective=cost.data_ptr(), row_lower=sup.data_ptr(), row_upper=sup.data_ptr(),
                     on_device=True)
        step(0)
        tk = session.time_kernels(3)
        print(json.dumps({"profile": tk}))
        session.close()
        return
    for k in range(args.warmup):
        step(k)
    launches = 0
    optimal = 0
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local_rank) as clocks:
        start.record()
        for k in range(args.warmup, args.warmup + args.steps):
            optimal += step(k)
            launches += session.last_timing()[1]
        end.record()
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    elapsed = start.elapsed_time(end) / 1e3
    t = torch.tensor([elapsed], device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    elapsed_max = float(t.item())
    value = world * args.batch * args.steps / elapsed_max

    # End to end through the C ABI: pinned host inputs copied in, solutions read back.
    pinned = [(torch.from_numpy(s).pin_memory(), torch.from_numpy(c).pin_memory()) for s, c in steps_in]
    out_x = torch.empty((args.batch, graph.arcs), dtype=torch.float64).pin_memory()
    out_y = torch.empty((args.batch, graph.nodes), dtype=torch.float64).pin_memory()
    h2d = args.batch * (graph.arcs + 2 * graph.nodes) * 8
    d2h = args.batch * (graph.arcs + graph.nodes) * 8
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    e2e_optimal = 0
    for k in range(args.warmup, args.warmup + args.steps):
        sup, cost = pinned[k]
        session.load(objective=cost.numpy(), row_lower=sup.numpy(), row_upper=sup.numpy())
        e2e_optimal += session.solve()
        res = session.read(primal=out_x.numpy(), dual=out_y.numpy())
    torch.cuda.synchronize()
    e2e_elapsed = time.perf_counter() - t0
    t = torch.tensor([e2e_elapsed], device=dev)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_value = world * args.batch * args.steps / float(t.item())

    # Dominant kernel, timed live with CUDA events on the library's stream.
    tk = session.time_kernels(20)
    kernel = "k_primal" if tk["primal_ms"] >= tk["dual_ms"] else "k_dual"
    ms = tk["primal_ms"] if kernel == "k_primal" else tk["dual_ms"]
    nbytes = tk["primal_bytes"] if kernel == "k_primal" else tk["dual_bytes"]
    peak, peak_kind = peaks()
    achieved = nbytes / (ms * 1e-3) / 1e9
    roofline = {"bound": "hbm", "kernel": kernel, "achieved": round(achieved, 1), "peak": peak,
                "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "traffic": ncu_traffic(kernel), "algorithmic_bytes_per_launch": nbytes,
                "launch_ms": round(ms, 5),
                "other_kernel": {"name": "k_dual" if kernel == "k_primal" else "k_primal",
                                 "launch_ms": round(tk["dual_ms"] if kernel == "k_primal" else tk["primal_ms"], 5),
                                 "gbs": round((tk["dual_bytes"] / tk["dual_ms"] if kernel == "k_primal"
                                               else tk["primal_bytes"] / tk["primal_ms"]) / 1e6, 1)}}

    line = {"metric": METRIC, "value": round(value, 2), "unit": "LPs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * elapsed_max / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 iterations, f64 checks"
            if args.precision == "mixed" else "f64", "data": "synthetic (seeded generators)",
            "config": config, "optimal_fraction": optimal / (args.batch * args.steps),
            "clocks": clocks.summary(), "gpu_launches": int(launches),
            "e2e": {"value": round(e2e_value, 2), "unit": "LPs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h, "optimal_fraction": e2e_optimal / (args.batch * args.steps)},
            "roofline": roofline}

    if rank == 0 and not args.no_extras:
        line["plain_gpu_fp64_single"] = plain_gpu(graph, steps_in[-1], args.tol)
        line["speedup_vs_plain_gpu_fp64"] = round(value / world / line["plain_gpu_fp64_single"]["lps_per_s"], 2)
    if rank == 0 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(args, graph, steps_in[-1])
    session.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))


def plain_gpu(graph, inputs, tol, count=6):
    """Plain FP64 single-instance GPU PDLP on the same instances, one LP per call."""
    from optimisation_solver_b200 import generators as g
    from optimisation_solver_b200.lp import PdlpOptions
    from optimisation_solver_b200.pdlp import PdlpSolver
    solver = PdlpSolver("fp64")
    opts = PdlpOptions().with_tolerance(tol)
    supply, cost = inputs
    solver.solve(g.flow_lp(graph, supply[0], cost[0]), opts)
    t0 = time.perf_counter()
    iters = []
    for i in range(1, count + 1):
        r = solver.solve(g.flow_lp(graph, supply[i], cost[i]), opts)
        iters.append(r.iterations)
    dt = time.perf_counter() - t0
    return {"lps_per_s": round(count / dt, 3), "instances": count, "mean_iterations": float(np.mean(iters))}


def cpu_baseline(args, graph, inputs):
    from oracle.oracle import available
    kind = "ref_fast" if available("ref_fast") else "port"
    threads = os.cpu_count() or 1
    supply, cost = inputs
    k = min(args.cpu_sample, supply.shape[0])
    seconds, statuses = cpu_solve_sample(kind, graph, supply[:k], cost[:k], args.tol, threads)
    return {"value": round(k / seconds, 3), "unit": "LPs/s", "cores": threads,
            "kind": "reference" if kind == "ref_fast" else "port",
            "sample": f"{k} instances of the same family and tolerance, instance-parallel, "
                      f"one solver thread each, {seconds:.1f} s",
            "optimal_fraction": statuses.count("optimal") / k}


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
        seconds, statuses = cpu_solve_sample(kind, graph, inputs[k][0], inputs[k][1], args.tol, threads)
        total += seconds
        optimal += statuses.count("optimal")
    value = per_step * args.steps / total
    line = {"metric": METRIC, "value": round(value, 3), "unit": "LPs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(1e3 * total / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generators)",
            "config": dict(config, batch=per_step), "impl": "reference",
            "optimal_fraction": optimal / (per_step * args.steps),
            "cpu_baseline": {"value": round(value, 3), "unit": "LPs/s", "cores": threads,
                             "kind": "reference" if kind == "ref_fast" else "port",
                             "sample": f"{per_step} instances per step, instance-parallel"},
            "e2e": {"value": round(value, 3), "unit": "LPs/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


if __name__ == "__main__":
    main()
