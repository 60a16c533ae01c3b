"""The multi-GPU path's host logic on CPU: two gloo ranks (one process each,
as torchrun launches them), nnz-balanced instance shards, disjoint seeds, the
max-over-ranks timing that bench.py reports, and a sharded solve whose
gathered results equal a single-process solve of the same instances (the
CPU oracle stands in for each rank's GPU)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from optimisation_solver_b200 import generators as g
from optimisation_solver_b200.sharding import balanced_shards, rank_seeds


def test_balanced_shards_cover_and_balance():
    sizes = g.uneven_batch_sizes(1024)
    weights = sizes * 16   # about 16 nonzeros per row in the uneven family
    for world in (1, 2, 3, 8):
        shards = balanced_shards(weights, world)
        assert len(shards) == world
        allidx = np.concatenate(shards)
        assert np.array_equal(allidx, np.arange(len(sizes)))
        loads = np.array([weights[s].sum() for s in shards])
        assert loads.max() - loads.min() <= 2 * weights.max()


def test_balanced_shards_fewer_instances_than_ranks():
    shards = balanced_shards([5, 1], 4)
    assert sorted(np.concatenate(shards).tolist()) == [0, 1]
    assert sum(len(s) == 0 for s in shards) == 2


def test_rank_seeds_disjoint():
    a, b = set(rank_seeds(0, 50)), set(rank_seeds(1, 50))
    assert not a & b and min(a | b) >= 100_000


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from optimisation_solver_b200.sharding import max_over_ranks, weak_scaling_rate
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        sizes = g.uneven_batch_sizes(64)
        mine = balanced_shards(sizes * 16, world)[rank]
        seconds = 1.0 + rank           # rank 1 is the slow one
        out[rank] = (len(mine), max_over_ranks(seconds),
                     weak_scaling_rate(len(mine), seconds), int(mine.min()), int(mine.max()))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_time():
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    n0, mx0, rate0, lo0, hi0 = out[0]
    n1, mx1, rate1, lo1, hi1 = out[1]
    assert n0 + n1 == 64 and hi0 + 1 == lo1
    assert mx0 == mx1 == 2.0                       # the slowest rank's time
    assert rate0 == rate1 == pytest.approx(64 / 2.0)


def _uneven_small(count=10):
    rng = np.random.default_rng(17)
    sizes = rng.integers(60, 240, count)
    return [g.planted_lp(int(m), 2 * int(m), seed=300 + i).lp for i, m in enumerate(sizes)]


def _solve_worker(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    from optimisation_solver_b200.sharding import gather_to_rank0
    from oracle.oracle import best_available
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        lps = _uneven_small()
        mine = balanced_shards([lp.nnz for lp in lps], world)[rank]
        orc = best_available()
        recs = []
        for i in mine:
            r = orc.solve(lps[i], dict(thread_count=1))
            recs.append((r.status, r.iterations, r.primal_objective))
        gathered = gather_to_rank0(mine, recs)
        if rank == 0:
            out["gathered"] = gathered
        out[f"count{rank}"] = len(mine)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_solve_shards_like_one_process():
    from oracle.oracle import best_available
    ctx = mp.get_context("spawn")
    manager = ctx.Manager()
    out = manager.dict()
    port = _free_port()
    procs = [ctx.Process(target=_solve_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs)
    assert out["count0"] > 0 and out["count1"] > 0
    orc = best_available()
    single = [orc.solve(lp, dict(thread_count=1)) for lp in _uneven_small()]
    gathered = out["gathered"]
    assert len(gathered) == len(single)
    for (status, iterations, objective), r in zip(gathered, single):
        assert status == r.status == "optimal"
        assert iterations == r.iterations and objective == r.primal_objective
