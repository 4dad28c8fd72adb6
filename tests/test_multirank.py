"""Multi-rank host logic (CPU, gloo, world size 2).

A single scene does not shard (one scene per GPU), so ``bench.py --gpus N``
runs N independent replicas and reports the whole-job rate from the slowest
rank's time. Batched worlds do shard: the worlds are split over the ranks by
particle count, with no collective in the step. These tests check the
aggregation, the barrier, the replica independence and the world split
with two CPU processes.
"""

from __future__ import annotations

import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    sys.path.insert(0, str(REPO))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta

    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        w, r, lr = bench.dist_env()
        assert (w, r, lr) == (world, rank, rank)
        # each replica builds the same scene independently (host side)
        model, cfg, wl = bench.make_scene("dam_break_32k", "cpu")
        t = 1.5 if rank == 0 else 2.5
        bench.barrier()
        mx = bench.max_over_ranks(t)
        out[rank] = (mx, model.particle_count, float(model.particle_q.sum()))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_replicas_time_is_max_over_ranks():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(240)
        assert p.exitcode == 0
    assert out[0][0] == 2.5 and out[1][0] == 2.5
    # identical replicas on every rank
    assert out[0][1:] == out[1][1:] and out[0][1] == 32768


def _worlds_worker(rank: int, world: int, port: int, out):
    sys.path.insert(0, str(REPO))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        # the first 64 worlds of the 4096-world workload, split over the ranks
        layout = bench.worlds_layout(bench.WORKLOADS["worlds_4096"])[:64]
        sizes = bench.world_sizes(layout)
        mine = bench.partition_worlds(sizes, world)[rank]
        model, cfgs, _ = bench.make_worlds_scene("worlds_4096", "cpu", max_worlds=64, subset=mine)
        assert model.world_count == len(mine) == len(cfgs)
        assert model.particle_count == sum(sizes[k] for k in mine)
        counts = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(counts, torch.tensor([model.particle_count], dtype=torch.int64))
        out[rank] = (mine, [int(c) for c in counts], sum(sizes))
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(300)
def test_worlds_split_over_ranks():
    """Every world on exactly one rank; the ranks' particles add up to the
    job's; the split is balanced to within the largest world."""
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worlds_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(240)
        assert p.exitcode == 0
    (m0, counts, total), (m1, counts1, _) = out[0], out[1]
    assert counts == counts1 and sum(counts) == total
    assert sorted(m0 + m1) == list(range(64))
    sys.path.insert(0, str(REPO))
    import bench

    sizes = bench.world_sizes(bench.worlds_layout(bench.WORKLOADS["worlds_4096"])[:64])
    assert abs(counts[0] - counts[1]) <= max(sizes)


def test_partition_worlds_greedy():
    sys.path.insert(0, str(REPO))
    import bench

    sizes = [5, 9, 1, 9, 3, 7, 2, 8]
    parts = bench.partition_worlds(sizes, 3)
    assert sorted(k for p in parts for k in p) == list(range(len(sizes)))
    loads = [sum(sizes[k] for k in p) for p in parts]
    assert max(loads) - min(loads) <= max(sizes)
    assert parts == bench.partition_worlds(sizes, 3)  # deterministic
    assert bench.partition_worlds(sizes, 1) == [list(range(len(sizes)))]
