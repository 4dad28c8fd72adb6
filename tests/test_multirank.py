"""Replica timing across ranks (CPU, gloo, world size 2).

The SPH step does not shard (one scene per GPU), so ``bench.py --gpus N``
runs N independent replicas and reports the whole-job rate from the slowest
rank's time. This checks that aggregation, the barrier and the replica
independence of the host logic with two CPU processes.
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
