"""The N > 1 path of bench.py (independent replicas, one per GPU): the
timing is the max over ranks and every rank takes the same collective steps.
Exercised with world_size 2 on the gloo backend, on the CPU."""
import os
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    from datetime import timedelta

    import bench

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        bench._barrier(world)
        ms = bench._max_over_ranks(10.0 + 5.0 * rank, world)  # rank 1 is slower
        e2e = bench._max_over_ranks(1.0 + rank, world)
        out.put((rank, ms, e2e))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_replicas():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=10) for _ in range(2))
    assert got == [(0, 15.0, 2.0), (1, 15.0, 2.0)]
