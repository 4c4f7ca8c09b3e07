"""The bench's multi-rank host logic (one process per GPU under torchrun), run as two gloo ranks on the CPU:
every rank keys its jobs differently (no two ranks compute the same RNG streams), the step time is the
maximum over ranks, and the whole-job throughput counts every rank's units over that maximum."""
from __future__ import annotations

import os
import socket

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import sys

    import torch.distributed as dist
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        keys = bench.rank_job_keys(rank, 20)
        gathered = [None] * world
        dist.all_gather_object(gathered, keys)
        my_ms = 100.0 + 37.5 * rank  # a slower second rank
        ms = bench.max_over_ranks(my_ms, dist, "cpu")
        value = bench.job_throughput(world, 497.664, 5, ms)
        q.put((rank, gathered, ms, value))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_and_time_like_the_bench():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    (r0, g0, ms0, v0), (r1, g1, ms1, v1) = out
    assert g0 == g1
    assert not set(g0[0]) & set(g0[1]), "ranks must key their jobs differently"
    assert len(set(k[1] for k in g0[0] + g0[1])) == 40
    assert ms0 == ms1 == 137.5, "both ranks report the slowest rank's time"
    assert v0 == v1 == pytest.approx(2 * 497.664 * 5 / 0.1375)
