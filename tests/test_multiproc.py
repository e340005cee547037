"""The N > 1 path of bench.py on CPU: two gloo ranks.

The GRRT path shards by rays with no exchange step (replicas: every rank
renders its own image), so the only cross-rank traffic is the timing
reduction -- the maximum of the per-rank times and the sum of the per-rank
ray-steps -- and the barriers around the timed region.
"""

from __future__ import annotations

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, q) -> None:
    import torch

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    td = bench.init_dist(world, "gloo")
    try:
        assert bench.dist_env() == (rank, world, rank)
        bench.barrier(world)
        t_max = bench.max_over_ranks(10.0 + rank * 5.0, world, torch.device("cpu"))
        steps = bench.sum_over_ranks(1000.0 * (rank + 1), world, torch.device("cpu"))
        bench.barrier(world)
        q.put((rank, t_max, steps))
    finally:
        td.destroy_process_group()


def test_two_rank_timing_reduction():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=5) for _ in range(2))
    for rank, t_max, steps in got:
        assert t_max == 15.0          # max over ranks
        assert steps == 3000.0        # whole-job ray-steps


def test_single_rank_reduction_is_identity():
    import bench

    assert bench.max_over_ranks(3.5, 1, None) == 3.5
    assert bench.sum_over_ranks(7.0, 1, None) == 7.0
