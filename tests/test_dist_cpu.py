"""Multi-process host logic of bench.py on CPU: two gloo ranks reduce their
timings (max) and counters (sum) the way the benchmark does across GPUs, and
the whole-job rate is computed from the slowest rank."""
from __future__ import annotations

import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took 100 + 10 r ms over its steps and saw r decrypt errors
        (t,), (e,) = bench.reduce_over_ranks([100.0 + 10 * rank], [float(rank)], "cpu")
        q.put((rank, t, e, bench.whole_job_rate(world, 1024, 20, t)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_reduce_like_the_benchmark():
    import torch.multiprocessing as mp
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    got = sorted(q.get(timeout=5) for _ in range(world))
    for rank, t, e, rate in got:
        assert t == 110.0                                   # the slowest rank's time
        assert e == 1.0                                     # errors summed over ranks
        assert rate == pytest.approx(2 * 1024 * 20 / 0.110)  # all ranks' units / slowest time


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_over_ranks([3.0, 4.0], [5.0], "cpu") == ([3.0, 4.0], [5.0])
    assert bench.whole_job_rate(1, 1024, 10, 1000.0) == pytest.approx(10240.0)
