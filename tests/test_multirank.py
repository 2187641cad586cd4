"""The N > 1 path on the CPU: world-size-2 gloo ranks run bench.py's
max-over-ranks timing and whole-job rate (one graph does not shard, so each
rank generates its own replica and the job's value counts all replicas over
the slowest rank's time)."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        slow = bench.max_over_ranks(1.0 + rank, world, "cpu")   # rank 1 is the slow one
        rate = bench.job_rate(1000, 5, world, slow)
        q.put((rank, slow, rate))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in procs)
    assert [g[1] for g in got] == [2.0, 2.0]
    assert all(g[2] == pytest.approx(2 * 1000 * 5 / 2.0) for g in got)


def test_single_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.job_rate(10, 2, 1, 4.0) == 5.0
