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


def _share_rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "cuppa-public_b200"))
    import torch
    import torch.distributed as dist
    import bench
    import cuppa_b200 as pa
    from cuppa_b200.workloads import batched_instances
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        inst = batched_instances(512)
        prms = [pa.make_params(x["n"], x["d"], x["p"], seed=x["seed"]) for x in inst]
        mine = bench.rank_share(pa, prms, world, rank)
        sizes = [None] * world
        dist.all_gather_object(sizes, mine)
        load = sum(pa.sizes(prms[i])[0] for i in mine)
        loads = [None] * world
        dist.all_gather_object(loads, load)
        q.put((rank, sizes, loads))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_split_a_batch_exactly_once():
    """Each rank derives its share of the batched workload on its own; together
    the shares cover every instance once, with balanced edge bytes."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_share_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = sorted(q.get(timeout=10) for _ in procs)
    shares = got[0][1]
    assert got[1][1] == shares                      # both ranks agree on the split
    allidx = sorted(shares[0] + shares[1])
    assert allidx == list(range(512))
    l0, l1 = got[0][2]
    assert abs(l0 - l1) / (l0 + l1) < 0.05


def test_single_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert bench.job_rate(10, 2, 1, 4.0) == 5.0
