"""Multi-rank host logic of bench.py on CPU (gloo, world size 2): independent
jobs dealt to ranks, whole-job throughput = all ranks' cell-updates over the
slowest rank's time.  No GPU and no data-path collective are involved."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        jobs = list(range(7))
        mine = bench.shard_jobs(jobs, rank, world)
        units = 1000.0 * len(mine)
        secs = 2.0 + rank            # rank 1 is the slow one
        rate, tot, mx = bench.aggregate(dist, units, secs, 0)
        q.put((rank, mine, rate, tot, mx, bench.max_over_ranks(dist, float(rank), 0)))
    finally:
        dist.destroy_process_group()


def test_two_rank_aggregation_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    (r0, m0, rate0, tot0, mx0, mr0), (r1, m1, rate1, tot1, mx1, mr1) = out
    assert sorted(m0 + m1) == list(range(7)) and not set(m0) & set(m1)
    assert tot0 == tot1 == 7000.0
    assert mx0 == mx1 == 3.0
    assert rate0 == rate1 == pytest.approx(7000.0 / 3.0)
    assert mr0 == mr1 == 1.0


def test_single_process_aggregation():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.aggregate(None, 10.0, 2.0, 0) == (5.0, 10.0, 2.0)
    assert bench.shard_jobs([1, 2, 3], 0, 1) == [1, 2, 3]
