"""The multi-rank host logic of bench.py (replicas, one process per GPU) on
CPU with gloo, world size 2: the timing taken is the max over ranks on every
rank, and throughput counts every replica's work."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, q):
    import datetime

    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank, 0.5 * (rank + 1)], dist, torch.device("cpu"))
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0] == out[1] == [2.0, 10.0, 1.0]


def test_replica_throughput_counts_every_rank():
    sys.path.insert(0, ROOT)
    import bench
    # 2 replicas of 1000 rays x 4 steps in 0.5 s (max over ranks)
    assert bench.replica_throughput(1000, 2, 4, 0.5) == pytest.approx(16000.0)
    assert bench.max_over_ranks([3.0], None, None) == [3.0]
