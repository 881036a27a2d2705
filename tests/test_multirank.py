"""The N > 1 host path of bench.py (replicas, max over ranks) with world_size
2 on the gloo backend (CPU)."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        q.put((rank, ms, bench.replica_throughput(world, 1000, 4, ms)))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_replica_throughput_gloo():
    world, port = 2, free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=worker, args=(r, world, port, q)) for r in range(world)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(world))
    for rank, ms, value in res:
        assert ms == 15.0                      # every rank sees the slowest rank's time
        assert value == 2 * 1000 * 4 / 15e-3   # all replicas' cells over that time


def test_single_rank_path():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(7.5) == 7.5
    assert bench.replica_throughput(1, 100, 2, 10.0) == 100 * 2 / 10e-3
