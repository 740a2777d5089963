"""Replica runs on several ranks (world size 2, gloo, CPU): every rank reports the
slowest rank's time, and all ranks agree. The bench runs one independent problem
per GPU with no data-path collective; this covers the reduction of its timings."""
from __future__ import annotations

import os
import socket

import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank: int, world: int, port: int, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        vals = bench.reduce_max([1.0 + rank, 10.0 - rank], "cpu")
        out.put((rank, vals))
    finally:
        dist.destroy_process_group()


def test_replica_times_reduce_to_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert results[0] == results[1] == [2.0, 10.0]
