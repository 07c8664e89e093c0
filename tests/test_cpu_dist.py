"""Replicas-only multi-GPU path, exercised on the CPU with gloo ranks: the
timing reduction takes the slowest rank and the whole-job value counts the
units of every rank."""
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


def _rank(rank, ws, port, q):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=ws, timeout=datetime.timedelta(seconds=60))
    import bench
    t = 1.0 + rank                          # rank 1 is the slow one
    slowest = bench.max_over_ranks(ws, t)
    value = bench.replica_value(ws, 10, t)
    bench.barrier(ws)
    q.put((rank, slowest, value))
    dist.destroy_process_group()


def test_replicas_take_the_slowest_rank():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, slowest, value in out:
        assert slowest == 2.0
        assert value == pytest.approx(10 * 2 / 2.0)
