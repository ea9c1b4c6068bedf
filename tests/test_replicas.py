"""Replica accounting of bench.py across ranks (two gloo ranks on CPU): the
job's time is the slowest rank's, its pair count the sum."""
import multiprocessing as mp
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as D

    import bench
    D.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                         timeout=datetime.timedelta(seconds=60))
    try:
        t, w = bench.combine_ranks(100.0 + 50.0 * rank, [1e12 * (rank + 1), 3.0])
        q.put((rank, t, w))
    finally:
        D.destroy_process_group()


def test_combine_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = [q.get(timeout=120) for _ in ps]
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, w in out:
        assert t == 150.0
        assert w == pytest.approx([3e12, 6.0])
