"""The replica path of bench.py: whole-job figures over ranks (the slowest
rank's time, the sum of the ranks' pair interactions), exercised with two
gloo ranks on the CPU."""
import os
import socket

import pytest
import torch.distributed as tdist
import torch.multiprocessing as mp

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    import sys

    sys.path.insert(0, REPO)
    import bench

    tdist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                             world_size=world)
    try:
        total, e2e, pairs = bench.combine_ranks(1.0 + rank, 0.5 * (2 - rank), 1000 * (rank + 1), tdist, "cpu")
        q.put((rank, total, e2e, pairs))
    finally:
        tdist.destroy_process_group()


def test_combine_ranks_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, total, e2e, pairs in got:
        assert total == 2.0          # max over ranks
        assert e2e == 1.0
        assert pairs == 3000.0       # sum over ranks


def test_combine_single_process():
    import sys

    sys.path.insert(0, REPO)
    import bench

    assert bench.combine_ranks(2.0, 3.0, 7, None, "cpu") == (2.0, 3.0, 7.0)
