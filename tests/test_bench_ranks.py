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


def test_plain_roofline_uses_committed_fp64_count():
    """The plain form's roofline: FP64 flops per pair from the committed ncu
    count, against the FP64 peak and the FP32 peak; no count, no figure."""
    import sys

    sys.path.insert(0, REPO)
    import bench

    f64 = bench.load_fp64_flops("c2")
    assert f64 and 100 < f64 < 400
    r = bench.plain_roofline("c2", 2.0e11, 2000.0, 34.0, 72.0)
    achieved = 2.0e11 / 2.0 * f64 / 1e12
    assert abs(r["achieved"] - achieved) < 1e-9 * achieved
    assert abs(r["frac"] - achieved / 34.0) < 1e-12 and abs(r["frac_of_fp32_peak"] - achieved / 72.0) < 1e-12
    assert bench.plain_roofline("no_such_workload", 1.0, 1.0, 34.0, 72.0)["flops_per_pair"] is None
