"""Multi-GPU runs of the renderer are replicas: every rank renders its own
stretch of the workload and the only exchange is the reduction of the
timings.  This checks that logic on the CPU with two gloo ranks: the ranks'
frame ranges are disjoint and adjacent, every rank sees the slowest rank's
time, and the whole-job throughput counts all ranks' rays over that time."""
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


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        warmup, steps = 3, 10
        f0 = bench.replica_first_frame(rank, warmup, steps)
        local = 100.0 + 25.0 * rank                       # this rank's device time, ms
        t_max = bench.max_over_ranks(dist, torch, local, "cpu")
        value = bench.replica_value(1000 * steps, world, t_max)
        out.put((rank, f0, t_max, value))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_replicas_share_only_their_timings():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(out.get(timeout=10) for _ in range(2))
    (r0, f0, t0, v0), (r1, f1, t1, v1) = res
    assert (r0, r1) == (0, 1)
    assert f0 == 0 and f1 == 13                         # [0, 13) and [13, 26): disjoint, adjacent
    assert t0 == t1 == pytest.approx(125.0)            # both see the slowest rank
    assert v0 == v1 == pytest.approx(2 * 1000 * 10 / 0.125)


def test_single_rank_needs_no_collective():
    sys.path.insert(0, ROOT)
    import torch

    import bench
    assert bench.max_over_ranks(None, torch, 42.0, "cpu") == 42.0
    assert bench.replica_first_frame(0, 3, 300) == 0
