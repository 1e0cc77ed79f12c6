"""Multi-rank bench runs share one host volume per node: local rank 0
creates and fills it, the other ranks map the same memory read-only, and
the backing file is gone once every rank has mapped it (no host memory is
left behind however the processes end).  Checked with two gloo ranks on
the CPU; also the per-rank host-tier budget."""
import os
import socket
import sys

import numpy as np
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

    import torch.distributed as dist

    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        shape, off = (64, 32, 48), 12
        calls = []

        def produce(a):
            calls.append(1)
            a[...] = np.arange(a.size, dtype=np.float32).reshape(a.shape)

        m, arr = bench.shared_host_array(dist, rank, "t", shape, np.float32, off, produce)
        ok = bool(np.array_equal(arr, np.arange(arr.size, dtype=np.float32).reshape(shape)))
        aligned = (arr.ctypes.data - off) % 4096 == 0
        leftover = [f for d in ("/dev/shm", "/tmp") if os.path.isdir(d)
                    for f in os.listdir(d) if f.startswith("vtbench_t_")]
        out.put((rank, ok, len(calls), aligned, arr.flags.writeable, leftover))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_ranks_share_one_volume_and_leave_no_file():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, ok0, calls0, al0, w0, left0), (r1, ok1, calls1, al1, w1, left1) = res
    assert ok0 and ok1                      # both ranks see the volume rank 0 produced
    assert calls0 == 1 and calls1 == 0      # produced once, by local rank 0
    assert al0 and al1                      # the requested offset past a page boundary
    assert w0 and not w1                    # the other ranks map it read-only
    assert not left0 and not left1          # the file is unlinked once mapped


def test_rank_host_tier_budget():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.rank_host_bytes(16 << 30, 0, 1) == 16 << 30
    total = os.sysconf("SC_PAGE_SIZE") * os.sysconf("SC_PHYS_PAGES")
    budget = (total - (8 << 30) - (16 << 30) - 2 * (6 << 30)) // 2
    if budget >= 1 << 30:
        assert bench.rank_host_bytes(1 << 50, 8 << 30, 2) == budget
        assert bench.rank_host_bytes(1 << 20, 8 << 30, 2) == 1 << 20
    with pytest.raises(RuntimeError):
        bench.rank_host_bytes(16 << 30, total, 2)
