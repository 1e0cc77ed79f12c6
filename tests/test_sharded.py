"""Camera-sharded batches (visualtur_b200/sharded.py) on the CPU: the view
split balances pixels and is the same on every rank, and the gather puts
every rank's images, in view order, on rank 0 -- two and three gloo ranks
with images standing in for the renders (each pixel encodes its view), so
a misplaced byte shows.  The render half runs through vt_render_batch and
is covered on one GPU by test_gpu_sharded.py."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from visualtur_b200.sharded import partition_views  # noqa: E402

RES = [(256, 256), (512, 512), (1024, 1024), (1920, 1080), (2048, 2048)]


def views(n, seed=3):
    rng = np.random.default_rng(seed)
    return [RES[int(k)] for k in rng.integers(len(RES), size=n)]


def test_partition_covers_every_view_once_and_balances_pixels():
    for world in (1, 2, 3, 8):
        wh = views(64)
        px = [w * h for w, h in wh]
        parts = partition_views(px, world)
        assert sorted(v for p in parts for v in p) == list(range(64))
        load = [sum(px[v] for v in p) for p in parts]
        assert max(load) - min(load) <= max(px)          # greedy bound: within one view
        assert parts == partition_views(px, world)      # deterministic


def test_partition_of_fewer_views_than_ranks():
    parts = partition_views([100, 50], 4)
    assert parts == [[0], [1], [], []]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _fake(v, w, h):
    import torch
    a = (np.arange(w * h * 3, dtype=np.int64) * 7 + v * 131) % 251
    return torch.from_numpy(a.astype(np.uint8))


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    from visualtur_b200.sharded import gather_images, partition_views
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        wh = views(23, seed=9)
        sizes = [w * h * 3 for w, h in wh]
        parts = partition_views([w * h for w, h in wh], world)
        mine = [_fake(v, *wh[v]) for v in parts[rank]]
        got = gather_images(dist, mine, sizes, parts, rank, "cpu")
        if rank == 0:
            ok = all(np.array_equal(got[v].numpy(), _fake(v, *wh[v]).numpy()) for v in range(len(wh)))
            out.put(("ok" if ok else "mismatch", [len(p) for p in parts]))
        else:
            assert got is None
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gather_puts_every_view_in_order_on_rank0(world):
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    status, counts = out.get(timeout=10)
    assert status == "ok" and sum(counts) == 23 and min(counts) > 0
