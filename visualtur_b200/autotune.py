"""Autotuner for the ray-casting kernels (no reference counterpart).

Sweeps the kernel schedule of a live renderer -- ray-tile size {32, 64,
128, 256 rays}, march unroll {1, 2, 4, 8}, one-ray-per-thread vs the
persistent ray queue and the queue's refill interval {8, ..., 128 steps}
-- and, through a caller-supplied factory, the brick
size {8, 16, 32} (which needs a new renderer: the cache layout changes).
Each point is timed with CUDA events over the same frames after a warm-up
that leaves the brick cache in the same state; the fastest is kept.
"""
import itertools

TILES = {32: (8, 4), 64: (8, 8), 128: (16, 8), 256: (16, 16)}
UNROLLS = (1, 2, 4, 8)
PERSIST = (0, 1)
POPS = (8, 16, 32, 64, 128)       # persistent queue: traversal steps between warp refills


def time_frames(torch, renderer, render_step, frames, warmup=2, stream=None):
    """Device ms per frame of render_step(renderer, i, stream) over `frames`
    frames, timed with CUDA events on `stream` (the launching stream)."""
    stream = stream or torch.cuda.Stream()
    with torch.cuda.stream(stream):
        for i in range(warmup):
            render_step(renderer, i, stream)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for i in range(frames):
            render_step(renderer, warmup + i, stream)
        b.record(stream)
        torch.cuda.synchronize()
    return a.elapsed_time(b) / frames


def tune_schedule(torch, renderer, render_step, frames=6, tiles=TILES, unrolls=UNROLLS, persist=PERSIST,
                  stream=None, pops=POPS):
    """Best (tile, unroll, persistent) for a renderer, then -- when the
    persistent queue wins -- its refill interval; returns (best, table)."""
    table = []
    for (rays, (tw, th)), u, p in itertools.product(sorted(tiles.items()), unrolls, persist):
        renderer.set_tuning(tile_w=tw, tile_h=th, unroll=u, persistent=p)
        ms = time_frames(torch, renderer, render_step, frames, stream=stream)
        table.append({"tile_rays": rays, "tile_w": tw, "tile_h": th, "unroll": u, "persistent": p,
                      "pops": renderer.tuning()["pops"], "ms": round(ms, 4)})
    best = min(table, key=lambda r: r["ms"])
    renderer.set_tuning(tile_w=best["tile_w"], tile_h=best["tile_h"], unroll=best["unroll"],
                        persistent=best["persistent"])
    if best["persistent"] and pops:
        # second stage: refill interval of the persistent queue at the best shape
        for pp in pops:
            renderer.set_tuning(pops=pp)
            ms = time_frames(torch, renderer, render_step, frames, stream=stream)
            table.append(dict(best, pops=pp, ms=round(ms, 4)))
        best = min(table, key=lambda r: r["ms"])
        renderer.set_tuning(pops=best.get("pops", renderer.tuning()["pops"]))
    return best, table


def tune(torch, make_renderer, render_step, brick_sizes=(8, 16, 32), frames=6, **kw):
    """Full sweep: make_renderer(brick) -> renderer for each brick size, then
    the schedule sweep on each; returns (best, table) over all points."""
    best, table = None, []
    for b in brick_sizes:
        r = make_renderer(b)
        if r is None:
            continue
        bb, t = tune_schedule(torch, r, render_step, frames, **kw)
        for row in t:
            row["brick"] = b
        table += t
        if best is None or bb["ms"] < best["ms"]:
            best = dict(bb, brick=b)
        r.close()
    return best, table
