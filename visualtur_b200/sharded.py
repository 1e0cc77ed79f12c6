"""Camera-sharded rendering on several GPUs (no reference counterpart: the
reference renders on the one device it selects, src/testVisualTur.cu:18-23).

Every ray and every view is independent, so a batch of views is split
across ranks -- one process per GPU, each with its own renderer (the
octree replicated, its own brick cache) -- and the finished RGB8 images are
gathered to rank 0.  Nothing else crosses between GPUs: there is no
exchange inside a frame, so the only collective is the final gather (NCCL
between GPUs; gloo in the CPU tests).

  partition_views(sizes, world)  -> the views each rank renders
  ShardedViews(renderer, group)  -> render(views) on every rank, images on rank 0
"""
import numpy as np


def partition_views(sizes, world):
    """Splits views of `sizes` pixels (a list) over `world` ranks, balancing
    pixels: largest view first onto the rank with the fewest pixels so far
    (ties to the lower rank).  Returns, per rank, the view indices in
    increasing order -- deterministic, so every rank computes the same
    split without communicating."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    parts = [[] for _ in range(world)]
    for v in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(v)
        load[r] += int(sizes[v])
    return [sorted(p) for p in parts]


def pack(images):
    """Concatenates a rank's images (uint8 tensors) into one flat tensor."""
    import torch
    if not images:
        return torch.zeros(0, dtype=torch.uint8)
    return torch.cat([im.reshape(-1) for im in images])


def gather_images(dist, images, sizes, parts, rank, device):
    """Gathers every rank's images to rank 0.  `images`: this rank's RGB8
    images (uint8 tensors on `device`, in the order of parts[rank]);
    `sizes`: bytes of every view; `parts`: partition_views' split.  Returns,
    on rank 0, all images in view order (CPU tensors); None elsewhere.
    Every rank takes part in the one gather (equal-length buffers, padded
    to the largest rank's bytes)."""
    import torch
    world = len(parts)
    nbytes = [sum(int(sizes[v]) for v in p) for p in parts]
    cap = max(max(nbytes), 1)
    buf = torch.zeros(cap, dtype=torch.uint8, device=device)
    flat = pack(images)
    if flat.numel() != nbytes[rank]:
        raise ValueError("rank %d has %d image bytes, its views need %d" % (rank, flat.numel(), nbytes[rank]))
    if flat.numel():
        buf[:flat.numel()].copy_(flat.to(device))
    if world == 1:
        got = [buf]
    else:
        got = [torch.empty_like(buf) for _ in range(world)] if rank == 0 else None
        dist.gather(buf, gather_list=got, dst=0)
    if rank != 0:
        return None
    out = [None] * len(sizes)
    for r, p in enumerate(parts):
        o = 0
        g = got[r].cpu()
        for v in p:
            n = int(sizes[v])
            out[v] = g[o:o + n].clone()
            o += n
    return out


class ShardedViews:
    """One rank's share of camera-sharded batches.  `renderer` is this
    rank's visualTur (its own device and brick cache); `dist` is
    torch.distributed with an initialised group (or None for one rank)."""

    def __init__(self, renderer, dist=None, rank=0, world=1, device=None, stream=None):
        self.r, self.dist, self.rank, self.world = renderer, dist, rank, world
        self.device, self.stream = device, stream
        self._bufs = {}

    def _buf(self, k, n):
        import torch
        b = self._bufs.get(k)
        if b is None or b.numel() < n:
            b = torch.empty(n, dtype=torch.uint8, device=self.device)
            self._bufs[k] = b
        return b[:n]

    def render(self, cams):
        """Renders the views `cams` (vt_camera list, the same on every rank):
        this rank renders its part in one vt_render_batch; rank 0 returns
        every view's RGB8 image (H*W*3 uint8, CPU), the others None."""
        from . import vt_view
        sizes = [c.W * c.H * 3 for c in cams]
        parts = partition_views([c.W * c.H for c in cams], self.world)
        mine = parts[self.rank]
        imgs = []
        if mine:
            views = []
            for i, v in enumerate(mine):
                b = self._buf(i, sizes[v])
                vv = vt_view()
                vv.cam, vv.dev_rgba, vv.dev_rgb8 = cams[v], None, b.data_ptr()
                views.append(vv)
                imgs.append(b)
            self.r.render_batch(views, stream=self.stream.cuda_stream if self.stream is not None else None)
            if self.stream is not None:
                self.stream.synchronize()
        return gather_images(self.dist, imgs, sizes, parts, self.rank, self.device)
