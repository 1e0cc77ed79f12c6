#!/usr/bin/env python
"""Benchmark: rays/s and ms/frame of the isosurface ray caster on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--config c2|c1|c3|c2s|c3s]
                  [--mode best|plain] [--impl ours|reference]   (also c4, c5, c5s)

A step is one rendered frame of the workload (one batch of views for c3):
  c2 (default): the 2048^3 float32 out-of-core fly-through -- 256 seeded
      anisotropic Gaussian blobs + 4-octave value noise, isovalue 0.6,
      16^3 bricks (apron 3), device brick cache 4 GB, pinned host tier
      16 GB, 1920x1080, orbit at radius 3000 voxels, 1.2 deg per frame.
      Inputs exceed L2 (32 GB volume), no flush between frames.
  c1: the 128^3 noisy sphere, fully resident in HBM, one 512x512 camera at
      distance 300; L2 flushed (256 MB write) between timed frames.
  c3: the c2 volume, 64 seeded views per launch at random poses on a
      sphere of radius 2500-3500 looking into the inner half, resolutions
      drawn from {256^2, 512^2, 1024^2, 1920x1080, 2048^2}; the autotuner
      also picks the brick edge {8, 16, 32}.
  c4: the c2 volume on a held-out 300-frame spline (the learned-prefetch
      evaluation: hit rate, stall per frame, same pixels as plain).
  c5: 4096^3 uint8 fractal, 32^3 bricks, 16 GB cache, 600-frame spline.
  c2s / c3s / c5s: c2 / c3 / c5 at half the edge (profiling and quick checks).
value = rays of all ranks / device time (CUDA events, max over ranks).
Multi-GPU: replicas only -- each rank renders its own frames, no
collective on the data path ("scaling": "weak").

--impl reference times the reference algorithm's CPU restatement (the
oracle port; the reference itself has no CPU path) on the host cores, on a
bounded sample of the same workload; rank 0 only.
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0

# DRAM bytes per ray of k_trace (dram__bytes_read.sum + dram__bytes_write.sum
# of one ncu capture of a full 1920x1080 frame of the c2s fly-through, warm
# cache; the c2 orbit is the same view of a volume twice the size, with the
# same samples per ray).  Scaled by the rays of a launch for roofline.traffic.
TRAFFIC_BYTES_PER_RAY = {"c2": 94.6, "c2s": 94.6}

CONFIGS = {
    "c1": dict(workload="128^3 f32 noisy sphere (|x-c|+N(0,0.25)), iso 40, resident, 512x512, FOV 60 deg, "
                        "distance 300, 8^3 bricks, 4^3 candidate nodes",
               gen="sphere", seed=1234, n=128, iso=40.0, levelC=4, levelO=5, inc=3, W=512, H=512, fov=30.0,
               dist=50.0, resident=1, l2flush=True, orbit=None, cam_pos=(63.5, 63.5, 363.5)),
    "c2": dict(workload="2048^3 f32 blobs+noise, iso 0.6, out-of-core: 16^3 bricks (apron 3), 4 GB device "
                        "cache, 16 GB pinned host tier, 1920x1080, orbit r=3000 at 1.2 deg/frame, timed from a cold cache",
               gen="blobs", seed=2048, n=2048, iso=0.6, levelC=7, levelO=9, inc=3, W=1920, H=1080, fov=30.0,
               dist=50.0, resident=0, l2flush=False, orbit=(3000.0, 1.2), dev_bytes=4 << 30,
               host_bytes=16 << 30, blobs=(256, 20.0, 120.0, 0.5, 1.5, 0.05)),
    # 64 seeded views per launch, mixed resolutions, on the c2 volume
    # the learned-prefetch evaluation: the c2 volume on a held-out spline
    "c4": dict(workload="2048^3 f32 blobs+noise (the c2 volume), held-out 300-frame Catmull-Rom spline through 12 "
                        "seeded control points at r 2500-3500 looking into the inner half, 1920x1080, 4 GB device "
                        "cache, 16 GB pinned host tier, prefetch network trained on 20 000 poses of other "
                        "fly-throughs, timed from a cold cache",
               gen="blobs", seed=2048, n=2048, iso=0.6, levelC=7, levelO=9, inc=3, W=1920, H=1080, fov=30.0,
               dist=50.0, resident=0, l2flush=False, orbit=None, dev_bytes=4 << 30, host_bytes=16 << 30,
               blobs=(256, 20.0, 120.0, 0.5, 1.5, 0.05), path=dict(frames=300, ctrl=12, r=(2500.0, 3500.0))),
    "c3": dict(workload="2048^3 f32 blobs+noise (the c2 volume), 64 views per launch at seeded random poses "
                        "on a sphere r in [2500,3500] looking into the inner half, resolutions drawn from "
                        "{256^2, 512^2, 1024^2, 1920x1080, 2048^2}; 4 GB device cache, 16 GB pinned host tier, "
                        "timed from a cold cache",
               gen="blobs", seed=2048, n=2048, iso=0.6, levelC=7, levelO=9, inc=3, W=1920, H=1080, fov=30.0,
               dist=50.0, resident=0, l2flush=False, orbit=None, dev_bytes=4 << 30, host_bytes=16 << 30,
               blobs=(256, 20.0, 120.0, 0.5, 1.5, 0.05),
               views=dict(n=64, r=(2500.0, 3500.0), res=((256, 256), (512, 512), (1024, 1024), (1920, 1080),
                                                         (2048, 2048)))),
    # c3 on the 1 GB volume (quick checks)
    "c3s": dict(workload="1024^3 f32 blobs+noise (c2 scaled by 1/2), 64 views per launch, r in [1250,1750], "
                         "mixed resolutions as c3",
                gen="blobs", seed=2048, n=1024, iso=0.6, levelC=6, levelO=8, inc=3, W=1920, H=1080, fov=30.0,
                dist=50.0, resident=0, l2flush=False, orbit=None, dev_bytes=2 << 30, host_bytes=4 << 30,
                blobs=(256, 10.0, 60.0, 0.5, 1.5, 0.05),
                views=dict(n=64, r=(1250.0, 1750.0), res=((256, 256), (512, 512), (1024, 1024), (1920, 1080),
                                                          (2048, 2048)))),
    # 4096^3 uint8 fractal with spheres, 32^3 bricks, 600-frame spline
    "c5": dict(workload="4096^3 u8 6-octave fractal value noise + 32 spheres (value 200, radius 50-400), iso 128, "
                        "out-of-core: 32^3 bricks (apron 3), 16 GB device cache, 64 GB pinned host tier, 1920x1080, "
                        "600-frame Catmull-Rom path through 12 seeded control points, timed from a cold cache",
               gen="fractal", seed=4096, n=4096, iso=128.0, levelC=7, levelO=10, inc=3, W=1920, H=1080, fov=30.0,
               dist=50.0, resident=0, l2flush=False, orbit=None, dev_bytes=16 << 30, host_bytes=64 << 30,
               spheres=(32, 50.0, 400.0, 200.0), path=dict(frames=600, ctrl=12, r=(3500.0, 5000.0))),
    # c5 scaled by 1/2 per axis (8 GB volume)
    "c5s": dict(workload="2048^3 u8 fractal + 32 spheres (c5 scaled by 1/2), iso 128, 32^3 bricks, 2 GB device "
                         "cache, 8 GB host tier, 1920x1080, 600-frame spline",
                gen="fractal", seed=4096, n=2048, iso=128.0, levelC=6, levelO=9, inc=3, W=1920, H=1080, fov=30.0,
                dist=50.0, resident=0, l2flush=False, orbit=None, dev_bytes=2 << 30, host_bytes=8 << 30,
                spheres=(32, 25.0, 200.0, 200.0), path=dict(frames=600, ctrl=12, r=(1750.0, 2500.0))),
    # profiling-sized version of c2 (1 GB volume) for ncu captures
    "c2s": dict(workload="1024^3 f32 blobs+noise (c2 scaled by 1/2), iso 0.6, 16^3 bricks, 1920x1080, orbit r=1500",
                gen="blobs", seed=2048, n=1024, iso=0.6, levelC=6, levelO=8, inc=3, W=1920, H=1080, fov=30.0,
                dist=50.0, resident=0, l2flush=False, orbit=(1500.0, 1.2), dev_bytes=2 << 30,
                host_bytes=4 << 30, blobs=(256, 10.0, 60.0, 0.5, 1.5, 0.05)),
}

# renderer modes: "plain" = the reference's scheme (one view per launch,
# demand LRU from a cold cache, no prefetch); "best" = the product: batches
# of 8 frames per persistent ray-queue launch, lookahead requests, learned
# prefetch hints for the next batch, kernel knobs from the autotuner
MODES = {
    "plain": dict(opts=dict(persistent=0, lookahead=0, use_graph=0), batch=1, learned=False, autotune=False),
    "best": dict(opts=dict(persistent=1, lookahead=2, use_graph=1, pops=32, blocks_per_sm=8), batch=8,
                 learned=True, autotune=True),
}


# demand loads copy x/y aprons from resident neighbours (both renderers)
SHARED_APRONS = 1


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# ----------------------------------------------------------------------------- clocks
class Clocks:
    """nvidia-smi sampling during the timed region (200 ms period)."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
        self.p = None

    def start(self):
        """Starts sampling and returns once the first sample is written:
        nvidia-smi's start-up takes driver locks that stall CUDA calls of
        this process for tens to hundreds of ms, which must not fall into
        the timed region."""
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
            return
        t_end = time.time() + 3.0
        while time.time() < t_end and self.p.poll() is None and os.path.getsize(self.f.name) == 0:
            time.sleep(0.01)

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = [r.split(", ") for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows if len(r) >= 9 for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------- workload
def huge_page_array(shape, dtype, offset=0):
    """Zero-filled-on-touch host array in anonymous memory advised for
    transparent huge pages (before first touch): random brick reads from a
    volume of many GB then miss the TLB far less often.  The first element
    sits `offset` bytes past a page boundary."""
    import ctypes
    import mmap
    nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
    m = mmap.mmap(-1, nbytes + 4096, flags=mmap.MAP_PRIVATE | mmap.MAP_ANONYMOUS)
    try:
        libc = ctypes.CDLL("libc.so.6")
        addr = ctypes.addressof(ctypes.c_char.from_buffer(m))
        libc.madvise(ctypes.c_void_p(addr), ctypes.c_size_t(nbytes + 4096), 14)   # MADV_HUGEPAGE
    except (OSError, AttributeError, TypeError):
        pass
    return m, np.frombuffer(m, dtype, count=int(np.prod(shape)), offset=offset).reshape(shape)


def _madvise_huge(addr, nbytes):
    import ctypes
    try:
        ctypes.CDLL("libc.so.6").madvise(ctypes.c_void_p(addr), ctypes.c_size_t(nbytes), 14)   # MADV_HUGEPAGE
    except (OSError, AttributeError, TypeError):
        pass


def shared_dir(nbytes):
    """A directory with room for a file of `nbytes` (shared memory first)."""
    for d in ("/dev/shm", tempfile.gettempdir()):
        try:
            st = os.statvfs(d)
        except OSError:
            continue
        if st.f_bavail * st.f_frsize >= nbytes + (2 << 30):
            return d
    return None


def shared_host_array(dist, local_rank, name, shape, dtype, offset, produce):
    """One host array for all ranks of the node: local rank 0 creates it
    in a file (shared memory where there is room) and fills it with
    `produce(array)`, the others map the same file read-only.  The file is
    unlinked once every rank has mapped it, so its memory goes with the
    last mapping, whatever way the processes end.  Returns (mmap, array)."""
    import mmap
    nbytes = int(np.prod(shape)) * np.dtype(dtype).itemsize
    size = offset + nbytes
    path = None
    if local_rank == 0:
        d = shared_dir(size)
        if d is None:
            raise RuntimeError("no room for a shared %.1f GB volume in /dev/shm or %s" %
                               (size / 1e9, tempfile.gettempdir()))
        path = os.path.join(d, "vtbench_%s_%d_%s" % (name, os.getpid(), os.environ.get("MASTER_PORT", "0")))
        with open(path, "wb") as f:
            f.truncate(size)
    paths = [path]
    dist.broadcast_object_list(paths, src=0)
    path = paths[0]
    if local_rank == 0:
        with open(path, "r+b") as f:
            m = mmap.mmap(f.fileno(), size, flags=mmap.MAP_SHARED, prot=mmap.PROT_READ | mmap.PROT_WRITE)
        arr = np.frombuffer(m, dtype, count=int(np.prod(shape)), offset=offset).reshape(shape)
        _madvise_huge(arr.ctypes.data - offset, size)
        produce(arr)
    dist.barrier()
    if local_rank != 0:
        with open(path, "rb") as f:
            m = mmap.mmap(f.fileno(), size, flags=mmap.MAP_SHARED, prot=mmap.PROT_READ)
        arr = np.frombuffer(m, dtype, count=int(np.prod(shape)), offset=offset).reshape(shape)
        _madvise_huge(arr.ctypes.data - offset, size)
    dist.barrier()
    if local_rank == 0:
        os.unlink(path)
    return m, arr


def rank_host_bytes(cfg_bytes, shared_bytes, local_world):
    """Pinned host-tier bytes for one of `local_world` ranks: the config's,
    unless the node's memory (after the shared volume and a reserve) does
    not hold that many tiers."""
    if local_world <= 1:
        return cfg_bytes
    try:
        with open("/proc/meminfo") as f:
            total = int(next(l for l in f if l.startswith("MemTotal")).split()[1]) * 1024
    except (OSError, StopIteration, ValueError):
        return cfg_bytes
    # a reserve for the system and 6 GB for each rank's own process
    budget = (total - shared_bytes - (16 << 30) - local_world * (6 << 30)) // local_world
    if budget < (1 << 30):
        raise RuntimeError("host memory too small for %d ranks' brick tiers" % local_world)
    return min(cfg_bytes, budget)


def volume_offset(cfg):
    """Where the host volume starts relative to a cache line: brick boxes
    start `inc` voxels before a brick boundary (a multiple of 64 bytes of z
    for 16^3 f32 bricks), so placing the volume `inc` voxels past a line
    boundary lets each box row begin on a line -- an 88-byte row of a 22^3
    f32 box then spans 2 cache lines instead of 3 (the reads of the host
    tier are bound by the lines they touch)."""
    es = 1 if cfg["gen"] == "fractal" else 4
    return (cfg["inc"] * es) % 64


# Poses of the workloads, as plain numbers: both arms turn them into their
# own camera (libvt's vt_camera for the product, the oracle's camera for the
# reference arm, which must not load libvt.so).  A pose is (W, H, position,
# look, up, right) in float32; h and w come from the camera's own init.
def _unit(v):
    v = np.asarray(v, np.float32)
    return (v / np.sqrt(np.float32((v * v).sum()))).astype(np.float32)


def look_at_pose(W, H, pos, target, up=(0.0, 1.0, 0.0)):
    """Pose at `pos` looking at `target` (right = cross(look, up), the
    reference's basis convention; up re-orthogonalised)."""
    pos = np.asarray(pos, np.float32)
    look = _unit(np.asarray(target, np.float32) - pos)
    upv = np.asarray(up, np.float32)
    right = np.cross(look, upv).astype(np.float32)
    if np.linalg.norm(right) < 1e-6:
        upv = np.array([1, 0, 0], np.float32)
        right = np.cross(look, upv).astype(np.float32)
    upv = np.cross(right, look).astype(np.float32)
    upv /= np.float32(np.linalg.norm(upv))
    right = np.cross(look, upv).astype(np.float32)
    return (W, H, pos, look, upv, right)


def orbit_pose(cfg, frame):
    """Pose on the orbit: position c + r (sin a, 0, cos a), looking at c, up +y,
    right = cross(look, up)."""
    r, step = cfg["orbit"]
    c = (cfg["n"] - 1) / 2.0
    a = math.radians(step * frame)
    pos = np.array([c + r * math.sin(a), c, c + r * math.cos(a)], np.float32)
    look = _unit(np.array([c, c, c], np.float32) - pos)
    up = np.array([0, 1, 0], np.float32)
    return (cfg["W"], cfg["H"], pos, look, up, np.cross(look, up).astype(np.float32))


def static_pose(cfg):
    """The reference camera's initial basis (look -z, up +y), moved to cam_pos."""
    look, up = np.array([0, 0, -1], np.float32), np.array([0, 1, 0], np.float32)
    return (cfg["W"], cfg["H"], np.asarray(cfg["cam_pos"], np.float32), look, up, np.cross(look, up).astype(np.float32))


def catmull_rom(points, frames):
    """Uniform Catmull-Rom spline through `points` (closed), `frames` samples."""
    P = np.asarray(points, np.float64)
    k = len(P)
    out = []
    for f in range(frames):
        u = f * k / frames
        i = int(u)
        t = u - i
        p0, p1, p2, p3 = P[(i - 1) % k], P[i % k], P[(i + 1) % k], P[(i + 2) % k]
        out.append(0.5 * ((2 * p1) + (-p0 + p2) * t + (2 * p0 - 5 * p1 + 4 * p2 - p3) * t * t +
                          (-p0 + 3 * p1 - 3 * p2 + p3) * t * t * t))
    return np.array(out)


def flythrough(rng, n, frames, r_lo, r_hi, ctrl):
    """Positions on a spline through `ctrl` random points at radius
    [r_lo, r_hi] around the volume centre, looking at points of a spline
    through random targets in the volume's inner half."""
    c = (n - 1) / 2.0
    v = rng.standard_normal((ctrl, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    pos = catmull_rom(c + v * rng.uniform(r_lo, r_hi, (ctrl, 1)), frames)
    tgt = catmull_rom(c + rng.uniform(-n / 4, n / 4, (ctrl, 3)), frames)
    return pos, tgt


_PATHS = {}


def path_pose(cfg, frame):
    """Pose `frame` of the workload's seeded Catmull-Rom fly-through (frames
    wrap around)."""
    spec, n = cfg["path"], cfg["n"]
    key = (cfg["seed"], n, spec["frames"])
    if key not in _PATHS:
        _PATHS[key] = flythrough(np.random.default_rng([cfg["seed"], 5]), n, spec["frames"], spec["r"][0],
                                 spec["r"][1], spec["ctrl"])
    pos, tgt = _PATHS[key]
    f = frame % spec["frames"]
    return look_at_pose(cfg["W"], cfg["H"], pos[f], tgt[f])


def frame_pose(cfg, frame):
    if cfg.get("path"):
        return path_pose(cfg, frame)
    return orbit_pose(cfg, frame) if cfg["orbit"] else static_pose(cfg)


def step_poses(cfg, step):
    """The seeded views of one batched step: positions uniform on a sphere
    shell around the volume centre, targets uniform in the inner half,
    resolution drawn uniformly from the config's list."""
    spec, n = cfg["views"], cfg["n"]
    rng = np.random.default_rng([cfg["seed"], 3, step])
    c = (n - 1) / 2.0
    out = []
    for _ in range(spec["n"]):
        v = rng.standard_normal(3)
        pos = c + v / np.linalg.norm(v) * rng.uniform(*spec["r"])
        tgt = c + rng.uniform(-n / 4.0, n / 4.0, 3)
        W, H = spec["res"][int(rng.integers(len(spec["res"])))]
        out.append(look_at_pose(W, H, pos, tgt))
    return out


def vt_cam(vt, cfg, pose):
    """libvt camera (vt_camera) of a pose."""
    W, H, pos, look, up, right = pose
    cam = vt.Camera(H, W, cfg["dist"], cfg["fov"], cfg["fov"]).c
    for i in range(3):
        cam.look[i], cam.up[i], cam.right[i], cam.position[i] = look[i], up[i], right[i], pos[i]
    return cam


def oracle_cam(orc, cfg, pose):
    """The oracle's camera of a pose."""
    W, H, pos, look, up, right = pose
    cam = orc.Camera(H, W, cfg["dist"], cfg["fov"], cfg["fov"])
    for name, v in (("look", look), ("up", up), ("right", right), ("position", pos)):
        setattr(cam.c, name, orc.orc_f3(float(v[0]), float(v[1]), float(v[2])))
    return cam


def frame_camera(vt, cfg, frame):
    return vt_cam(vt, cfg, frame_pose(cfg, frame))


def step_views(cfg, step):
    import visualtur_b200 as vt
    return [vt_cam(vt, cfg, p) for p in step_poses(cfg, step)]


class Workload:
    """Volume (device generated), octree (GPU builder) and renderer."""

    def __init__(self, cfg, torch, device, workdir, need_renderer=True, mode="best", warm=False, share=None):
        """share: None (one process), or (dist, local_rank, local_world) of a
        multi-rank job: the node's ranks then share one host volume (local
        rank 0 generates it and the octree), each rank's pinned brick tier
        fits the node's memory next to the others', and each rank's host
        reads use its share of the cores."""
        import visualtur_b200 as vt
        self.vt, self.cfg = vt, cfg
        n = cfg["n"]
        u8 = cfg["gen"] == "fractal"
        self.esize = 1 if u8 else 4
        vdt = torch.uint8 if u8 else torch.float32
        ndt = np.uint8 if u8 else np.float32
        dist_, local_rank, local_world = share if share else (None, 0, 1)
        vol_bytes = n * n * n * self.esize
        self.host_bytes = rank_host_bytes(cfg.get("host_bytes", 0), vol_bytes if local_world > 1 else 0, local_world)
        self.host_threads = 0 if local_world <= 1 else max(1, (os.cpu_count() or 1) // local_world)
        t0 = time.time()
        times = [t0, t0, t0]
        octree_name = "vol_%s.oct" % cfg["gen"]

        def produce(arr):
            """generate on this GPU, build the octree, copy to `arr`"""
            dvol = torch.empty(n * n * n, dtype=vdt, device=device)
            if cfg["gen"] == "sphere":
                c = (n - 1) / 2.0
                vt.generate_volume(vt.VT_GEN_SPHERE, cfg["seed"], (n, n, n), (c, c, c, 0.25),
                                   device_ptr=dvol.data_ptr())
            elif u8:
                vt.generate_volume(vt.VT_GEN_FRACTAL_U8, cfg["seed"], (n, n, n), cfg["spheres"],
                                   device_ptr=dvol.data_ptr())
            else:
                vt.generate_volume(vt.VT_GEN_BLOBS, cfg["seed"], (n, n, n), cfg["blobs"], device_ptr=dvol.data_ptr())
            torch.cuda.synchronize()
            times[0] = time.time()
            vt.build_octree_device(dvol.data_ptr(), vt.VT_U8 if u8 else vt.VT_F32, (n, n, n), cfg["iso"],
                                   self.octree_path)
            times[1] = time.time()
            torch.from_numpy(arr.reshape(-1)).copy_(dvol)
            torch.cuda.synchronize()
            del dvol
            torch.cuda.empty_cache()
            times[2] = time.time()

        # host copy of the volume: the out-of-core source and the CPU baseline's input
        if local_world <= 1:
            self.octree_path = os.path.join(workdir, octree_name)
            self._host_map, arr = huge_page_array((n * n * n,), ndt, volume_offset(cfg))
            produce(arr)
            octree_bytes = None
        else:
            # the octree file travels from local rank 0 as bytes
            self.octree_path = os.path.join(workdir, octree_name)
            self._host_map, arr = shared_host_array(dist_, local_rank, "vol", (n * n * n,), ndt, volume_offset(cfg),
                                                    produce)
            blob = [open(self.octree_path, "rb").read() if local_rank == 0 else None]
            dist_.broadcast_object_list(blob, src=0)
            if local_rank != 0:
                with open(self.octree_path, "wb") as f:
                    f.write(blob[0])
            octree_bytes = len(blob[0])
        self.volume = arr.reshape(n, n, n)
        t1, t2, t3 = times
        log("setup: generate %.1fs octree %.1fs host copy %.1fs%s" %
            (t1 - t0, t2 - t1, t3 - t2, "" if octree_bytes is None else
             " (volume shared by %d ranks, %d host threads and %.1f GB pinned tier each)" %
             (local_world, self.host_threads, self.host_bytes / 2 ** 30)))
        self.r = None
        if need_renderer:
            self.fm = vt.FileManager.wrap(self.volume)
            self.oc = vt.Octree(self.octree_path)
            self.brick = 1 << (self.oc.nLevels - cfg["levelC"])
            t4 = time.time()
            self.r = self.renderer(mode, warm)
            log("setup: renderer %.1fs (device slots %d, host slots %d, %d B/brick)" %
                ((time.time() - t4,) + self.slots))

    def params(self, brick=None):
        """Renderer parameters for brick edge `brick` (default: the config's
        levelCubes); cache slots from the config's device / host bytes."""
        vt, cfg = self.vt, self.cfg
        edge = brick or self.brick
        levelC = self.oc.nLevels - int(round(math.log2(edge)))
        D = edge + 2 * cfg["inc"]
        slot = (D ** 3 * self.esize + 15) // 16 * 16
        dev = cfg.get("dev_bytes", 0) // slot or 8 ** levelC
        host = self.host_bytes // slot or 8 ** levelC
        self.slots = (dev, host, slot)
        return vt.make_params(W=cfg["W"], H=cfg["H"], octreeFile=None, hdf5File=None, octreeLevel=cfg["levelO"],
                              levelCubes=levelC, dimCube=edge, cubeInc=cfg["inc"], distance=cfg["dist"],
                              fov_H=cfg["fov"], fov_W=cfg["fov"], maxElementsCache=dev, maxElementsCache_CPU=host)

    def renderer(self, mode, warm=False, brick=None):
        """A renderer in `mode` (cold cache unless the workload is resident
        or `warm`: every needed brick preloaded, for steady-state profiles)."""
        opt = self.vt.default_options(resident=self.cfg["resident"], record_hits=0, host_threads=self.host_threads,
                                      preload=1 if (self.cfg["resident"] or warm) else 0,
                                      shared_aprons=SHARED_APRONS, **MODES[mode]["opts"])
        return self.vt.visualTur(self.params(brick), opt, volume=self.fm, octree=self.oc)

    def train_prefetcher(self, torch, poses=20000, paths=100, W=240, H=135, epochs=30):
        """Learned prefetch: traces from random fly-throughs (radius
        2500-3500 scaled to the volume) rendered at W x H by a resident
        renderer with the access log, then GPU training of the network."""
        from visualtur_b200 import prefetch as pf
        vt, cfg, n = self.vt, self.cfg, self.cfg["n"]
        t0 = time.time()
        p = vt.make_params(W=W, H=H, octreeFile=None, hdf5File=None, octreeLevel=cfg["levelO"],
                           levelCubes=cfg["levelC"], dimCube=1 << (self.oc.nLevels - cfg["levelC"]),
                           cubeInc=cfg["inc"], distance=cfg["dist"], fov_H=cfg["fov"], fov_W=cfg["fov"])
        tr = vt.visualTur(p, vt.default_options(resident=1, record_trace=1, trace_level=pf.TRACE_LEVEL,
                                                record_hits=0), volume=self.fm, octree=self.oc)
        scale = n / 2048.0
        X, Y = pf.collect_traces(tr, n, W, H, cfg["fov"], np.random.default_rng(7), paths, poses // paths,
                                 *(cfg["path"]["r"] if cfg.get("path") else (2500 * scale, 3500 * scale)),
                                 dist=cfg["dist"])
        bricks = tr.brick_list()
        tr.close()
        torch.cuda.empty_cache()
        t1 = time.time()
        P = pf.Prefetcher(n, cfg["fov"], cfg["levelC"], bricks, seed=11)
        hist = P.train(torch, X, Y, epochs=epochs, batch=256, lr=1e-3)
        t2 = time.time()
        self.train_info = {"poses": int(X.shape[0]), "trace_res": [W, H], "positive_frac": round(float(Y.mean()), 4),
                           "epochs": epochs, "loss_first": round(hist[0], 4), "loss_last": round(hist[-1], 4),
                           "trace_s": round(t1 - t0, 1), "train_s": round(t2 - t1, 1)}
        log("prefetch: %d traces in %.1fs, training %.1fs, loss %.4f -> %.4f" %
            (X.shape[0], t1 - t0, t2 - t1, hist[0], hist[-1]))
        return P


def roofline(stats_frames, trace_ms, pixels, traffic_per_ray=None, esize=4):
    """Algorithmic bytes of the march (4 B voxels, 8 taps per sample, 6 extra
    samples per hit for the normal) + 4 B per output pixel, over the trace
    kernels' device time."""
    samples = sum(s["samples"] for s in stats_frames)
    hits = sum(s["hits"] for s in stats_frames)
    b_alg = esize * 8 * (samples + 6 * hits) + 4 * pixels
    peak, src = HBM_FALLBACK_GBS, "fallback"
    try:
        mp = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
        peak, src = float(mp["hbm_gbs"]), "measured"
    except Exception:
        pass
    ach = b_alg / (trace_ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": round(ach, 1), "peak": peak, "peak_source": src, "unit": "GB/s",
            "frac": round(ach / peak, 4),
            "traffic": round(traffic_per_ray * pixels / len(stats_frames)) if traffic_per_ray else None,
            "bytes_alg_per_launch": b_alg / len(stats_frames),
            "kernel": "k_trace"}


def workload_config(cfg, name, world):
    """The `config` of both arms' lines: what the workload is, nothing the
    renderer chose (the product's tuned settings go under "renderer")."""
    conf = {"workload": cfg["workload"], "name": name,
            "l2": "flushed (256 MB write) between frames" if cfg["l2flush"] else "inputs larger than L2",
            "parallelism": "replicas" if world > 1 else "single GPU"}
    if "views" in cfg:
        conf.update(views_per_launch=cfg["views"]["n"], resolutions=[list(r) for r in cfg["views"]["res"]])
    else:
        conf.update(W=cfg["W"], H=cfg["H"])
    return conf


def hint_use(P, conf):
    """How the timed run uses the learned prefetcher: a network is trained
    for every out-of-core workload, and the paging tuner decides whether its
    hints are sent (threshold) or not."""
    if P is None:
        return "off"
    thr = conf.get("hint_threshold")
    if thr is None:
        return "trained; hints off (tuner's choice)" if "hint_threshold" in conf else "trained; no hints on batched views"
    return "hints on (threshold %g)" % thr


def sample_pose(cfg, step):
    """The pose the CPU baseline renders for `step`: the frame's pose, or the
    first view of a batched step."""
    return step_poses(cfg, step)[0] if "views" in cfg else frame_pose(cfg, step)


def cpu_baseline(cfg, wl, octree_path, budget_s, nthreads=0, step=0, octree=None, per_ray=None, keep=False):
    """Oracle (CPU restatement of the reference algorithm) on a bounded ray
    sample of step `step`'s camera; returns rays/s (with "per_ray_s", the
    probe's seconds per ray, to size later samples without probing)."""
    from oracle import oracle as orc
    o = octree if octree is not None else orc.Octree(octree_path)
    cam = oracle_cam(orc, cfg, sample_pose(cfg, step))
    c = cam.c
    n = c.W * c.H
    stride = 1
    # probe a sparse sample, then size the sample to the time budget
    if per_ray is None:
        t0 = time.perf_counter()
        orc.render(o, wl.volume, cam, cfg["levelO"], cfg["levelC"], cfg["inc"], nthreads=nthreads, ray_stride=257)
        dt = max(time.perf_counter() - t0, 1e-6)
        per_ray = dt / (n // 257 + 1)
    stride = max(1, int(math.ceil(n * per_ray / budget_s)))
    t0 = time.perf_counter()
    reps = 0
    rays = 0
    while True:
        out = orc.render(o, wl.volume, cam, cfg["levelO"], cfg["levelC"], cfg["inc"], nthreads=nthreads,
                         ray_stride=stride)
        rays += (n + stride - 1) // stride
        reps += 1
        if time.perf_counter() - t0 > budget_s * 0.5 or stride > 1:
            break
    el = time.perf_counter() - t0
    threads = nthreads or os.cpu_count()
    res = {"value": round(rays / el, 1), "unit": "rays/s", "cores": threads, "kind": "port",
           "sample": "%d x every %d-th ray of a %dx%d view of step %d (%d rays, %.1f s)" %
                     (reps, stride, c.W, c.H, step, rays, el), "per_ray_s": el / max(rays, 1)}
    if keep:
        res["_oracle"] = (out, stride)
    return res


def oracle_mismatch(product_rgba, oracle):
    """Rays of the oracle's sample whose product RGBA differs in any bit; a
    NaN colour (a 0/0 refinement on integer voxels, on both sides) counts as
    equal to a NaN, whatever the NaN's bits."""
    out, stride = oracle
    pa, pb = product_rgba[::stride], out["rgba"][::stride]
    nan_a, nan_b = np.isnan(pa), np.isnan(pb)
    diff = (pa.view(np.uint32) != pb.view(np.uint32)) & ~(nan_a & nan_b)
    return {"oracle_checked_rays": int(pa.shape[0]), "oracle_mismatch_rays": int(diff.any(axis=1).sum()),
            "oracle_nan_rays": int(nan_b.any(axis=1).sum()), "oracle_hits": int((out["node"][::stride] != 0).sum())}


# ----------------------------------------------------------------------------- arms
class Launcher:
    """Renders consecutive orbit frames in launches of `batch` views; with a
    predictor, hands the renderer the predicted bricks of this launch and the
    next one: their host-tier reads overlap this launch's first pass, and
    those still absent after its last pass are filled for the next launch."""

    def __init__(self, wl, r, cfg, torch, dev, stream, batch=1, predictor=None, threshold=0.25, warm=False):
        self.wl, self.r, self.cfg, self.torch, self.stream = wl, r, cfg, torch, stream
        self.warm = warm
        self.batch, self.P, self.thr = batch, predictor, threshold
        W, H = cfg["W"], cfg["H"]
        # two sets of output buffers: a launch renders into one while the
        # images of the launch before are copied out of the other
        self.sets = [[(torch.empty(W * H * 4, dtype=torch.float32, device=dev),
                       torch.empty(W * H * 3, dtype=torch.uint8, device=dev)) for _ in range(batch)]
                     for _ in range(2)]
        self.cur = 0

    @property
    def bufs(self):
        return self.sets[self.cur]

    def cams(self, f0, n):
        return [frame_camera(self.wl.vt, self.cfg, f0 + i) for i in range(n)]

    def rays(self, cams):
        return sum(c.W * c.H for c in cams)

    def outputs(self, cams):
        """(device RGB8 buffer, bytes) of each frame of the last launch"""
        return [(self.bufs[b][1], c.W * c.H * 3) for b, c in enumerate(cams)]

    hint_s = 0.0

    def hint(self, cams, f=None):
        """The network's prediction for `cams` (this launch's frames and the
        next launch's) on the device: vt_prefetch_predict requests the
        predicted absent bricks, which load on the cache's side stream while
        the launch renders -- no synchronisation or host-side selection."""
        if self.P is None or not cams or self.thr is None:
            return
        t0 = time.perf_counter()
        self.r.prefetch_predict(self.P.mlp, list(cams), self.cfg["n"], self.cfg["fov"], self.thr,
                                stream=self.stream.cuda_stream)
        self.hint_s += time.perf_counter() - t0

    def launch(self, cams, next_cams=(), f=None):
        self.hint(list(cams) + list(next_cams), f)
        sp = self.stream.cuda_stream
        if self.batch == 1:
            self.r.set_camera(cams[0])
            self.r.updateVisibleCubes(self.bufs[0][0], self.bufs[0][1], stream=sp)
            return
        views = []
        for c, (a, b) in zip(cams, self.bufs):
            v = self.wl.vt.vt_view()
            v.cam, v.dev_rgba, v.dev_rgb8 = c, a.data_ptr(), b.data_ptr()
            views.append(v)
        self.r.render_batch(views, stream=sp)


class ViewLauncher:
    """Batched workload: each step is one launch of that step's views (mixed
    resolutions, RGB8 output); `plain` renders the same views one per launch
    instead.  With a predictor, the hint names the predicted bricks of this
    step's and the next step's views."""
    batch = 1

    def __init__(self, wl, r, cfg, torch, dev, stream, predictor=None, threshold=0.25, warm=False, plain=False):
        self.wl, self.r, self.cfg, self.torch, self.stream = wl, r, cfg, torch, stream
        self.warm, self.plain, self.P, self.thr = warm, plain, predictor, threshold
        spec = cfg["views"]
        maxpix = max(w * h for w, h in spec["res"])
        self.sets = [[torch.empty(maxpix * 3, dtype=torch.uint8, device=dev) for _ in range(spec["n"])]
                     for _ in range(2)]
        self.cur = 0

    @property
    def bufs(self):
        return self.sets[self.cur]

    def cams(self, f0, n):
        return [step_views(self.cfg, f0 + i) for i in range(n)]

    def rays(self, items):
        return sum(c.W * c.H for views in items for c in views)

    def outputs(self, items):
        return [(b, c.W * c.H * 3) for c, b in zip(items[-1], self.bufs)]

    hint_s = 0.0

    def hint(self, items):
        if self.P is None or not items or self.thr is None:
            return
        t0 = time.perf_counter()
        self.r.prefetch_predict(self.P.mlp, [c for views in items for c in views], self.cfg["n"], self.cfg["fov"],
                                self.thr, stream=self.stream.cuda_stream)
        self.hint_s += time.perf_counter() - t0

    def launch(self, items, next_items=(), f=None):
        self.hint(list(items) + list(next_items))
        sp = self.stream.cuda_stream
        views = []
        for c, b in zip(items[0], self.bufs):
            v = self.wl.vt.vt_view()
            v.cam, v.dev_rgba, v.dev_rgb8 = c, None, b.data_ptr()
            views.append(v)
        if self.plain:
            for v in views:
                self.r.render_batch([v], stream=sp)
        else:
            self.r.render_batch(views, stream=sp)


def product_frame_rgba(vtm, r, cam, torch, dev, stream):
    """RGBA of one view rendered by renderer `r` (any resolution)."""
    buf = torch.empty(cam.W * cam.H * 4, dtype=torch.float32, device=dev)
    v = vtm.vt_view()
    v.cam, v.dev_rgba, v.dev_rgb8 = cam, buf.data_ptr(), None
    with torch.cuda.stream(stream):
        r.render_batch([v], stream=stream.cuda_stream)
    torch.cuda.synchronize()
    return buf.cpu().numpy().reshape(-1, 4)


def launch_split(start, frames, batch):
    """The launches that render frames [start, start + frames) `batch` at a
    time: (first frame, frames in it, frames in the next launch)."""
    out = []
    f, end = start, start + frames
    while f < end:
        n = min(batch, end - f)
        out.append((f, n, min(batch, end - f - n)))
        f += n
    return out


def timed_frames(L, frame0, warmup, steps, dist, clocks=None, flush_l2=False, label="timed", e2e=None):
    """Renders `warmup` then `steps` consecutive frames in launches of
    L.batch; returns device ms (CUDA events on the launching stream) and
    stats per launch, and the number of frames in each.

    With `e2e` (a dict, filled in): the end-to-end view of the same timed
    steps -- every launch's RGB8 images are copied into pinned host memory
    on a copy stream (overlapping the next launch, which renders into the
    other set of output buffers), and the host wall clock runs from the
    first launch to the last image on the host."""
    torch, r, stream = L.torch, L.r, L.stream
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=stream.device) if flush_l2 else None
    with torch.cuda.stream(stream):
        f = frame0
        while f < frame0 + warmup:
            # whole launches, as timed: buffers sized by the views per launch
            # are allocated here, not in the first timed launch
            n = L.batch
            L.launch(L.cams(f, n), L.cams(f + n, n), f)
            f += n
        torch.cuda.synchronize()
        if not L.cfg["resident"] and not L.warm:
            r.drop_cache()     # every timed run starts from a cold cache: all loading is timed
            if L.P is not None:
                L.P.reset_hints()
        r.reset_stats()
        launches = [(f, n, L.cams(f, n), L.cams(f + n, nxt))
                    for f, n, nxt in launch_split(frame0 + warmup, steps, L.batch)]
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in launches]
        per = []
        if e2e is not None:
            cs = torch.cuda.Stream(device=stream.device)
            copied = [torch.cuda.Event() for _ in launches]
            maxb = max(b.numel() for b, _ in L.outputs(launches[0][2]))
            host8 = [torch.empty(maxb, dtype=torch.uint8, pin_memory=True) for _ in range(64)]
            d2h = rays = 0
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        if clocks:
            clocks.start()
        L.hint_s = 0.0
        torch.cuda.nvtx.range_push(label)     # the timed region, for launch lists (ncu --nvtx-include)
        t0 = time.perf_counter()
        for k, (f0, n, cams, nxt) in enumerate(launches):
            L.cur = k % 2
            if e2e is not None and k >= 2:
                stream.wait_event(copied[k - 2])      # its output buffers are free again
            if flush is not None:
                flush.zero_()
            ev[k][0].record(stream)
            L.launch(cams, nxt, f0)
            ev[k][1].record(stream)
            if e2e is not None:
                cs.wait_event(ev[k][1])
                with torch.cuda.stream(cs):
                    for i, (b, nb) in enumerate(L.outputs(cams)):
                        host8[i][:nb].copy_(b[:nb], non_blocking=True)
                        d2h += nb
                copied[k].record(cs)
                rays += L.rays(cams)
            per.append(r.stats())
        torch.cuda.synchronize()
        wall_ms = (time.perf_counter() - t0) * 1e3
        torch.cuda.nvtx.range_pop()
        L.cur = 0
        L.timed_hint_s = L.hint_s
        if dist:
            dist.barrier()
    clk = clocks.stop() if clocks else None
    if e2e is not None:
        e2e.update(wall_ms=max_over_ranks(dist, torch, wall_ms, stream.device), rays=rays, d2h=d2h)
    return [a.elapsed_time(b) for a, b in ev], per, launches, clk


def frame_deltas(per_frame):
    out, prev = [], None
    for s in per_frame:
        out.append(dict(s) if prev is None else {k: (s[k] - prev[k]) if isinstance(s[k], int) else s[k] for k in s})
        prev = s
    return out


# ----------------------------------------------------------------------------- replicas
def replica_first_frame(rank, warmup, steps):
    """Replicas render disjoint stretches of the workload: rank r starts at
    frame r * (warmup + steps) (no data is exchanged between GPUs)."""
    return rank * (warmup + steps)


def max_over_ranks(dist, torch, value, device):
    """The largest of the ranks' values (a time in ms): a job is as slow as
    its slowest replica.  Every rank must call it at the same point."""
    if not dist:
        return value
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(rays_per_rank, world, t_max_ms):
    """Whole-job throughput: every rank's rays over the slowest rank's time."""
    return rays_per_rank * world / (t_max_ms * 1e-3)


def frame_digest(r, cam):
    """SHA-256 of the float RGBA frame renderer `r` makes from `cam`."""
    import hashlib
    r.set_camera(cam)
    rgba, _ = r.render_host(rgb8=False)
    return hashlib.sha256(rgba.tobytes()).hexdigest()


def make_launcher(wl, r, cfg, torch, dev, stream, batch, predictor=None, warm=False, plain=False):
    if "views" in cfg:
        return ViewLauncher(wl, r, cfg, torch, dev, stream, predictor=predictor, warm=warm, plain=plain)
    return Launcher(wl, r, cfg, torch, dev, stream, batch=batch, predictor=predictor, warm=warm)


# (frames per launch, lookahead, absent-brick candidates a ray may set aside)
PAGING_CANDIDATES = ((8, 2, 0), (4, 2, 0), (2, 2, 0), (1, 2, 0), (1, 0, 0),
                     (16, 0, 0), (8, 0, 0), (4, 0, 0), (2, 0, 0), (4, 1, 0),
                     (4, 2, 4), (2, 2, 4), (4, 0, 4), (2, 0, 4), (1, 0, 4), (4, 0, 2))
HINT_THRESHOLDS = (None, 0.25, 0.8)                             # besides 0.5; None = no hints
DEMAND_BATCHES = (8192,)                                        # besides 0 = no bound
VIEWS_PAGING = ((2, 0), (0, 0), (2, 2), (0, 2))                 # batched views: (lookahead, skip)


def tune_paging(wl, cfg, torch, dev, stream, P, f0, frames=96):
    """Frames per launch, lookahead, absent-brick candidates set aside per
    pass and the prefetch-hint threshold for an out-of-core fly-through:
    each candidate renders the same `frames` frames (another stretch of the
    path than the timed one, as long as it) from a cold cache; the fastest
    total device time wins.  Batching more frames per
    launch amortises launches and host work but needs their joint working
    set in the device cache, and hints help only while the cache has room
    for them -- a small cache thrashes, which only a cold-cache run shows."""
    def run(b, la, thr, sk=0, sa=SHARED_APRONS, db=0, start=None):
        s0 = f0 if start is None else start
        wl.r.set_tuning(lookahead=la, skip=sk, shared_aprons=sa, demand_batch=db)
        L = make_launcher(wl, wl.r, cfg, torch, dev, stream, b, predictor=P)
        L.thr = thr
        wl.r.drop_cache()
        if P is not None:
            P.reset_hints()
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            torch.cuda.synchronize()
            a.record(stream)
            # the last launch holds the frames that are left, as in the timed
            # run (a full one would charge larger batches for frames past the
            # stretch)
            for f, n, nxt in launch_split(s0, frames, b):
                L.launch(L.cams(f, n), L.cams(f + n, nxt), f)
            e.record(stream)
            torch.cuda.synchronize()
        ms = a.elapsed_time(e)
        log("autotune: %d frames/launch, lookahead %d, hints %s, skip %d, shared aprons %d, demand batch %d "
            "-> %.1f ms for %d frames" % (b, la, thr, sk, sa, db, ms, frames))
        return {"frames_per_launch": b, "lookahead": la, "hint_threshold": thr, "skip": sk, "shared_aprons": sa,
                "demand_batch": db, "ms": round(ms, 2)}

    thr0 = 0.5 if P is not None else None
    rows = [run(b, la, thr0, sk) for b, la, sk in PAGING_CANDIDATES]
    # one cold stretch varies by a few per cent and favours what suits it:
    # the three fastest also run on a second stretch and are ranked by the
    # sum of both
    f1 = f0 + frames + 53
    for r0 in sorted(rows, key=lambda x: x["ms"])[:3]:
        again = run(r0["frames_per_launch"], r0["lookahead"], thr0, r0["skip"], start=f1)
        r0["ms2"] = again["ms"]
    rank = lambda x: x["ms"] + x.get("ms2", x["ms"] * 10)
    best = min(rows, key=rank)
    for r0 in rows:
        r0.pop("ms2", None)
    # the settings below vary the chosen schedule and compete with it alone
    # (on the first stretch, where all of them ran)
    cands = [best]

    def add(r):
        rows.append(r)
        cands.append(r)
        return min(cands, key=lambda x: x["ms"])

    if P is not None:
        for t in HINT_THRESHOLDS:
            best = add(run(best["frames_per_launch"], best["lookahead"], t, best["skip"]))
    if best["skip"]:
        best = add(run(best["frames_per_launch"], best["lookahead"], best["hint_threshold"], 2))
    if SHARED_APRONS:
        # under eviction churn a brick loaded without its x/y aprons may have
        # to read them later (its neighbours gone): whole bricks can win
        best = add(run(best["frames_per_launch"], best["lookahead"], best["hint_threshold"], best["skip"], 0))
    if wl.r.tuning()["spec_async"]:
        # a cold start's demand bricks past a batch load on the side stream
        # while the next pass runs
        for db in DEMAND_BATCHES:
            best = add(run(best["frames_per_launch"], best["lookahead"], best["hint_threshold"], best["skip"],
                           best["shared_aprons"], db))
    wl.r.set_tuning(lookahead=best["lookahead"], skip=best["skip"], shared_aprons=best["shared_aprons"],
                    demand_batch=best["demand_batch"])
    wl.r.drop_cache()
    return best, rows


def autotune(args, wl, cfg, torch, dev, stream, frame0, batch):
    """Kernel schedule sweep (tile x unroll x persistent) on the renderer;
    for the batched workload first the brick edge {8, 16, 32} at the
    default schedule, keeping the fastest renderer."""
    from visualtur_b200 import autotune as at
    bricks = None
    if "views" in cfg and not args.no_brick_sweep:
        L0 = make_launcher(wl, wl.r, cfg, torch, dev, stream, batch)
        items = L0.cams(frame0, 1)
        rows = []
        for b in (8, 16, 32):
            r = wl.r if b == wl.brick else wl.renderer(args.mode, brick=b)
            L = make_launcher(wl, r, cfg, torch, dev, stream, batch)
            ms = at.time_frames(torch, r, lambda rr, i, s_: L.launch(items), frames=1, warmup=1, stream=stream)
            rows.append({"brick": b, "ms": round(ms, 3)})
            log("autotune: brick %d -> %.2f ms" % (b, ms))
            if r is not wl.r:
                r.close()
        best_b = min(rows, key=lambda x: x["ms"])["brick"]
        if best_b != wl.brick:
            wl.r.close()
            wl.brick = best_b
            wl.r = wl.renderer(args.mode)
        bricks = rows
    Lt = make_launcher(wl, wl.r, cfg, torch, dev, stream, batch)
    items = Lt.cams(frame0, batch)
    frames = 1 if "views" in cfg else 3
    best, table = at.tune_schedule(torch, wl.r, lambda rr, i, s_: Lt.launch(items), frames=frames, stream=stream)
    if bricks:
        best = dict(best, brick=wl.brick)
    if "views" in cfg and not cfg["resident"] and args.skip is None:
        # lookahead requests and set-aside candidates, from a cold cache on
        # two batches of another stretch of the workload
        stretch = [Lt.cams(frame0 + 50 + k, batch) for k in range(2)]
        prow = []
        for la, sk in VIEWS_PAGING:
            wl.r.set_tuning(lookahead=la, skip=sk)
            wl.r.drop_cache()
            a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            with torch.cuda.stream(stream):
                torch.cuda.synchronize()
                a.record(stream)
                for it in stretch:
                    Lt.launch(it)
                e.record(stream)
                torch.cuda.synchronize()
            prow.append({"lookahead": la, "skip": sk, "ms": round(a.elapsed_time(e), 2)})
            log("autotune: lookahead %d, skip %d -> %.1f ms for 2 batches" % (la, sk, prow[-1]["ms"]))
        bp = min(prow, key=lambda x: x["ms"])
        wl.r.set_tuning(lookahead=bp["lookahead"], skip=bp["skip"])
        best = dict(best, lookahead=bp["lookahead"], skip=bp["skip"])
        table = table + prow
    log("autotune: best %s" % best)
    if not cfg["resident"]:
        wl.r.drop_cache()
    return {"best": best, "points": len(table) + len(bricks or []), "bricks": bricks, "table": table}


def run_ours(args, cfg, rank, world, torch, dist):
    dev = torch.device("cuda", int(os.environ.get("LOCAL_RANK", 0)))
    torch.cuda.set_device(dev)
    work = tempfile.mkdtemp(prefix="vtbench_")
    M = MODES[args.mode]
    local_world = int(os.environ.get("LOCAL_WORLD_SIZE", world))
    share = (dist, int(os.environ.get("LOCAL_RANK", 0)), local_world) if (dist is not None and local_world > 1) else None
    wl = Workload(cfg, torch, dev, work, mode=args.mode, warm=args.warm, share=share)
    stream = torch.cuda.Stream(device=dev)
    frame0 = replica_first_frame(rank, args.warmup, args.steps)
    batch = 1 if (cfg["resident"] or "views" in cfg) else M["batch"]
    P = wl.train_prefetcher(torch) if (M["learned"] and not cfg["resident"] and not args.no_learned) else None
    tune = None
    paging = None
    if args.paging and not cfg["resident"] and "views" not in cfg:
        v = args.paging.split(",")
        fixed = {"frames_per_launch": int(v[0]), "lookahead": int(v[1]),
                 "hint_threshold": float(v[2]) if len(v) > 2 and v[2] not in ("", "none") else None,
                 "skip": int(v[3]) if len(v) > 3 else 0}
        wl.r.set_tuning(lookahead=fixed["lookahead"], skip=fixed["skip"])
        batch = fixed["frames_per_launch"]
        paging = {"best": fixed, "table": []}
    elif M["autotune"] and not args.no_autotune and not cfg["resident"] and "views" not in cfg:
        # a stretch of the fly-through away from the timed frames
        # as many frames as the timed region, from a cold cache: how much
        # speculation pays depends on the horizon it is judged over
        paging, prow = tune_paging(wl, cfg, torch, dev, stream, P, frame0 + args.warmup + args.steps + 97,
                                   frames=max(args.steps, 8))
        batch = paging["frames_per_launch"]
        paging = {"best": paging, "table": prow}
    if args.skip is not None:
        wl.r.set_tuning(skip=args.skip)
    if not cfg["resident"]:
        wl.r.set_tuning(spec_async=args.spec_async, wavefront=args.wavefront)
        if args.demand_batch is not None:
            wl.r.set_tuning(demand_batch=args.demand_batch)
    if M["autotune"] and not args.no_autotune:
        tune = autotune(args, wl, cfg, torch, dev, stream, frame0, batch)
        if args.skip is not None:      # the brick sweep may have built a new renderer
            wl.r.set_tuning(skip=args.skip)
        if not cfg["resident"]:
            wl.r.set_tuning(spec_async=args.spec_async, wavefront=args.wavefront)
            if args.demand_batch is not None:
                wl.r.set_tuning(demand_batch=args.demand_batch)
    if P is not None:
        P.set_bricks(wl.r.brick_list(), wl.oc.nLevels - int(round(math.log2(wl.brick))))
    L = make_launcher(wl, wl.r, cfg, torch, dev, stream, batch, predictor=P, warm=args.warm)
    if paging and P is not None:
        L.thr = paging["best"]["hint_threshold"]
    skip_used = wl.r.tuning()["skip"]
    wave_used = wl.r.tuning()["wavefront"]
    aprons_used = wl.r.tuning()["shared_aprons"]
    batch_used = wl.r.tuning()["demand_batch"]
    e2e_raw = {}
    ms, per, launches, clk = timed_frames(L, frame0, args.warmup, args.steps, dist, Clocks(dev.index),
                                          cfg["l2flush"], e2e=e2e_raw)
    tot_ms = sum(ms)
    st = wl.r.stats()
    ld = frame_deltas(per)
    slow = sorted(range(len(per)), key=lambda k: -per[k]["ms_last_frame"])[:3]
    log("timed: slowest launches (index: host ms, stall ms, wait ms, trace ms, device ms) " + ", ".join(
        "%d: %.2f %.2f %.2f %.2f %.2f" % (k, per[k]["ms_last_frame"], per[k]["ms_stall_last_frame"],
                                          per[k]["ms_wait_last_frame"], per[k]["ms_trace_last_frame"], ms[k])
        for k in slow))
    trace_tot = sum(s["ms_trace_last_frame"] for s in per)
    rays_rank = sum(L.rays(cams) for _, _, cams, _ in launches)
    t_max = max_over_ranks(dist, torch, tot_ms, dev)
    value = replica_value(rays_rank, world, t_max)
    # end to end through the public API over the timed steps themselves:
    # poses in, every RGB8 image back in pinned host memory (wall clock from
    # the first launch to the last image, max over ranks)
    import ctypes
    e2e_steps = args.steps
    e2e = {"value": round(e2e_raw["rays"] * world / (e2e_raw["wall_ms"] * 1e-3), 1), "unit": "rays/s",
           "h2d_bytes_per_step": ctypes.sizeof(wl.vt.vt_camera) * (cfg["views"]["n"] if "views" in cfg else 1),
           "d2h_bytes_per_step": int(e2e_raw["d2h"] / e2e_steps),
           "ms_per_step": round(e2e_raw["wall_ms"] / e2e_steps, 4), "steps": e2e_steps,
           "note": "the timed steps themselves: host wall clock from the first render call (vt_render / "
                   "vt_render_batch; camera poses in, brick transfers inside) to the last RGB8 image copied to "
                   "pinned host memory (copies on a second stream, overlapping the next launch)"}
    # one frame of the timed workload through the product renderer, for the
    # oracle comparison of the CPU baseline's ray sample
    product_sample = product_frame_rgba(wl.vt, wl.r, vt_cam(wl.vt, cfg, sample_pose(cfg, frame0 + args.warmup)),
                                        torch, dev, stream)
    # with hints on, the same timed stretch with them off: what the learned
    # prefetch gains on this workload (stall, device-cache hit rate, time)
    learned_gain = None
    if P is not None and getattr(L, "thr", None) is not None and "views" not in cfg:
        thr = L.thr
        L.thr = None
        offms, offper, _, _ = timed_frames(L, frame0, args.warmup, args.steps, dist, label="hints_off")
        L.thr = thr
        so = wl.r.stats()
        learned_gain = {
            "hint_threshold": thr,
            "ms_per_step_on": round(t_max / args.steps, 4),
            "ms_per_step_off": round(max_over_ranks(dist, torch, sum(offms), dev) / args.steps, 4),
            "stall_ms_per_step_on": round(sum(x["ms_stall_last_frame"] for x in per) / args.steps, 4),
            "stall_ms_per_step_off": round(sum(x["ms_stall_last_frame"] for x in offper) / args.steps, 4),
            "device_hit_rate_on": round(st["device_hits"] / max(1, st["device_hits"] + st["device_misses"]), 5),
            "device_hit_rate_off": round(so["device_hits"] / max(1, so["device_hits"] + so["device_misses"]), 5),
            "passes_per_launch_on": round(sum(x["passes"] for x in per) / len(per), 3),
            "passes_per_launch_off": round(sum(x["passes"] for x in offper) / len(offper), 3)}
    # the plain LRU renderer on the same steps, for comparison
    plain = None
    check = None
    if args.mode != "plain" and not cfg["resident"] and not args.no_plain:
        # the same frames from both renderers must be identical
        check = {"frames": [frame0 + args.warmup + k * max(1, args.steps // 4) for k in range(4)]}
        if "views" not in cfg:
            check["best"] = [frame_digest(wl.r, frame_camera(wl.vt, cfg, f)) for f in check["frames"]]
        wl.r.close()
        rp = wl.renderer("plain")
        if "views" not in cfg:
            check["plain"] = [frame_digest(rp, frame_camera(wl.vt, cfg, f)) for f in check["frames"]]
            rp.drop_cache()
            rp.reset_stats()
        Lp = make_launcher(wl, rp, cfg, torch, dev, stream, 1, plain=True)
        pms, pper, _, _ = timed_frames(Lp, frame0, args.warmup, args.steps, dist, label="plain")
        ps = rp.stats()
        p_max = max_over_ranks(dist, torch, sum(pms), dev)
        plain = {"value": round(replica_value(rays_rank, world, p_max), 1), "unit": "rays/s",
                 "ms_per_step": round(p_max / args.steps, 4),
                 "stall_ms_per_step": round(sum(s["ms_stall_last_frame"] for s in pper) / args.steps, 4),
                 "passes_per_step": round(sum(s["passes"] for s in pper) / args.steps, 3),
                 "device_hit_rate": round(ps["device_hits"] / max(1, ps["device_hits"] + ps["device_misses"]), 5),
                 "bricks_loaded": ps["bricks_loaded_disk"]}
        rp.close()
    if rank != 0:
        return None
    W, H = cfg["W"], cfg["H"]
    if "views" in cfg:
        conf = {"views_per_launch": cfg["views"]["n"], "resolutions": [list(r) for r in cfg["views"]["res"]],
                "rays_per_step": round(rays_rank / args.steps), "skip": skip_used}
    else:
        conf = {"W": W, "H": H, "frames_per_launch": batch, "skip": skip_used,
                "wavefront": wave_used}
    if not cfg["resident"]:
        conf["shared_aprons"] = aprons_used
        conf["demand_batch"] = batch_used
        conf["host_tier_bytes"] = wl.host_bytes
        if P is not None and "views" not in cfg:
            conf["hint_threshold"] = getattr(L, "thr", None)
    line = {
        "metric": "rays/s & ms/frame on 1 B200 (%s)" % (
            "resident march" if cfg["resident"] else
            ("batched views, %s renderer; a step is one batch of views" % args.mode) if "views" in cfg else
            "out-of-core fly-through, %s renderer" % args.mode),
        "value": round(value, 1), "unit": "rays/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(t_max / args.steps, 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8" if wl.esize == 1 else "f32",
        "data": "synthetic (seeded generators, device-generated)",
        "config": workload_config(cfg, args.config, world),
        "renderer": dict(conf, mode=args.mode, learned_prefetch=hint_use(P, conf), brick=wl.brick),
        "roofline": roofline(ld, trace_tot, rays_rank, TRAFFIC_BYTES_PER_RAY.get(args.config), wl.esize),
        "e2e": e2e,
        "clocks": clk,
        "gpu_launches": int(st["launches"]),
        "frame_stats": {"passes_per_launch": round(sum(s["passes"] for s in per) / len(per), 3),
                        "stall_ms_per_step": round(sum(s["ms_stall_last_frame"] for s in per) / args.steps, 4),
                        "prefetch_ms_per_step": round(sum(s["ms_prefetch_last_frame"] for s in per) / args.steps, 4),
                        "trace_ms_per_step": round(trace_tot / args.steps, 4),
                        "hint_host_ms_per_step": round(getattr(L, "timed_hint_s", 0.0) * 1e3 / args.steps, 4),
                        "host_ms_per_step": round(sum(s["ms_last_frame"] for s in per) / args.steps, 4),
                        "device_hit_rate": round(st["device_hits"] / max(1, st["device_hits"] + st["device_misses"]), 5),
                        "bricks_requested": st["bricks_requested"], "bricks_loaded": st["bricks_loaded_disk"],
                        "bricks_prefetched": st["bricks_prefetched"], "bricks_hinted": st["bricks_hinted"],
                        "bricks_staged": st["bricks_staged"],
                        "bricks_speculative": st["bricks_speculative"],
                        "first_launch_stall_ms": round(per[0]["ms_stall_last_frame"], 3),
                        "host_read_ms_total": round(st["ms_host_read_total"], 2),
                        "fill_wait_ms_total": round(st["ms_fill_wait_total"], 2),
                        "h2d_gb_total": round(sum(s["bytes_h2d_last_frame"] for s in per) / 1e9, 4),
                        "hits": st["hits"], "samples": st["samples"], "candidates": st["candidates"],
                        "expansions": st["expansions"]},
    }
    if plain:
        line["plain_lru"] = plain
        if check and "best" in check:
            plain["same_pixels"] = check["best"] == check["plain"]
            plain["pixels_checked_frames"] = check["frames"]
    if P is not None:
        line["learned_prefetch"] = dict(wl.train_info, **({"timed_gain": learned_gain} if learned_gain else {}))
    if tune:
        line["autotune"] = {"best": tune["best"], "points": tune["points"]}
        if paging:
            line["autotune"]["paging"] = paging
        if tune["bricks"]:
            line["autotune"]["bricks"] = tune["bricks"]
    if not args.no_cpu_baseline:
        cb = cpu_baseline(cfg, wl, wl.octree_path, args.cpu_budget, step=frame0 + args.warmup, keep=True)
        cb.pop("per_ray_s")
        # the product's pixels of the same rays against the oracle's
        line["oracle_check"] = dict(oracle_mismatch(product_sample, cb.pop("_oracle")),
                                    frame="step %d (the first timed step)" % (frame0 + args.warmup))
        one = cpu_baseline(cfg, wl, wl.octree_path, max(1.0, args.cpu_budget / 3), nthreads=1,
                           step=frame0 + args.warmup)
        cb["value_1thread"] = one["value"]
        cb["sample_1thread"] = one["sample"]
        line["cpu_baseline"] = cb
    return line


class RefWorkload:
    """The reference arm's inputs, made without libvt: the volume by the
    torch restatement of the seeded generators (oracle/volumes.py, equal to
    libvt's device generator bit for bit), the octree by the oracle's CPU
    builder (the reference's algorithm, byte-identical files)."""

    def __init__(self, cfg, torch, dev, workdir):
        from oracle import oracle as orc
        from oracle import volumes as V
        n = cfg["n"]
        u8 = cfg["gen"] == "fractal"
        t0 = time.time()
        self._host_map, arr = huge_page_array((n, n, n), np.uint8 if u8 else np.float32, volume_offset(cfg))
        host = torch.from_numpy(arr)
        if cfg["gen"] == "sphere":
            c = (n - 1) / 2.0
            kind, prm = "sphere", (c, c, c, 0.25)
        elif u8:
            kind, prm = "fractal", cfg["spheres"]
        else:
            kind, prm = "blobs", cfg["blobs"]
        V.generate(torch, kind, cfg["seed"], (n, n, n), prm, host, dev, slab=max(1, (256 << 20) // (n * n)))
        if dev.type == "cuda":
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
        self.volume = arr
        t1 = time.time()
        self.octree_path = os.path.join(workdir, "vol_%s.oct" % cfg["gen"])
        orc.build_octree(self.volume, cfg["iso"], self.octree_path)
        t2 = time.time()
        log("reference setup: generate %.1fs (torch), octree %.1fs (oracle builder, CPU)" % (t1 - t0, t2 - t1))


def run_reference(args, cfg, rank, world, torch):
    """The reference's path is CUDA code with no CPU implementation; this
    arm times its CPU restatement -- the oracle port of the reference's
    camera, octree traversal, brick addressing and march -- on all host
    threads, a bounded ray sample of every step's camera."""
    if rank != 0:
        return None
    # the generators run on the GPU where there is one (the bench's boxes),
    # else on the CPU (exact for the sphere and fractal volumes)
    dev = torch.device("cuda", 0) if torch.cuda.is_available() else torch.device("cpu")
    work = tempfile.mkdtemp(prefix="vtbench_ref_")
    wl = RefWorkload(cfg, torch, dev, work)
    if "views" in cfg:
        n = sum(p[0] * p[1] for p in step_poses(cfg, args.warmup))
    else:
        n = cfg["W"] * cfg["H"]
    # the whole run samples about --ref-total seconds of CPU rendering
    from oracle import oracle as orc
    octree = orc.Octree(wl.octree_path)
    budget = max(0.1, min(args.ref_budget, args.ref_total / (args.warmup + args.steps)))
    vals, per_ray = [], None
    for i in range(args.warmup + args.steps):
        cb = cpu_baseline(cfg, wl, wl.octree_path, budget, step=i, octree=octree, per_ray=per_ray)
        per_ray = cb.pop("per_ray_s")
        if i >= args.warmup:
            vals.append(cb)
    rays_s = statistics.median(v["value"] for v in vals)
    line = {
        "impl": "reference",
        "metric": "rays/s & ms/frame on 1 B200 (%s)" % (
            "resident march" if cfg["resident"] else
            ("batched views, best renderer; a step is one batch of views" if "views" in cfg else
             "out-of-core fly-through, best renderer")),
        "value": rays_s, "unit": "rays/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(n / rays_s * 1e3, 3), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8" if cfg["gen"] == "fractal" else "f32", "data": "synthetic (seeded generators)",
        "config": workload_config(cfg, args.config, world),
        "cpu_baseline": dict(vals[-1], value=rays_s),
        "e2e": {"value": rays_s, "unit": "rays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "vs CPU port: the reference's path is CUDA-only, so this arm times the reference algorithm's CPU "
                "restatement (oracle/vt_oracle.cpp) on all host threads over a bounded ray sample per step; "
                "inputs made without libvt (torch restatement of the generators, oracle CPU octree builder)",
    }
    return line


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--config", default=os.environ.get("VT_BENCH_CONFIG", "c2"), choices=sorted(CONFIGS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-budget", type=float, default=10.0)
    ap.add_argument("--ref-budget", type=float, default=6.0, help="reference arm: CPU seconds per step at most")
    ap.add_argument("--ref-total", type=float, default=150.0, help="reference arm: CPU seconds over all steps")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--mode", default="best", choices=sorted(MODES))
    ap.add_argument("--no-plain", action="store_true", help="skip the plain-LRU comparison run")
    ap.add_argument("--no-learned", action="store_true", help="best mode without the learned prefetch")
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--no-brick-sweep", action="store_true", help="batched configs: keep the config's brick size")
    ap.add_argument("--paging", default=None, help="fly-throughs: fixed FRAMES,LOOKAHEAD[,HINT_THRESHOLD[,SKIP]] "
                                                   "instead of the paging autotune")
    ap.add_argument("--warm", action="store_true", help="profiling: preloaded cache, no cold start")
    ap.add_argument("--wavefront", type=int, default=0,
                    help="wavefront rounds per pass (0: the fused trace kernel; slab mode, in-order traversal)")
    ap.add_argument("--spec-async", type=int, default=1, choices=(0, 1),
                    help="1: lookahead bricks load on the cache's side stream while passes run; 0: with the demand "
                         "requests of the same service")
    ap.add_argument("--skip", type=int, default=None,
                    help="absent-brick candidates a ray may set aside per pass (default: tuned on fly-throughs, 0 on "
                         "batched views)")
    ap.add_argument("--demand-batch", type=int, default=None,
                    help="fixed demand batch (bricks a service loads itself before queuing the rest on the side "
                         "stream; 0: no bound) instead of the tuner's choice")
    ap.add_argument("--shared-aprons", type=int, default=1, choices=(0, 1),
                    help="1: demand loads copy x/y aprons from resident neighbours' slots; 0: whole bricks")
    args = ap.parse_args()
    global SHARED_APRONS
    SHARED_APRONS = args.shared_aprons
    if args.warmup < 3:
        args.warmup = 3
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    dist = None
    if world > 1 and args.impl == "reference":
        if rank != 0:
            return                  # the reference arm runs on rank 0's host cores only
    elif world > 1:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", 0)))
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    cfg = CONFIGS[args.config]
    if args.steps is None:
        args.steps = (300 if cfg["orbit"] else cfg["path"]["frames"] if cfg.get("path") else
                      6 if "views" in cfg else 200)
    if args.impl == "reference":
        line = run_reference(args, cfg, rank, world, torch)
    else:
        line = run_ours(args, cfg, rank, world, torch, dist)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
