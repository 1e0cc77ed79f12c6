"""Renders of the benchmark workloads themselves against the oracle.

The fixture cases of test_gpu_parity.py are small spheres; these are the
bench's workloads (bench.CONFIGS): the 128^3 resident sphere at its stated
512x512, the 2048^3 blobs fly-through (nLevels 11: the flat node array's
index field and the page table at full size) and its 1024^3 version, and
the 2048^3 uint8 fractal with 32^3 bricks.  Each is generated on the device
by libvt's seeded generators, its octree built by libvt's GPU builder, and
rendered through vt_render from a cold brick cache with the product's
settings (persistent ray queue, lookahead requests, with and without
set-aside candidates, fused and wavefront passes); the oracle renders the same frames from the same
volume and octree.  Bar: hit node and brick ids bit-exact, t within 1e-3
voxel, normals within 1e-3 rad, RGB8 within 1 LSB (and in fact every RGBA
bit equal).  The oracle's own CPU builder must write the same octree file
as the GPU builder (nLevels 10 and 11)."""
import filecmp
import math
import os
import sys

import numpy as np
import pytest

import visualtur_b200 as vt
from oracle import oracle as orc
from test_gpu_parity import assert_parity

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402

pytestmark = pytest.mark.gpu

_WL = {}


def workload(name, torch, workdir):
    """bench's Workload (device generation, GPU octree build, host copy of
    the volume), kept for the module's tests."""
    if name not in _WL:
        for k in list(_WL):           # one large volume in host memory at a time
            del _WL[k]
        cfg = bench.CONFIGS[name]
        d = os.path.join(workdir, name)
        os.makedirs(d, exist_ok=True)
        wl = bench.Workload(cfg, torch, torch.device("cuda", 0), d, need_renderer=False)
        wl.fm = vt.FileManager.wrap(wl.volume)
        wl.oc = vt.Octree(wl.octree_path)
        wl.brick = 1 << (wl.oc.nLevels - cfg["levelC"])
        _WL[name] = wl
    return _WL[name]


def oracle_frame(wl, cfg, cam):
    o = orc.Octree(wl.octree_path)
    oc = orc.Camera(cam.H, cam.W, cfg["dist"], cfg["fov"], cfg["fov"])
    for f in ("look", "up", "right", "position"):
        v = getattr(cam, f)
        setattr(oc.c, f, orc.orc_f3(v[0], v[1], v[2]))
    return orc.render(o, wl.volume, oc, cfg["levelO"], cfg["levelC"], cfg["inc"])


def product_frames(wl, cfg, frames, **opt):
    o = dict(resident=cfg["resident"], preload=cfg["resident"], record_hits=1, host_threads=0)
    o.update(opt)
    r = vt.visualTur(wl.params(), vt.default_options(**o), volume=wl.fm, octree=wl.oc)
    out = []
    for f in frames:
        cam = bench.frame_camera(vt, cfg, f)
        r.set_camera(cam)
        rgba, rgb8 = r.render_host()
        node, brick, t, nrm = r.debug_hits()
        out.append((cam, dict(rgba=rgba, rgb8=rgb8, node=node, brick=brick, t=t, normal=nrm, stats=r.stats())))
    r.close()
    return out


BEST = dict(persistent=1, lookahead=2, pops=32, blocks_per_sm=8, use_graph=1)


@pytest.mark.parametrize("mode", ["resident", "paged"])
def test_c1_sphere_at_512(mode, workdir, cuda):
    """BASELINE config 1 as stated: 128^3 noisy sphere, iso 40, 8^3 bricks,
    512x512, FOV 60 deg, distance 300."""
    cfg = dict(bench.CONFIGS["c1"])
    wl = workload("c1", cuda, workdir)
    if mode == "paged":
        cfg["resident"] = 0
    for cam, got in product_frames(wl, cfg, [0], **(BEST if mode == "paged" else {})):
        assert cam.W == 512 and cam.H == 512
        want = oracle_frame(wl, cfg, cam)
        assert_parity(got, want)
        assert got["stats"]["hits"] == want["agg"]["hits"] > 10000


def check_blobs(name, cuda, workdir):
    cfg = bench.CONFIGS[name]
    wl = workload(name, cuda, workdir)
    assert wl.oc.nLevels == int(math.log2(cfg["n"])) and wl.brick == 16
    for skip, wave in ((0, 0), (2, 0), (0, 2)):
        for cam, got in product_frames(wl, cfg, [0, 37], skip=skip, wavefront=wave, **BEST):
            want = oracle_frame(wl, cfg, cam)
            assert_parity(got, want)
            assert want["agg"]["hits"] > 100000
            assert got["stats"]["bricks_loaded_disk"] > 1000     # the frames were paged in
    return wl


def test_blobs_1024_frames_and_octree(workdir, cuda):
    """The 1024^3 blobs (nLevels 10), 16^3 bricks with a 3-voxel apron,
    1920x1080 orbit frames from a cold cache, with and without set-aside
    candidates; and the GPU builder's octree file equals the oracle's (the
    reference's algorithm on the CPU), byte for byte."""
    wl = check_blobs("c2s", cuda, workdir)
    p = os.path.join(workdir, "c2s_oracle.oct")
    orc.build_octree(wl.volume, bench.CONFIGS["c2s"]["iso"], p)
    assert filecmp.cmp(p, wl.octree_path, shallow=False)


def test_blobs_2048_frames(workdir, cuda):
    """The 2048^3 blobs of the out-of-core fly-through (nLevels 11: the flat
    node array's index field and the page table at full size)."""
    check_blobs("c2", cuda, workdir)


def test_u8_fractal_frames(workdir, cuda):
    """The 2048^3 uint8 fractal + spheres volume, iso 128, 32^3 bricks,
    1920x1080 frames of its Catmull-Rom path from a cold cache, with and
    without set-aside candidates."""
    cfg = bench.CONFIGS["c5s"]
    wl = workload("c5s", cuda, workdir)
    assert wl.volume.dtype == np.uint8 and wl.brick == 32
    for skip, wave in ((0, 0), (2, 0), (0, 3)):
        for cam, got in product_frames(wl, cfg, [0, 211], skip=skip, wavefront=wave, **BEST):
            want = oracle_frame(wl, cfg, cam)
            assert_parity(got, want)
            assert want["agg"]["hits"] > 100000
