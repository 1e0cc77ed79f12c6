"""GPU parity: libvt.so (through its C ABI) against the CPU oracle on the
same seeded inputs.

Bar (from the task): hit-node Morton codes and brick ids bit-exact; hit t
within 1e-3 voxel; normals within 1e-3 rad; RGB8 within 1 LSB.  The kernels
are compiled without contraction and with IEEE division/sqrt, so in
practice t, normals and RGBA come out bit-identical; the tolerances below
are the stated bar.
"""
import os

import numpy as np
import pytest

import vt_fixtures as F
import visualtur_b200 as vt
from oracle import oracle as orc

pytestmark = pytest.mark.gpu

T_TOL = 1e-3        # voxels
N_TOL = 1e-3        # radians
RGB8_TOL = 1        # LSB


def product_render(case, workdir, mode, vol=None, extra_ops=(), refine=0):
    c = F.CASES[case]
    vol = F.case_volume(case) if vol is None else vol
    fm = vt.FileManager.wrap(vol)
    oc = vt.Octree(F.case_octree(case, workdir))
    nb = 8 ** c["levelC"]
    dev, host = nb, nb
    if mode.startswith("demand"):
        dev, host = 24, 16
    opt = vt.default_options(resident=1 if mode in ("resident", "persist") else 0, record_hits=1,
                             persistent=1 if mode in ("persist", "demand_la", "demand_skip") else 0,
                             lookahead={"demand_la": 3, "demand_skip": 2, "demand_la_sync": 3,
                                        "demand_wave": 2}.get(mode, 0), pops=3,
                             spec_async=0 if mode == "demand_la_sync" else 1,
                             wavefront={"wave": 2, "demand_wave": 3, "wave1": 1}.get(mode, 0),
                             unroll={"persist": 4, "demand_la": 2, "slab": 8}.get(mode, 1), refine=refine,
                             skip={"demand_skip": 4, "demand_skip_np": 2}.get(mode, 0))
    p = vt.make_params(W=c["W"], H=c["H"], octreeFile=None, hdf5File=None, octreeLevel=c["levelO"],
                       levelCubes=c["levelC"], dimCube=1 << (int(np.log2(c["n"])) - c["levelC"]),
                       cubeInc=c["inc"], distance=c["dist"], fov_H=c["fov"], fov_W=c["fov"],
                       maxElementsCache=dev, maxElementsCache_CPU=host)
    r = vt.visualTur(p, opt, volume=fm, octree=oc)
    m = {"mv": r.camera_Move, "rx": r.camera_RotateX, "ry": r.camera_RotateY, "rz": r.camera_RotateZ,
         "mf": r.camera_MoveForward, "mu": r.camera_MoveUpward, "sr": r.camera_StrafeRight}
    for op, v in list(c["ops"]) + list(extra_ops):
        m[op](v)
    rgba, rgb8 = r.render_host()
    node, brick, t, nrm = r.debug_hits()
    st = r.stats()
    r.close()
    return dict(rgba=rgba, rgb8=rgb8, node=node, brick=brick, t=t, normal=nrm, stats=st)


def oracle_render(case, workdir, vol=None, extra_ops=(), refine=0):
    c = F.CASES[case]
    vol = F.case_volume(case) if vol is None else vol
    o = orc.Octree(F.case_octree(case, workdir))
    cam = F.oracle_camera(case)
    orc.apply_ops(cam, extra_ops)
    return orc.render(o, vol, cam, c["levelO"], c["levelC"], c["inc"], refine=refine)


def assert_parity(a, b):
    """The bar, plus bit equality.  A crossing where the previous sample,
    the crossing sample and the isovalue are all equal (integer voxels of a
    uint8 volume) refines with 0/0 in the reference (src/rayCaster.cu:
    227-228): t, the normal and the colour are NaN there, on both sides."""
    assert np.array_equal(a["node"], b["node"]), "node ids differ at %d rays" % (a["node"] != b["node"]).sum()
    assert np.array_equal(a["brick"], b["brick"])
    hit = b["node"] != 0
    ta, tb = a["t"][hit], b["t"][hit]
    assert np.array_equal(np.isnan(ta), np.isnan(tb))
    fin = ~np.isnan(tb)
    assert np.abs(ta[fin] - tb[fin]).max(initial=0) <= T_TOL
    na, nb = a["normal"][hit], b["normal"][hit]
    assert np.array_equal(np.isnan(na), np.isnan(nb))
    fin = ~np.isnan(nb).any(axis=1)
    dots = np.clip((na[fin] * nb[fin]).sum(axis=1), -1, 1)
    assert np.arccos(dots).max(initial=0) <= N_TOL
    assert np.abs(a["rgb8"].astype(int) - b["rgb8"].astype(int)).max() <= RGB8_TOL
    # stronger than the bar: the evaluation is IEEE-exact on both sides
    # (NaN colours compare as NaN: the GPU's and the host's NaN bit
    # patterns differ)
    ra, rb = a["rgba"], b["rgba"]
    assert np.array_equal(np.isnan(ra), np.isnan(rb))
    fin = ~np.isnan(rb)
    assert np.array_equal(ra[fin].view(np.uint32), rb[fin].view(np.uint32))
    assert np.array_equal(a["rgb8"], b["rgb8"])


@pytest.mark.parametrize("mode", ["resident", "slab", "demand", "persist", "demand_la", "demand_la_sync",
                                  "demand_skip", "demand_skip_np", "wave", "wave1", "demand_wave"])
@pytest.mark.parametrize("case", sorted(F.CASES))
def test_render_parity(case, mode, workdir, cuda):
    a = product_render(case, workdir, mode)
    b = oracle_render(case, workdir)
    assert_parity(a, b)
    assert a["stats"]["hits"] == b["agg"]["hits"]
    if "skip" in mode:
        # candidates set aside behind an absent brick let a ray march past
        # its final hit: more work, the same image
        assert a["stats"]["samples"] >= b["agg"]["samples"]
        assert a["stats"]["candidates"] >= b["agg"]["candidates"]
    else:
        assert a["stats"]["samples"] == b["agg"]["samples"]
        assert a["stats"]["candidates"] == b["agg"]["candidates"]
    if mode.startswith("demand"):
        assert a["stats"]["passes"] > 1 and a["stats"]["bricks_requested"] > 24


@pytest.mark.parametrize("mode", ["resident", "demand_la"])
@pytest.mark.parametrize("case", ["c1", "s64rot"])
def test_bisection_mode_parity(case, mode, workdir, cuda):
    """Bisection refinement (5 steps) against the oracle in the same mode;
    node and brick ids equal those of the reference refinement."""
    a = product_render(case, workdir, mode, refine=5)
    b = oracle_render(case, workdir, refine=5)
    assert_parity(a, b)
    assert a["stats"]["samples"] == b["agg"]["samples"]
    base = oracle_render(case, workdir)
    assert np.array_equal(a["node"], base["node"]) and np.array_equal(a["brick"], base["brick"])
    hit = base["node"] != 0
    assert b["agg"]["samples"] == base["agg"]["samples"] + 5 * int(hit.sum())
    assert not np.array_equal(a["t"][hit], base["t"][hit])


def test_camera_rays_bitwise(cuda, workdir):
    torch = cuda
    cam = vt.Camera(72, 80, 50.0, 25.0, 27.5)
    oc = orc.Camera(72, 80, 50.0, 25.0, 27.5)
    for c in (cam, oc):
        c.Move((31.5, 31.5, 181.5)); c.RotateY(10.0); c.RotateX(-8.0); c.StrafeRight(3.0)
    d = torch.empty(72 * 80 * 3, dtype=torch.float32, device="cuda")
    cam.rays_into(d)
    torch.cuda.synchronize()
    got = d.cpu().numpy().reshape(-1, 3)
    assert np.array_equal(got.view(np.uint32), oc.rays().view(np.uint32))


@pytest.mark.parametrize("inc", [3, 2])
def test_render_cube_parity(inc, cuda):
    torch = cuda
    vol = F.case_volume("s64")
    dim = 32
    b0 = np.array([16, 16, 16]) - inc
    D = dim + 2 * inc
    brick = orc.read_voxels(vol, tuple(b0), tuple(b0 + D))
    W, H = 96, 80
    for mv in [(16.0, 16.0, 110.0), (40.0, 20.0, -60.0)]:
        cam, ocam = vt.Camera(H, W, 50.0, 30.0, 35.0), orc.Camera(H, W, 50.0, 30.0, 35.0)
        cam.Move(mv)
        ocam.Move(mv)
        if mv[2] < 0:
            cam.RotateY(180.0)
            ocam.RotateY(180.0)
        db = torch.from_numpy(brick.ravel()).cuda()
        out = torch.empty(W * H * 4, dtype=torch.float32, device="cuda")
        vt.rayCaster(20.0).renderCube(cam, db, (0, 0, 0), (dim,) * 3, (inc,) * 3, out)
        torch.cuda.synchronize()
        got = out.cpu().numpy().reshape(-1, 4)
        exp, oob = orc.render_cube(ocam, brick, (0, 0, 0), (dim,) * 3, (inc,) * 3, 20.0)
        assert np.array_equal(got.view(np.uint32), exp.view(np.uint32)), "inc %d oob %d" % (inc, oob)


def test_device_generator_matches_host(cuda):
    torch = cuda
    for shape, c in [((64, 64, 64), (31.5, 31.5, 31.5)), ((50, 40, 33), (20.0, 18.5, 16.0))]:
        d = torch.empty(int(np.prod(shape)), dtype=torch.float32, device="cuda")
        vt.generate_volume(vt.VT_GEN_SPHERE, 77, shape, c + (0.25,), device_ptr=d.data_ptr())
        torch.cuda.synchronize()
        h = vt.generate_volume(vt.VT_GEN_SPHERE, 77, shape, c + (0.25,))
        assert np.array_equal(d.cpu().numpy().view(np.uint32), h.ravel().view(np.uint32))


def test_render_into_device_buffers_and_repeat(workdir, cuda):
    torch = cuda
    c = F.CASES["c1"]
    fm = vt.FileManager.wrap(F.case_volume("c1"))
    oc = vt.Octree(F.case_octree("c1", workdir))
    p = vt.make_params(W=c["W"], H=c["H"], octreeFile=None, hdf5File=None, octreeLevel=5, levelCubes=4, dimCube=8,
                       distance=50.0, fov_H=30.0, fov_W=30.0)
    r = vt.visualTur(p, vt.default_options(resident=1), volume=fm, octree=oc)
    r.camera_Move((63.5, 63.5, 363.5))
    rgba = torch.empty(c["W"] * c["H"] * 4, dtype=torch.float32, device="cuda")
    rgb8 = torch.empty(c["W"] * c["H"] * 3, dtype=torch.uint8, device="cuda")
    outs = []
    for _ in range(3):
        r.updateVisibleCubes(rgba, rgb8)
        torch.cuda.synchronize()
        outs.append((rgba.cpu().numpy().copy(), rgb8.cpu().numpy().copy()))
    assert all(np.array_equal(outs[0][0], o[0]) and np.array_equal(outs[0][1], o[1]) for o in outs)
    exp = oracle_render("c1", workdir)
    assert np.array_equal(outs[0][1].reshape(-1, 3), exp["rgb8"])
    st = r.stats()
    assert st["frames"] == 3 and st["passes"] == 1


def _views(vt_, torch, cams):
    views, bufs = [], []
    for cam in cams:
        n = cam.W * cam.H
        rgba = torch.empty(n * 4, dtype=torch.float32, device="cuda")
        rgb8 = torch.empty(n * 3, dtype=torch.uint8, device="cuda")
        v = vt.vt_view()
        v.cam = cam
        v.dev_rgba, v.dev_rgb8 = rgba.data_ptr(), rgb8.data_ptr()
        views.append(v)
        bufs.append((rgba, rgb8))
    return views, bufs


BATCH = [((96, 96), [("mv", (31.5, 31.5, 181.5))]),
         ((50, 37), [("mv", (31.5, 31.5, 181.5)), ("ry", 20.0), ("mf", 30.0)]),
         ((128, 72), [("mv", (31.5, 31.5, 181.5)), ("rx", -12.0), ("rz", 33.0), ("sr", 4.0)]),
         ((33, 65), [("mv", (-80.0, 40.0, 31.5)), ("ry", -90.0)])]


@pytest.mark.parametrize("mode", ["resident", "demand", "persist", "demand_la"])
def test_batch_parity(mode, workdir, cuda):
    """Several views of different sizes in one launch equal per-view oracle renders."""
    torch = cuda
    c = F.CASES["s64"]
    fm, oc = vt.FileManager.wrap(F.case_volume("s64")), vt.Octree(F.case_octree("s64", workdir))
    dev, host = (24, 16) if mode.startswith("demand") else (512, 512)
    opt = vt.default_options(resident=1 if mode in ("resident", "persist") else 0, record_hits=0,
                             persistent=1 if mode in ("persist", "demand_la") else 0,
                             lookahead=2 if mode == "demand_la" else 0, pops=2, tile_w=16, tile_h=16,
                             unroll=4 if mode == "persist" else 1)
    p = vt.make_params(W=96, H=96, octreeFile=None, hdf5File=None, octreeLevel=4, levelCubes=3, dimCube=8,
                       distance=50.0, fov_H=30.0, fov_W=30.0, maxElementsCache=dev, maxElementsCache_CPU=host)
    r = vt.visualTur(p, opt, volume=fm, octree=oc)
    cams = []
    for (W, H), ops in BATCH:
        cam = vt.Camera(H, W, 50.0, 30.0, 27.0)
        for op, v in ops:
            {"mv": cam.Move, "rx": cam.RotateX, "ry": cam.RotateY, "rz": cam.RotateZ, "mf": cam.MoveForward,
             "sr": cam.StrafeRight}[op](v)
        cams.append(cam)
    views, bufs = _views(vt, torch, [cm.c for cm in cams])
    r.render_batch(views)
    torch.cuda.synchronize()
    o = orc.Octree(F.case_octree("s64", workdir))
    vol = F.case_volume("s64")
    for ((W, H), ops), (rgba, rgb8) in zip(BATCH, bufs):
        ocam = orc.Camera(H, W, 50.0, 30.0, 27.0)
        orc.apply_ops(ocam, ops)
        exp = orc.render(o, vol, ocam, c["levelO"], c["levelC"], c["inc"])
        assert np.array_equal(rgba.cpu().numpy().reshape(-1, 4).view(np.uint32), exp["rgba"].view(np.uint32))
        assert np.array_equal(rgb8.cpu().numpy().reshape(-1, 3), exp["rgb8"])
    if mode.startswith("demand"):
        assert r.stats()["passes"] > 1


def test_trace_log_and_prefetch(workdir, cuda):
    c = F.CASES["c1"]
    fm, oc = vt.FileManager.wrap(F.case_volume("c1")), vt.Octree(F.case_octree("c1", workdir))
    opt = vt.default_options(resident=0, preload=0, record_trace=1, trace_level=2, record_hits=1)
    p = vt.make_params(W=c["W"], H=c["H"], octreeFile=None, hdf5File=None, octreeLevel=5, levelCubes=4, dimCube=8,
                       distance=50.0, fov_H=30.0, fov_W=30.0, maxElementsCache=4096, maxElementsCache_CPU=4096)
    r = vt.visualTur(p, opt, volume=fm, octree=oc)
    r.camera_Move((63.5, 63.5, 363.5))
    rgba1, _ = r.render_host(rgb8=False)
    st1 = r.stats()
    assert st1["passes"] > 1                       # cold cache: demand passes
    node = r.debug_hits()[0]
    bits = r.trace(2)
    touched = {64 + k for k in range(64) if (bits[k // 32] >> (k % 32)) & 1}
    hit_anc = {int(n) >> 9 for n in node[node != 0]}     # level-5 code -> level-2 ancestor
    assert hit_anc and hit_anc <= touched
    # second frame of the same pose: every brick now resident, one pass
    r.reset_stats()
    rgba2, _ = r.render_host(rgb8=False)
    assert r.stats()["passes"] == 1 and np.array_equal(rgba1, rgba2)
    # a fresh cold handle with every brick prefetched renders in one pass
    r2 = vt.visualTur(p, vt.default_options(resident=0, preload=0), volume=fm, octree=oc)
    r2.camera_Move((63.5, 63.5, 363.5))
    assert r2.prefetch(r2.brick_list()) > 0
    rgba3, _ = r2.render_host(rgb8=False)
    assert r2.stats()["passes"] == 1 and np.array_equal(rgba1, rgba3)


def test_autotune_changes_speed_not_pixels(workdir, cuda):
    torch = cuda
    from visualtur_b200 import autotune as at
    c = F.CASES["s64"]
    vol = F.case_volume("s64")
    fm, oc = vt.FileManager.wrap(vol), vt.Octree(F.case_octree("s64", workdir))
    exp = oracle_render("s64", workdir)

    def make(brick):
        lc = {8: 3, 16: 2}[brick]
        p = vt.make_params(W=c["W"], H=c["H"], octreeFile=None, hdf5File=None, octreeLevel=4, levelCubes=lc,
                           dimCube=brick, distance=50.0, fov_H=30.0, fov_W=30.0, maxElementsCache=512,
                           maxElementsCache_CPU=512)
        r = vt.visualTur(p, vt.default_options(resident=0, record_hits=1), volume=fm, octree=oc)
        r.camera_Move(c["ops"][0][1])
        return r

    def step(r, i, stream):
        r.updateVisibleCubes(None, stream=stream.cuda_stream)

    best, table = at.tune(torch, make, step, brick_sizes=(8, 16), frames=2,
                          tiles={32: (8, 4), 256: (16, 16)}, unrolls=(1, 4), persist=(0, 1))
    # 16 shape points, plus the refill-interval stage for each brick size
    # whose best shape used the persistent queue
    extra = len(table) - 2 * 2 * 2 * 2
    assert extra in (0, len(at.POPS), 2 * len(at.POPS)) and best["ms"] == min(t["ms"] for t in table)
    for row in table[::3]:
        r = make(row["brick"])
        r.set_tuning(tile_w=row["tile_w"], tile_h=row["tile_h"], unroll=row["unroll"], persistent=row["persistent"],
                     pops=row["pops"])
        rgba, rgb8 = r.render_host()
        node = r.debug_hits()[0]
        r.close()
        assert np.array_equal(rgb8, exp["rgb8"]) and np.array_equal(node, exp["node"])


@pytest.mark.parametrize("case", ["c1", "s64rot"])
def test_side_stream_lookahead_loads_keep_pixels(case, workdir, cuda):
    """Lookahead bricks queued and loaded on the cache's side stream while
    later passes and frames run: frames after the first start with bricks
    that landed meanwhile, and every frame equals the oracle's."""
    c = F.CASES[case]
    vol = F.case_volume(case)
    fm, oc = vt.FileManager.wrap(vol), vt.Octree(F.case_octree(case, workdir))
    nb = 8 ** c["levelC"]
    p = vt.make_params(W=c["W"], H=c["H"], octreeFile=None, hdf5File=None, octreeLevel=c["levelO"],
                       levelCubes=c["levelC"], dimCube=1 << (int(np.log2(c["n"])) - c["levelC"]),
                       cubeInc=c["inc"], distance=c["dist"], fov_H=c["fov"], fov_W=c["fov"],
                       maxElementsCache=nb, maxElementsCache_CPU=nb)
    r = vt.visualTur(p, vt.default_options(resident=0, preload=0, record_hits=1, persistent=1, lookahead=4,
                                           pops=3, spec_async=1), volume=fm, octree=oc)
    m = {"mv": r.camera_Move, "rx": r.camera_RotateX, "ry": r.camera_RotateY, "rz": r.camera_RotateZ,
         "mf": r.camera_MoveForward, "mu": r.camera_MoveUpward, "sr": r.camera_StrafeRight}
    for op, v in c["ops"]:
        m[op](v)
    for k, extra in enumerate([(), (("ry", 4.0),), (("ry", 4.0), ("rx", 3.0)), (("ry", 4.0), ("rx", 3.0), ("mf", 5.0))]):
        if k:
            op, v = extra[-1]
            m[op](v)
        rgba, rgb8 = r.render_host()
        node, brick, t, nrm = r.debug_hits()
        a = dict(rgba=rgba, rgb8=rgb8, node=node, brick=brick, t=t, normal=nrm)
        assert_parity(a, oracle_render(case, workdir, extra_ops=extra))
    st = r.stats()
    assert st["bricks_speculative"] > 0 and st["bricks_spec_loaded"] > 0
    r.close()


@pytest.mark.parametrize("case", ["c1", "s64rot"])
def test_deferred_demand_loads_keep_pixels(case, workdir, cuda):
    """A service that loads only a few demand bricks itself (demand_batch)
    and hands the rest to the cache's side stream, which loads them while
    the next pass runs: rays that find them absent request them again, and
    every frame equals the oracle's."""
    c = F.CASES[case]
    vol = F.case_volume(case)
    fm, oc = vt.FileManager.wrap(vol), vt.Octree(F.case_octree(case, workdir))
    nb = 8 ** c["levelC"]
    p = vt.make_params(W=c["W"], H=c["H"], octreeFile=None, hdf5File=None, octreeLevel=c["levelO"],
                       levelCubes=c["levelC"], dimCube=1 << (int(np.log2(c["n"])) - c["levelC"]),
                       cubeInc=c["inc"], distance=c["dist"], fov_H=c["fov"], fov_W=c["fov"],
                       maxElementsCache=nb, maxElementsCache_CPU=nb)
    r = vt.visualTur(p, vt.default_options(resident=0, preload=0, record_hits=1, persistent=1, lookahead=0,
                                           pops=3, spec_async=1, demand_batch=4, max_passes=100000),
                     volume=fm, octree=oc)
    m = {"mv": r.camera_Move, "rx": r.camera_RotateX, "ry": r.camera_RotateY, "rz": r.camera_RotateZ,
         "mf": r.camera_MoveForward, "mu": r.camera_MoveUpward, "sr": r.camera_StrafeRight}
    for op, v in c["ops"]:
        m[op](v)
    for k, extra in enumerate([(), (("ry", 4.0),), (("ry", 4.0), ("rx", 3.0))]):
        if k:
            op, v = extra[-1]
            m[op](v)
        rgba, rgb8 = r.render_host()
        node, brick, t, nrm = r.debug_hits()
        a = dict(rgba=rgba, rgb8=rgb8, node=node, brick=brick, t=t, normal=nrm)
        assert_parity(a, oracle_render(case, workdir, extra_ops=extra))
    r.close()
