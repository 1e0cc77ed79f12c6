"""A device slot must hold exactly the zero-padded box
[min - inc, min + edge + inc) of the volume (lruCache's brick,
src/lruCache.cu:224-226), whichever way the service filled it (whole
bricks or some parts from the packed host tier, x/y aprons copied from
neighbouring slots, slots reused within a service, lookahead bricks on the
side stream or with the demand ones).  Checked slot by slot against the volume (vt_debug_slot) and
frame by frame against the resident renderer, for float32 and uint8
voxels, a non-cubic volume (bricks on its faces and beyond it), an apron
wider than the brick, and device caches small enough that slots are reused
within a frame."""
import math
import os

import numpy as np
import pytest

import visualtur_b200 as vt
from visualtur_b200 import prefetch as pf

pytestmark = pytest.mark.gpu

SHAPE = (96, 80, 112)          # brick grid of 128^3 (nLevels 7)
W = H = 96


def volume(dtype, seed=3):
    rng = np.random.default_rng(seed)
    x, y, z = np.meshgrid(*[np.arange(n, dtype=np.float32) for n in SHAPE], indexing="ij")
    r = np.sqrt((x - 47.5) ** 2 + (y - 41.0) ** 2 + (z - 60.0) ** 2)
    v = r + rng.normal(0.0, 0.6, SHAPE).astype(np.float32)
    if dtype == np.uint8:
        return np.clip(v * 4.0, 0, 255).astype(np.uint8), 120.0
    return v.astype(np.float32), 30.0


def padded_box(vol, lo, D):
    out = np.zeros((D, D, D), vol.dtype)
    s = [max(0, l) for l in lo]
    e = [min(n, l + D) for l, n in zip(lo, vol.shape)]
    if all(a < b for a, b in zip(s, e)):
        out[s[0] - lo[0]:e[0] - lo[0], s[1] - lo[1]:e[1] - lo[1], s[2] - lo[2]:e[2] - lo[2]] = \
            vol[s[0]:e[0], s[1]:e[1], s[2]:e[2]]
    return out


def decode(code, Lc):
    """brick Morton code at level Lc -> brick coordinates"""
    c = [0, 0, 0]
    for b in range(Lc):
        c[0] |= ((code >> (3 * b + 2)) & 1) << b
        c[1] |= ((code >> (3 * b + 1)) & 1) << b
        c[2] |= ((code >> (3 * b)) & 1) << b
    return c


@pytest.mark.parametrize("dtype,levelC,inc,dev,opts", [
    (np.float32, 4, 3, 4096, {}),     # every brick fits
    (np.float32, 4, 3, 60, {}),       # slots reused within a frame's services
    (np.uint8, 4, 4, 90, {}),         # byte voxels, wider apron
    (np.float32, 5, 5, 300, {}),      # apron wider than the brick (inc 5 > edge 4)
    (np.float32, 4, 3, 60, {"shared_aprons": 0}),                  # whole bricks only
    (np.uint8, 4, 3, 4096, {"spec_async": 0}),                     # lookahead with the demand loads
    (np.float32, 3, 3, 200, {"spec_async": 0, "lookahead": 0}),    # 16^3 bricks, demand loads only
    (np.float32, 4, 3, 4096, {"lookahead": 0, "demand_batch": 8}),  # most demand bricks via the side stream
])
def test_slots_hold_the_padded_box(dtype, levelC, inc, dev, opts, tmp_path, cuda):
    vol, iso = volume(dtype)
    fm = vt.FileManager.wrap(vol)
    path = os.path.join(str(tmp_path), "vol.oct")
    vt.build_octree(fm, iso, path)
    oc = vt.Octree(path)
    edge = 1 << (oc.nLevels - levelC)
    D = edge + 2 * inc

    def make(resident, nslots):
        p = vt.make_params(W=W, H=H, octreeFile=None, hdf5File=None, octreeLevel=levelC + 1, levelCubes=levelC,
                           dimCube=edge, cubeInc=inc, distance=50.0, fov_H=30.0, fov_W=30.0,
                           maxElementsCache=nslots, maxElementsCache_CPU=max(nslots, 64))
        o = dict(resident=resident, record_hits=0, preload=0, lookahead=2, max_passes=4096)
        if not resident:
            o.update(opts)
        return vt.visualTur(p, vt.default_options(**o), volume=fm, octree=oc)

    ref = make(1, 8)
    dem = make(0, dev)
    bricks = dem.brick_list()
    c = (47.5, 41.0, 60.0)
    checked = 0
    for f in range(3):
        a = math.radians(50.0 * f + 10.0)
        eye = (c[0] + 260.0 * math.sin(a), c[1] + 40.0, c[2] + 260.0 * math.cos(a))
        cam = pf.look_at(W, H, 50.0, 30.0, eye, c)
        ref.set_camera(cam)
        dem.set_camera(cam)
        ra, _ = ref.render_host(rgb8=False)
        da, _ = dem.render_host(rgb8=False)
        assert np.array_equal(ra.view(np.uint32), da.view(np.uint32)), "frame %d differs" % f
        for code in bricks:
            slot = dem.debug_slot(code, D, vol.dtype)
            if slot is None:
                continue
            bx, by, bz = decode(int(code), levelC)
            want = padded_box(vol, (bx * edge - inc, by * edge - inc, bz * edge - inc), D)
            assert np.array_equal(slot, want), "slot of brick %d (%d, %d, %d) differs" % (code, bx, by, bz)
            checked += 1
    assert checked > 0
    ref.close()
    dem.close()
