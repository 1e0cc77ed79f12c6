"""The bisection refinement mode of the oracle (the renderer's `refine`
option; the reference's own refinement loop is compiled out, so this mode
has no reference output to pin against).  Checked by properties: it finds
the same hit nodes and bricks as the reference refinement, every hit stays
within the bracketing half-voxel step, and the hit point lies closer to the
isosurface of the trilinear field than the single linear step puts it."""
import os

import numpy as np

import vt_fixtures as F
from oracle import oracle as orc


def trilinear(vol, p):
    """Zero-padded trilinear interpolation of vol ([x][y][z]) at points p."""
    n = np.array(vol.shape)
    f = np.floor(p).astype(np.int64)
    w = (p - f).astype(np.float64)
    out = np.zeros(len(p))
    for dx in (0, 1):
        for dy in (0, 1):
            for dz in (0, 1):
                q = f + np.array([dx, dy, dz])
                ok = np.all((q >= 0) & (q < n), axis=1)
                v = np.zeros(len(p))
                v[ok] = vol[q[ok, 0], q[ok, 1], q[ok, 2]]
                wx = w[:, 0] if dx else 1 - w[:, 0]
                wy = w[:, 1] if dy else 1 - w[:, 1]
                wz = w[:, 2] if dz else 1 - w[:, 2]
                out += v * wx * wy * wz
    return out


def ball_volume(n=64, radius=18.0):
    """v = radius - |x - c| (float32), c the volume centre: the isosurface
    v = 8 is a sphere of radius 10 whose curvature the single linear step
    misses, and every value outside it is below 8, so the zero padding adds
    no crossing at the volume's faces."""
    x, y, z = np.meshgrid(*(np.arange(n, dtype=np.float32),) * 3, indexing="ij")
    c = np.float32((n - 1) / 2.0)
    return (np.float32(radius) - np.sqrt((x - c) ** 2 + (y - c) ** 2 + (z - c) ** 2)).astype(np.float32)


def test_bisection_refines_toward_the_isosurface(workdir):
    vol, iso = ball_volume(), 8.0
    path = os.path.join(workdir, "ball64.oct")
    orc.build_octree(vol, iso, path)
    o = orc.Octree(path)
    cam = orc.Camera(96, 96, 50.0, 30.0, 30.0)
    orc.apply_ops(cam, [("mv", (31.5, 31.5, 61.5))])
    lin = orc.render(o, vol, cam, 4, 3, 3)
    bis = orc.render(o, vol, cam, 4, 3, 3, refine=5)
    assert np.array_equal(lin["node"], bis["node"]) and np.array_equal(lin["brick"], bis["brick"])
    hit = lin["node"] != 0
    assert hit.sum() > 1000
    assert bis["agg"]["samples"] == lin["agg"]["samples"] + 5 * int(hit.sum())
    assert np.abs(bis["t"][hit] - lin["t"][hit]).max() <= 0.5 + 1e-4
    d = cam.rays()[hit].astype(np.float64)
    pos = np.array(cam.state()["position"], np.float64)
    res = {}
    for name, r in (("linear", lin), ("bisection", bis)):
        x = pos + d * r["t"][hit, None].astype(np.float64)
        res[name] = np.abs(trilinear(vol, x) - iso)
    # five halvings of the bracket: the residual drops by far more than 10x
    assert res["bisection"].mean() < 0.1 * res["linear"].mean()
    assert res["bisection"].max() < 0.1 * res["linear"].max()
