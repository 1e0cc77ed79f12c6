"""Shared test inputs: seeded volumes (numpy restatement of the sphere
generator), raw volume files, and the fixture cases used by the golden
vectors in tests/golden/ and by the parity tests.

Test infrastructure: imports the oracle (oracle/oracle.py) to build octrees.
"""
import os
import struct
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(z):
    z = z + np.uint64(0x9E3779B97F4A7C15)
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def sphere_volume(seed, n, c, sigma=0.25):
    """Cubic n^3 version of sphere_volume_shape."""
    return sphere_volume_shape(seed, (n, n, n), c, sigma)


def sphere_volume_shape(seed, shape, c, sigma=0.25):
    """v(x) = |x - c| + sigma * g, g a 4-term Irwin-Hall N(0,1) draw from
    splitmix64 counters 2k, 2k+1 of voxel k = (x*ny + y)*nz + z; float32
    arithmetic, left to right (the VT_GEN_SPHERE generator of libvt.so)."""
    nx, ny, nz = shape
    with np.errstate(over="ignore"):
        x, y, z = np.meshgrid(np.arange(nx, dtype=np.int64), np.arange(ny, dtype=np.int64),
                              np.arange(nz, dtype=np.int64), indexing="ij")
        k = ((x * ny + y) * nz + z).astype(np.uint64)
        s = np.uint64(seed)
        r0 = splitmix64(s + np.uint64(2) * k)
        r1 = splitmix64(s + np.uint64(2) * k + np.uint64(1))
        m24 = np.uint64(0xFFFFFF)
        S = (r0 >> np.uint64(40)) + ((r0 >> np.uint64(16)) & m24) + (r1 >> np.uint64(40)) + \
            ((r1 >> np.uint64(16)) & m24)
    g = (S.astype(np.float32) * np.float32(5.9604644775390625e-08) - np.float32(2.0)) * np.float32(1.7320508075688772)
    dx = x.astype(np.float32) - np.float32(c[0])
    dy = y.astype(np.float32) - np.float32(c[1])
    dz = z.astype(np.float32) - np.float32(c[2])
    r = np.sqrt(dx * dx + dy * dy + dz * dz)
    return (r + np.float32(sigma) * g).astype(np.float32)


def write_raw(path, vol):
    """Raw volume file: 64-byte header "VTVOL001", u32 1, u32 type, i64 dims[3],
    u64 offset 64, then voxels (x slowest)."""
    vol = np.ascontiguousarray(vol)
    vt = 1 if vol.dtype == np.uint8 else 0
    h = b"VTVOL001" + struct.pack("<II", 1, vt) + struct.pack("<qqq", *vol.shape) + struct.pack("<Q", 64)
    h = h + b"\0" * (64 - len(h))
    with open(path, "wb") as f:
        f.write(h)
        f.write(vol.tobytes())


# Fixture cases.  Camera ops follow the reference API (visualTur::camera_*).
CASES = {
    # 64^3 sphere, 8^3 bricks (levelCubes 3), 4^3 candidate nodes (octreeLevel 4)
    "s64": dict(seed=7, n=64, c=(31.5, 31.5, 31.5), sigma=0.25, iso=20.0, levelC=3, levelO=4, inc=3,
                W=96, H=96, fov=30.0, dist=50.0, ops=[("mv", (31.5, 31.5, 181.5))]),
    # same volume, every camera operation exercised
    "s64rot": dict(seed=7, n=64, c=(31.5, 31.5, 31.5), sigma=0.25, iso=20.0, levelC=3, levelO=4, inc=3,
                   W=80, H=72, fov=25.0, dist=50.0,
                   ops=[("mv", (31.5, 31.5, 181.5)), ("ry", 10.0), ("rx", -8.0), ("rz", 5.0), ("mf", 20.0),
                        ("sr", 3.0), ("mu", -2.0)]),
    # the 128^3 noisy-sphere volume of the resident benchmark, 8^3 bricks
    "c1": dict(seed=1234, n=128, c=(63.5, 63.5, 63.5), sigma=0.25, iso=40.0, levelC=4, levelO=5, inc=3,
               W=128, H=128, fov=30.0, dist=50.0, ops=[("mv", (63.5, 63.5, 363.5))]),
    # camera on node planes (x = y = 64) with an odd screen: slab products of
    # exactly 0, coincident events and infinite reciprocals exercise the
    # traversal's exact-tie paths
    "c1plane": dict(seed=1234, n=128, c=(63.5, 63.5, 63.5), sigma=0.25, iso=40.0, levelC=4, levelO=5, inc=3,
                    W=65, H=65, fov=20.0, dist=50.0, ops=[("mv", (64.0, 64.0, 200.0))]),
    # camera inside the volume's bounding box (tnear clamped to 0 paths)
    "c1in": dict(seed=1234, n=128, c=(63.5, 63.5, 63.5), sigma=0.25, iso=40.0, levelC=4, levelO=5, inc=3,
                 W=64, H=64, fov=40.0, dist=50.0, ops=[("mv", (63.5, 70.25, 120.0)), ("ry", 17.0)]),
}


def case_volume(case):
    c = CASES[case]
    return sphere_volume(c["seed"], c["n"], c["c"], c["sigma"])


def case_octree(case, workdir):
    """Builds (with the oracle) and returns the octree file of a case."""
    from oracle import oracle as orc
    c = CASES[case]
    path = os.path.join(workdir, "%s_n%d_iso%g.oct" % (case, c["n"], c["iso"]))
    if not os.path.exists(path):
        orc.build_octree(case_volume(case), c["iso"], path)
    return path


def oracle_camera(case):
    from oracle import oracle as orc
    c = CASES[case]
    cam = orc.Camera(c["H"], c["W"], c["dist"], c["fov"], c["fov"])
    orc.apply_ops(cam, c["ops"])
    return cam
