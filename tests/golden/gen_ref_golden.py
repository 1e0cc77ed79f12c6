"""Generates the golden vectors in tests/golden/ from the reference itself.

Runs the reference's own code, built from its sources by oracle/ref_build.sh
into oracle/_ref/ (test infrastructure):
  * volumeToOctree (its octree builder CLI, host code)  -> ref_octree_sha256.json
  * vtref render (visualTur + camera ops + updateVisibleCubes, GPU)
                                                       -> ref_render_<case>.npz
  * vtref cube (rayCaster::renderCube, GPU)            -> ref_cube.npz
  * vtref lru (lruCache::updateCache, GPU memory)      -> ref_lru.npz
Inputs are the seeded volumes of tests/vt_fixtures.py.

    python tests/golden/gen_ref_golden.py OUTDIR [--cpu-only]

--cpu-only produces only the builder hashes (no GPU needed).
"""
import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import vt_fixtures as F  # noqa: E402

REF = os.path.join(F.ROOT, "oracle", "_ref")

# builder pins: fixture volumes plus non-cubic / non-power-of-two shapes
BUILD_CASES = {
    "s64_iso20": dict(seed=7, shape=(64, 64, 64), c=(31.5, 31.5, 31.5), iso=20.0),
    "c1_iso40": dict(seed=1234, shape=(128, 128, 128), c=(63.5, 63.5, 63.5), iso=40.0),
    "odd_50x40x33": dict(seed=5, shape=(50, 40, 33), c=(20.0, 18.5, 16.0), iso=12.0),
    "wide_96x32x48": dict(seed=11, shape=(96, 32, 48), c=(47.5, 15.5, 23.5), iso=14.5),
    "tiny_17": dict(seed=3, shape=(17, 17, 17), c=(8.0, 8.0, 8.0), iso=5.0),
}


def build_volume(bc):
    """Sphere volume of arbitrary shape (same formula, linear index over the shape)."""
    nx, ny, nz = bc["shape"]
    n = max(nx, ny, nz)
    full = F.sphere_volume_shape(bc["seed"], bc["shape"], bc["c"])
    assert full.shape == (nx, ny, nz) and n > 0
    return full


def run(cmd, **kw):
    r = subprocess.run(cmd, capture_output=True, text=True, **kw)
    if r.returncode != 0:
        raise RuntimeError("%s failed (%d): %s" % (cmd[0], r.returncode, r.stdout[-2000:]))
    return r


def ref_octree(raw, out, iso):
    run([os.path.join(REF, "volumeToOctree"), raw, out], input="%r\n" % iso)


def builder_hashes(work):
    res = {}
    for name, bc in BUILD_CASES.items():
        vol = build_volume(bc)
        raw = os.path.join(work, name + ".raw")
        F.write_raw(raw, vol)
        oct_ = os.path.join(work, name + ".oct")
        ref_octree(raw, oct_, bc["iso"])
        data = open(oct_, "rb").read()
        res[name] = dict(bc, shape=list(bc["shape"]), c=list(bc["c"]), bytes=len(data),
                         sha256=hashlib.sha256(data).hexdigest())
    return res


def load(path, dtype, shape=None):
    a = np.fromfile(path, dtype)
    return a.reshape(shape) if shape else a


def render_case(case, work, outdir):
    c = F.CASES[case]
    vol = F.case_volume(case)
    raw = os.path.join(work, case + ".raw")
    F.write_raw(raw, vol)
    oct_ = os.path.join(work, case + ".oct")
    ref_octree(raw, oct_, c["iso"])
    nb = (c["n"] // (1 << (int(np.log2(c["n"])) - c["levelC"]))) ** 3
    ops = []
    for op, v in c["ops"]:
        ops.append("%s:%s" % (op, ",".join(repr(float(x)) for x in v)) if op == "mv" else "%s:%r" % (op, float(v)))
    prefix = os.path.join(work, case)
    r = run([os.path.join(REF, "vtref"), "render", raw, oct_, str(c["W"]), str(c["H"]), repr(c["fov"]),
             repr(c["fov"]), repr(c["dist"]), str(c["levelC"]), str(c["levelO"]), str(c["inc"]), str(nb),
             str(nb), prefix] + ops)
    n = c["W"] * c["H"]
    iters = [ln for ln in r.stdout.splitlines() if ln.startswith("Iterations")]
    np.savez_compressed(os.path.join(outdir, "ref_render_%s.npz" % case),
                        rgba=load(prefix + ".rgba", np.float32, (n, 4)),
                        ids=load(prefix + ".ids", np.uint64),
                        cube=load(prefix + ".cube", np.uint64),
                        state=load(prefix + ".state", np.uint8),
                        dirs=load(prefix + ".dirs", np.float32, (n, 3)),
                        cam=load(prefix + ".cam", np.float32),
                        octree_sha256=np.array(hashlib.sha256(open(oct_, "rb").read()).hexdigest()),
                        iterations=np.array(iters[-1] if iters else ""))


CUBE = dict(case="s64", W=96, H=80, dist=50.0, fovH=30.0, fovW=35.0, pos=(16.0, 16.0, 110.0),
            brick=(16, 16, 16), dim=32, inc=3, iso=20.0)


def cube_case(work, outdir):
    cc = CUBE
    vol = F.case_volume(cc["case"])
    raw = os.path.join(work, "cube.raw")
    F.write_raw(raw, vol)
    prefix = os.path.join(work, "cube")
    run([os.path.join(REF, "vtref"), "cube", raw, str(cc["W"]), str(cc["H"]), repr(cc["dist"]), repr(cc["fovH"]),
         repr(cc["fovW"])] + [repr(x) for x in cc["pos"]] + [str(x) for x in cc["brick"]] +
        [str(cc["dim"]), str(cc["inc"]), repr(cc["iso"]), prefix])
    n = cc["W"] * cc["H"]
    D = cc["dim"] + 2 * cc["inc"]
    np.savez_compressed(os.path.join(outdir, "ref_cube.npz"), rgba=load(prefix + ".rgba", np.float32, (n, 4)),
                        dirs=load(prefix + ".dirs", np.float32, (n, 3)),
                        brick=load(prefix + ".brick", np.float32, (D, D, D)))


LRU = dict(case="s64", nGPU=6, nCPU=10, levelO=4, levelC=3, nLevels=6, inc=3, rounds=14, m=40, seed=2024)


def lru_sequence(lc):
    rng = np.random.default_rng(lc["seed"])
    base = 8 ** lc["levelO"]
    pool = rng.choice(np.arange(base, 2 * base, dtype=np.uint64), size=48, replace=False)
    ids = rng.choice(pool, size=(lc["rounds"], lc["m"])).astype(np.uint64)
    states = rng.choice(np.array([0, 1, 2, 4, 8], np.uint8), p=[0.1, 0.2, 0.1, 0.1, 0.5],
                        size=(lc["rounds"], lc["m"])).astype(np.uint8)
    return ids, states


def lru_case(work, outdir):
    lc = LRU
    vol = F.case_volume(lc["case"])
    raw = os.path.join(work, "lru.raw")
    F.write_raw(raw, vol)
    ids, states = lru_sequence(lc)
    seq = os.path.join(work, "lru.seq")
    with open(seq, "wb") as f:
        f.write(np.array([lc["rounds"], lc["m"]], np.int32).tobytes())
        for r in range(lc["rounds"]):
            for i in range(lc["m"]):
                f.write(ids[r, i].tobytes())
                f.write(states[r, i].tobytes())
    out = os.path.join(work, "lru.out")
    run([os.path.join(REF, "vtref"), "lru", raw, str(lc["nGPU"]), str(lc["nCPU"]), str(lc["levelO"]),
         str(lc["levelC"]), str(lc["nLevels"]), str(lc["inc"]), seq, out])
    rec = np.fromfile(out, np.dtype([("state", "u1"), ("slot", "<i4"), ("cube", "<u8")]))
    np.savez_compressed(os.path.join(outdir, "ref_lru.npz"), ids=ids, states=states,
                        out_state=rec["state"].reshape(ids.shape), out_slot=rec["slot"].reshape(ids.shape),
                        out_cube=rec["cube"].reshape(ids.shape), stats=np.fromfile(out + ".stats", np.int64))


def main():
    outdir = sys.argv[1]
    os.makedirs(outdir, exist_ok=True)
    with tempfile.TemporaryDirectory() as work:
        with open(os.path.join(outdir, "ref_octree_sha256.json"), "w") as f:
            json.dump(builder_hashes(work), f, indent=1, sort_keys=True)
        if "--cpu-only" in sys.argv:
            return
        for case in F.CASES:
            render_case(case, work, outdir)
            print("rendered", case, flush=True)
        cube_case(work, outdir)
        lru_case(work, outdir)
    print("golden vectors written to", outdir)


if __name__ == "__main__":
    main()
