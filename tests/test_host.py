"""Host-side logic of libvt.so that needs no GPU: exported ABI, camera
semantics, seeded generators, octree file reading, parameter validation and
error statuses."""
import ctypes
import os
import re

import numpy as np
import pytest

import vt_fixtures as F
import visualtur_b200 as vt
from oracle import oracle as orc


def test_library_exports_every_declared_symbol():
    hdr = open(os.path.join(F.ROOT, "include", "vt.h")).read()
    names = sorted(set(re.findall(r"^\s*(?:[\w\*]+\s+)+\**(vt_\w+)\s*\(", hdr, re.M)))
    assert len(names) > 30
    L = ctypes.CDLL(vt.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert vt.lib().vt_api_version() == 2


OPS = [("mv", (31.5, 31.5, 181.5)), ("ry", 10.0), ("rx", -8.0), ("rz", 5.0), ("mf", 20.0), ("sr", 3.0),
       ("mu", -2.0), ("rx", 33.0), ("ry", -71.5), ("mv", (1.0, -2.0, 0.25))]


def test_camera_ops_bitwise_match_oracle():
    a = vt.Camera(72, 80, 50.0, 25.0, 27.5)
    b = orc.Camera(72, 80, 50.0, 25.0, 27.5)
    m = {"mv": "Move", "rx": "RotateX", "ry": "RotateY", "rz": "RotateZ", "mf": "MoveForward", "mu": "MoveUpward",
         "sr": "StrafeRight"}
    for op, v in OPS:
        getattr(a, m[op])(v)
        getattr(b, m[op])(v)
        sa, sb = a.state(), b.state()
        for k in ("look", "up", "right", "position", "h", "w"):
            assert np.array_equal(np.float32(sa[k]).view(np.uint32), np.float32(sb[k]).view(np.uint32)), (op, k)


@pytest.mark.parametrize("shape,c", [((64, 64, 64), (31.5, 31.5, 31.5)), ((50, 40, 33), (20.0, 18.5, 16.0)),
                                     ((9, 130, 7), (-3.0, 64.25, 100.0))])
def test_sphere_generator_matches_numpy(shape, c):
    a = F.sphere_volume_shape(99, shape, c, 0.25)
    b = vt.generate_volume(vt.VT_GEN_SPHERE, 99, shape, c + (0.25,))
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_other_generators_are_seeded():
    a = vt.generate_volume(vt.VT_GEN_BLOBS, 5, (24, 20, 16), (16, 2.0, 6.0, 0.5, 1.5, 0.05))
    b = vt.generate_volume(vt.VT_GEN_BLOBS, 5, (24, 20, 16), (16, 2.0, 6.0, 0.5, 1.5, 0.05))
    c = vt.generate_volume(vt.VT_GEN_BLOBS, 6, (24, 20, 16), (16, 2.0, 6.0, 0.5, 1.5, 0.05))
    assert np.array_equal(a, b) and not np.array_equal(a, c) and a.dtype == np.float32
    f = vt.generate_volume(vt.VT_GEN_FRACTAL_U8, 5, (32, 32, 32), (4, 3.0, 6.0, 200.0))
    assert f.dtype == np.uint8 and (f == 200).any() and f.min() < 128 < f.max()


def test_octree_reader_matches_oracle(workdir):
    p = F.case_octree("s64", workdir)
    a, b = vt.Octree(p), orc.Octree(p)
    assert (a.isosurface, a.dimension, a.nLevels, a.realDim) == (b.iso, b.dimension, b.nLevels, b.realDim)
    for l in range(a.nLevels + 1):
        assert np.array_equal(a.level(l), b.level(l))


def test_error_statuses(workdir):
    with pytest.raises(vt.VtError) as e:
        vt.FileManager(os.path.join(workdir, "missing.raw"))
    assert e.value.status == vt.VT_ERR_IO
    bad = os.path.join(workdir, "bad.oct")
    open(bad, "wb").write(b"\0" * 64)
    with pytest.raises(vt.VtError) as e:
        vt.Octree(bad)
    assert e.value.status == vt.VT_ERR_FORMAT
    vol = F.case_volume("s64")
    raw = os.path.join(workdir, "s64.raw")
    F.write_raw(raw, vol)
    oct_ = F.case_octree("s64", workdir)
    for kw, status in [(dict(cubeInc=2), vt.VT_ERR_INVALID), (dict(dimCube=16), vt.VT_ERR_INVALID),
                       (dict(octreeLevel=9), vt.VT_ERR_INVALID), (dict(levelCubes=5), vt.VT_ERR_INVALID)]:
        args = dict(W=32, H=32, octreeFile=oct_, hdf5File=raw, octreeLevel=4, levelCubes=3, dimCube=8)
        args.update(kw)
        with pytest.raises(vt.VtError) as e:
            vt.visualTur(vt.make_params(**args))
        assert e.value.status == status, kw
    p = vt.make_params(W=32, H=32, octreeFile=oct_, hdf5File=raw, octreeLevel=4, levelCubes=3, dimCube=8)
    p.numRayPx = 2
    with pytest.raises(vt.VtError) as e:
        vt.visualTur(p)
    assert e.value.status == vt.VT_ERR_UNSUPPORTED


def test_raw_volume_roundtrip(workdir):
    vol = F.case_volume("s64")
    path = os.path.join(workdir, "rt.raw")
    vt.FileManager.CreateFile(vol, path, fmt=0)
    fm = vt.FileManager(path)
    assert fm.dims == (64, 64, 64) and np.array_equal(fm.readHDF5(), vol)
    u8 = (np.arange(4 * 5 * 6) % 251).astype(np.uint8).reshape(4, 5, 6)
    vt.FileManager.CreateFile(u8, path, fmt=0)
    fm = vt.FileManager(path)
    assert fm.vtype == vt.VT_U8 and np.array_equal(fm.readHDF5(), u8)
    assert np.array_equal(fm.readHDF5_Voxel_Array((-1, 0, 2), (3, 5, 8)),
                          orc.read_voxels(u8.astype(np.float32), (-1, 0, 2), (3, 5, 8)))


LAYOUT_STRUCTS = ("vt_camera", "vt_params", "vt_options", "vt_stats", "vt_h5_info", "vt_tuning", "vt_view")


def test_ctypes_mirrors_match_the_header(workdir):
    """Every ctypes mirror of a vt.h struct has the C compiler's size and
    field offsets (a field added on one side only shifts the rest)."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "vt.h"', "int main(void) {"]
    for s in LAYOUT_STRUCTS:
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (s, s))
        for name, _ in getattr(vt, s)._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (s, name, s, name))
    lines.append("return 0; }")
    src = os.path.join(workdir, "layout.c")
    exe = os.path.join(workdir, "layout")
    open(src, "w").write("\n".join(lines) + "\n")
    subprocess.run([cc, "-std=c11", "-I", os.path.join(F.ROOT, "include"), src, "-o", exe], check=True)
    out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {tuple(l.split()[:2]): int(l.split()[2]) for l in out if l.strip()}
    for s in LAYOUT_STRUCTS:
        T = getattr(vt, s)
        assert got[(s, "size")] == ctypes.sizeof(T), s
        for name, _ in T._fields_:
            assert got[(s, name)] == getattr(T, name).offset, (s, name)


def test_default_options_keep_the_reference_order():
    """Defaults: demand paging without lookahead or set-aside candidates
    (the reference's in-order scheme), single linear refinement."""
    o = vt.default_options()
    assert o.lookahead == 0 and o.skip == 0 and o.refine == 0 and o.resident == 0
