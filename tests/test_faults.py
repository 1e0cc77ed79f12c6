"""Host-side failures, injected on the host (no GPU): files that are
missing or short, a volume whose reads fail, option bounds.  The reference
exit(0)s on an HDF5 error (src/FileManager.cu:15-36) and throws on a bad
octree magic (src/Octree.cu:781-785); libvt returns a status and a message
instead.  The render-time forms of these failures are in
test_gpu_faults.py."""
import os
import struct

import numpy as np
import pytest

import vt_fixtures as F
import visualtur_b200 as vt
from oracle import oracle as orc


def test_missing_volume_file_is_an_io_error(tmp_path):
    with pytest.raises(vt.VtError) as e:
        vt.FileManager(str(tmp_path / "nope.vtvol"))
    assert e.value.status == vt.VT_ERR_IO and "nope.vtvol" in str(e.value)


def test_short_volume_file_is_a_format_error(tmp_path):
    vol = F.sphere_volume(3, 16, (7.5, 7.5, 7.5))
    p = str(tmp_path / "short.vtvol")
    F.write_raw(p, vol)
    with open(p, "r+b") as f:            # a short read: the file ends early
        f.truncate(64 + vol.nbytes // 2)
    with pytest.raises(vt.VtError) as e:
        vt.FileManager(p)
    assert e.value.status == vt.VT_ERR_FORMAT and "truncated" in str(e.value)


def test_bad_octree_magic_is_a_format_error(tmp_path):
    p = str(tmp_path / "bad.oct")
    with open(p, "wb") as f:
        f.write(struct.pack("<ifiiiii", 1234, 0.5, 16, 16, 16, 16, 4))
    with pytest.raises(vt.VtError) as e:
        vt.Octree(p)
    assert e.value.status == vt.VT_ERR_FORMAT


def test_reader_volume_reads_through_the_function_and_reports_failures():
    vol = F.sphere_volume(5, 24, (11.5, 11.5, 11.5))
    fail = {"on": False}
    calls = []

    def read(s, e):
        calls.append((s, e))
        if fail["on"]:
            return None                   # a missing brick / short read
        return orc.read_voxels(vol, s, e)
    fm = vt.FileManager.from_reader(read, vol.shape)
    assert fm.dims == vol.shape
    got = fm.readHDF5_Voxel_Array((-3, 4, 20), (9, 30, 27))
    assert np.array_equal(got, orc.read_voxels(vol, (-3, 4, 20), (9, 30, 27)))
    assert calls[-1] == ((-3, 4, 20), (9, 30, 27))
    fail["on"] = True
    with pytest.raises(vt.VtError) as e:
        fm.readHDF5_Voxel_Array((0, 0, 0), (4, 4, 4))
    assert e.value.status == vt.VT_ERR_IO and "failed" in str(e.value)
    fail["on"] = False
    assert np.array_equal(fm.readHDF5(), vol)


def test_reader_volume_cannot_feed_the_octree_builder(tmp_path):
    vol = F.sphere_volume(5, 16, (7.5, 7.5, 7.5))
    fm = vt.FileManager.from_reader(lambda s, e: orc.read_voxels(vol, s, e), vol.shape)
    with pytest.raises(vt.VtError) as e:
        vt.build_octree(fm, 5.0, str(tmp_path / "x.oct"))
    assert e.value.status == vt.VT_ERR_UNSUPPORTED


@pytest.mark.parametrize("field,value", [("max_passes", 0), ("max_suspended", -1), ("max_requests", -2),
                                         ("pool_per_ray", -1)])
def test_queue_bounds_are_validated(field, value, tmp_path):
    c = F.CASES["s64"]
    vol = F.case_volume("s64")
    fm, oc = vt.FileManager.wrap(vol), vt.Octree(F.case_octree("s64", str(tmp_path)))
    p = vt.make_params(W=c["W"], H=c["H"], octreeFile=None, hdf5File=None, octreeLevel=c["levelO"],
                       levelCubes=c["levelC"], dimCube=8, maxElementsCache=64, maxElementsCache_CPU=64)
    with pytest.raises(vt.VtError) as e:
        vt.visualTur(p, vt.default_options(**{field: value}), volume=fm, octree=oc)
    assert e.value.status == vt.VT_ERR_INVALID
