"""HDF5 volume files (libvt's own reader and writer, written from the HDF5
file-format specification; there is no libhdf5 in this environment).

The writer must produce what libhdf5 writes by default for one contiguous
dataset, and the reader must read it back and read files libhdf5 wrote.
A libhdf5-written file ships with scipy (a MATLAB v7.3 file: HDF5 after a
512-byte user block); where it is installed it is read as an external
check.  FileManager semantics (zero padding outside the volume) are
checked against the oracle's restatement of the reference's reader."""
import os
import struct

import numpy as np
import pytest

import vt_fixtures as F
import visualtur_b200 as vt
from oracle import oracle as orc

SIG = b"\x89HDF\r\n\x1a\n"


def test_hdf5_roundtrip_f32_and_u8(workdir):
    vol = F.case_volume("s64")
    path = os.path.join(workdir, "s64.h5")
    vt.FileManager.CreateFile(vol, path, "value")
    fm = vt.FileManager(path, "value")
    assert fm.dims == (64, 64, 64) and fm.vtype == vt.VT_F32
    assert np.array_equal(fm.readHDF5(), vol)
    for s, e in (((-3, 5, 60), (9, 20, 70)), ((0, 0, 0), (64, 64, 64)), ((62, -2, 1), (70, 3, 2))):
        assert np.array_equal(fm.readHDF5_Voxel_Array(s, e), orc.read_voxels(vol, s, e))
    fm.close()
    u8 = (np.arange(5 * 6 * 7) % 253).astype(np.uint8).reshape(5, 6, 7)
    vt.FileManager.CreateFile(u8, path, "/density")
    fm = vt.FileManager(path, "density")
    assert fm.vtype == vt.VT_U8 and fm.dims == (5, 6, 7) and np.array_equal(fm.readHDF5(), u8)


def test_hdf5_file_structure(workdir):
    """Independent reading of the written file's key structures."""
    vol = np.arange(2 * 3 * 4, dtype=np.float32).reshape(2, 3, 4)
    path = os.path.join(workdir, "small.h5")
    vt.FileManager.CreateFile(vol, path, "value")
    b = open(path, "rb").read()
    assert b[:8] == SIG and b[8] == 0                      # superblock version 0
    assert b[13] == 8 and b[14] == 8                       # 8-byte offsets and lengths
    leaf_k, inner_k = struct.unpack_from("<HH", b, 16)
    assert (leaf_k, inner_k) == (4, 16)
    base, free, eof, drv = struct.unpack_from("<QQQQ", b, 24)
    assert base == 0 and free == 2 ** 64 - 1 and drv == 2 ** 64 - 1 and eof == len(b)
    _, root_oh, cache, _, btree, heap = struct.unpack_from("<QQIIQQ", b, 56)
    assert cache == 1 and b[btree:btree + 4] == b"TREE" and b[heap:heap + 4] == b"HEAP"
    hsize, hfree, hdata = struct.unpack_from("<QQQ", b, heap + 8)
    assert b[hdata + 8:hdata + 14] == b"value\x00"
    nxt, fsize = struct.unpack_from("<QQ", b, hdata + hfree)
    assert nxt == 1 and hfree + fsize == hsize             # free list ends with offset 1
    info = vt.FileManager.h5_describe(path, "value")
    assert info["rank"] == 3 and info["dims"] == (2, 3, 4) and info["class"] == "float" and info["size"] == 4
    assert info["offset"] % 512 == 0 and info["bytes"] == vol.nbytes
    assert np.array_equal(np.frombuffer(b, np.float32, 24, info["offset"]).reshape(2, 3, 4), vol)


def _patch_type(path, out, code, props, esize, values):
    """Rewrites a float32 (2,3,4) file written by libvt as another element
    type: datatype message, layout size and data (appended at the same
    offset)."""
    b = bytearray(open(path, "rb").read())
    f32 = bytes([0x11, 0x20, 31, 0]) + struct.pack("<I", 4)
    i = b.index(f32)
    new = bytes(code) + struct.pack("<I", esize) + props
    b[i:i + 20] = new.ljust(20, b"\x00")
    info = vt.FileManager.h5_describe(path, "value")
    lay = b.index(bytes([3, 1]) + struct.pack("<QQ", info["offset"], info["bytes"]))
    n = values.size
    b[lay + 10:lay + 18] = struct.pack("<Q", n * esize)
    b = b[:info["offset"]] + values.tobytes()
    struct.pack_into("<Q", b, 40, len(b))
    open(out, "wb").write(bytes(b))


def test_hdf5_other_types_convert_to_float32(workdir):
    vol = np.zeros((2, 3, 4), np.float32)
    path = os.path.join(workdir, "t.h5")
    vt.FileManager.CreateFile(vol, path, "value")
    # float64: class 1 version 1, LE, sign bit 63, exponent 52/11, mantissa 0/52, bias 1023
    d = (np.arange(24, dtype=np.float64) * np.pi / 4).reshape(2, 3, 4)
    p64 = os.path.join(workdir, "f64.h5")
    _patch_type(path, p64, [0x11, 0x20, 63, 0], struct.pack("<HHBBBBI", 0, 64, 52, 11, 0, 52, 1023), 8, d)
    assert vt.FileManager.h5_describe(p64, "value")["size"] == 8
    fm = vt.FileManager(p64, "value")
    assert fm.vtype == vt.VT_F32 and np.array_equal(fm.readHDF5(), d.astype(np.float32))
    # signed 16-bit integers: class 0 version 1, bit 3 = signed
    s16 = (np.arange(24, dtype=np.int16) * -1234).reshape(2, 3, 4)
    p16 = os.path.join(workdir, "i16.h5")
    _patch_type(path, p16, [0x10, 0x08, 0, 0], struct.pack("<HH", 0, 16), 2, s16)
    fm = vt.FileManager(p16, "value")
    assert np.array_equal(fm.readHDF5(), s16.astype(np.float32))


def test_hdf5_errors(workdir):
    vol = np.zeros((2, 3, 4), np.float32)
    path = os.path.join(workdir, "e.h5")
    vt.FileManager.CreateFile(vol, path, "value")
    with pytest.raises(vt.VtError) as e:
        vt.FileManager(path, "missing")
    assert e.value.status == vt.VT_ERR_FORMAT and "missing" in str(e.value)
    b = bytearray(open(path, "rb").read())
    bad = os.path.join(workdir, "trunc.h5")
    open(bad, "wb").write(bytes(b[:len(b) - 8]))
    with pytest.raises(vt.VtError) as e:
        vt.FileManager(bad, "value")
    assert e.value.status == vt.VT_ERR_FORMAT


MAT73 = os.path.join(os.path.dirname(np.__file__), "..", "scipy", "io", "matlab", "tests", "data",
                     "testhdf5_7.4_GLNX86.mat")


@pytest.mark.skipif(not os.path.exists(MAT73), reason="libhdf5-written sample file not installed")
def test_reads_a_file_written_by_libhdf5():
    """MATLAB v7.3 file (libhdf5 1.8): HDF5 after a 512-byte user block,
    variable `testdouble` = [0, pi/4, ..., 2 pi] stored as a (9, 1) float64
    dataset with a version-2 layout message."""
    info = vt.FileManager.h5_describe(MAT73, "testdouble")
    assert info["rank"] == 2 and info["dims"] == (9, 1)
    assert info["class"] == "float" and info["size"] == 8 and not info["big_endian"]
    raw = open(MAT73, "rb").read()
    vals = np.frombuffer(raw, "<f8", 9, info["offset"])
    assert np.allclose(vals, np.arange(9) * np.pi / 4)
    with pytest.raises(vt.VtError):
        vt.FileManager(MAT73, "testdouble")   # not 3-D
