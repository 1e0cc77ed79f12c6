"""Headless frame files and the volume converter (the reference's GLUT
viewer / FreeImage dumps and src/cutFile.cu)."""
import os

import numpy as np
import pytest

import vt_fixtures as F
import visualtur_b200 as vt
from oracle import oracle as orc
from visualtur_b200 import convert, frames


def test_png_and_ppm_round_trip(workdir):
    W, H = 37, 21
    rgb = (np.arange(W * H * 3) % 251).astype(np.uint8)
    p = os.path.join(workdir, "f.png")
    frames.write_png(p, rgb, W, H)
    img = frames.read_png(p)
    assert img.shape == (H, W, 3)
    assert np.array_equal(img, rgb.reshape(H, W, 3)[::-1])          # top row first
    q = os.path.join(workdir, "f.ppm")
    frames.write_ppm(q, rgb, W, H, bottom_up=False)
    raw = open(q, "rb").read()
    head = b"P6\n%d %d\n255\n" % (W, H)
    assert raw.startswith(head) and raw[len(head):] == rgb.tobytes()


def test_convert_raw_hdf5_and_crop(workdir):
    vol = F.case_volume("s64")
    raw = os.path.join(workdir, "v.raw")
    vt.FileManager.CreateFile(vol, raw, fmt=0)
    h5 = os.path.join(workdir, "v.h5")
    assert convert.convert(raw, h5, fmt="hdf5")[0] == (64, 64, 64)
    back = os.path.join(workdir, "back.raw")
    convert.convert(h5, back, fmt="raw")
    assert np.array_equal(vt.FileManager(back).readHDF5(), vol)
    # cutFile: a 24^3 cube reaching past the volume's corner, zero padded
    cut = os.path.join(workdir, "cut.h5")
    convert.main([h5, cut, "--crop", "50,-4,30,24"])
    got = vt.FileManager(cut).readHDF5()
    assert got.shape == (24, 24, 24) and got.dtype == np.float32
    assert np.array_equal(got, orc.read_voxels(vol, (50, -4, 30), (74, 20, 54)))
    u8 = (np.arange(6 * 7 * 8) % 250).astype(np.uint8).reshape(6, 7, 8)
    src = os.path.join(workdir, "u8.raw")
    vt.FileManager.CreateFile(u8, src, fmt=0)
    dst = os.path.join(workdir, "u8.h5")
    assert convert.convert(src, dst)[1] == np.uint8                  # type kept without a crop
    assert np.array_equal(vt.FileManager(dst).readHDF5(), u8)


@pytest.mark.gpu
def test_frames_cli_matches_render(workdir, cuda):
    c = F.CASES["s64"]
    vol = F.case_volume("s64")
    h5 = os.path.join(workdir, "s64_frames.h5")
    vt.FileManager.CreateFile(vol, h5)
    oct_path = F.case_octree("s64", workdir)
    out = os.path.join(workdir, "frames")
    paths = frames.main(["--volume", h5, "--octree", oct_path, "--levelO", str(c["levelO"]),
                         "--levelC", str(c["levelC"]), "--W", str(c["W"]), "--H", str(c["H"]),
                         "--fov", str(c["fov"]), "--distance", str(c["dist"]),
                         "--move", ",".join(str(v) for v in c["ops"][0][1]), "--strafe", "0.5",
                         "--frames", "2", "--out", out])
    assert len(paths) == 2
    cam = orc.Camera(c["H"], c["W"], c["dist"], c["fov"], c["fov"])
    orc.apply_ops(cam, c["ops"])
    o = orc.Octree(oct_path)
    for k, p in enumerate(paths):
        ref = orc.render(o, vol, cam, c["levelO"], c["levelC"], c["inc"])["rgb8"].reshape(c["H"], c["W"], 3)
        assert np.array_equal(frames.read_png(p), ref[::-1])
        cam.StrafeRight(0.5)
