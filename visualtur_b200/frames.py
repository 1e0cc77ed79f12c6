"""Headless frame output: PNG / PPM files instead of a window.

The reference shows frames in a GLUT window (src/drawPixel.cu) and its test
programs save PNGs through FreeImage (src/testVisualTur.cu:52-116); neither
library exists here.  This module writes the RGB8 frames libvt renders as
plain files, with the standard library only.

Row order: the renderer's pixel (i, j) has i = 0 at the bottom of the
screen (src/Camera.cu:59-72), so images are written top row first by
flipping rows (bottom_up=True).

    python -m visualtur_b200.frames --volume vol.h5 --dataset value \\
        --octree vol.oct --levelO 5 --levelC 4 --W 512 --H 512 \\
        --move 63.5,63.5,363.5 --strafe 0.5 --frames 10 --out frames/

renders like src/testVisualTur.cu:73-110 (a camera move, then a right
strafe of 0.5 between frames) and saves frames/frame0000.png, ...
"""
import argparse
import os
import struct
import zlib

import numpy as np


def _rows(rgb8, W, H, bottom_up):
    img = np.asarray(rgb8, np.uint8).reshape(H, W, 3)
    return img[::-1] if bottom_up else img


def write_ppm(path, rgb8, W, H, bottom_up=True):
    """Binary PPM (P6) of a W x H RGB8 frame."""
    img = _rows(rgb8, W, H, bottom_up)
    with open(path, "wb") as f:
        f.write(b"P6\n%d %d\n255\n" % (W, H))
        f.write(np.ascontiguousarray(img).tobytes())


def write_png(path, rgb8, W, H, bottom_up=True):
    """8-bit RGB PNG (no filtering, zlib level 6) of a W x H RGB8 frame."""
    img = _rows(rgb8, W, H, bottom_up)
    raw = b"".join(b"\x00" + img[r].tobytes() for r in range(H))

    def chunk(tag, data):
        return struct.pack(">I", len(data)) + tag + data + struct.pack(">I", zlib.crc32(tag + data) & 0xFFFFFFFF)

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", W, H, 8, 2, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(chunk(b"IEND", b""))


def read_png(path):
    """Inverse of write_png (8-bit RGB, filter type 0 rows): H x W x 3."""
    with open(path, "rb") as f:
        data = f.read()
    assert data[:8] == b"\x89PNG\r\n\x1a\n", "not a PNG"
    pos, idat, W, H = 8, b"", 0, 0
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag, body = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        if tag == b"IHDR":
            W, H, depth, ctype = struct.unpack(">IIBB", body[:10])
            assert depth == 8 and ctype == 2, "only 8-bit RGB"
        elif tag == b"IDAT":
            idat += body
        pos += 12 + n
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(H, 1 + 3 * W)
    assert (raw[:, 0] == 0).all(), "only filter type 0"
    return raw[:, 1:].reshape(H, W, 3)


def main(argv=None):
    import visualtur_b200 as vt
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--volume", required=True)
    ap.add_argument("--dataset", default="value")
    ap.add_argument("--octree", required=True)
    ap.add_argument("--levelO", type=int, required=True)
    ap.add_argument("--levelC", type=int, required=True)
    ap.add_argument("--inc", type=int, default=3)
    ap.add_argument("--W", type=int, default=512)
    ap.add_argument("--H", type=int, default=512)
    ap.add_argument("--fov", type=float, default=30.0, help="half-angle, degrees (the reference's fov)")
    ap.add_argument("--distance", type=float, default=50.0)
    ap.add_argument("--move", default="0,0,0", help="camera Move before the first frame")
    ap.add_argument("--strafe", type=float, default=0.0, help="StrafeRight between frames")
    ap.add_argument("--frames", type=int, default=1)
    ap.add_argument("--format", choices=("png", "ppm"), default="png")
    ap.add_argument("--out", required=True)
    a = ap.parse_args(argv)
    fm, oc = vt.FileManager(a.volume, a.dataset), vt.Octree(a.octree)
    p = vt.make_params(W=a.W, H=a.H, octreeFile=None, hdf5File=None, octreeLevel=a.levelO, levelCubes=a.levelC,
                       dimCube=1 << (oc.nLevels - a.levelC), cubeInc=a.inc, distance=a.distance, fov_H=a.fov,
                       fov_W=a.fov)
    r = vt.visualTur(p, vt.default_options(record_hits=0), volume=fm, octree=oc)
    r.camera_Move(tuple(float(v) for v in a.move.split(",")))
    os.makedirs(a.out, exist_ok=True)
    write = write_png if a.format == "png" else write_ppm
    paths = []
    for k in range(a.frames):
        _, rgb8 = r.render_host(rgb8=True)
        path = os.path.join(a.out, "frame%04d.%s" % (k, a.format))
        write(path, rgb8, a.W, a.H)
        paths.append(path)
        if a.strafe:
            r.camera_StrafeRight(a.strafe)
    r.close()
    return paths


if __name__ == "__main__":
    for p in main():
        print(p)
