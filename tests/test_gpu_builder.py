"""GPU octree builder (vt_octree_build) against the reference's own builder:
byte-identical files (SHA-256 of the reference's volumeToOctree output in
tests/golden/ref_octree_sha256.json) and equal to the oracle's builder."""
import hashlib
import json
import os

import numpy as np
import pytest

import vt_fixtures as F
import visualtur_b200 as vt
from oracle import oracle as orc

pytestmark = pytest.mark.gpu
GOLD = json.load(open(os.path.join(F.GOLDEN, "ref_octree_sha256.json")))


@pytest.mark.parametrize("name", sorted(GOLD))
def test_gpu_builder_matches_reference_bytes(name, workdir, cuda):
    g = GOLD[name]
    vol = F.sphere_volume_shape(g["seed"], tuple(g["shape"]), tuple(g["c"]))
    path = os.path.join(workdir, "gpu_%s.oct" % name)
    vt.build_octree(vt.FileManager.wrap(vol), g["iso"], path)
    data = open(path, "rb").read()
    assert hashlib.sha256(data).hexdigest() == g["sha256"]


@pytest.mark.parametrize("iso", [0.6, 0.9])
def test_gpu_builder_matches_oracle_on_blobs(iso, workdir, cuda):
    vol = vt.generate_volume(vt.VT_GEN_BLOBS, 42, (96, 80, 72), (24, 4.0, 16.0, 0.5, 1.5, 0.05))
    a, b = os.path.join(workdir, "blob_gpu.oct"), os.path.join(workdir, "blob_orc.oct")
    vt.build_octree(vt.FileManager.wrap(vol), iso, a)
    orc.build_octree(vol, iso, b)
    assert open(a, "rb").read() == open(b, "rb").read()


def test_gpu_builder_uint8(workdir, cuda):
    vol = vt.generate_volume(vt.VT_GEN_FRACTAL_U8, 9, (64, 64, 64), (6, 4.0, 12.0, 200.0))
    a, b = os.path.join(workdir, "u8_gpu.oct"), os.path.join(workdir, "u8_orc.oct")
    vt.build_octree(vt.FileManager.wrap(vol), 128.0, a)
    orc.build_octree(vol, 128.0, b)
    assert open(a, "rb").read() == open(b, "rb").read()
