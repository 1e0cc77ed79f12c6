"""Pins the oracle's octree builder (src/CreateOctree.cu) against the
reference's own builder: tests/golden/ref_octree_sha256.json holds the
SHA-256 of octree files written by the reference's volumeToOctree, built
from its sources, for these seeded volumes."""
import hashlib
import json
import os

import pytest

import vt_fixtures as F
from oracle import oracle as orc

GOLD = json.load(open(os.path.join(F.GOLDEN, "ref_octree_sha256.json")))


@pytest.mark.parametrize("name", sorted(GOLD))
def test_oracle_builder_matches_reference_bytes(name, workdir):
    g = GOLD[name]
    vol = F.sphere_volume_shape(g["seed"], tuple(g["shape"]), tuple(g["c"]))
    path = os.path.join(workdir, "orc_%s.oct" % name)
    orc.build_octree(vol, g["iso"], path)
    data = open(path, "rb").read()
    assert len(data) == g["bytes"]
    assert hashlib.sha256(data).hexdigest() == g["sha256"]


def test_octree_file_roundtrip_header(workdir):
    g = GOLD["odd_50x40x33"]
    vol = F.sphere_volume_shape(g["seed"], tuple(g["shape"]), tuple(g["c"]))
    path = os.path.join(workdir, "hdr.oct")
    orc.build_octree(vol, g["iso"], path)
    o = orc.Octree(path)
    # dimension is the next power of two of the largest extent (src/CreateOctree.cu:308-319)
    assert (o.iso, o.dimension, o.nLevels, o.realDim) == (g["iso"], 64, 6, (50, 40, 33))
    lv = [o.level(l) for l in range(o.nLevels + 1)]
    assert list(lv[0]) == [1, 1]
    for l, words in enumerate(lv):
        assert words.size % 2 == 0
        if words.size:   # sorted inclusive ranges of level-l codes
            assert (words[1:] >= words[:-1]).all()
            assert words[0] >= 8 ** l and words[-1] < 2 * 8 ** l
