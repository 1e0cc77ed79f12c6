"""The bench's workload table and tuner candidates, checked on the CPU:
the plain renderer stays the reference's scheme, and every paging
candidate is a setting the library accepts."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_plain_mode_is_the_reference_scheme():
    o = bench.MODES["plain"]["opts"]
    assert o["lookahead"] == 0 and o.get("skip", 0) == 0 and o["persistent"] == 0 and o["use_graph"] == 0
    assert bench.MODES["plain"]["batch"] == 1 and not bench.MODES["plain"]["learned"]


def test_paging_candidates_are_valid_settings():
    seen = set()
    for b, la, sk in bench.PAGING_CANDIDATES:
        assert b >= 1 and 0 <= la <= 64 and 0 <= sk <= 4
        assert (b, la, sk) not in seen
        seen.add((b, la, sk))
    assert any(sk == 0 for _, _, sk in bench.PAGING_CANDIDATES)   # the in-order traversal is always a candidate
    for t in bench.HINT_THRESHOLDS:
        assert t is None or 0.0 < t < 1.0


def test_every_workload_names_its_shape():
    for name, c in bench.CONFIGS.items():
        assert c["workload"] and c["W"] > 0 and c["H"] > 0, name
        assert c["inc"] >= 3 and c["levelC"] <= c["levelO"], name
        assert c["resident"] or c["dev_bytes"] > 0, name


def test_views_paging_candidates_are_valid_settings():
    assert (2, 0) in bench.VIEWS_PAGING          # the mode's own setting stays a candidate
    for la, sk in bench.VIEWS_PAGING:
        assert 0 <= la <= 64 and 0 <= sk <= 4


@pytest.mark.parametrize("frames,batch", [(20, 8), (20, 16), (20, 4), (300, 16), (7, 1), (3, 8)])
def test_launch_split_covers_the_stretch_once(frames, batch):
    """Timed runs and tuner trials render exactly the frames of their
    stretch: the last launch holds only what is left (a trial that rendered
    whole batches charged large batches for frames past the stretch)."""
    out = bench.launch_split(40, frames, batch)
    got = [f for f0, n, _ in out for f in range(f0, f0 + n)]
    assert got == list(range(40, 40 + frames))
    assert all(0 < n <= batch for _, n, _ in out)
    assert [nxt for _, _, nxt in out] == [n for _, n, _ in out[1:]] + [0]
