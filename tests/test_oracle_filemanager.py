"""Known-answer checks of the zero-padded hyperslab read, mirroring the
reference's only self-checking test (src/testFileManager.cu:8-100): a box
shifted to negative offsets reads 0 outside the volume and the reference
values inside.  Applied to the oracle and to libvt.so's host reader."""
import numpy as np
import pytest

import vt_fixtures as F
from oracle import oracle as orc

INC, DIM = 2, 32
DIM2 = DIM + 2 * INC


def check_values(d1, d2, minBox, maxBox):
    """checkValues (src/testFileManager.cu:8-36)."""
    for i in range(abs(minBox[0])):
        for j in range(abs(minBox[1])):
            for k in range(abs(minBox[2])):
                assert d2[i, j, k] == 0.0
    ax, ay, az = abs(minBox[0]), abs(minBox[1]), abs(minBox[2])
    sub2 = d2[ax:maxBox[0], ay:maxBox[1], az:maxBox[2]]
    sub1 = d1[ax + minBox[0]:maxBox[0] + minBox[0], ay + minBox[1]:maxBox[1] + minBox[1],
              az + minBox[2]:maxBox[2] + minBox[2]]
    assert np.array_equal(sub1, sub2)


SHIFTS = [(-2 * INC, -2 * INC, -2 * INC), (-2 * INC, 0, 0), (0, -2 * INC, 0), (0, 0, 0)]


def readers():
    import visualtur_b200 as vt
    vol = F.sphere_volume(7, 64, (31.5, 31.5, 31.5))
    fm = vt.FileManager.wrap(vol)
    return vol, [("oracle", lambda s, e: orc.read_voxels(vol, s, e)),
                 ("libvt", lambda s, e: fm.readHDF5_Voxel_Array(s, e))], fm


@pytest.mark.parametrize("shift", SHIFTS)
def test_filemanager_kat(shift):
    vol, rs, fm = readers()
    for name, rd in rs:
        d1 = rd((0, 0, 0), (DIM2, DIM2, DIM2))
        assert np.array_equal(d1, vol[:DIM2, :DIM2, :DIM2]), name
        mn = shift
        mx = tuple(mn[a] + DIM2 for a in range(3))
        d2 = rd(mn, mx)
        check_values(d1, d2, mn, mx)


def test_filemanager_outside_and_far_edges():
    vol, rs, fm = readers()
    for name, rd in rs:
        assert not rd((64, 0, 0), (70, 6, 6)).any(), name            # completely outside (+x)
        assert not rd((-10, 0, 0), (-1, 5, 5)).any(), name           # completely outside (-x)
        d = rd((60, 61, 62), (68, 69, 70))                            # straddles the + faces
        assert np.array_equal(d[:4, :3, :2], vol[60:, 61:, 62:])
        assert not d[4:].any() and not d[:, 3:].any() and not d[:, :, 2:].any()
