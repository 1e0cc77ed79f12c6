"""Demand paging at scale: a cold first pass that requests more bricks than
one transfer chunk, so the host-tier reads of one chunk run while the GPU
copies the chunk before.  The brick cache only decides when a candidate is
marched, never what it shows: every frame must equal, bit for bit, the
frame of a renderer that holds the whole volume in device memory."""
import math

import numpy as np
import pytest

import visualtur_b200 as vt
from visualtur_b200 import prefetch as pf

pytestmark = pytest.mark.gpu

N, ISO, LC, LO = 512, 0.6, 6, 7          # 8^3 bricks: 262 144 pages
W = H = 1024


def test_chunked_service_matches_resident(cuda):
    torch = cuda
    dvol = torch.empty(N ** 3, dtype=torch.float32, device="cuda")
    s = N / 2048.0
    vt.generate_volume(vt.VT_GEN_BLOBS, 2048, (N, N, N), (256, 20 * s, 120 * s, 0.5, 1.5, 0.05),
                       device_ptr=dvol.data_ptr())
    import tempfile, os
    path = os.path.join(tempfile.mkdtemp(), "blobs512.oct")
    vt.build_octree_device(dvol.data_ptr(), vt.VT_F32, (N, N, N), ISO, path)
    vol = dvol.cpu().numpy().reshape(N, N, N)
    del dvol
    fm, oc = vt.FileManager.wrap(vol), vt.Octree(path)
    bricks = 8 ** LC

    def make(resident, **opt):
        p = vt.make_params(W=W, H=H, octreeFile=None, hdf5File=None, octreeLevel=LO, levelCubes=LC, dimCube=8,
                           distance=50.0, fov_H=30.0, fov_W=30.0, maxElementsCache=bricks,
                           maxElementsCache_CPU=bricks)
        return vt.visualTur(p, vt.default_options(resident=resident, record_hits=0, preload=0, **opt),
                            volume=fm, octree=oc)

    res = make(1)
    dem = make(0, lookahead=4)
    skp = make(0, skip=4, persistent=1)      # candidates behind absent bricks marched in the same pass
    c = (N - 1) / 2.0
    first = None
    for f in range(3):
        a = math.radians(20.0 * f)
        cam = pf.look_at(W, H, 50.0, 30.0, (c + 1.4 * N * math.sin(a), c + 0.2 * N, c + 1.4 * N * math.cos(a)),
                         (c, c, c))
        res.set_camera(cam)
        dem.set_camera(cam)
        skp.set_camera(cam)
        ra, _ = res.render_host(rgb8=False)
        da, _ = dem.render_host(rgb8=False)
        sa, _ = skp.render_host(rgb8=False)
        st = dem.stats()
        if first is None:
            first = st["bricks_requested"]
        assert np.array_equal(ra.view(np.uint32), da.view(np.uint32)), "frame %d differs" % f
        assert np.array_equal(ra.view(np.uint32), sa.view(np.uint32)), "frame %d differs (skip)" % f
    assert first > 8192, "first pass requested only %d bricks" % first
    res.close()
    dem.close()
    skp.close()
