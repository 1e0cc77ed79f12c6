"""Camera-sharded batches on one GPU: with one rank the shard is the whole
batch, rendered by one vt_render_batch, and the images equal the same
views rendered one at a time (and the first view equals the oracle's)."""
import numpy as np
import pytest

import vt_fixtures as F
import visualtur_b200 as vt
from visualtur_b200 import prefetch as pf
from visualtur_b200.sharded import ShardedViews
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def test_single_rank_shard_equals_view_by_view(workdir, cuda):
    torch = cuda
    case = "c1"
    c = F.CASES[case]
    vol = F.case_volume(case)
    fm, oc = vt.FileManager.wrap(vol), vt.Octree(F.case_octree(case, workdir))
    p = vt.make_params(W=c["W"], H=c["H"], octreeFile=None, hdf5File=None, octreeLevel=c["levelO"],
                       levelCubes=c["levelC"], dimCube=8, distance=c["dist"], fov_H=c["fov"], fov_W=c["fov"],
                       maxElementsCache=4096, maxElementsCache_CPU=4096)
    r = vt.visualTur(p, vt.default_options(persistent=1), volume=fm, octree=oc)
    rng = np.random.default_rng(4)
    cams = []
    for k in range(7):
        v = rng.standard_normal(3)
        pos = 63.5 + v / np.linalg.norm(v) * rng.uniform(180, 260)
        W, H = [(64, 48), (96, 96), (40, 72)][k % 3]
        cams.append(pf.look_at(W, H, c["dist"], c["fov"], pos, 63.5 + rng.uniform(-20, 20, 3)))
    sv = ShardedViews(r, None, 0, 1, device=torch.device("cuda"), stream=torch.cuda.Stream())
    imgs = sv.render(cams)
    assert len(imgs) == len(cams)
    for cam, im in zip(cams, imgs):
        buf = torch.empty(cam.W * cam.H * 3, dtype=torch.uint8, device="cuda")
        v = vt.vt_view()
        v.cam, v.dev_rgba, v.dev_rgb8 = cam, None, buf.data_ptr()
        r.render_batch([v])
        torch.cuda.synchronize()
        assert np.array_equal(im.numpy(), buf.cpu().numpy())
    o = orc.Octree(F.case_octree(case, workdir))
    ocam = orc.Camera(cams[0].H, cams[0].W, c["dist"], c["fov"], c["fov"])
    for f in ("look", "up", "right", "position"):
        v = getattr(cams[0], f)
        setattr(ocam.c, f, orc.orc_f3(v[0], v[1], v[2]))
    want = orc.render(o, vol, ocam, c["levelO"], c["levelC"], c["inc"])
    assert np.array_equal(imgs[0].numpy().reshape(-1, 3), want["rgb8"])
    r.close()
