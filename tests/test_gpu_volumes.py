"""The torch restatement of the seeded generators (oracle/volumes.py), run
on the GPU as the bench's reference arm runs it, equals libvt's device
generator bit for bit: the reference arm renders exactly the product's
volumes without loading libvt.so."""
import numpy as np
import pytest

import visualtur_b200 as vt
from oracle import volumes as V

pytestmark = pytest.mark.gpu

CASES = [("sphere", vt.VT_GEN_SPHERE, (63.5, 60.0, 70.25, 0.25), (128, 120, 136)),
         ("fractal", vt.VT_GEN_FRACTAL_U8, (32, 25.0, 200.0, 200.0), (160, 144, 152)),
         ("blobs", vt.VT_GEN_BLOBS, (256, 10.0, 60.0, 0.5, 1.5, 0.05), (160, 176, 144))]


@pytest.mark.parametrize("kind,code,prm,dims", CASES)
def test_torch_generators_match_libvt_device(kind, code, prm, dims, cuda):
    torch = cuda
    dt = torch.uint8 if kind == "fractal" else torch.float32
    want = torch.empty(dims, dtype=dt, device="cuda")
    vt.generate_volume(code, 2048, dims, prm, device_ptr=want.data_ptr())
    got = torch.empty(dims, dtype=dt, device="cuda")
    V.generate(torch, kind, 2048, dims, prm, got, torch.device("cuda"), slab=37)
    torch.cuda.synchronize()
    a, b = want.cpu().numpy(), got.cpu().numpy()
    assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), "%d voxels differ" % (a != b).sum()
