"""oracle/volumes.py (the torch restatement of libvt's seeded generators,
the reference arm's inputs) against libvt's host generators: bit-exact for
the sphere and the fractal volumes, within a few ulp of the blob term's
exp for the blobs (the GPU test pins all three bit for bit against the
device generator, which the bench uses)."""
import numpy as np
import pytest
import torch

import visualtur_b200 as vt
from oracle import volumes as V

CASES = [("sphere", vt.VT_GEN_SPHERE, (20.5, 19.5, 21.0, 0.25), (40, 37, 45)),
         ("fractal", vt.VT_GEN_FRACTAL_U8, (5, 3.0, 12.0, 200.0), (48, 50, 56)),
         ("blobs", vt.VT_GEN_BLOBS, (16, 2.0, 9.0, 0.5, 1.5, 0.05), (48, 40, 56))]


@pytest.mark.parametrize("kind,code,prm,dims", CASES)
def test_torch_generators_match_libvt_host(kind, code, prm, dims):
    want = vt.generate_volume(code, 2048, dims, prm)
    out = torch.empty(dims, dtype=torch.uint8 if kind == "fractal" else torch.float32)
    V.generate(torch, kind, 2048, dims, prm, out, torch.device("cpu"), slab=7)
    got = out.numpy()
    if kind == "blobs":
        assert np.abs(got - want).max() <= 2e-6 * max(1.0, float(np.abs(want).max()))
    else:
        assert np.array_equal(got.view(np.uint8), want.view(np.uint8))
