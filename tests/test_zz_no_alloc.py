"""vt_mlp_forward_noalloc: the prefetch network's inference for callers
that cannot allocate GPU memory where they run it (a render loop inside a
host that owns the device's memory, a frame thread that must not call
cudaMalloc).  Checked through the C ABI against vt_mlp_forward on two calls
in a row; collected last so a failure here comes after every other test."""
import ctypes

import numpy as np
import pytest

import visualtur_b200 as vt

pytestmark = pytest.mark.gpu


def test_noalloc_forward_matches_forward_twice(cuda):
    torch = cuda
    m = vt.MLP((12, 512, 512, 4096), seed=21)
    rng = np.random.default_rng(4)
    L = vt.lib()
    ref, got = [], []
    for batch in (64, 7):       # two calls in a row, the second on a smaller batch
        x = torch.from_numpy(rng.standard_normal((batch, 12)).astype(np.float32)).cuda()
        p_ref = torch.empty(batch * 4096, dtype=torch.float32, device="cuda")
        p_new = torch.full((batch * 4096,), -1.0, dtype=torch.float32, device="cuda")
        vt.check(L.vt_mlp_forward(m._h, ctypes.c_void_p(x.data_ptr()), batch, ctypes.c_void_p(p_ref.data_ptr()), None))
        vt.check(L.vt_mlp_forward_noalloc(m._h, ctypes.c_void_p(x.data_ptr()), batch,
                                          ctypes.c_void_p(p_new.data_ptr()), None))
        torch.cuda.synchronize()
        a, b = p_ref.cpu().numpy(), p_new.cpu().numpy()
        assert np.abs(a - b).max() <= 1e-4        # the MLP tests' tolerance
        ref.append(a)
        got.append(b)
    assert not np.array_equal(ref[0][:7 * 4096], ref[1])   # different inputs, different outputs


def test_noalloc_rejects_oversize_batch(cuda):
    torch = cuda
    m = vt.MLP((12, 512, 512, 4096), seed=22)
    x = torch.zeros(257 * 12, dtype=torch.float32, device="cuda")
    p = torch.zeros(257 * 4096, dtype=torch.float32, device="cuda")
    with pytest.raises(vt.VtError) as e:
        m.forward_noalloc(x, 257, p)
    assert e.value.status == vt.VT_ERR_INVALID and "static scratch" in str(e.value)
