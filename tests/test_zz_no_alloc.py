"""vt_mlp_forward_noalloc: the prefetch network's inference for callers
that cannot allocate GPU memory where they run it -- a render loop inside a
host application that owns the device's memory budget, or a frame thread
that must not call cudaMalloc (it synchronises the device and stalls the
frame).  Checked through the C ABI against vt_mlp_forward of a second
network with the same weights, on calls in a row; collected last so that a
failure here comes after every other test has run."""
import ctypes

import numpy as np
import pytest

import visualtur_b200 as vt

pytestmark = pytest.mark.gpu

DIMS = (12, 512, 512, 4096)
TOL = 1e-4          # the MLP tests' tolerance


def _call(L, fn, m, x, batch, p):
    vt.check(getattr(L, fn)(m._h, ctypes.c_void_p(x.data_ptr()), batch, ctypes.c_void_p(p.data_ptr()), None))


def test_noalloc_forward_matches_forward(cuda):
    torch = cuda
    L = vt.lib()
    m_new = vt.MLP(DIMS, seed=21)     # only ever runs the allocation-free path
    m_ref = vt.MLP(DIMS, seed=21)     # same weights, the allocating path
    rng = np.random.default_rng(4)
    outs = []
    # the first call comes before any vt_mlp_forward on its handle, so it
    # cannot lean on activation buffers that call would have allocated;
    # batch 256 fills the static scratch exactly (256 x (512 + 512) floats)
    for k, batch in enumerate((64, 7, 256)):
        x = torch.from_numpy(rng.standard_normal((batch, DIMS[0])).astype(np.float32)).cuda()
        p_new = torch.full((batch * DIMS[3],), -1.0, dtype=torch.float32, device="cuda")
        p_ref = torch.empty(batch * DIMS[3], dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        _call(L, "vt_mlp_forward_noalloc", m_new, x, batch, p_new)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info()[0]
        if k > 0:
            # after the first call (which may load libvt's device code and
            # its static array) no call takes device memory
            assert free1 == free0, "free device memory changed by %d bytes" % (free0 - free1)
        _call(L, "vt_mlp_forward", m_ref, x, batch, p_ref)
        torch.cuda.synchronize()
        a, b = p_ref.cpu().numpy(), p_new.cpu().numpy()
        assert np.isfinite(b).all() and (b >= 0).all() and (b <= 1).all()
        assert np.abs(a - b).max() <= TOL
        outs.append(b)
    assert not np.array_equal(outs[0][:7 * DIMS[3]], outs[1])   # different inputs, different outputs


def test_noalloc_rejects_oversize_batch(cuda):
    torch = cuda
    m = vt.MLP(DIMS, seed=22)
    x = torch.zeros(257 * DIMS[0], dtype=torch.float32, device="cuda")
    p = torch.zeros(257 * DIMS[3], dtype=torch.float32, device="cuda")
    with pytest.raises(vt.VtError) as e:
        m.forward_noalloc(x, 257, p)
    assert e.value.status == vt.VT_ERR_INVALID and "static scratch" in str(e.value)
