"""Prefetch network kernels (vt_mlp_*) against a CPU FP32 implementation.

The GPU forward and backward GEMMs read BF16 weights and accumulate in FP32.
On the tensor cores (tcgen05, the default) every GEMM input -- activations
and gradients too -- is rounded to BF16 as it is staged; on the SIMT path
the activations stay FP32.  The CPU reference rounds the same operands the
same way and multiplies in float32 numpy, so gradients agree up to FP32
summation order (rtol 2e-3 below)."""
import numpy as np
import pytest

import visualtur_b200 as vt

pytestmark = pytest.mark.gpu


def bf16(a):
    u = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def cpu_grads(layers, x, y, tc=True):
    """mean BCE of sigmoid(relu(relu(x W1 + b1) W2 + b2) W3 + b3) and its
    grads; tc: GEMM inputs rounded to BF16 as the tensor-core path stages them"""
    W = [bf16(w) for w, _ in layers]
    b = [bb for _, bb in layers]
    q = bf16 if tc else (lambda a: a)
    a0 = x
    a1 = np.maximum(q(a0) @ W[0] + b[0], 0)
    a2 = np.maximum(q(a1) @ W[1] + b[1], 0)
    p = 1 / (1 + np.exp(-(q(a2) @ W[2] + b[2])))
    B = x.shape[0]
    pc = np.clip(p, 1e-7, 1 - 1e-7)
    loss = -(y * np.log(pc) + (1 - y) * np.log(1 - pc)).sum() / B
    d3 = (p - y) / B
    g = [None, None, None]
    g[2] = (q(a2).T @ q(d3), d3.sum(0))
    d2 = (q(d3) @ W[2].T) * (a2 > 0)
    g[1] = (q(a1).T @ q(d2), d2.sum(0))
    d1 = (q(d2) @ W[1].T) * (a1 > 0)
    g[0] = (q(a0).T @ q(d1), d1.sum(0))
    return g, loss, p


@pytest.mark.parametrize("tc", [True, False])
@pytest.mark.parametrize("dims,batch", [((12, 512, 512, 4096), 64), ((12, 512, 512, 4096), 256),
                                        ((12, 40, 33, 70), 19), ((12, 200, 130, 300), 133)])
def test_mlp_gradients_match_cpu(dims, batch, tc, cuda):
    torch = cuda
    m = vt.MLP(dims, seed=3)
    m.use_tensor_cores(tc)
    rng = np.random.default_rng(0)
    x = rng.standard_normal((batch, dims[0])).astype(np.float32)
    y = (rng.random((batch, dims[3])) < 0.2).astype(np.float32)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    layers = m.weights()
    # He init: std sqrt(2/fan_in), zero bias
    for l, (w, b) in enumerate(layers):
        assert abs(w.std() / np.sqrt(2.0 / dims[l]) - 1) < 0.1 and not b.any()
    g, loss = m.gradients(dx, dy, batch)
    gc, lc, p = cpu_grads(layers, x.astype(np.float64).astype(np.float32), y, tc)
    assert abs(loss - lc) <= 1e-4 * max(1, abs(lc))
    for (gw, gb), (cw, cb) in zip(g, gc):
        scale = np.abs(cw).max() + 1e-12
        assert np.abs(gw - cw).max() <= 2e-3 * scale
        assert np.abs(gb - cb).max() <= 2e-3 * (np.abs(cb).max() + 1e-12)
    dp = torch.empty(batch * dims[3], dtype=torch.float32, device="cuda")
    m.forward(dx, batch, dp)
    torch.cuda.synchronize()
    # probabilities: FP32 activations agree to summation order (1e-4); on the
    # tensor cores an activation within an FP32 rounding of a BF16 rounding
    # boundary can round to the neighbouring BF16 value on one side only,
    # which moves an output by up to a few 1e-4 (bar 2e-3)
    assert np.abs(dp.cpu().numpy().reshape(batch, -1) - p).max() < (2e-3 if tc else 1e-4)


@pytest.mark.parametrize("tc", [True, False])
def test_mlp_training_reduces_loss(tc, cuda):
    """Learns a pose -> node-set style mapping: output k on iff a fixed
    random projection of the input exceeds a threshold."""
    torch = cuda
    rng = np.random.default_rng(1)
    n, din, dout = 4096, 12, 256
    x = rng.standard_normal((n, din)).astype(np.float32)
    proj = rng.standard_normal((din, dout)).astype(np.float32)
    y = (x @ proj > 0.8).astype(np.float32)
    m = vt.MLP((din, 128, 128, dout), seed=5)
    m.use_tensor_cores(tc)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    first = m.train_step(dx[:256], dy[:256], 256, 2e-3)
    for ep in range(30):
        for i in range(0, n, 256):
            last = m.train_step(dx[i:i + 256], dy[i:i + 256], 256, 2e-3, want_loss=False)
    final = m.train_step(dx[:256], dy[:256], 256, 0.0)
    assert final < 0.25 * first, (first, final)
    # weight round trip
    w = m.weights()
    m2 = vt.MLP((din, 128, 128, dout), seed=6)
    m2.use_tensor_cores(tc)
    m2.set_weights(w)
    p1 = torch.empty(256 * dout, device="cuda")
    p2 = torch.empty(256 * dout, device="cuda")
    m.forward(dx[:256], 256, p1)
    m2.forward(dx[:256], 256, p2)
    torch.cuda.synchronize()
    assert torch.equal(p1, p2)


def test_baseline_network_trains_on_20k_poses_on_the_tensor_cores(cuda):
    """The learned-prefetch network at its stated size (12 -> 512 -> 512 ->
    4096) trained for 30 epochs of 20 000 poses, batch 256, by the
    tcgen05 kernels: reports the time, and the loss falls."""
    import time
    torch = cuda
    rng = np.random.default_rng(2)
    n = 20000
    x = rng.standard_normal((n, 12)).astype(np.float32)
    proj = rng.standard_normal((12, 4096)).astype(np.float32)
    y = (x @ proj > 1.0).astype(np.float32)
    m = vt.MLP((12, 512, 512, 4096), seed=9)
    dx, dy = torch.from_numpy(x).cuda(), torch.from_numpy(y).cuda()
    first = m.train_step(dx[:256], dy[:256], 256, 1e-3)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for ep in range(30):
        for i in range(0, n - 255, 256):
            m.train_step(dx[i:i + 256], dy[i:i + 256], 256, 1e-3, want_loss=False)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    final = m.train_step(dx[:256], dy[:256], 256, 0.0)
    print("\n20k-pose training, 30 epochs of batch 256 on the tensor cores: %.2f s (loss %.4f -> %.4f)"
          % (dt, first, final))
    assert final < 0.5 * first
