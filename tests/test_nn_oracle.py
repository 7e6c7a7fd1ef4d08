"""The CPU oracle of the learned network, checked on the CPU: with BF16
rounding switched off its hand-written backward pass equals torch autograd
of the same network (periodic 3x3x3 convolutions, pooling, upsampling,
skip additions)."""
import numpy as np
import pytest

from oracle import nn_oracle as O


def _torch_net(params, x):
    import torch
    import torch.nn.functional as F
    P = [(torch.tensor(w, requires_grad=True), torch.tensor(b, requires_grad=True)) for w, b in O.unpack(params)]

    def conv(i, inp, skip=None):
        cin, cout, lev, up, relu = O.LAYERS[i]
        w, b = P[i]
        xx = inp.permute(0, 4, 1, 2, 3)
        if up:
            xx = F.interpolate(xx, scale_factor=2, mode="nearest")
        wt = w.reshape(cout, 3, 3, 3, cin).permute(0, 4, 1, 2, 3)
        z = F.conv3d(F.pad(xx, (1, 1, 1, 1, 1, 1), mode="circular"), wt).permute(0, 2, 3, 4, 1) + b
        if skip is not None:
            z = z + skip
        return torch.relu(z) if relu else z

    def pool(a):
        return F.avg_pool3d(a.permute(0, 4, 1, 2, 3), 2).permute(0, 2, 3, 4, 1)

    a0 = conv(0, x)
    s0 = conv(1, a0)
    a1 = conv(2, pool(s0))
    s1 = conv(3, a1)
    a2 = conv(4, pool(s1))
    b2 = conv(5, a2)
    c1 = conv(6, b2, s1)
    d1 = conv(7, c1)
    c0 = conv(8, d1, s0)
    d0 = conv(9, c0)
    return conv(10, d0), P


def test_oracle_backward_equals_autograd_without_rounding():
    import torch
    rng = np.random.default_rng(4)
    sizes = [27 * cin * cout + cout for cin, cout, *_ in O.LAYERS]
    params = np.concatenate([rng.normal(0, 0.2, n) for n in sizes]).astype(np.float32)
    x = rng.standard_normal((1, 8, 8, 8, 8)).astype(np.float32)
    gy = rng.standard_normal((1, 8, 8, 8, 4)).astype(np.float32)
    O.ROUND[0] = False
    try:
        y, g = O.gradients(params, x, gy)
    finally:
        O.ROUND[0] = True
    yt, P = _torch_net(params, torch.tensor(x))
    (yt * torch.tensor(gy)).sum().backward()
    ref = np.concatenate([np.concatenate([w.grad.numpy().ravel(), b.grad.numpy().ravel()]) for w, b in P])
    np.testing.assert_allclose(y, yt.detach().numpy(), rtol=1e-4, atol=1e-4 * np.abs(y).max())
    for li, sl in enumerate(O.layer_slices()):
        rel = np.linalg.norm(g[sl] - ref[sl]) / np.linalg.norm(ref[sl])
        assert rel < 1e-4, f"layer {li}: {rel:.2e}"


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 3.0e-3], np.float32)
    r = O.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == np.float32(1.0 + 2 ** -7) and r[3] == -2.5
    assert abs(r[4] - 3.0e-3) <= 3.0e-3 * 2 ** -8
