"""CPU oracle of the learned preconditioner network (numpy).

TEST INFRASTRUCTURE ONLY: tests/ use it to check the GPU network's forward
pass and parameter gradients; the library never calls it.  The learned stage
has no counterpart in the reference (its preconditioner is multigrid only,
src_gmres/apply_precon.f90), so this restates the network as the library
defines it: a 3-level periodic convolutional encoder-decoder, 3x3x3 kernels,
16/32/64 channels, activations stored in BF16 after every layer and FP32
arithmetic, with the backward pass in the same order and the same BF16
roundings as the GPU kernels.

Layout: channels-last [batch, z, y, x, C]; weights [Cout][27][Cin] with tap
t = (dz+1)*9 + (dy+1)*3 + (dx+1); parameters per layer = weights then biases.
"""
from __future__ import annotations

import numpy as np

# (cin, cout, level, up, relu): E0a E0b E1a E1b E2a E2b D1a D1b D0a D0b Out
LAYERS = [(8, 16, 0, 0, 1), (16, 16, 0, 0, 1), (16, 32, 1, 0, 1), (32, 32, 1, 0, 1), (32, 64, 2, 0, 1), (64, 64, 2, 0, 1),
          (64, 32, 1, 1, 1), (32, 32, 1, 0, 1), (32, 16, 0, 1, 1), (16, 16, 0, 0, 1), (16, 4, 0, 0, 0)]
TAPS = [(t // 9 - 1, (t // 3) % 3 - 1, t % 3 - 1) for t in range(27)]  # (dz, dy, dx)


ROUND = [True]  # False: keep FP32 everywhere (used to check the oracle against autograd)


def bf16(a):
    """round float32 to the nearest BF16 (ties to even), returned as float32"""
    if not ROUND[0]:
        return np.asarray(a, dtype=np.float32)
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    r = ((u >> 16) & 1) + np.uint32(0x7FFF)
    return ((u + r) & np.uint32(0xFFFF0000)).view(np.float32)


def unpack(params):
    out, o = [], 0
    for cin, cout, *_ in LAYERS:
        w = params[o:o + 27 * cin * cout].reshape(cout, 27, cin)
        o += 27 * cin * cout
        b = params[o:o + cout]
        o += cout
        out.append((w, b))
    return out


def up2(x):
    return x.repeat(2, axis=1).repeat(2, axis=2).repeat(2, axis=3)


def shift(x, dz, dy, dx):
    """xs[v] = x[v + (dz, dy, dx)] (periodic)"""
    return np.roll(x, shift=(-dz, -dy, -dx), axis=(1, 2, 3))


def conv(x, w, up):
    if up:
        x = up2(x)
    cout = w.shape[0]
    out = np.zeros(x.shape[:4] + (cout,), np.float32)
    for t, (dz, dy, dx) in enumerate(TAPS):
        out += shift(x, dz, dy, dx) @ w[:, t, :].T
    return out


def dgrad(g, w):
    """adjoint of conv (no upsampling) with respect to its input"""
    cin = w.shape[2]
    out = np.zeros(g.shape[:4] + (cin,), np.float32)
    for t, (dz, dy, dx) in enumerate(TAPS):
        out += shift(g, -dz, -dy, -dx) @ w[:, t, :]
    return out


def wgrad(x, g, up):
    if up:
        x = up2(x)
    cout, cin = g.shape[-1], x.shape[-1]
    dw = np.zeros((cout, 27, cin), np.float32)
    gf = g.reshape(-1, cout)
    for t, (dz, dy, dx) in enumerate(TAPS):
        dw[:, t, :] = gf.T @ shift(x, dz, dy, dx).reshape(-1, cin)
    return dw


def pool(x):
    B, Z, Y, X, C = x.shape
    return bf16(x.reshape(B, Z // 2, 2, Y // 2, 2, X // 2, 2, C).mean(axis=(2, 4, 6), dtype=np.float32))


def downsum(x):
    B, Z, Y, X, C = x.shape
    return bf16(x.reshape(B, Z // 2, 2, Y // 2, 2, X // 2, 2, C).sum(axis=(2, 4, 6), dtype=np.float32))


def forward(params, x):
    P = unpack(params)

    def layer(i, inp, skip=None):
        cin, cout, lev, up, relu = LAYERS[i]
        w, b = P[i]
        z = conv(inp, bf16(w), up) + b
        if skip is not None:
            z = z + skip
        return bf16(np.maximum(z, 0)) if relu else z

    A = {}
    A["a0"] = layer(0, x)
    A["s0"] = layer(1, A["a0"])
    A["p0"] = pool(A["s0"])
    A["a1"] = layer(2, A["p0"])
    A["s1"] = layer(3, A["a1"])
    A["p1"] = pool(A["s1"])
    A["a2"] = layer(4, A["p1"])
    A["b2"] = layer(5, A["a2"])
    A["c1"] = layer(6, A["b2"], A["s1"])
    A["d1"] = layer(7, A["c1"])
    A["c0"] = layer(8, A["d1"], A["s0"])
    A["d0"] = layer(9, A["c0"])
    A["y"] = layer(10, A["d0"])
    return A


def gradients(params, x, gy):
    """gradients of sum(gy * y) with respect to every parameter (flat)"""
    P = unpack(params)
    A = forward(params, x)
    W = [bf16(w) for w, _ in P]
    grads = [None] * len(LAYERS)

    def record(i, inp, g):
        grads[i] = (wgrad(inp, g, LAYERS[i][3]), g.reshape(-1, g.shape[-1]).sum(axis=0, dtype=np.float32))

    def mask(g, act):
        return bf16(np.where(act > 0, g, 0).astype(np.float32))

    gy = bf16(gy)
    record(10, A["d0"], gy)
    g_d0 = mask(dgrad(gy, W[10]), A["d0"])
    record(9, A["c0"], g_d0)
    g_c0 = mask(dgrad(g_d0, W[9]), A["c0"])
    record(8, A["d1"], g_c0)
    g_d1 = mask(downsum(bf16(dgrad(g_c0, W[8]))), A["d1"])
    record(7, A["c1"], g_d1)
    g_c1 = mask(dgrad(g_d1, W[7]), A["c1"])
    record(6, A["b2"], g_c1)
    g_b2 = mask(downsum(bf16(dgrad(g_c1, W[6]))), A["b2"])
    record(5, A["a2"], g_b2)
    g_a2 = mask(dgrad(g_b2, W[5]), A["a2"])
    record(4, A["p1"], g_a2)
    g_p1 = bf16(dgrad(g_a2, W[4]))
    g_s1 = mask(g_c1 + up2(g_p1) * np.float32(0.125), A["s1"])
    record(3, A["a1"], g_s1)
    g_a1 = mask(dgrad(g_s1, W[3]), A["a1"])
    record(2, A["p0"], g_a1)
    g_p0 = bf16(dgrad(g_a1, W[2]))
    g_s0 = mask(g_c0 + up2(g_p0) * np.float32(0.125), A["s0"])
    record(1, A["a0"], g_s0)
    g_a0 = mask(dgrad(g_s0, W[1]), A["a0"])
    record(0, x, g_a0)
    flat = []
    for dw, db in grads:
        flat += [dw.ravel(), db.ravel()]
    return A["y"], np.concatenate(flat)


def layer_slices():
    out, o = [], 0
    for cin, cout, *_ in LAYERS:
        n = 27 * cin * cout + cout
        out.append(slice(o, o + n))
        o += n
    return out
