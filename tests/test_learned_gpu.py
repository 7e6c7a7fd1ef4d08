"""tcgen05 tensor-core kernels of the learned preconditioner stage, checked
against FP32 matrix products of the same BF16-rounded operands."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _gemm(A, B):
    import torch

    from lowmachmixtures_b200 import _native
    lib = _native.load()
    M, K = A.shape
    N = B.shape[0]
    D = torch.empty(M, N, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.lmm_nn_gemm_bf16(C.c_void_p(A.data_ptr()), C.c_void_p(B.data_ptr()), C.c_void_p(D.data_ptr()), M, N, K,
                              C.c_void_p(err.data_ptr()), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    return D


@pytest.mark.parametrize("M,N,K", [(128, 16, 64), (300, 48, 200), (1000, 64, 432), (256, 256, 128), (64, 32, 8)])
def test_gemm_bf16_matches_fp32_product(M, N, K):
    import torch
    g = torch.Generator().manual_seed(M + N + K)
    A = torch.randn(M, K, generator=g).to(torch.bfloat16).cuda()
    B = torch.randn(N, K, generator=g).to(torch.bfloat16).cuda()
    D = _gemm(A, B)
    ref = A.float() @ B.float().t()
    np.testing.assert_allclose(D.cpu().numpy(), ref.cpu().numpy(), rtol=1e-4, atol=1e-3 * np.sqrt(K))


# ---------------------------------------------------------------- conv layers
def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def _ref_conv(x_cl, w, up):
    """circular 3x3x3 conv of channels-last x [B,z,y,x,C] with w [Cout][27][Cin]"""
    import torch
    import torch.nn.functional as F
    x = x_cl.float().permute(0, 4, 1, 2, 3)
    if up:
        x = F.interpolate(x, scale_factor=2, mode="nearest")
    co, _, cin = w.shape
    wt = w.float().reshape(co, 3, 3, 3, cin).permute(0, 4, 1, 2, 3)
    return F.conv3d(F.pad(x, (1, 1, 1, 1, 1, 1), mode="circular"), wt).permute(0, 2, 3, 4, 1)


def _packed(w, with_t=False):
    import torch
    from lowmachmixtures_b200 import _native
    lib = _native.load()
    co, _, cin = w.shape
    r16 = lambda v: (v + 15) // 16 * 16  # noqa: E731
    wf = torch.zeros(r16(co), 27 * cin, dtype=torch.bfloat16, device="cuda")
    wt = torch.zeros(r16(cin), 27 * ((co + 7) // 8 * 8), dtype=torch.bfloat16, device="cuda") if with_t else None
    assert lib.lmm_nn_pack_weights(_p(w), _p(wf), _p(wt), co, cin, _stream()) == 0
    return wf, wt


# grids whose x tiles by 8 and y by 16 run the shifted-view tile kernel
# (conv_tile.cuh) when its weights fit in shared memory; the others the
# gathered implicit GEMM
@pytest.mark.parametrize("B,n,cin,cout,up,relu", [(2, (16, 8, 8), 16, 32, 0, 1), (1, (16, 16, 8), 32, 16, 1, 1),
                                                  (1, (8, 8, 8), 64, 64, 0, 0), (1, (32, 16, 16), 8, 16, 0, 1),
                                                  (2, (16, 32, 8), 16, 16, 0, 1), (1, (32, 32, 8), 64, 32, 1, 1),
                                                  (1, (16, 16, 16), 32, 64, 0, 1), (1, (24, 16, 6), 16, 48, 0, 0),
                                                  (1, (16, 16, 4), 64, 64, 0, 1), (1, (16, 16, 8), 8, 16, 0, 0),
                                                  # more planes than resident CTAs: runs of several planes that
                                                  # cross tile boundaries
                                                  (1, (64, 64, 64), 16, 16, 0, 1), (2, (32, 48, 40), 32, 16, 1, 1),
                                                  (1, (64, 32, 64), 64, 32, 1, 1), (3, (8, 16, 5), 16, 32, 0, 1),
                                                  (1, (128, 128, 24), 16, 16, 0, 0),
                                                  # output channels in slices: 2 x 32 and 3 x 16
                                                  (1, (32, 32, 32), 64, 64, 0, 1), (1, (16, 32, 12), 64, 48, 0, 1),
                                                  # 8 input channels: x taps paired in one K = 16 step
                                                  (1, (64, 64, 32), 8, 16, 0, 1), (2, (32, 32, 16), 8, 32, 0, 1)])
def test_conv3d_matches_torch(B, n, cin, cout, up, relu):
    import torch
    from lowmachmixtures_b200 import _native
    lib = _native.load()
    nx, ny, nz = n
    g = torch.Generator().manual_seed(cin * cout + up)
    sh = (B, nz >> up, ny >> up, nx >> up, cin)
    x = torch.randn(sh, generator=g).to(torch.bfloat16).cuda()
    w = (torch.randn(cout, 27, cin, generator=g) / np.sqrt(27 * cin)).cuda()
    bias = torch.randn(cout, generator=g).cuda() * 0.1
    skip = torch.randn(B, nz, ny, nx, cout, generator=g).to(torch.bfloat16).cuda()
    wf, _ = _packed(w)
    out = torch.empty(B, nz, ny, nx, cout, dtype=torch.bfloat16, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.lmm_nn_conv3d(_p(x), _p(wf), _p(bias), _p(skip), None, _p(out), None, B, nx, ny, nz, up, cin, cout, cout, relu,
                           _p(err), _stream())
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref = _ref_conv(x, w.to(torch.bfloat16), up) + bias + skip.float()
    if relu:
        ref = torch.relu(ref)
    scale = ref.abs().max().item()
    np.testing.assert_allclose(out.float().cpu().numpy(), ref.cpu().numpy(), rtol=1e-2, atol=1e-2 * scale)


@pytest.mark.parametrize("n", [16, 64])
def test_conv3d_fp32_output_and_mask(n):
    import torch
    from lowmachmixtures_b200 import _native
    lib = _native.load()
    B, nx, ny, nz, cin, cout = 1, n, n, n, 16, 4
    g = torch.Generator().manual_seed(5)
    x = torch.randn(B, nz, ny, nx, cin, generator=g).to(torch.bfloat16).cuda()
    w = (torch.randn(cout, 27, cin, generator=g) / 20).cuda()
    wf, _ = _packed(w)
    out32 = torch.empty(B, nz, ny, nx, cout, dtype=torch.float32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    assert lib.lmm_nn_conv3d(_p(x), _p(wf), None, None, None, None, _p(out32), B, nx, ny, nz, 0, cin, cout, cout, 0, _p(err),
                             _stream()) == 0
    torch.cuda.synchronize()
    ref = _ref_conv(x, w.to(torch.bfloat16), 0)
    np.testing.assert_allclose(out32.cpu().numpy(), ref.cpu().numpy(), rtol=1e-4, atol=1e-4)
    # masked BF16 output with padded channel rows (Cs = 8 > Cout = 4)
    mask = torch.randn(B, nz, ny, nx, 8, generator=g).to(torch.bfloat16).cuda()
    out = torch.full((B, nz, ny, nx, 8), 7.0, dtype=torch.bfloat16, device="cuda")
    assert lib.lmm_nn_conv3d(_p(x), _p(wf), None, None, _p(mask), _p(out), None, B, nx, ny, nz, 0, cin, cout, 8, 0, _p(err),
                             _stream()) == 0
    torch.cuda.synchronize()
    exp = torch.where(mask[..., :4].float() > 0, ref, torch.zeros_like(ref))
    np.testing.assert_allclose(out[..., :4].float().cpu().numpy(), exp.cpu().numpy(), rtol=1e-2, atol=1e-2)
    assert (out[..., 4:].float() == 0).all()


@pytest.mark.parametrize("B,n,cin,cout,up", [(2, (16, 8, 8), 16, 32, 0), (1, (16, 16, 16), 32, 16, 1), (1, (32, 32, 32), 8, 16, 0),
                                             (1, (16, 16, 16), 16, 4, 0)])
def test_conv3d_gradients_match_torch_autograd(B, n, cin, cout, up):
    import torch
    from lowmachmixtures_b200 import _native
    lib = _native.load()
    nx, ny, nz = n
    g = torch.Generator().manual_seed(cin + 3 * cout + up)
    x = torch.randn(B, nz >> up, ny >> up, nx >> up, cin, generator=g).to(torch.bfloat16).cuda()
    w = (torch.randn(cout, 27, cin, generator=g) / np.sqrt(27 * cin)).cuda()
    coutp = (cout + 7) // 8 * 8
    gy = torch.zeros(B, nz, ny, nx, coutp, dtype=torch.bfloat16, device="cuda")
    gy[..., :cout] = torch.randn(B, nz, ny, nx, cout, generator=g).to(torch.bfloat16).cuda()
    # torch reference gradients of sum(conv(x, w) * gy)
    xr = x.float().clone().requires_grad_(True)
    wr = w.to(torch.bfloat16).float().clone().requires_grad_(True)
    y = _ref_conv(xr, wr, up)
    (y * gy[..., :cout].float()).sum().backward()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    dw = torch.zeros(cout, 27, cin, dtype=torch.float32, device="cuda")
    assert lib.lmm_nn_conv3d_wgrad(_p(x), _p(gy), _p(dw), B, nx, ny, nz, up, cin, coutp, cout, _p(err), _stream()) == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    ref_dw = wr.grad
    np.testing.assert_allclose(dw.cpu().numpy(), ref_dw.cpu().numpy(), rtol=2e-3, atol=2e-3 * ref_dw.abs().max().item())
    if up == 0:
        # data gradient: the same convolution kernel with the flipped, transposed weights
        _, wt = _packed(w, with_t=True)
        dx = torch.empty(B, nz, ny, nx, cin, dtype=torch.float32, device="cuda")
        assert lib.lmm_nn_conv3d(_p(gy), _p(wt), None, None, None, None, _p(dx), B, nx, ny, nz, 0, coutp, cin, cin, 0, _p(err),
                                 _stream()) == 0
        torch.cuda.synchronize()
        ref_dx = xr.grad
        np.testing.assert_allclose(dx.cpu().numpy(), ref_dx.cpu().numpy(), rtol=2e-3, atol=2e-3 * ref_dx.abs().max().item())


# ---------------------------------------------------------------- the network
def _net(n, batch, seed):
    from lowmachmixtures_b200 import _native
    lib = _native.load()
    h = C.c_void_p()
    assert lib.lmm_net_create(n[0], n[1], n[2], batch, seed, C.byref(h)) == 0
    return lib, h


def test_net_forward_and_gradients_match_cpu_oracle():
    """Parameter gradients of the whole encoder-decoder (hand-written
    backward pass on the tensor cores) against the numpy oracle."""
    import torch
    from oracle import nn_oracle as O
    lib, h = _net((8, 8, 8), 2, 3)
    try:
        npar = lib.lmm_net_num_params(h)
        params = np.zeros(npar, np.float32)
        assert lib.lmm_net_params(h, params.ctypes.data_as(C.c_void_p), 0) == 0
        # biases are initialised to zero; give them values so their gradients matter
        rng = np.random.default_rng(0)
        for sl, (cin, cout, *_) in zip(O.layer_slices(), O.LAYERS):
            params[sl][27 * cin * cout:] = rng.normal(0, 0.1, cout).astype(np.float32)
        assert lib.lmm_net_params(h, params.ctypes.data_as(C.c_void_p), 1) == 0
        x = np.zeros((2, 8, 8, 8, 8), np.float32)
        x[..., :5] = rng.standard_normal((2, 8, 8, 8, 5))
        x = O.bf16(x)
        gy = rng.standard_normal((2, 8, 8, 8, 4)).astype(np.float32)
        xd = torch.from_numpy(x).to(torch.bfloat16).cuda()
        gyd = torch.from_numpy(gy).cuda()
        yd = torch.empty(2, 8, 8, 8, 4, dtype=torch.float32, device="cuda")
        assert lib.lmm_net_forward(h, _p(xd), _p(yd)) == 0
        grads = np.zeros(npar, np.float32)
        assert lib.lmm_net_gradients(h, _p(xd), _p(gyd), grads.ctypes.data_as(C.c_void_p)) == 0
        y_ref, g_ref = O.gradients(params, x, gy)
        y = yd.cpu().numpy()
        assert np.linalg.norm(y - y_ref) <= 2e-2 * np.linalg.norm(y_ref)
        for li, sl in enumerate(O.layer_slices()):
            a, b = grads[sl], g_ref[sl]
            rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            assert rel < 3e-2, f"layer {li}: relative gradient error {rel:.3e}"
    finally:
        lib.lmm_net_destroy(h)


def test_net_training_reduces_loss():
    """Adam steps on a fixed smooth target decrease the mean squared error."""
    import torch
    lib, h = _net((16, 16, 16), 2, 11)
    try:
        g = torch.Generator().manual_seed(1)
        x = torch.zeros(2, 16, 16, 16, 8)
        x[..., :5] = torch.randn(2, 16, 16, 16, 5, generator=g)
        t = torch.stack([x[..., 0] + 0.5 * torch.roll(x[..., 1], 1, 1), x[..., 2] * 0.3, -x[..., 3], x[..., 4] * 0.7], -1)
        xd = x.to(torch.bfloat16).cuda()
        td = t.float().contiguous().cuda()
        losses = []
        for _ in range(150):
            loss = C.c_float()
            assert lib.lmm_net_train_step(h, _p(xd), _p(td), 3e-3, C.byref(loss)) == 0
            losses.append(loss.value)
        assert np.isfinite(losses).all()
        # the weight gradients accumulate with float atomics, so the path
        # differs slightly run to run: check a clear, not an exact, decrease
        assert np.mean(losses[-10:]) < 0.6 * losses[0], losses[::15]
    finally:
        lib.lmm_net_destroy(h)


def test_learned_stage_dry_run_changes_nothing_and_stage_converges():
    """learned_stage = 2 computes every correction but accepts none: the
    solve equals the stage-free solve bit for bit.  With the stage on
    (an untrained network) FGMRES still reaches the tolerance."""
    import torch
    from lowmachmixtures_b200 import learned, synth
    prob = synth.make_problem(3, 32, 100.0, 21)
    with learned.Net((32, 32, 32), 1, 5) as net:
        plain = learned.solve_with(prob, None)
        dry = learned.solve_with(prob, net, knobs=learned.mixed_knobs(learned_stage=2))
        on = learned.solve_with(prob, net)
    assert dry[0] == plain[0] and dry[2] == plain[2]
    assert dry[3] == 0 and dry[4] > 0
    assert on[2] <= 1e-9 and on[4] > 0


def test_judged_stage_drops_a_network_that_does_not_help():
    """learned_stage = 4: the GMRES residual judges the network.  A network
    whose weights are all zero returns a zero correction, so every network
    column is dropped as a miss: the solve stops asking it after two forward
    passes and goes on with the plain V-cycle, reaching the tolerance in the
    stage-free iteration count.  Always on (learned_stage = 1) the same
    network is asked once per V-cycle application and never kept."""
    from lowmachmixtures_b200 import learned, synth
    prob = synth.make_problem(3, 32, 100.0, 23)
    with learned.Net((32, 32, 32), 1, 5) as net:
        net.set_params(np.zeros(net.num_params, np.float32))
        plain = learned.solve_with(prob, None)
        judged = learned.solve_with(prob, net, knobs=learned.mixed_knobs(learned_stage=4))
        always = learned.solve_with(prob, net, knobs=learned.mixed_knobs(learned_stage=1))
    assert plain[0] >= 3
    assert judged[2] <= 1e-9 and always[2] <= 1e-9
    assert judged[0] == plain[0] and always[0] == plain[0]
    assert judged[3] == 0 and judged[4] == 2
    assert always[3] == 0 and always[4] == always[0]


def test_trained_stage_gains_on_held_out_seeds():
    """What training gains, on held-out seeds of the learned-stage family
    (32^3, steady, contrast log-uniform in [10, 1000]).  The network trained
    on the GPU by the library's own kernels, on pairs the solver's operators
    make, removes a clear share of the residual one FP32 V-cycle
    application leaves (|r1 - A c| / |r1| below 0.9), where the same network
    untrained removes at least 0.1 less.  Used as extra FGMRES directions
    (learned_stage = 1) it keeps every solve at the FP64 tolerance, with at
    most two V-cycle applications more per seed and 10% more in all than the
    method without it (the V-cycle alone already removes about 99% of that
    residual, so the network's share does not lower the count)."""
    from lowmachmixtures_b200 import learned, synth
    net, hist, _ = learned.train(n=32, fields=40, steps=400, batch=4)
    rows = []
    try:
        assert np.mean(hist[-20:]) < hist[0]
        with learned.Net((32, 32, 32), 1, 0) as raw:
            for f in range(7001, 7007):
                prob = synth.make_problem(3, 32, learned.field_contrast(f), f)
                rt = learned.residual_ratios(net, prob, [f])[0][1]
                ru = learned.residual_ratios(raw, prob, [f])[0][1]
                a = learned.solve_with(prob, None)
                b = learned.solve_with(prob, net)
                rows.append(dict(seed=f, net_ratio=rt, untrained_ratio=ru, it_plain=a[0], it_learned=b[0], res_plain=a[2],
                                 res_learned=b[2], kept=b[3], tried=b[4]))
    finally:
        net.close()
    msg = repr(rows)
    assert np.mean([r["net_ratio"] for r in rows]) < 0.9, msg
    assert np.mean([r["untrained_ratio"] for r in rows]) >= np.mean([r["net_ratio"] for r in rows]) + 0.1, msg
    for r in rows:
        assert r["res_plain"] <= 1e-9 and r["res_learned"] <= 1e-9, msg
        assert r["it_learned"] <= r["it_plain"] + 2, msg
        assert r["tried"] == r["it_learned"], msg  # one correction per V-cycle application
    assert sum(r["it_learned"] for r in rows) <= 1.1 * sum(r["it_plain"] for r in rows), msg


def test_weight_file_round_trip_through_the_library(tmp_path):
    """lmm_net_save / lmm_net_load against the format's Python reader and
    writer (test_learned_weights_cpu.py); the file does not depend on the
    grid the network was created for"""
    from lowmachmixtures_b200 import learned
    a = learned.Net((16, 16, 16), 1, 3)
    p = a.params()
    assert p.size == learned.num_params()
    a.save(str(tmp_path / "a.bin"))
    assert np.array_equal(learned.read_weights(str(tmp_path / "a.bin")).view(np.uint32), p.view(np.uint32))
    q = np.random.default_rng(5).standard_normal(p.size).astype(np.float32)
    learned.write_weights(str(tmp_path / "q.bin"), q)
    b = learned.Net((32, 32, 16), 2, 0)
    b.load(str(tmp_path / "q.bin"))
    assert np.array_equal(b.params().view(np.uint32), q.view(np.uint32))
    b.load(str(tmp_path / "a.bin"))
    assert np.array_equal(b.params().view(np.uint32), p.view(np.uint32))
    # a damaged file leaves the weights as they were
    d = bytearray((tmp_path / "q.bin").read_bytes())
    d[-3] ^= 0x10
    (tmp_path / "bad.bin").write_bytes(bytes(d))
    with pytest.raises(RuntimeError, match="checksum"):
        b.load(str(tmp_path / "bad.bin"))
    with pytest.raises(RuntimeError, match="cannot open"):
        b.load(str(tmp_path / "missing.bin"))
    assert np.array_equal(b.params().view(np.uint32), p.view(np.uint32))
    a.close()
    b.close()
