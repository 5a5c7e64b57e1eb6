"""The surrogate's CUDA kernels (csrc/surrogate.cu, through the C ABI of
include/dsmc_surrogate.h) against the NumPy FP64 restatement in
oracle/surrogate_ref.py, on small shapes.

Inputs are bf16-representable, so the references see the kernels' exact
operands.  Tolerances: FP32 results (forward with an FP32 output, weight and
bias gradients) to 1e-4 relative to the result's scale (FP32 accumulation of
at most a few thousand terms); bf16 results to 2^-7 relative (one bf16
rounding) plus the same accumulation allowance.  The whole network, with the
restatement rounding to bf16 where the kernels store bf16: output to 1% and
weight gradients to 3% of each tensor's scale (the FP32 accumulation order
still differs, and a value near a rounding boundary or a ReLU's zero can
land on the other side), and one Adam step matches its formula to 1e-5
(FP32).
"""
from __future__ import annotations

import numpy as np
import pytest

from oracle import surrogate_ref as ref

pytestmark = pytest.mark.gpu


def _bf16(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16).cuda()


def _np(t):
    return t.float().cpu().numpy().astype(np.float64)


def _rand(rng, *shape, scale=1.0):
    return rng.standard_normal(shape) * scale


def _close(got, want, rtol, what):
    scale = max(np.abs(want).max(), 1e-30)
    err = np.abs(got - want).max() / scale
    assert err <= rtol, f"{what}: max error {err:.3e} of scale {scale:.3e}"


# Cin 32 with one channel tile on images of 16-pixel columns and 8-pixel
# rows takes the halo boxes (16 x 8-pixel tiles: (1, 32, 32, 32, 64),
# (2, 16, 32, 32, 32), (3, 8, 16, 32, 32), (2, 128, 128, 32, 128)); other
# shapes whose 128-pixel tiles are rectangles of one image take the TMA tap
# loads (Cin 32: two 64-byte-swizzled taps a chunk; Cin a multiple of 64:
# 128-byte-swizzled boxes); the others, and Cin 96, the cp.async gather.
@pytest.mark.parametrize("n,h,w,cin,cout", [(2, 8, 8, 32, 32), (1, 12, 20, 64, 96),
                                            (3, 16, 16, 128, 64), (2, 16, 8, 32, 32),
                                            (1, 32, 32, 32, 64), (1, 4, 256, 64, 128),
                                            (2, 8, 16, 96, 32), (1, 2, 128, 256, 32),
                                            (1, 160, 128, 64, 128), (1, 150, 130, 32, 128),
                                            (2, 16, 32, 32, 32), (3, 8, 16, 32, 32),
                                            (2, 128, 128, 32, 128), (1, 24, 40, 32, 64),
                                            (2, 8, 130, 32, 32), (1, 16, 14, 32, 32),
                                            (1, 8, 3, 32, 32)])
def test_conv_forward(cuda, n, h, w, cin, cout):
    from dsmc_erlend_b200.surrogate import lib, ptr

    torch = cuda
    rng = np.random.default_rng(n * 100 + cin)
    x = _bf16(torch, _rand(rng, n, h, w, cin))
    wt = _bf16(torch, _rand(rng, cout, 3, 3, cin, scale=0.1))
    b = torch.from_numpy(rng.standard_normal(cout).astype(np.float32)).cuda()
    res = _bf16(torch, _rand(rng, n, h, w, cout))
    y = torch.empty(n, h, w, cout, dtype=torch.bfloat16, device="cuda")
    y32 = torch.empty(n, h, w, cout, dtype=torch.float32, device="cuda")
    assert lib().dsmc_sg_conv_fwd(ptr(x), ptr(wt), ptr(b), None, None, ptr(y32), n, h, w, cin,
                                  cout, 0, None) == 0
    torch.cuda.synchronize()
    want = ref.conv3x3(_np(x), _np(wt), b.cpu().numpy())
    _close(_np(y32), want, 1e-4, "forward fp32")
    assert lib().dsmc_sg_conv_fwd(ptr(x), ptr(wt), ptr(b), ptr(res), ptr(y), None, n, h, w, cin,
                                  cout, 1, None) == 0
    torch.cuda.synchronize()
    _close(_np(y), np.maximum(want, 0.0) + _np(res), 2 ** -7 + 1e-4, "forward relu + res bf16")
    # No bounded wait of the tensor-core kernel gave up.
    assert lib().dsmc_sg_check(None) == 0


@pytest.mark.parametrize("n,h,w,cin,cout", [(2, 8, 8, 32, 32), (1, 10, 6, 64, 32),
                                            (2, 12, 9, 128, 128), (1, 7, 13, 64, 96),
                                            (1, 9, 11, 96, 64), (1, 5, 9, 32, 160),
                                            (1, 6, 10, 128, 256), (2, 16, 16, 64, 32),
                                            (1, 8, 32, 32, 128), (1, 8, 16, 128, 256),
                                            (2, 4, 64, 32, 160), (2, 16, 32, 32, 32),
                                            (1, 8, 16, 32, 64), (3, 16, 16, 32, 32)])
def test_conv_dgrad_and_wgrad(cuda, n, h, w, cin, cout):
    from dsmc_erlend_b200.surrogate import lib, ptr

    torch = cuda
    rng = np.random.default_rng(7 + cin)
    x = _bf16(torch, _rand(rng, n, h, w, cin))
    wt = _bf16(torch, _rand(rng, cout, 3, 3, cin, scale=0.1))
    dy = _bf16(torch, _rand(rng, n, h, w, cout))
    w_rot = torch.empty(9 * cin * cout, dtype=torch.bfloat16, device="cuda")
    dx = torch.empty(n, h, w, cin, dtype=torch.bfloat16, device="cuda")
    dw = torch.zeros(cout, 3, 3, cin, dtype=torch.float32, device="cuda")
    db = torch.zeros(cout, dtype=torch.float32, device="cuda")
    L = lib()
    assert L.dsmc_sg_conv_dgrad(ptr(dy), ptr(wt), ptr(w_rot), ptr(dx), n, h, w, cin, cout,
                                None) == 0
    assert L.dsmc_sg_conv_wgrad(ptr(dy), ptr(x), ptr(dw), ptr(db), n, h, w, cin, cout, None) == 0
    torch.cuda.synchronize()
    _close(_np(dx), ref.conv3x3_dgrad(_np(dy), _np(wt)), 2 ** -7 + 1e-4, "dgrad")
    _close(_np(dw), ref.conv3x3_wgrad(_np(dy), _np(x)), 1e-4, "wgrad")
    _close(_np(db), _np(dy).sum(axis=(0, 1, 2)), 1e-4, "bias grad")
    assert L.dsmc_sg_check(None) == 0


@pytest.mark.parametrize("cin,cout", [(32, 64), (64, 128), (128, 32), (32, 32), (64, 32)])
def test_wgrad_large_pixel_count_splits(cuda, cin, cout):
    # Enough pixels for several pixel splits, and accumulation into dw.
    from dsmc_erlend_b200.surrogate import lib, ptr

    torch = cuda
    rng = np.random.default_rng(3)
    n, h, w = 4, 64, 64
    x = _bf16(torch, _rand(rng, n, h, w, cin))
    dy = _bf16(torch, _rand(rng, n, h, w, cout, scale=0.05))
    dw = torch.ones(cout, 3, 3, cin, dtype=torch.float32, device="cuda")
    assert lib().dsmc_sg_conv_wgrad(ptr(dy), ptr(x), ptr(dw), None, n, h, w, cin, cout,
                                    None) == 0
    torch.cuda.synchronize()
    _close(_np(dw) - 1.0, ref.conv3x3_wgrad(_np(dy), _np(x)), 1e-4, "wgrad split")
    assert lib().dsmc_sg_check(None) == 0


@pytest.mark.parametrize("n,h,w,cout", [(5, 64, 160, 32), (3, 64, 128, 64)])
def test_wgrad_halo_tile_ranges(cuda, n, h, w, cout):
    # Cin 32 on 16 x 8-pixel tiles: several tiles a CTA, a short last
    # range (400 tiles: on 148 SMs 133 CTAs of 3 and one of 1), accumulation
    # into dw.
    from dsmc_erlend_b200.surrogate import lib, ptr

    torch = cuda
    rng = np.random.default_rng(11)
    x = _bf16(torch, _rand(rng, n, h, w, 32))
    dy = _bf16(torch, _rand(rng, n, h, w, cout, scale=0.05))
    dw = torch.ones(cout, 3, 3, 32, dtype=torch.float32, device="cuda")
    assert lib().dsmc_sg_conv_wgrad(ptr(dy), ptr(x), ptr(dw), None, n, h, w, 32, cout,
                                    None) == 0
    torch.cuda.synchronize()
    _close(_np(dw) - 1.0, ref.conv3x3_wgrad(_np(dy), _np(x)), 1e-4, "wgrad halo")
    assert lib().dsmc_sg_check(None) == 0


def test_wgrad_wide_input_pixel_splits(cuda):
    # Cin 128: several pixel splits, a ragged last split, and accumulation
    # into dw.
    from dsmc_erlend_b200.surrogate import lib, ptr

    torch = cuda
    rng = np.random.default_rng(5)
    n, h, w, cin, cout = 3, 45, 37, 128, 64
    x = _bf16(torch, _rand(rng, n, h, w, cin))
    dy = _bf16(torch, _rand(rng, n, h, w, cout, scale=0.05))
    dw = torch.ones(cout, 3, 3, cin, dtype=torch.float32, device="cuda")
    assert lib().dsmc_sg_conv_wgrad(ptr(dy), ptr(x), ptr(dw), None, n, h, w, cin, cout,
                                    None) == 0
    torch.cuda.synchronize()
    _close(_np(dw) - 1.0, ref.conv3x3_wgrad(_np(dy), _np(x)), 1e-4, "wgrad wide split")
    assert lib().dsmc_sg_check(None) == 0


def test_resampling_and_loss_kernels(cuda):
    from dsmc_erlend_b200.surrogate import lib, ptr

    torch = cuda
    L = lib()
    rng = np.random.default_rng(11)
    n, h, w, c = 2, 8, 12, 32
    x = _bf16(torch, _rand(rng, n, h, w, c))
    p = torch.empty(n, h // 2, w // 2, c, dtype=torch.bfloat16, device="cuda")
    u = torch.empty(n, 2 * h, 2 * w, c, dtype=torch.bfloat16, device="cuda")
    assert L.dsmc_sg_pool_fwd(ptr(x), ptr(p), n, h, w, c, None) == 0
    assert L.dsmc_sg_up_fwd(ptr(x), ptr(u), n, h, w, c, None) == 0
    pb = torch.empty_like(x)
    ub = torch.empty_like(x)
    assert L.dsmc_sg_pool_bwd(ptr(p), ptr(pb), n, h, w, c, None) == 0
    assert L.dsmc_sg_up_bwd(ptr(u), ptr(ub), n, h, w, c, None) == 0
    torch.cuda.synchronize()
    _close(_np(p), ref.pool2(_np(x)), 2 ** -8, "pool")
    assert np.array_equal(_np(u), ref.up2(_np(x)))
    _close(_np(pb), ref.pool2_bwd(_np(p)), 2 ** -8, "pool bwd")
    _close(_np(ub), ref.up2_bwd(_np(u)), 2 ** -7, "up bwd")
    # ReLU gradient and add.
    y = _bf16(torch, _rand(rng, n, h, w, c))
    g = _bf16(torch, _rand(rng, n, h, w, c))
    g0 = _np(g)
    assert L.dsmc_sg_relu_bwd(ptr(g), ptr(y), g.numel(), None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(_np(g), g0 * (_np(y) > 0))
    # Masked MSE.
    out = torch.from_numpy(rng.standard_normal((n, h, w, c)).astype(np.float32)).cuda()
    tgt = torch.from_numpy(rng.standard_normal((n, h, w, 4)).astype(np.float32)).cuda()
    mask = torch.from_numpy((rng.random((n, h, w)) > 0.3).astype(np.float32)).cuda()
    dy = torch.empty(n, h, w, c, dtype=torch.bfloat16, device="cuda")
    loss = torch.zeros(2, device="cuda")
    assert L.dsmc_sg_mse(ptr(out), ptr(tgt), ptr(mask), ptr(dy), ptr(loss), n * h * w, c, 4,
                         None) == 0
    torch.cuda.synchronize()
    lw, gw = ref.mse(out.cpu().numpy().astype(np.float64), tgt.cpu().numpy(),
                     mask.cpu().numpy(), 4)
    assert abs(loss[0].item() - lw) <= 1e-5 * lw
    _close(_np(dy), gw, 2 ** -8, "mse grad")


def test_conv_forward_with_skip(cuda):
    # y and y + skip from one pass equal the convolution followed by the add.
    from dsmc_erlend_b200.surrogate import lib, ptr

    torch = cuda
    L = lib()
    rng = np.random.default_rng(21)
    for n, h, w, cin, cout in [(2, 16, 32, 32, 32), (1, 8, 16, 64, 64), (1, 16, 16, 128, 128)]:
        x = _bf16(torch, _rand(rng, n, h, w, cin))
        wt = _bf16(torch, _rand(rng, cout, 3, 3, cin, scale=0.1))
        b = torch.from_numpy(rng.standard_normal(cout).astype(np.float32)).cuda()
        skip = _bf16(torch, _rand(rng, n, h, w, cout))
        y = torch.empty(n, h, w, cout, dtype=torch.bfloat16, device="cuda")
        ysum, y0, ysum0 = torch.empty_like(y), torch.empty_like(y), torch.empty_like(y)
        assert L.dsmc_sg_conv_fwd_skip(ptr(x), ptr(wt), ptr(b), ptr(skip), ptr(y), ptr(ysum),
                                       n, h, w, cin, cout, 1, None) == 0
        assert L.dsmc_sg_conv_fwd(ptr(x), ptr(wt), ptr(b), None, ptr(y0), None, n, h, w, cin,
                                  cout, 1, None) == 0
        ysum0.copy_(y0)
        assert L.dsmc_sg_add(ptr(ysum0), ptr(skip), ysum0.numel(), None) == 0
        torch.cuda.synchronize()
        assert torch.equal(y, y0) and torch.equal(ysum, ysum0)
    assert L.dsmc_sg_check(None) == 0


def test_rotate_layers(cuda):
    # Several layers' rotated weights in one launch, at their offsets.
    import ctypes as C

    from dsmc_erlend_b200.surrogate import lib, ptr

    torch = cuda
    rng = np.random.default_rng(8)
    shapes = [(32, 32), (64, 32), (128, 64)]  # (cout, cin)
    offs, off = [], 16
    for co, ci in shapes:
        offs.append(off)
        off += 9 * co * ci + 32
    w = _bf16(torch, _rand(rng, off))
    rot = torch.zeros(off, dtype=torch.bfloat16, device="cuda")
    n = len(shapes)
    assert lib().dsmc_sg_rotate_layers(
        ptr(w), ptr(rot), (C.c_int64 * n)(*offs), (C.c_int * n)(*[ci for _, ci in shapes]),
        (C.c_int * n)(*[co for co, _ in shapes]), n, None) == 0
    torch.cuda.synchronize()
    wn, rn = _np(w), _np(rot)
    for (co, ci), o in zip(shapes, offs):
        k = 9 * co * ci
        want = wn[o:o + k].reshape(co, 9, ci)[:, ::-1, :].transpose(2, 1, 0).ravel()
        assert np.array_equal(rn[o:o + k], want)


def _round_bf16(torch, a):
    return torch.from_numpy(np.asarray(a, np.float32)).to(torch.bfloat16).float().numpy()


@pytest.mark.parametrize("c", [32, 128])
def test_fused_backward_passes(cuda, c):
    # dsmc_sg_relu_bias_bwd (skip copy or add, ReLU mask, bias gradient) and
    # the accumulating pooling / upsampling gradients, against the separate
    # passes they replace.
    from dsmc_erlend_b200.surrogate import lib, ptr

    torch = cuda
    L = lib()
    rng = np.random.default_rng(c)
    n, h, w = 2, 8, 12
    y = _bf16(torch, _rand(rng, n, h, w, c))
    g = _bf16(torch, _rand(rng, n, h, w, c))
    s0 = _bf16(torch, _rand(rng, n, h, w, c))
    g0, y0, s00 = _np(g), _np(y), _np(s0)
    masked = g0 * (y0 > 0)
    # ReLU with the skip source's first gradient (a copy).
    skip = torch.empty_like(g)
    db = torch.ones(c, device="cuda")
    assert L.dsmc_sg_relu_bias_bwd(ptr(g), ptr(y), ptr(skip), 0, ptr(db), n * h * w, c,
                                   None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(_np(skip), g0)
    assert np.array_equal(_np(g), masked)
    _close(db.cpu().numpy() - 1.0, masked.sum(axis=(0, 1, 2)), 1e-5, "bias grad")
    # No ReLU, the skip gradient added.
    g2 = _bf16(torch, g0)
    db2 = torch.zeros(c, device="cuda")
    assert L.dsmc_sg_relu_bias_bwd(ptr(g2), None, ptr(s0), 1, ptr(db2), n * h * w, c,
                                   None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(_np(g2), g0)
    assert np.array_equal(_np(s0), _round_bf16(torch, s00 + g0))
    _close(db2.cpu().numpy(), g0.sum(axis=(0, 1, 2)), 1e-5, "bias grad, no relu")
    # Pooling and upsampling gradients added to what dx holds.
    p = _bf16(torch, _rand(rng, n, h // 2, w // 2, c))
    u = _bf16(torch, _rand(rng, n, 2 * h, 2 * w, c))
    d0 = _rand(rng, n, h, w, c)
    pb, ub = _bf16(torch, d0), _bf16(torch, d0)
    base = _np(pb)
    assert L.dsmc_sg_pool_bwd_acc(ptr(p), ptr(pb), n, h, w, c, 1, None) == 0
    assert L.dsmc_sg_up_bwd_acc(ptr(u), ptr(ub), n, h, w, c, 1, None) == 0
    pw, uw = torch.empty_like(pb), torch.empty_like(ub)
    assert L.dsmc_sg_pool_bwd(ptr(p), ptr(pw), n, h, w, c, None) == 0
    assert L.dsmc_sg_up_bwd(ptr(u), ptr(uw), n, h, w, c, None) == 0
    torch.cuda.synchronize()
    assert np.array_equal(_np(pb), _round_bf16(torch, base + _np(pw)))
    assert np.array_equal(_np(ub), _round_bf16(torch, base + _np(uw)))


def test_adam_step(cuda):
    from dsmc_erlend_b200.surrogate import lib, ptr

    torch = cuda
    rng = np.random.default_rng(5)
    w = rng.standard_normal(1000).astype(np.float32)
    g = rng.standard_normal(1000).astype(np.float32)
    m = rng.standard_normal(1000).astype(np.float32) * 0.1
    v = rng.random(1000).astype(np.float32) * 0.1
    tw, tg, tm, tv = (torch.from_numpy(a.copy()).cuda() for a in (w, g, m, v))
    wb = torch.empty(1000, dtype=torch.bfloat16, device="cuda")
    assert lib().dsmc_sg_adam(ptr(tw), ptr(wb), ptr(tg), ptr(tm), ptr(tv), 1000, 1e-3, 0.9,
                              0.999, 1e-8, 3, None) == 0
    torch.cuda.synchronize()
    # The kernel's constants are the float32 roundings of 0.9 and 0.999.
    b1, b2 = np.float32(0.9), np.float32(0.999)
    m1 = b1 * m + (np.float32(1) - b1) * g
    v1 = b2 * v + (np.float32(1) - b2) * g * g
    w1 = w - 1e-3 * (m1 / (1 - b1 ** 3)) / (np.sqrt(v1 / (1 - b2 ** 3)) + 1e-8)
    assert np.allclose(tw.cpu().numpy(), w1, rtol=1e-5, atol=1e-7)
    # FP32 with contraction on the GPU: within a few ulp of the moments' terms.
    assert np.allclose(tm.cpu().numpy(), m1, rtol=1e-5, atol=1e-7)
    assert np.allclose(tv.cpu().numpy(), v1, rtol=1e-5, atol=1e-9)
    assert np.allclose(wb.float().cpu().numpy(), w1, rtol=2 ** -7)


def test_network_gradients_match_restatement(cuda):
    from dsmc_erlend_b200.surrogate import LAYERS, Surrogate

    torch = cuda
    n, res = 2, 32
    net = Surrogate(n, res=res, seed=4)
    rng = np.random.default_rng(9)
    # Nonzero biases, so every ReLU sees both signs.
    for name in net.b32:
        net.b32[name].copy_(torch.from_numpy(rng.standard_normal(net.b32[name].numel())
                                             .astype(np.float32) * 0.1))
    x = _bf16(torch, _rand(rng, n, res, res, 32))
    out = net.forward(x)
    torch.cuda.synchronize()
    params = {}
    for name in net.w32:
        params[name + ".w"] = net.wb[name].float().cpu().numpy().astype(np.float64)
        params[name + ".b"] = net.b32[name].cpu().numpy().astype(np.float64)
    acts = ref.network_forward(params, _np(x), LAYERS)
    _close(out.cpu().numpy(), acts[LAYERS[-1][0]], 0.01, "network output")
    dout = _bf16(torch, _rand(rng, n, res, res, 32, scale=1e-2))
    net.backward(dout)
    torch.cuda.synchronize()
    # The backward is checked on the kernels' own forward activations (bf16,
    # as stored): with the restatement's, the few pre-activations within a
    # rounding of zero would switch ReLU masks between the two sides and
    # their differences, not the backward kernels', would dominate 18 layers
    # down.
    gpu_acts = {"x": _np(x)}
    for name, src, op, *_ in LAYERS:
        gpu_acts[name + ".relu"] = _np(net.relu_out[name])
        gpu_acts[name + ".in"] = _np(net.a_in[name]) if op else _np(net._acts[src])
    grads = ref.network_backward(params, gpu_acts, _np(dout), LAYERS)
    # Each weight tensor is held to 4% relative L2, each bias (a sum over
    # every pixel, where terms cancel) to 8%, and every element to 10% of its
    # tensor's scale.
    errs = {}
    for name in net.w32:
        for kind, got in (("w", net.gw[name]), ("b", net.gb[name])):
            want = grads[f"{name}.{kind}"]
            g = got.cpu().numpy()
            errs[f"{name}.{kind}"] = (float(np.linalg.norm(g - want) /
                                            max(np.linalg.norm(want), 1e-30)),
                                      float(np.abs(g - want).max() /
                                            max(np.abs(want).max(), 1e-30)))
    print({k: (round(a, 4), round(b, 4)) for k, (a, b) in errs.items()})
    for k, (l2, worst) in errs.items():
        assert l2 <= (0.04 if k.endswith(".w") else 0.08) and worst <= 0.10, (k, l2, worst)


def test_trained_surrogate_beats_freestream_and_shortens_transient(cuda, engine_lib):
    """What the network gains over the method without it: trained on fields
    the engine generates (small ensemble), its held-out predictions are
    closer to DSMC than the freestream (density and temperature each, and the
    four quantities together), and a warm start from its prediction is closer
    to the converged field after a short window than the cold start after the
    same window."""
    from dsmc_erlend_b200 import Engine, setup
    from dsmc_erlend_b200.sgdata import case_input, generate, prediction_field, surrogate_cases
    from dsmc_erlend_b200.surrogate import Surrogate, predict, relative_errors, train
    from dsmc_erlend_b200.fields import weighted_errors
    from dsmc_erlend_b200.timetofield import merged_field, reference_field, warm_array

    cases = surrogate_cases(96, seed=77, steps=1500, grid_range=(64, 96))
    x, t, m, _ = generate(cases, chunk=48)
    net, hist = train(x[:80], t[:80], m[:80], epochs=150, batch=16, lr=2e-3, seed=1)
    assert hist[-1][1] < 0.5 * hist[0][1]
    pred = predict(net, x[80:])
    got = relative_errors(pred, t[80:], m[80:])
    free = np.zeros_like(t[80:])
    for i, p in enumerate(cases[80:]):
        d = setup(p)
        free[i, ..., 0] = 1.0
        free[i, ..., 1] = d.ux_free / d.u_free
        free[i, ..., 2] = d.uy_free / d.u_free
        free[i, ..., 3:7] = p.t_free / (p.t_free * (1.0 + p.ma_free ** 2 / 3.0))
    base = relative_errors(free, t[80:], m[80:])
    # Density and temperature, where the freestream is far off, each improve;
    # over n, ux, uy and T together the error falls well below the
    # freestream's.
    assert got["n"] < base["n"] and got["t"] < base["t"], (got, base)
    main = ("n", "ux", "uy", "t")
    assert sum(got[k] for k in main) < 0.7 * sum(base[k] for k in main), (got, base)

    # Transient: one held-out case (dense enough that the local Maxwellian is
    # a fair start), converged reference from replicas, then cold and warm
    # runs compared after the same short window.
    p = cases[90].copy(n_free=1e18, first_sampling_step=0)
    d = setup(p)
    ref = reference_field(p.copy(first_sampling_step=1500), 4, transient=1500, steps=1500)
    one = Surrogate(1)
    one.load_state_dict(net.state_dict())
    warm_f = prediction_field(p, d, predict(one, case_input(p)[None])[0])
    window = 300
    errs = {}
    kinds = {"warm": "moments", "warm_tensor": "tensor", "warm_mixture": "mixture_tensor"}
    for start in ("cold", *kinds):
        e = Engine(p)
        if start in kinds:
            e.init_warm(warm_array(p, d, warm_f, kinds[start]))
        else:
            e.InitialConditions()
        e.step(window)
        errs[start] = weighted_errors(merged_field(e, 1), ref, p, d.u_free)
        e.close()
    # After the same window the warm starts are closer to the converged
    # field than the cold start: in density, in temperature and summed over
    # n, ux, uy and T.
    for w in ("warm", "warm_tensor"):
        assert errs[w]["n"] < errs["cold"]["n"], errs
        assert errs[w]["t"] < errs["cold"]["t"], errs
        assert sum(errs[w].values()) < sum(errs["cold"].values()), errs
    # The two-population seed (freestream plus the rest of the predicted
    # tensor) gains over the cold start as well.
    assert sum(errs["warm_mixture"].values()) < sum(errs["cold"].values()), errs
    print("errors after the window:", errs)


def test_graph_train_step_matches_eager(cuda):
    # The captured step (device-side learning rate and bias corrections)
    # gives the weights of the eager step, with a changing learning rate.
    from dsmc_erlend_b200.surrogate import OUT_CH, Surrogate, lib

    torch = cuda
    res = 32
    rng = np.random.default_rng(11)
    x = torch.from_numpy(rng.standard_normal((2, res, res, 32)).astype(np.float32))
    x = x.to(torch.bfloat16).cuda()
    tgt = torch.from_numpy(rng.standard_normal((2, res, res, OUT_CH)).astype(np.float32)).cuda()
    mask = torch.ones(2, res, res, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    eager = Surrogate(2, res=res, seed=3, stream=s1.cuda_stream)
    graph = Surrogate(2, res=res, seed=3, stream=s2.cuda_stream)
    lrs = [1e-3, 5e-4, 2e-4]
    with torch.cuda.stream(s1):
        for lr in lrs:
            eager.train_step(x, tgt, mask, lr=lr)
    for lr in lrs:
        graph.train_step_graph(x, tgt, mask, lr=lr)
    torch.cuda.synchronize()
    for name in eager.w32:
        a, b = eager.w32[name].cpu().numpy(), graph.w32[name].cpu().numpy()
        assert np.allclose(a, b, rtol=1e-5, atol=1e-7), name
        # The bf16 copies are the FP32 masters rounded: equal, or one bf16
        # rounding apart where the masters differ in their last bits (the
        # weight gradients are summed with FP32 atomics, in any order).  One
        # bf16 unit in the last place of v in [2^e, 2^(e+1)) is 2^(e - 7).
        wa = eager.wb[name].float().cpu().numpy()
        wg = graph.wb[name].float().cpu().numpy()
        big = np.maximum(np.abs(wa), np.abs(wg))
        ulp = np.ldexp(1.0, np.frexp(big)[1] - 8)  # frexp: big = m 2^k, m in [0.5, 1)
        assert np.all(np.abs(wa - wg) <= ulp), name
    assert lib().dsmc_sg_check(None) == 0
