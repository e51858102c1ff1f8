"""The denoiser's kernels and network against the numpy FP64 oracle
(oracle/unet.py), and its training on the card.

One convolution: the forward output, the input gradient and the weight and
bias gradients of the BF16 tensor-core kernels equal the FP64 results on the
same BF16-rounded operands up to FP32 accumulation and the BF16 rounding of
the outputs (y, dx: 1/128 of the largest value; dw, db: 1e-3 relative).
The whole network's parameter gradient: per layer, cosine > 0.99 and
relative error < 0.1 against the FP64 oracle run on the same parameters
(the card stores every activation and activation gradient in BF16).
"""
import numpy as np
import pytest

import mb3dcu
import unet

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("cin,cout,n,h,w", [(16, 32, 2, 9, 13), (32, 32, 2, 9, 13), (48, 64, 2, 9, 13),
                                             (80, 48, 2, 9, 13), (32, 96, 2, 9, 13), (112, 16, 2, 9, 13),
                                             (176, 80, 2, 9, 13), (16, 128, 2, 9, 13),
                                             # more tiles than blocks: each block's accumulators
                                             # take several tiles through the stage ring
                                             (16, 32, 8, 100, 124), (64, 48, 3, 61, 77)])
def test_conv_kernels_match_fp64(card, cin, cout, n, h, w):
    rng = np.random.default_rng(cin * 1000 + cout + h)
    # (9 x 13: ragged, partial pixel tiles, every border)
    x = unet.bf16(rng.standard_normal((n, h, w, cin)))
    wt = unet.bf16(rng.standard_normal((cout, 9, cin)) * np.sqrt(2.0 / (9 * cin)))
    b = rng.standard_normal(cout).astype(np.float32)
    dy = unet.bf16(rng.standard_normal((n, h, w, cout)))
    y, dx, dw, db = mb3dcu.conv_check(card, x, wt, b, dy)
    ye = unet.conv(x.astype(np.float64), wt.astype(np.float64), b.astype(np.float64))
    dxe, dwe, dbe = unet.conv_bwd(x.astype(np.float64), wt.astype(np.float64), dy.astype(np.float64))
    assert np.abs(y - ye).max() <= np.abs(ye).max() / 128, (cin, cout)
    assert np.abs(dx - dxe).max() <= np.abs(dxe).max() / 128, (cin, cout)
    assert np.abs(dw - dwe).max() <= 1e-3 * np.abs(dwe).max(), (cin, cout)
    assert np.abs(db - dbe).max() <= 1e-3 * np.abs(dbe).max(), (cin, cout)


def test_tensor_core_wait_runs_out_and_the_context_stays_usable(card):
    """The convolution's pipeline waits are bounded by a launch parameter:
    with its TMA and MMA lanes told to issue nothing, the epilogue's first
    accumulator wait runs out after 2 ms (nothing in flight), the kernel
    frees its tensor memory and the host reads an error status; the next
    convolutions on the same context work."""
    L = mb3dcu.lib()
    assert L.mb3d_cu_dn_wait_check(card._ctx, 2000.0, 1) == mb3dcu.EIO
    assert "wait ran out" in L.mb3d_cu_last_error().decode()
    assert L.mb3d_cu_dn_wait_check(card._ctx, 2000.0, 0) == 0
    rng = np.random.default_rng(11)
    x = unet.bf16(rng.standard_normal((1, 9, 13, 16)))
    wt = unet.bf16(rng.standard_normal((32, 9, 16)) * 0.1)
    b = rng.standard_normal(32).astype(np.float32)
    dy = unet.bf16(rng.standard_normal((1, 9, 13, 32)))
    y = mb3dcu.conv_check(card, x, wt, b, dy)[0]
    ye = unet.conv(x.astype(np.float64), wt.astype(np.float64), b.astype(np.float64))
    assert np.abs(y - ye).max() <= np.abs(ye).max() / 128


def _batch(rng, n, h, w):
    rad = rng.gamma(1.0, 0.4, (n, h, w, 3)).astype(np.float32)
    alb = rng.uniform(0, 1, (n, h, w, 3)).astype(np.float32)
    nrm = rng.standard_normal((n, h, w, 3)).astype(np.float32)
    nrm /= np.linalg.norm(nrm, axis=-1, keepdims=True)
    dep = rng.uniform(0.2, 1.0, (n, h, w)).astype(np.float32)
    tgt = (rad * rng.uniform(0.5, 1.5, rad.shape)).astype(np.float32)
    return rad, alb, nrm, dep, tgt


def test_network_gradient_matches_fp64_oracle(card):
    rng = np.random.default_rng(5)
    dn = mb3dcu.Denoiser(card, seed=3)
    try:
        p = dn.get_params()
        # non-zero biases, so that every ReLU sees both signs
        p = p + np.where(np.arange(p.size) % 7 == 0, 0.01, 0.0).astype(np.float32)
        dn.set_params(p)
        rad, alb, nrm, dep, tgt = _batch(rng, 2, 32, 48)
        loss, g = dn.gradient(rad, tgt, alb, nrm, dep, depth_scale=1.0)
        x = unet.pack_input(rad.astype(np.float64), alb, nrm, dep, 1.0)
        pred, cache = unet.forward(p, x)
        le, dpred = unet.l1_loss(pred, tgt.astype(np.float64))
        ge = unet.backward(p, cache, dpred)
        assert abs(loss - le) <= 0.02 * le, (loss, le)
        o = 0
        for i, (cin, cout, _) in enumerate(unet.layers()):
            k = cout * 9 * cin + cout
            a, e = g[o:o + k].astype(np.float64), ge[o:o + k]
            o += k
            if i == 18:  # the output layer: only channels 0..2 have a gradient
                a = a.reshape(-1)
            cos = a @ e / (np.linalg.norm(a) * np.linalg.norm(e) + 1e-30)
            rel = np.linalg.norm(a - e) / (np.linalg.norm(e) + 1e-30)
            assert cos > 0.99 and rel < 0.1, (i, cos, rel)
    finally:
        dn.close()


def test_training_lowers_the_loss(card):
    rng = np.random.default_rng(9)
    dn = mb3dcu.Denoiser(card, seed=4)
    try:
        rad, alb, nrm, dep, tgt = _batch(rng, 4, 64, 64)
        first = dn.train_step(rad, tgt, alb, nrm, dep, lr=2e-3)
        for _ in range(60):
            last = dn.train_step(rad, tgt, alb, nrm, dep, lr=2e-3)
        assert last < 0.7 * first, (first, last)
        out = dn.denoise(rad, alb, nrm, dep)
        assert out.shape == rad.shape and np.isfinite(out).all() and out.min() >= 0.0
        # a picture whose size is not a multiple of 16
        odd = dn.denoise(rad[:1, :50, :37].copy(), alb[:1, :50, :37].copy(), nrm[:1, :50, :37].copy(),
                         dep[:1, :50, :37].copy())
        assert odd.shape == (1, 50, 37, 3) and np.isfinite(odd).all()
    finally:
        dn.close()


def test_device_inputs_made_by_torch_are_ready(card):
    """Inputs that torch has only just computed on its own stream: the binding
    orders torch's stream before the library's, so the denoised picture is
    the one of the finished inputs (the same as from host arrays)."""
    import torch
    rng = np.random.default_rng(11)
    dn = mb3dcu.Denoiser(card, seed=2)
    try:
        rad, alb, nrm, dep, _ = _batch(rng, 2, 64, 96)
        want = dn.denoise(rad, alb, nrm, dep, depth_scale=1.0)
        big = torch.randn(4096, 4096, device="cuda")
        for _ in range(4):
            big = big @ big  # (keeps torch's stream busy)
        t = [torch.from_numpy(a).cuda(non_blocking=True) * 1.0 + 0.0 * big[0, 0] for a in (rad, alb, nrm, dep)]
        got = dn.denoise(*t, depth_scale=1.0)
        assert np.array_equal(got.cpu().numpy(), want)
    finally:
        dn.close()


def test_trained_network_beats_the_plain_trace(card):
    """What the trained network gains over the method without it: on a
    picture it was not trained on (the hybrid scene at 240x135), the 4-ray
    trace denoised with the committed weights is closer to an independent
    256-ray trace than the 4-ray trace itself (PSNR of x/(1+x), +2 dB at
    least); the 16-ray trace denoised stays within 0.5 dB of the plain one
    or above it (the network is trained for 4 and 16 rays)."""
    import os
    import train_denoiser as T
    import scenes
    if not os.path.exists(T.WEIGHTS):
        pytest.skip("no trained weights")
    sc = scenes.scaled(scenes.c2_hybrid(), 240, 135)
    lv = mb3dcu.mc_light_default(sc)
    ref = card.mc_render(sc, mb3dcu.mc_opts(256, depth=4, ray0=4096), lv)["radiance"]
    r4 = card.mc_render(sc, mb3dcu.mc_opts(4, depth=4), lv)
    r16 = card.mc_render(sc, mb3dcu.mc_opts(16, depth=4), lv)["radiance"]
    dn = mb3dcu.Denoiser(card)
    try:
        dn.set_params(np.fromfile(T.WEIGHTS, "<f4"))
        g = [r4[k][None].copy() for k in ("albedo", "normal", "depth")]
        den4 = dn.denoise(r4["radiance"][None].copy(), *g)[0]
        den16 = dn.denoise(r16[None].copy(), *g)[0]
    finally:
        dn.close()
    p4, pd4, p16, pd16 = (T.psnr(a, ref) for a in (r4["radiance"], den4, r16, den16))
    assert pd4 >= p4 + 2.0 and pd16 >= p16 - 0.5, (p4, pd4, p16, pd16)
