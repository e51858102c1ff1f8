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


@pytest.mark.parametrize("kind", [mb3dcu.Denoiser.LOSS_L1_LOG, mb3dcu.Denoiser.LOSS_TONE_MSE,
                                  mb3dcu.Denoiser.LOSS_TONE_DISPLAY])
def test_network_gradient_matches_fp64_oracle(card, kind):
    rng = np.random.default_rng(5)
    dn = mb3dcu.Denoiser(card, seed=3)
    try:
        dn.set_loss(kind)
        p = dn.get_params()
        # non-zero biases, so that every ReLU sees both signs
        p = p + np.where(np.arange(p.size) % 7 == 0, 0.01, 0.0).astype(np.float32)
        if kind != mb3dcu.Denoiser.LOSS_L1_LOG:
            # the output layer scaled down: the untrained network's outputs
            # (about +-50) would put the tone's exp(-pred) far out of range
            k_out = unet.layers()[-1][1] * 9 * unet.layers()[-1][0] + unet.layers()[-1][1]
            p[-k_out:] *= 0.02
        dn.set_params(p)
        rad, alb, nrm, dep, tgt = _batch(rng, 2, 32, 48)
        loss, g = dn.gradient(rad, tgt, alb, nrm, dep, depth_scale=1.0)
        x = unet.pack_input(rad.astype(np.float64), alb, nrm, dep, 1.0)
        pred, cache = unet.forward(p, x)
        if kind == mb3dcu.Denoiser.LOSS_L1_LOG:
            le, dpred = unet.l1_loss(pred, tgt.astype(np.float64))
        else:
            le, dpred = unet.tone_mse_loss(pred, tgt.astype(np.float64), kind == mb3dcu.Denoiser.LOSS_TONE_DISPLAY)
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


def _fallback_np(a, b, den, tile, k):
    """The fallback rule in FP64 numpy: per tile x tile piece (ragged at the
    right and bottom), the keep-the-plain-trace decision and its margin."""
    def tone(x):
        x = np.maximum(x.astype(np.float64), 0.0)
        return x / (1.0 + x)
    h, w, _ = den.shape
    m = 0.5 * (a + b)  # (float32, as the card forms it)
    out = den.copy()
    keep, margin = [], []
    for y in range(0, h, tile):
        for x in range(0, w, tile):
            sl = (slice(y, y + tile), slice(x, x + tile))
            cnt = den[sl].size
            sigma = np.sqrt(np.sum((tone(a[sl]) - tone(b[sl])) ** 2) / cnt / 4.0 / cnt) + 1e-3
            dev = abs(np.sum(tone(den[sl]) - tone(m[sl])) / cnt)
            keep.append(dev > k * sigma)
            margin.append(abs(dev - k * sigma) / (k * sigma))
            if keep[-1]:
                out[sl] = m[sl]
    return out, np.array(keep), np.array(margin)


def test_fallback_keeps_the_plain_trace_where_the_denoised_picture_is_off(card):
    """The plain trace as the fallback and judge (mb3d_cu_dn_fallback): two
    noisy halves of a smooth picture and a 'denoised' picture equal to the
    smooth one except in two pieces made 60 % brighter (one of them the
    ragged corner piece): exactly those keep the plain trace; the decisions
    and the composite equal the FP64 rule's; device buffers and out == den
    give the same."""
    rng = np.random.default_rng(21)
    h, w, tile = 50, 70, 16
    yy, xx = np.mgrid[0:h, 0:w]
    truth = (0.4 + 0.3 * np.sin(xx / 9.0)[..., None] * np.cos(yy / 7.0)[..., None] * np.array([1.0, 0.8, 0.6]))
    truth = truth.astype(np.float32)
    a = (truth * rng.gamma(8.0, 1 / 8.0, truth.shape)).astype(np.float32)
    b = (truth * rng.gamma(8.0, 1 / 8.0, truth.shape)).astype(np.float32)
    den = truth.copy()
    den[16:32, 32:48] *= 1.6
    den[48:50, 64:70] *= 1.6
    want, keep, margin = _fallback_np(a, b, den, tile, 3.0)
    assert margin.min() > 1e-4  # (no decision at the threshold's edge)
    tiles_x = (w + tile - 1) // tile
    assert keep[1 * tiles_x + 2] and keep[3 * tiles_x + 4]
    dn = mb3dcu.Denoiser(card, seed=1)
    try:
        got, share = dn.fallback(a, b, den, tile=tile, k=3.0)
        assert share == pytest.approx(keep.mean(), abs=1e-6)
        assert np.array_equal(got, want)
        import torch
        t = [torch.from_numpy(v).cuda() for v in (a, b, den)]
        got_d, share_d = dn.fallback(*t, tile=tile, k=3.0, out=t[2])
        assert share_d == share and np.array_equal(got_d.cpu().numpy(), want)
        # a denoised picture equal to the truth: few pieces, the rule's own
        _, keep0, _ = _fallback_np(a, b, truth, tile, 3.0)
        assert dn.fallback(a, b, truth, tile=tile)[1] == pytest.approx(keep0.mean(), abs=1e-6) and keep0.mean() < 0.2
        with pytest.raises(mb3dcu.CardError):
            dn.fallback(a, b, den, tile=0)
    finally:
        dn.close()


def test_unknown_loss_is_refused(card):
    dn = mb3dcu.Denoiser(card, seed=1)
    try:
        with pytest.raises(mb3dcu.CardError):
            dn.set_loss(7)
    finally:
        dn.close()


@pytest.mark.parametrize("kind", [mb3dcu.Denoiser.LOSS_L1_LOG, mb3dcu.Denoiser.LOSS_TONE_DISPLAY])
def test_training_lowers_the_loss(card, kind):
    rng = np.random.default_rng(9)
    dn = mb3dcu.Denoiser(card, seed=4)
    try:
        dn.set_loss(kind)
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
    least), and the 16-ray trace denoised gains too (0.3 dB at least; on
    the whole C5 frame the committed network gains 2.0 dB there)."""
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
    assert pd4 >= p4 + 2.0 and pd16 >= p16 + 0.3, (p4, pd4, p16, pd16)
