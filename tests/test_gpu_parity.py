"""Parity of the card's kernels with the oracle (the C++ FP64 restatement of
the reference CPU march), through the C ABI.

The plain FP64 march is the drop-in: its records agree with the oracle up
to the last bits of FMA contraction and of the device's log/sin/cos.  The
mixed march (FP32 bulk, FP64 origin, t and finish) is held to the targets:
>= 99.9 % hit/miss agreement and <= 1e-4 relative depth error on the
pixels both hit (the median; at least 98 % of the pixels within 1e-4 --
the rest are grazing rays where the single precision bulk's sample points,
a fraction of a step away from the FP64 march's, meet the near or the far
surface of an edge), normals within the reference's own card tolerance
(mean cosine > 0.97, src/gpu.rs:4177-4248).
"""
import ctypes

import numpy as np
import pytest

import mb3dcu
import oracle_py as O
import scenes
from gbcompare import compare

pytestmark = pytest.mark.gpu


def zc(sc):
    p = O.params(sc)
    return p[7], p[6]


def test_de_probe_matches_oracle(card):
    rng = np.random.default_rng(1)
    for name in ("Integer Power", "Amazing Box", "Bulbox", "Tricorn", "Real Power", "Folding Int Pow", "Quaternion",
                 "Aexion C"):
        sc = scenes.preset(name, 96, 72)
        pts = rng.uniform(-1.6, 1.6, size=(2000, 3))
        d0, i0 = O.de_at(sc, pts)
        d1, i1 = card.de_probe(sc, pts, mb3dcu.FP64)
        assert (i0 == i1).mean() > 0.999, name
        rel = np.abs(d0 - d1) / np.maximum(np.abs(d0), 1e-300)
        assert np.median(rel) < 1e-12 and (rel < 1e-6).mean() > 0.999, (name, np.max(rel))
        d2, i2 = card.de_probe(sc, pts, mb3dcu.FP32_FP64)
        rel2 = np.abs(d0 - d2) / np.maximum(np.abs(d0), 1e-300)
        assert np.median(rel2) < 1e-2, (name, np.median(rel2))


@pytest.mark.parametrize("name", scenes.PRESETS)
def test_fp64_march_matches_oracle(card, name):
    sc = scenes.preset(name, 160, 120)
    ref = O.march(sc, mb3dcu.SILIGHT)
    g = card.march(sc, mb3dcu.FP64)
    r = compare(g, ref, *zc(sc))
    assert r["hit_agree"] >= 0.999, r
    assert r["exact"] >= 0.95, r
    assert r.get("depth_rel_p99", 0.0) < 1e-6, r


def _ipol_scenes():
    a = scenes.interpolated("Integer Power", "Tricorn", (0.7, 0.3), 160, 120)
    b = scenes.interpolated("Amazing Box", "Amazing Box", (0.5, 0.5), 160, 120)
    b.slots[1].options[0] = 2.5  # (two boxes: the analytic DE's blend)
    c = scenes.interpolated("Integer Power", "Folding Int Pow", (0.5, 0.5), 160, 120)
    d = scenes.interpolated("Quaternion", "Quaternion", (0.5, 0.5), 160, 120)
    d.slots[1].options[1] = 0.1  # (two Quaternions: the 4D interpolation, doInterpolHybridPas4D)
    return [("ip8+tricorn", a), ("box+box", b), ("ip8+fip", c), ("quat+quat 4d", d)]


def test_interpolation_hybrid_matches_oracle(card):
    """Interpolation hybrids (doInterpolHybridPas[DE], src/iteration.rs:347-
    455): the numerical DE's blend (Integer Power with Tricorn, with Folding
    Int Pow) and the analytic one's (two Amazing Boxes), the FP64 march
    against the oracle with the same bounds as the single formulas; the
    mixed mode marches them in FP64 (the precision rule sends every pixel
    there) and gives the same records; the DE probe at points."""
    for name, sc in _ipol_scenes():
        ref = O.march(sc, mb3dcu.SILIGHT)
        g = card.march(sc, mb3dcu.FP64)
        r = compare(g, ref, *zc(sc))
        assert r["hit_agree"] >= 0.999 and r["exact"] >= 0.95, (name, r)
        assert r.get("depth_rel_p99", 0.0) < 1e-6, (name, r)
        gm = card.march(sc, mb3dcu.FP32_FP64)
        assert card.stats()["fp64_pixels"] == sc.width * sc.height
        assert gm.tobytes() == g.tobytes(), name
        pts = np.array([[0.3, 0.2, -2.0], [0.7, -0.4, 0.5], [0.1, 0.9, -0.3], [1.2, -0.2, 0.4]])
        d0, i0 = O.de_at(sc, pts)
        d1, i1 = card.de_probe(sc, pts, mb3dcu.FP64)
        assert np.array_equal(i0, i1), (name, i0, i1)
        assert np.all(np.abs(d1 - d0) <= 1e-6 * np.maximum(np.abs(d0), 1e-3)), (name, d0, d1)


def test_quaternion_4d_rotation_and_hybrid(card):
    """The 4D hybrid (doHybrid4DPas, src/iteration.rs:757-772): the Quaternion
    preset turned in 4D (BuildSMatrix4 of three plane angles), and the
    Quaternion in a 3D alternating hybrid with Integer Power (the DE options
    combine to the 3D numerical DE), the FP64 march against the oracle."""
    a = scenes.preset("Quaternion", 160, 120)
    a.rot_4d[0], a.rot_4d[1], a.rot_4d[2] = 0.3, -0.15, 0.2
    b = scenes.preset("Quaternion", 160, 120)
    scenes.set_slots(b, [scenes.slot(mb3dcu.F_QUATERNION, 1, -1.0, 0.0), scenes.intpow(8, -1.0, 1)])
    for name, sc in (("4d-rotated", a), ("quaternion+ip8", b)):
        ref = O.march(sc, mb3dcu.SILIGHT)
        assert (~mb3dcu.is_background(ref)).mean() > 0.02, name
        g = card.march(sc, mb3dcu.FP64)
        r = compare(g, ref, *zc(sc))
        assert r["hit_agree"] >= 0.999 and r["exact"] >= 0.95, (name, r)
        assert card.march(sc, mb3dcu.FP32_FP64).tobytes() == g.tobytes(), name


def _decomb_scenes():
    out = [("two objects (min)", scenes.two_objects("min"))]
    for kind in ("max", "max_inverted", "smooth_linear", "smooth"):
        out.append((kind, scenes.two_objects(kind, place=False)))
    return out


def test_de_combinations_match_oracle(card):
    """DE combinations (CalcDEfull with FormulaType > 0, src/calc.rs:1365-
    1455): the reference's scene of two objects (a Mandelbulb and an Amazing
    Box moved, turned and scaled as part 2, combined by min) and the bulb with
    a box over it combined by max, max with the inverted box and the two
    smooth minima: the FP64 march against the oracle with the single
    formulas' bounds, the mixed mode giving the same records (every pixel in
    FP64), and the DE probe with its iteration counts at points of both
    parts (the reference's grid of both_parts_of_a_de_combination_use_their
    _compiled_loops, tests/render.rs:345-382)."""
    i = np.arange(8000)
    grid = np.stack([(i % 20) * 0.25 - 1.3, ((i // 20) % 20) * 0.14 - 1.3, (i // 400) * 0.14 - 1.3], 1)
    for name, sc in _decomb_scenes():
        ref = O.march(sc, mb3dcu.SILIGHT)
        assert (~mb3dcu.is_background(ref)).mean() > 0.03, name
        g = card.march(sc, mb3dcu.FP64)
        r = compare(g, ref, *zc(sc))
        assert r["hit_agree"] >= 0.999 and r["exact"] >= 0.95, (name, r)
        assert r.get("depth_rel_p99", 0.0) < 1e-6, (name, r)
        assert card.march(sc, mb3dcu.FP32_FP64).tobytes() == g.tobytes(), name
        d0, i0 = O.de_at(sc, grid)
        d1, i1 = card.de_probe(sc, grid, mb3dcu.FP64)
        assert (i0 == i1).mean() > 0.999, name
        rel = np.abs(d0 - d1) / np.maximum(np.abs(d0), 1e-300)
        assert np.median(rel) < 1e-12 and (rel < 1e-6).mean() > 0.999, (name, np.max(rel))


def test_de_combination_shadows_and_ao(card):
    """Hard shadows and DE AO on the scene of two objects (their DEs are the
    combination's, their surface tests take the ruling part's iteration
    limit): the card's FP64 render against the oracle's passes."""
    sc = scenes.two_objects("min")
    sc.shadow_lights, sc.deao_quality = 1, 1
    ref = O.deao(sc, O.shadows(sc, O.march(sc, mb3dcu.SILIGHT), per_pixel=True))
    g = card.render(sc, mb3dcu.FP64)
    obj = ~mb3dcu.is_background(ref) & ~mb3dcu.is_background(g)
    assert obj.mean() > 0.1
    sh = (g["shadow"][obj] >> 10) == (ref["shadow"][obj] >> 10)
    da = np.abs(g["amb_shadow"][obj].astype(np.int64) - ref["amb_shadow"][obj].astype(np.int64))
    assert sh.mean() >= 0.98 and (da <= 16).mean() >= 0.97, (sh.mean(), (da <= 16).mean())


def test_interpolation_hybrid_shadows_and_ao(card):
    """The post passes on an interpolation hybrid (their DEs blend too): hard
    shadows and DE AO of the card's FP64 render against the oracle's passes
    on the oracle's G-buffer."""
    name, sc = _ipol_scenes()[0]
    sc.shadow_lights, sc.deao_quality = 1, 1
    ref = O.deao(sc, O.shadows(sc, O.march(sc, mb3dcu.SILIGHT), per_pixel=True))
    g = card.render(sc, mb3dcu.FP64)
    obj = ~mb3dcu.is_background(ref) & ~mb3dcu.is_background(g)
    assert obj.mean() > 0.1
    sh = (g["shadow"][obj] >> 10) == (ref["shadow"][obj] >> 10)
    da = np.abs(g["amb_shadow"][obj].astype(np.int64) - ref["amb_shadow"][obj].astype(np.int64))
    assert sh.mean() >= 0.98 and (da <= 16).mean() >= 0.97, (sh.mean(), (da <= 16).mean())


def test_menger_hybrid_fp64_and_mixed(card):
    sc = scenes.scaled(scenes.c4_frames(8)[0], 160, 90)
    ref = O.march(sc, mb3dcu.SILIGHT)
    g = card.march(sc, mb3dcu.FP64)
    r = compare(g, ref, *zc(sc))
    assert r["hit_agree"] >= 0.999 and r["exact"] >= 0.95, r
    m = card.march(sc, mb3dcu.FP32_FP64)
    rm = compare(m, ref, *zc(sc))
    assert rm["hit_agree"] >= 0.99, rm


@pytest.mark.parametrize("name", ["Integer Power", "Amazing Box", "Bulbox"])
def test_mixed_march_matches_oracle(card, name):
    sc = scenes.preset(name, 320, 240)
    ref = O.march(sc, mb3dcu.SILIGHT)
    g = card.march(sc, mb3dcu.FP32_FP64)
    r = compare(g, ref, *zc(sc))
    assert r["hit_agree"] >= 0.995, r
    assert r["depth_rel_median"] <= 1e-4, r
    assert r["normal_cos_mean"] > 0.97, r


def test_c1_full_size_both_precisions(card):
    sc = scenes.c1_plain_bulb()
    ref = O.march(sc, mb3dcu.SILIGHT)
    g64 = card.march(sc, mb3dcu.FP64)
    r64 = compare(g64, ref, *zc(sc))
    assert r64["hit_agree"] >= 0.9995, r64
    g32 = card.march(sc, mb3dcu.FP32_FP64)
    r32 = compare(g32, ref, *zc(sc))
    assert r32["hit_agree"] >= 0.999, r32
    assert r32["depth_rel_median"] <= 1e-4, r32
    assert r32["depth_rel_1e4"] >= 0.98, r32
    assert r32["normal_cos_mean"] > 0.97, r32


def test_c2_shadows_and_deao(card):
    sc = scenes.scaled(scenes.c2_hybrid(), 480, 270)
    ref = O.march(sc, mb3dcu.SILIGHT)
    for prec, agree in ((mb3dcu.FP64, 0.999), (mb3dcu.FP32_FP64, 0.99)):
        g = card.march(sc, prec)
        # post passes on the oracle's own G-buffer: the pass compared alone
        a = card.post_on_card(sc, ref.copy(), mb3dcu.POST_SHADOW | mb3dcu.POST_DEAO, prec)
        b = O.deao(sc, O.shadows(sc, ref.copy(), per_pixel=True))
        obj = mb3dcu.hit_mask(ref)
        sh = ((a["shadow"] & 0x400) == (b["shadow"] & 0x400))[obj].mean()
        assert sh >= agree, (prec, sh)
        dao = np.abs(a["amb_shadow"].astype(np.int64) - b["amb_shadow"].astype(np.int64))[obj] / 16383.0
        assert dao.mean() < 0.01 and (dao > 0.1).mean() < 0.01, (prec, dao.mean(), (dao > 0.1).mean())
        r = compare(g, ref, *zc(sc))
        assert r["hit_agree"] >= agree, (prec, r)


def test_menger_shadows_iteration_limited_surfaces(card):
    """The shadow pass where the iteration count limits the surfaces (the
    Menger IFS hybrid of the animation): its start points come from
    RMdoBinSearchIt, in double precision in both modes."""
    sc = scenes.scaled(scenes.c4_frames(8)[3], 160, 90)
    ref = O.march(sc, mb3dcu.SILIGHT)
    obj = mb3dcu.hit_mask(ref)
    assert obj.mean() > 0.2
    b = O.shadows(sc, ref.copy(), per_pixel=True)
    for prec, agree in ((mb3dcu.FP64, 0.999), (mb3dcu.FP32_FP64, 0.99)):
        a = card.post_on_card(sc, ref.copy(), mb3dcu.POST_SHADOW, prec)
        sh = ((a["shadow"] & 0x400) == (b["shadow"] & 0x400))[obj].mean()
        assert sh >= agree, (prec, sh)
        if prec == mb3dcu.FP64:
            assert (a["shadow"] == b["shadow"])[obj].mean() >= 0.999


def _painted_psnr(sc, a, b):
    pa, pb = O.paint(sc, a).astype(np.float64), O.paint(sc, b).astype(np.float64)
    return 10 * np.log10(255.0 ** 2 / max(float(np.mean((pa - pb) ** 2)), 1e-12))


def test_painted_pictures_match_the_oracle(card):
    """The parity of the pictures: the oracle's painter (render::paint,
    default lighting) applied to the card's G-buffer and to the oracle's.
    The FP64 drop-in paints the oracle's picture (measured 99-168 dB); the
    mixed mode's surfaces lie a fraction of a step away and its normals
    follow the rough fractal surface there (measured 30.6-37.2 dB)."""
    c1 = scenes.c1_plain_bulb()
    ref = O.march(c1, mb3dcu.SILIGHT)
    assert _painted_psnr(c1, card.march(c1, mb3dcu.FP64), ref) >= 60.0
    assert _painted_psnr(c1, card.march(c1, mb3dcu.FP32_FP64), ref) >= 35.0
    # the whole C2 frame: march, hard shadows, DE AO
    c2 = scenes.scaled(scenes.c2_hybrid(), 480, 270)
    ref = O.deao(c2, O.shadows(c2, O.march(c2, mb3dcu.SILIGHT), per_pixel=True))
    assert _painted_psnr(c2, card.render(c2, mb3dcu.FP64), ref) >= 60.0
    assert _painted_psnr(c2, card.render(c2, mb3dcu.FP32_FP64), ref) >= 29.5
    c4 = scenes.scaled(scenes.c4_frames(8)[0], 320, 180)
    ref = O.march(c4, mb3dcu.SILIGHT)
    assert _painted_psnr(c4, card.march(c4, mb3dcu.FP64), ref) >= 60.0
    assert _painted_psnr(c4, card.march(c4, mb3dcu.FP32_FP64), ref) >= 33.0


def test_card_painter_matches_the_oracle(card):
    """mb3d_cu_paint (render::paint on the card) against the oracle's
    painter on the same records: both single precision and unfused; the
    card's sinf/cosf of the view vector may move a channel by one step."""
    import torch
    cases = []
    c2 = scenes.scaled(scenes.c2_hybrid(), 480, 270)
    cases.append((c2, card.render(c2, mb3dcu.FP64)))
    c4 = scenes.scaled(scenes.c4_frames(8)[3], 320, 180)
    cases.append((c4, card.render(c4, mb3dcu.FP32_FP64)))
    c1 = scenes.scaled(scenes.c1_plain_bulb(), 320, 240)
    cases.append((c1, card.march(c1, mb3dcu.FP32_FP64)))
    for sc, g in cases:
        want = O.paint(sc, g).astype(np.int64)
        got = card.paint(sc, g).astype(np.int64)
        d = np.abs(got - want)
        assert (d == 0).mean() >= 0.999 and d.max() <= 1, ((d == 0).mean(), d.max())
        # a band of rows, on device buffers
        r0, rows = sc.height // 3, sc.height // 4
        band = g[r0 * sc.width:(r0 + rows) * sc.width]
        dg = torch.from_numpy(band.view(np.uint8).copy()).cuda()
        dout = torch.zeros((rows, sc.width, 3), dtype=torch.uint8, device="cuda")
        card.paint(sc, dg, row0=r0, out=dout)
        torch.cuda.synchronize()
        assert np.array_equal(dout.cpu().numpy(), got[r0:r0 + rows])
    with pytest.raises(mb3dcu.CardError) as e:
        card.paint(c1, cases[2][1], row0=10)
    assert e.value.status == mb3dcu.EINVAL


def test_ssao_matches_the_oracle(card):
    """gpu::ssao24 (the 24-bit SSAO, regular sampling) against the oracle's
    ssao::ssao24 on the same G-buffer: the angles are the reference's bit
    for bit (single precision, unfused); the sum of their arctangents uses
    the card's atanf, so a pixel may land one step away from the oracle's
    where the sum sits at a rounding boundary."""
    import torch
    c2 = scenes.scaled(scenes.c2_hybrid(), 480, 270)
    g = O.march(c2, mb3dcu.SILIGHT)
    zm, zr = zc(c2)
    obj = ~mb3dcu.is_background(g)
    assert obj.mean() > 0.2
    cases = [dict(), dict(threshold=1.5, t0=True), dict(border_mirror=0.3), dict(wrap_x=True, threshold=3.0)]
    for kw in cases:
        o = mb3dcu.ssao_default()
        for k, v in kw.items():
            setattr(o, k, v)
        want = O.ssao24(g, c2.width, c2.height, zm, zr, **kw)
        got = card.ssao24(c2, g, o)
        d = np.abs(got["amb_shadow"].astype(np.int64) - want["amb_shadow"].astype(np.int64))[obj]
        assert (d == 0).mean() >= 0.99 and d.max() <= 1, (kw, (d == 0).mean(), d.max())
        assert np.array_equal(got["amb_shadow"][~obj], g["amb_shadow"][~obj])
        assert np.array_equal(got["zpos_fine"], g["zpos_fine"])
    # a device G-buffer, changed in place, equals the host one
    dev = torch.from_numpy(g.view(np.uint8).copy()).cuda()
    card.ssao24(c2, dev)
    torch.cuda.synchronize()
    host = card.ssao24(c2, g)
    assert dev.cpu().numpy().tobytes() == host.tobytes()


def test_ssao15_matches_the_oracle(card):
    """gpu::ssao15 (the older 15-bit SSAO) against the oracle's
    ssao15::ssao15 on the same G-buffers (the hybrid frame at 480x270, and
    a small 37x23 picture where every pixel is near a border): the levels
    and the slopes are the reference's bit for bit, the arctangents' sum
    uses the card's atanf (one step apart where the sum sits at a rounding
    boundary); the t0 variant, the threshold and the panorama's wrap."""
    import torch
    c2 = scenes.scaled(scenes.c2_hybrid(), 480, 270)
    small = scenes.scaled(scenes.c2_hybrid(), 37, 23)
    for sc in (c2, small):
        g = O.march(sc, mb3dcu.SILIGHT)
        zm, zr = zc(sc)
        obj = ~mb3dcu.is_background(g)
        assert obj.mean() > 0.2
        for kw in [dict(), dict(threshold=1.5, t0=True), dict(wrap_x=True, threshold=3.0)]:
            o = mb3dcu.ssao_default()
            for k, v in kw.items():
                setattr(o, k, v)
            want = O.ssao15(g, sc.width, sc.height, zm, zr, **kw)
            got = card.ssao15(sc, g, o)
            d = np.abs(got["amb_shadow"].astype(np.int64) - want["amb_shadow"].astype(np.int64))[obj]
            assert (d == 0).mean() >= 0.99 and d.max() <= 1, (sc.width, kw, (d == 0).mean(), d.max())
            assert np.array_equal(got["amb_shadow"][~obj], g["amb_shadow"][~obj])
            assert np.array_equal(got["zpos_fine"], g["zpos_fine"])
    # a device G-buffer, changed in place, equals the host one
    g = O.march(c2, mb3dcu.SILIGHT)
    dev = torch.from_numpy(g.view(np.uint8).copy()).cuda()
    card.ssao15(c2, dev)
    torch.cuda.synchronize()
    assert dev.cpu().numpy().tobytes() == card.ssao15(c2, g).tobytes()
    # pictures below 4 x 4 stay as they are
    tiny = scenes.scaled(scenes.c2_hybrid(), 3, 3)
    gt = O.march(tiny, mb3dcu.SILIGHT)
    assert card.ssao15(tiny, gt).tobytes() == gt.tobytes()


def test_render_device_buffer_equals_host_buffer(card):
    import torch
    sc = scenes.scaled(scenes.c2_hybrid(), 240, 136)
    host = card.render(sc, mb3dcu.FP32_FP64)
    dev = torch.zeros(sc.width * sc.height * 20, dtype=torch.uint8, device="cuda")
    card.render(sc, mb3dcu.FP32_FP64, out=dev)
    torch.cuda.synchronize()
    got = np.frombuffer(dev.cpu().numpy().tobytes(), dtype=mb3dcu.SILIGHT)
    assert got.tobytes() == host.tobytes()
    # the same picture twice (no state left between calls)
    assert card.render(sc, mb3dcu.FP32_FP64).tobytes() == host.tobytes()


def test_bands_equal_whole_picture(card):
    sc = scenes.preset("Integer Power", 128, 96)
    whole = card.march(sc, mb3dcu.FP32_FP64)
    parts = [card.march(sc, mb3dcu.FP32_FP64, row0=r, rows=32) for r in (0, 32, 64)]
    assert np.concatenate(parts).tobytes() == whole.tobytes()


def test_errors_and_cancel(card):
    sc = scenes.preset("Integer Power", 64, 48)
    with pytest.raises(mb3dcu.CardError) as e:
        card.march(sc, mb3dcu.FP64, row0=40, rows=20)
    assert e.value.status == mb3dcu.EINVAL
    flag = ctypes.c_int(1)
    with pytest.raises(mb3dcu.CardError) as e:
        card.march(sc, mb3dcu.FP64, cancel=flag)
    assert e.value.status == mb3dcu.ECANCELED
    # the context still works after the failures
    assert mb3dcu.hit_mask(card.march(sc, mb3dcu.FP64)).mean() > 0.05


def _six_lights(sc):
    """All six lights on, spread around the object; every light casts shadows."""
    import math
    for i in range(6):
        sc.lights[i] = mb3dcu.Light(1, 0, (i * 60.0 - 150.0) * math.pi / 180.0, (35.0 - 12.0 * i) * math.pi / 180.0)
    sc.shadow_lights = 0x3F
    return sc


def test_six_light_hard_shadows(card):
    """The hard shadow pass with six lights (one shadow bit each,
    0x400 << light) on the oracle's G-buffer, against hard_shadow_row of
    the oracle (src/calc.rs:2777-2898) per light."""
    sc = _six_lights(scenes.scaled(scenes.c2_hybrid(), 240, 135))
    ref = O.march(sc, mb3dcu.SILIGHT)
    obj = mb3dcu.hit_mask(ref)
    b = O.shadows(sc, ref.copy(), per_pixel=True)
    assert all(0.05 < ((b["shadow"] & (0x400 << k)) != 0)[obj].mean() < 0.999 for k in range(6))
    for prec, agree in ((mb3dcu.FP64, 0.999), (mb3dcu.FP32_FP64, 0.99)):
        a = card.post_on_card(sc, ref.copy(), mb3dcu.POST_SHADOW, prec)
        for light in range(6):
            bit = 0x400 << light
            same = ((a["shadow"] & bit) == (b["shadow"] & bit))[obj].mean()
            assert same >= agree, (prec, light, same)
        assert ((a["shadow"] & 0x3FF) == (ref["shadow"] & 0x3FF)).all()  # the step count is kept


@pytest.mark.parametrize("radius", [1.0, 3.0])
def test_soft_shadow(card, radius):
    """The soft shadow (calcHSsoft, src/calc.rs:2901-2979): a 6-bit light
    value in bits 10..15 for the last selected light, against the oracle."""
    sc = scenes.scaled(scenes.c2_hybrid(), 240, 135)
    sc.shadow_soft, sc.soft_radius = 1, radius
    ref = O.march(sc, mb3dcu.SILIGHT)
    obj = mb3dcu.hit_mask(ref)
    b = O.shadows(sc, ref.copy(), per_pixel=True)
    vb = (b["shadow"] >> 10).astype(np.int64)
    assert (vb[obj] < 63).mean() > 0.05  # some pixels are in (part) shadow
    for prec, tol, share in ((mb3dcu.FP64, 1, 0.999), (mb3dcu.FP32_FP64, 2, 0.98)):
        a = card.post_on_card(sc, ref.copy(), mb3dcu.POST_SHADOW, prec)
        va = (a["shadow"] >> 10).astype(np.int64)
        d = np.abs(va - vb)[obj]
        assert (d <= tol).mean() >= share, (prec, radius, (d <= tol).mean(), d.max())
        assert d.mean() < 0.5, (prec, radius, d.mean())


def test_random_ssao_matches_the_oracle(card):
    """The 24-bit SSAO with random sampling (SsaoParams::random passes,
    TAmbHiQCalcR, src/ssao.rs:207-247): the card keeps each row's number
    chain exactly (a warp per row), so its samples are the oracle's; each
    pass's sum may land one step away (the card's atanf)."""
    c2 = scenes.scaled(scenes.c2_hybrid(), 480, 270)
    g = O.march(c2, mb3dcu.SILIGHT)
    zm, zr = zc(c2)
    obj = ~mb3dcu.is_background(g)
    cases = [dict(random=1), dict(random=3, border_mirror=0.3), dict(random=2, t0=True, threshold=1.5),
             dict(random=2, wrap_x=True)]
    for kw in cases:
        o = mb3dcu.ssao_default()
        for k, v in kw.items():
            setattr(o, k, v)
        want = O.ssao24(g, c2.width, c2.height, zm, zr, **kw)
        got = card.ssao24(c2, g, o)
        d = np.abs(got["amb_shadow"].astype(np.int64) - want["amb_shadow"].astype(np.int64))[obj]
        assert (d == 0).mean() >= 0.99 and d.max() <= kw["random"], (kw, (d == 0).mean(), d.max())
        assert np.array_equal(got["amb_shadow"][~obj], g["amb_shadow"][~obj])
    # random sampling differs from regular sampling, but not by much on average
    reg = card.ssao24(c2, g)["amb_shadow"][obj].astype(np.float64)
    o = mb3dcu.ssao_default()
    o.random = 4
    rnd = card.ssao24(c2, g, o)["amb_shadow"][obj].astype(np.float64)
    assert (reg != rnd).mean() > 0.3 and abs(rnd.mean() - reg.mean()) < 0.1 * reg.mean()
