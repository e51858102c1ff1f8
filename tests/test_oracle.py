"""The oracle against the reference's own known-answer tests (CPU only).

Each test restates one of mb3d-rs's tests for this path; the citation is
in its docstring.  These pin the oracle, since the reference binary cannot
run here.
"""
import math

import numpy as np
import pytest

import mb3dcu
import oracle_py as O
import scenes


def triplex(n, v):
    """The spherical triplex power (src/formulas.rs:915-921)."""
    r = math.sqrt(sum(c * c for c in v))
    th = math.atan2(v[1], v[0]) * n
    ph = math.atan2(v[2], math.hypot(v[0], v[1])) * n
    rn = r ** n
    return [rn * math.cos(th) * math.cos(ph), rn * math.sin(th) * math.cos(ph), -rn * math.sin(ph)]


@pytest.mark.parametrize("n", range(2, 9))
def test_int_powers_match_spherical_triplex(n):
    """src/formulas.rs:923-941."""
    p = [0.31, -0.42, 0.27]
    v, _ = O.formula_iterate(mb3dcu.F_INTPOW, [n, -1.0], p + [0.0], [0, 0, 0, 0])
    exp = triplex(n, p)
    for k in range(3):
        assert abs(v[k] - exp[k]) < 1e-9, (n, k, v[k], exp[k])


def test_real_power_matches_int_power8():
    """src/formulas.rs:943-954."""
    p = [0.31, -0.42, 0.27]
    rout = sum(c * c for c in p)
    a, _ = O.formula_iterate(mb3dcu.F_INTPOW, [8, -1.0], p + [0.0], [0] * 4, rout)
    b, _ = O.formula_iterate(mb3dcu.F_REALPOWER, [8.0, -1.0], p + [0.0], [0] * 4, rout)
    assert np.all(np.abs(a[:3] - b[:3]) < 1e-9)


def test_box_scales_derivative():
    """src/formulas.rs:956-966: r < min_r^2, w *= scale / min_r^2."""
    v, _ = O.formula_iterate(mb3dcu.F_AMAZINGBOX, [2.0, 0.5, 1.0], [0.1, 0.1, 0.1, 1.0], [0] * 4, 0.0, ade=True)
    assert abs(v[3] - 8.0) < 1e-12


def test_a_negative_min_r_acts_as_zero():
    """src/formulas.rs:863-875."""
    for ade in (False, True):
        for p in ([0.1, 0.1, 0.1, 1.0], [0.8, -0.3, 0.2, 1.0], [0.01, 0.02, -0.01, 1.0]):
            neg, _ = O.formula_iterate(mb3dcu.F_AMAZINGBOX, [1.7, -0.6, 0.3], p, [0] * 4, 0.0, ade)
            zero, _ = O.formula_iterate(mb3dcu.F_AMAZINGBOX, [1.7, 0.0, 0.3], p, [0] * 4, 0.0, ade)
            pos, _ = O.formula_iterate(mb3dcu.F_AMAZINGBOX, [1.7, 0.6, 0.3], p, [0] * 4, 0.0, ade)
            assert np.array_equal(neg, zero)
            assert not np.array_equal(neg, pos)


def test_pixel_seed_steps_along_the_row():
    """src/calc.rs:2986-2996 (the jump-ahead equals stepping the LCG)."""
    for y in (0, 7, 1499):
        s = ((0x24563487 + (y + 1) * 0x324594A1) + 2 ** 31) % 2 ** 32 - 2 ** 31
        for x in range(3000):
            assert O.pixel_seed(y, x) == s, (y, x)
            s = ((s * 214013 + 2531011) + 2 ** 31) % 2 ** 32 - 2 ** 31


def test_bulb_distance_estimate_is_sane():
    """tests/render.rs:47-60."""
    s = scenes.preset("Integer Power", 96, 72)
    de, its = O.de_at(s, [[0.0, 0.0, 0.0], [0.3, 0.2, -2.0]])
    assert its[0] == s.iterations
    assert its[1] < s.iterations
    assert 0.2 < de[1] < 1.5


def test_analytic_box_de_is_sane():
    """tests/render.rs:63-71."""
    s = scenes.preset("Amazing Box", 96, 72)
    p = O.params(s)
    assert p[29] == 1.0  # is_custom_de
    de, _ = O.de_at(s, [[0.0, 0.0, -9.0]])
    assert 0.5 < de[0] < 6.0


@pytest.mark.parametrize("name", scenes.PRESETS)
def test_every_preset_hits_the_object(name):
    """tests/render.rs:24-30."""
    g = O.march(scenes.preset(name, 96, 72), mb3dcu.SILIGHT)
    cov = 1.0 - mb3dcu.is_background(g).mean()
    assert 0.05 < cov < 0.995, (name, cov)


def test_deterministic_and_thread_independent():
    """tests/render.rs:11-21 (byte-exact across thread counts)."""
    s = scenes.preset("Integer Power", 96, 72)
    a = O.march(s, mb3dcu.SILIGHT, threads=1)
    b = O.march(s, mb3dcu.SILIGHT, threads=3)
    assert a.tobytes() == b.tobytes()


def test_shadows_darken():
    """tests/render.rs:118-139: some pixel in shadow; the per-pixel form of the
    card pass agrees with the row pass on most pixels."""
    s = scenes.preset("Integer Power", 96, 72)
    s.shadow_lights = 0x3F
    s.soft_radius = 2.0
    g = O.march(s, mb3dcu.SILIGHT)
    a = O.shadows(s, g.copy(), per_pixel=False)
    b = O.shadows(s, g.copy(), per_pixel=True)
    obj = ~mb3dcu.is_background(a)
    assert ((a["shadow"] & 0x400) != 0)[obj].sum() > 0
    assert ((a["shadow"] & 0x400) == (b["shadow"] & 0x400))[obj].mean() > 0.95


def test_deao_occludes():
    """tests/render.rs:162-177 (DE AO quality 1: some pixel > 2000)."""
    s = scenes.preset("Integer Power", 96, 72)
    s.deao_quality = 1
    g = O.deao(s, O.march(s, mb3dcu.SILIGHT))
    obj = ~mb3dcu.is_background(g)
    assert (g["amb_shadow"][obj] > 2000).sum() > 0


def test_deao_ray_counts():
    """src/deao.rs:462-470."""
    assert len(O.ao_rays(0)) == 3
    r1, r3 = len(O.ao_rays(1)), len(O.ao_rays(3))
    assert 5 <= r1 and r3 <= 33 and r3 > r1
    assert len(O.ao_rays(2)) == 17


def test_catmull_rom_passes_through_keyframes():
    """src/anim.rs:692-700: weight 1 on keyframe 1 at t=0, on keyframe 2 at t=1."""
    assert scenes.catmull_rom_weights(0.0) == [0.0, 1.0, 0.0, 0.0]
    w = scenes.catmull_rom_weights(1.0)
    assert abs(w[2] - 1.0) < 1e-15 and abs(w[0]) + abs(w[1]) + abs(w[3]) < 1e-15
    for t in (0.1, 0.5, 0.9):
        assert abs(sum(scenes.catmull_rom_weights(t)) - 1.0) < 1e-12


def test_configs_see_the_object():
    """The synthetic workloads show the fractal (not empty, not all inside)."""
    for sc in (scenes.scaled(scenes.c1_plain_bulb(), 160, 120), scenes.scaled(scenes.c2_hybrid(), 160, 90),
               scenes.scaled(scenes.c4_frames(8)[0], 160, 90)):
        g = O.march(sc, mb3dcu.SILIGHT)
        h = mb3dcu.hit_mask(g).mean()
        assert 0.05 < h < 0.99, h


def test_deep_zoom_fixture_point():
    """The deep zoom's point is on the surface and its camera outside the set."""
    import json
    import os
    f = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c3_point.json")))
    assert f["camera_outside"]
    sc = scenes.c3_deep_zoom(f["point"], f["view_dir"], 64, 36)
    de, its = O.de_at(sc, [f["point"]])
    assert de[0] < 1e-8


def _seed_of(x, y, b):
    """seed_of (src/mc.rs:1107-1116) in Python."""
    def mix(h):
        h &= 0xFFFFFFFF
        h ^= h >> 16
        h = (h * 0x7FEB352D) & 0xFFFFFFFF
        h ^= h >> 15
        h = (h * 0x846CA68B) & 0xFFFFFFFF
        return h ^ (h >> 16)
    v = mix(((x * 0x9E3779B1) & 0xFFFFFFFF) ^ mix(((y * 0x85EBCA77) & 0xFFFFFFFF) ^ mix(b + 0x165667B1)))
    return v - (1 << 32) if v >= 1 << 31 else v


def test_mc_seed_and_halton():
    """seed_of and halton_seq (src/mc.rs:103-128, 1107-1116) as Python
    restates them; the first Halton numbers of bases 2 and 3 are the van der
    Corput fractions 1/2, 1/4, 3/4 and 1/3, 2/3, 1/9."""
    for x, y, b in ((1, 0, 0), (1920, 1079, 3), (17, 5, 1023), (-3, 7, 2 ** 31)):
        assert O.mc_seed_of(x, y, b & 0xFFFFFFFF) == _seed_of(x, y, b), (x, y, b)
    for i, (f2, f3) in enumerate(((0.5, 1 / 3), (0.25, 2 / 3), (0.75, 1 / 9))):
        rec, _ = O.mc_halton(i, 1, 0)
        assert rec[0] == round(f2 * 65535) and rec[1] == round(f3 * 65535)
    _, sh = O.mc_halton(0, 5, 9)
    assert all(0.0 <= s < 1.0 for s in sh)


def test_mc_light_values_of_the_startup_lighting():
    """LightVals::build (src/lighting.rs:978-1190) of Lighting::default
    (src/lighting.rs:290-391): light 0 colour $A0E8FF as r, g, b; specular
    function 53 & 7 -> power 2 << 5; diffuse 120 x 0.02; specular 50 x 0.02;
    depth fog 27 x 0.8e-6; the palette at 0, 10922, 21844, 32200 + 84 k."""
    sc = scenes.c2_hybrid()
    lv = mb3dcu.mc_light_default(sc)
    assert lv.n_lights == 1
    assert list(lv.col[0]) == [255.0, 232.0, 160.0]
    assert lv.pow_func[0] == 64
    assert abs(lv.s_diff - 2.4) < 1e-6 and abs(lv.s_spec - 1.0) < 1e-7
    assert abs(lv.s_depth - 2.16e-5) < 1e-11
    assert list(lv.col_pos) == [0, 10922, 21844] + [32200 + 84 * k for k in range(7)]
    assert abs(lv.col_dif[0][0] - 0xE1 / 255) < 1e-7  # 5873889 = $59A0E1: r = $E1
    assert abs(lv.lmax_l[0] - 800.0 * (255 + 232 + 160 + 128)) < 1e-3
    ln = np.array(list(lv.ln[0]))
    assert abs(np.linalg.norm(ln) - 1.0) < 1e-6


def test_mc_oracle_is_deterministic_and_sane():
    """The Monte Carlo oracle: thread-independent, lights the object, every
    pixel's light finite and within the clamp."""
    sc = scenes.scaled(scenes.c2_hybrid(), 64, 36)
    lv = mb3dcu.mc_light_default(sc)
    o = mb3dcu.mc_opts(4, depth=3)
    a = O.mc_render(sc, lv, o, threads=1)
    b = O.mc_render(sc, lv, o, threads=4)
    assert a["radiance"].tobytes() == b["radiance"].tobytes()
    assert 0.05 < a["hit"].mean() < 0.99
    assert np.isfinite(a["radiance"]).all() and a["radiance"].min() >= 0.0 and a["radiance"].max() <= 400.0
    # the first surface's normal is a unit vector where there is one
    n = np.linalg.norm(a["normal"], axis=2)
    assert np.all(np.abs(n[a["depth"] > 0] - 1.0) < 1e-9)


def test_mc_painter_lab_round_trip():
    """mc.rs lab_roundtrip (src/mc.rs:4187-4195): RGB -> Lab -> RGB within
    1e-3 for its three colours, seen through the painter with the default
    settings (exposure 1, no gamma curve, no soft clip, saturation 1), which
    squares, converts there and back and takes the square root."""
    opts = mb3dcu.mc_paint_default()
    assert (opts.contrast, opts.saturation, opts.options, opts.gamma) == (128, 32, 2, 32.0)
    for v in ([0.2, 0.5, 0.8], [1.0, 1.0, 1.0], [0.01, 0.0, 0.3]):
        c = np.sqrt(np.array([v], np.float32))
        rgb = O.mc_paint(c, opts)[0].astype(np.float64)
        # |sqrt(v + e) - sqrt(v)| * 255 with |e| <= 1e-3, plus the rounding
        tol = 255 * np.max(np.sqrt(np.array(v) + 1e-3) - np.sqrt(v)) + 0.5
        assert np.abs(rgb - 255 * c[0]).max() <= tol, (v, rgb)


def test_mc_painter_default_settings_and_rays():
    """With the default settings the painted picture is the clipped colour in
    8 bits up to the round trip's last bits; pixels without rays are black;
    the gamma slider and the exposure move the picture the way they say."""
    rng = np.random.default_rng(11)
    c = rng.uniform(-0.2, 2.0, (20000, 3)).astype(np.float32)
    opts = mb3dcu.mc_paint_default()
    p = O.mc_paint(c, opts).astype(int)
    e = np.round(np.clip(c, 0, 1) * 255).astype(int)
    assert np.abs(p - e).max() <= 1 and (p == e).mean() > 0.99
    rays = (np.arange(len(c)) % 3 != 0).astype(np.uint8)
    q = O.mc_paint(c, opts, rays)
    assert (q[rays == 0] == 0).all() and (q[rays == 1] == p[rays == 1]).all()
    mid = rng.uniform(0.05, 0.6, (2000, 3)).astype(np.float32)
    base = O.mc_paint(mid, opts).astype(int).sum()
    bright, dark, expo = mb3dcu.mc_paint_default(), mb3dcu.mc_paint_default(), mb3dcu.mc_paint_default()
    bright.gamma, dark.gamma, expo.contrast = 63.0, 0.0, 200
    assert O.mc_paint(mid, bright).astype(int).sum() > base > O.mc_paint(mid, dark).astype(int).sum()
    assert O.mc_paint(mid, expo).astype(int).sum() > base


def test_painter_background_shadows_and_occlusion():
    """The oracle's Calculate 3D painter (render::paint, default lighting):
    with the default dynamic fog the background is the depth colour gradient
    (top depth_col to bottom depth_col2, src/lighting.rs:1791) up to
    rounding; a hard shadow bit and the ambient occlusion only darken."""
    sc = scenes.scaled(scenes.c2_hybrid(), 96, 54)
    g = O.deao(sc, O.shadows(sc, O.march(sc, mb3dcu.SILIGHT), per_pixel=True))
    img = O.paint(sc, g).astype(int)
    h, w = sc.height, sc.width
    bg = ((g["zpos_fine"] >> 16) >= 32768).reshape(h, w)
    obj = mb3dcu.hit_mask(g).reshape(h, w)
    assert bg.mean() > 0.2 and obj.mean() > 0.1
    yp = (np.arange(h, dtype=np.float32) / np.float32(h))[:, None, None]
    top = np.array([0x1D, 0x49, 0x8B], np.float32)
    bottom = np.array([0x9F, 0xC4, 0xFF], np.float32)
    want = np.round(top + yp * (bottom - top)) * np.ones((1, w, 1))
    assert np.abs(img[bg] - want[bg]).max() <= 1
    lit = g.copy()
    lit["shadow"] &= 0x3FF
    a = O.paint(sc, lit).astype(int).sum(-1)
    shadowed = ((g["shadow"] & 0x400) != 0).reshape(h, w) & obj
    assert shadowed.sum() > 20
    assert (img.sum(-1)[shadowed] <= a[shadowed]).all() and (img.sum(-1)[shadowed] < a[shadowed]).mean() > 0.95
    open_ = g.copy()
    open_["amb_shadow"] = 0
    c = O.paint(sc, open_).astype(int).sum(-1)
    assert (img.sum(-1)[obj] <= c[obj]).mean() > 0.99


def test_unet_oracle_backward_matches_finite_differences():
    """The denoiser oracle's backward pass (oracle/unet.py) against central
    differences of its forward pass, FP64, on a 1 x 16 x 16 input."""
    import unet
    rng = np.random.default_rng(2)
    n_par = sum(co * 9 * ci + co for ci, co, _ in unet.layers())
    p = np.zeros(n_par)
    o = 0
    for ci, co, _ in unet.layers():
        p[o:o + co * 9 * ci] = rng.standard_normal(co * 9 * ci) * np.sqrt(2.0 / (9 * ci))
        o += co * 9 * ci
        p[o:o + co] = rng.standard_normal(co) * 0.05
        o += co
    rad = rng.gamma(1.0, 0.4, (1, 16, 16, 3))
    x = unet.pack_input(rad, rng.uniform(0, 1, (1, 16, 16, 3)), rng.standard_normal((1, 16, 16, 3)),
                        rng.uniform(0, 1, (1, 16, 16)), 1.0)
    tgt = rad * 1.3

    def loss(q):
        # a smooth loss (squared error) keeps the check away from L1's kinks
        pred, _ = unet.forward(q, x)
        e = pred[..., :3] - np.log1p(tgt)
        return 0.5 * np.sum(e * e)

    pred, cache = unet.forward(p, x)
    dpred = np.zeros_like(pred)
    dpred[..., :3] = pred[..., :3] - np.log1p(tgt)
    g = unet.backward(p, cache, dpred)
    idx = rng.choice(n_par, 40, replace=False)
    for i in idx:
        e = np.zeros(n_par)
        e[i] = 1e-6
        num = (loss(p + e) - loss(p - e)) / 2e-6
        assert abs(num - g[i]) <= 1e-4 * max(1.0, abs(num)), (i, num, g[i])


def test_unet_oracle_tone_loss_gradient_matches_finite_differences():
    """The tone-space squared error's gradient with respect to the
    prediction (oracle/unet.py tone_mse_loss) against central differences."""
    import unet
    rng = np.random.default_rng(4)
    pred = rng.normal(0.3, 0.6, (1, 4, 5, 16))
    tgt = rng.gamma(1.0, 0.5, (1, 4, 5, 3))
    tgt[0, 0, 0, 0] = -0.2  # a negative sample counts as 0
    loss, d = unet.tone_mse_loss(pred, tgt)
    assert np.all(d[..., 3:] == 0.0)
    for idx in [(0, 0, 0, 0), (0, 1, 2, 1), (0, 3, 4, 2), (0, 2, 1, 0)]:
        e = np.zeros_like(pred)
        e[idx] = 1e-6
        num = (unet.tone_mse_loss(pred + e, tgt)[0] - unet.tone_mse_loss(pred - e, tgt)[0]) / 2e-6
        assert abs(num - d[idx]) <= 1e-6 * max(1.0, abs(num)), (idx, num, d[idx])
    # the tone of the exact prediction log(1 + y) is y / (1 + y): no loss
    exact = np.zeros_like(pred)
    exact[..., :3] = np.log1p(np.maximum(tgt, 0.0))
    assert unet.tone_mse_loss(exact, tgt)[0] < 1e-30
    assert unet.tone_mse_loss(exact, tgt, display=True)[0] < 1e-30
    # the display term: the true gradient where the clamp is open (0 < x < 1)
    inner = rng.uniform(0.05, 0.65, pred.shape)
    ld, dd = unet.tone_mse_loss(inner, tgt, display=True)
    for idx in [(0, 0, 0, 0), (0, 1, 2, 1), (0, 3, 4, 2)]:
        e = np.zeros_like(inner)
        e[idx] = 1e-6
        num = (unet.tone_mse_loss(inner + e, tgt, True)[0] - unet.tone_mse_loss(inner - e, tgt, True)[0]) / 2e-6
        assert abs(num - dd[idx]) <= 1e-6 * max(1.0, abs(num)), (idx, num, dd[idx])
    # a prediction above 1 for a target below 1 is pulled down, though clamped
    hi = np.full((1, 1, 1, 16), 3.0)
    assert unet.tone_mse_loss(hi, np.full((1, 1, 1, 3), 0.5), True)[1][0, 0, 0, 0] > \
        unet.tone_mse_loss(hi, np.full((1, 1, 1, 3), 0.5))[1][0, 0, 0, 0]


# ---- the screen space ambient occlusion (ssao::ssao24), the reference's own
# tests restated (src/ssao.rs:338-417)

def test_ssao_rne_matches_round_ties_even():
    vals = [0.0, -0.0, 0.5, -0.5, 1.5, 2.5, -2.5, 8388607.5, 4194304.5, -4194303.5, 1e10, -1e10, math.inf, -math.inf]
    rng = np.random.default_rng(12345)
    bits = rng.integers(0, 2 ** 32, 20000, dtype=np.uint64).astype(np.uint32)
    f = bits.view(np.float32)
    f = np.fmod(f[np.isfinite(f)], np.float32(1e8))
    vals += [float(x) for x in f]
    for x in vals:
        want = np.rint(np.float32(x))
        got = np.float32(O.ssao_rne(x))
        assert got.tobytes() == want.tobytes(), x
    assert math.isnan(O.ssao_rne(math.nan))


def test_ssao_levels():
    assert O.ssao_levels(100, 100) == 5
    assert O.ssao_levels(6000, 6000) <= 15


def _depth_gbuf(w, h, depth):
    g = np.zeros(w * h, dtype=mb3dcu.SILIGHT)
    g["zpos_fine"] = (np.asarray(depth, np.int64).reshape(-1).astype(np.uint32) << 8)
    return g


def test_ssao_flat_plane_has_no_occlusion_and_a_pit_has():
    w = h = 64
    y, x = np.mgrid[0:h, 0:w] - 32
    pit = np.where(x * x + y * y < 36, 20000, 0)
    g = O.ssao24(_depth_gbuf(w, h, 4_000_000 - pit), w, h, 300.0, 0.001)
    center, far = int(g["amb_shadow"][32 * w + 32]), int(g["amb_shadow"][5 * w + 5])
    assert center > far + 1000, (center, far)


def test_ssao_wrapped_occlusion_turns_with_the_picture():
    """A panorama has no left or right border: the occlusion of the picture
    turned sideways by an even number of columns is the turned occlusion."""
    w, h = 96, 48

    def scene(shift):
        yy, xx = np.mgrid[0:h, 0:w]
        xs = (xx + shift) % w
        pit = ((xs - 3) ** 2 + (yy - 24) ** 2 < 30) | ((xs - 60) ** 2 + (yy - 10) ** 2 < 20)
        depth = np.where(pit, 20000, (xs * 37 % 11) * 300)
        return _depth_gbuf(w, h, 4_000_000 - depth)

    a = O.ssao24(scene(0), w, h, 300.0, 0.001, wrap_x=True)["amb_shadow"].reshape(h, w)
    k = 38
    b = O.ssao24(scene(k), w, h, 300.0, 0.001, wrap_x=True)["amb_shadow"].reshape(h, w)
    assert np.array_equal(b, np.roll(a, -k, axis=1))


def test_ssao_leaves_the_background_and_stays_in_range():
    w, h = 80, 60
    yy, xx = np.mgrid[0:h, 0:w]
    depth = 4_000_000 - ((xx * 7919 + yy * 104729) % 5000)
    g = _depth_gbuf(w, h, depth)
    g["zpos_fine"][:w * 5] = np.uint32(0xFFFFFF00)  # background rows (zpos >= 32768)
    g["amb_shadow"] = 777
    for t0 in (False, True):
        for mirror in (0.0, 0.3):
            o = O.ssao24(g, w, h, 300.0, 0.001, threshold=1.5, border_mirror=mirror, t0=t0)
            assert (o["amb_shadow"][:w * 5] == 777).all()
            assert (o["amb_shadow"][w * 5:] <= 16383).all()


def test_mc_passes_converge():
    """mc.rs's passes_converge (src/mc.rs:4197-4221) on the oracle's pass:
    the bulb at 48x36, the first pass gives every pixel 4 rays, later passes
    add rays where the picture is noisy, the painted picture is lit, and the
    thread count does not change the records."""
    import mb3dcu
    sc = scenes.preset("Integer Power", 48, 36)
    lv = mb3dcu.mc_light_default(sc)
    opts = mb3dcu.mc_opts(1, depth=3)
    recs = np.zeros(48 * 36, mb3dcu.MC_RECORD)
    O.mc_pass(sc, lv, opts, 0, recs, threads=2)
    assert (recs["ray_count"] == 4).all()
    hits = int(recs["hit"].sum())
    assert 200 < hits < 48 * 36, hits
    avg1 = recs["ray_count"].mean()
    O.mc_pass(sc, lv, opts, 1, recs, threads=2)
    O.mc_pass(sc, lv, opts, 2, recs, threads=2)
    assert recs["ray_count"].mean() > avg1
    rgb = O.mc_paint(recs["col"].copy(), mb3dcu.mc_paint_default(), (recs["ray_count"] > 0).astype(np.uint8))
    lit = int((rgb.reshape(-1, 3) > 20).any(axis=1).sum())
    assert lit > 500, lit
    a = np.zeros(48 * 36, mb3dcu.MC_RECORD)
    b = np.zeros(48 * 36, mb3dcu.MC_RECORD)
    for k in range(2):
        O.mc_pass(sc, lv, opts, k, a, threads=1)
        O.mc_pass(sc, lv, opts, k, b, threads=3)
    assert a.tobytes() == b.tobytes()


def _dof_checker(w, h):
    """dof.rs's test scene (src/dof.rs:671-685): left half near, right half
    far, a 2-pixel checker pattern."""
    import mb3dcu
    rgb = np.zeros((h, w, 3), np.uint8)
    g = np.zeros(w * h, mb3dcu.SILIGHT)
    for y in range(h):
        for x in range(w):
            v = 255 if (x // 2 + y // 2) % 2 == 0 else 0
            rgb[y, x] = v
            g[y * w + x]["zpos_fine"] = (8_000_000 if x < w // 2 else 6_000_000) << 8
    return rgb, g


def _contrast(rgb, x0, x1):
    a = rgb[1:-1, x0 + 1:x1 - 1, 0].astype(np.float64)
    b = rgb[1:-1, x0 + 2:x1, 0].astype(np.float64)
    return float(np.abs(a - b).sum())


def test_dof_focus_keeps_one_depth_sharp():
    """dof.rs's focus_keeps_one_depth_sharp (src/dof.rs:700-722) on the
    oracle's depth of field, both variants."""
    import mb3dcu
    w, h = 64, 32
    for forward in (0, 1):
        rgb, g = _dof_checker(w, h)
        before_far = _contrast(rgb, w // 2, w)
        a = (8388352 - 8_000_000) / 300.0 + 1.0
        near_z = np.float32((a * a - 1.0) / 0.001)
        o = mb3dcu.DofOpts(near_z / w, near_z / w, 0.5, 20.0, 1, forward)
        out = O.dof_raw(g, rgb, w, h, 300.0, 0.001, 30.0, o)
        near, far = _contrast(out, 4, w // 2 - 4), _contrast(out, w // 2 + 4, w)
        assert far < before_far * 0.5, (forward, far, before_far)
        assert near > far * 2.0, (forward, near, far)


def test_ssao_random_sampling_sees_the_pit_too():
    """Random sampling (SsaoParams::random, TAmbHiQCalcR) on the pit of the
    reference's flat_plane_has_no_occlusion_and_a_pit_has: the pit is
    occluded, the plane is not, and the passes' mean stays near the regular
    sampling's occlusion."""
    w = h = 64
    y, x = np.mgrid[0:h, 0:w] - 32
    pit = np.where(x * x + y * y < 36, 20000, 0)
    gb = _depth_gbuf(w, h, 4_000_000 - pit)
    reg = O.ssao24(gb, w, h, 300.0, 0.001)["amb_shadow"].astype(np.int64)
    for passes in (1, 4):
        g = O.ssao24(gb, w, h, 300.0, 0.001, random=passes)["amb_shadow"].astype(np.int64)
        center, far = int(g[32 * w + 32]), int(g[5 * w + 5])
        assert center > far + 1000, (passes, center, far)
        assert abs(center - int(reg[32 * w + 32])) < 0.25 * int(reg[32 * w + 32]), (passes, center)
    a = O.ssao24(gb, w, h, 300.0, 0.001, random=2)
    b = O.ssao24(gb, w, h, 300.0, 0.001, random=2)
    assert a.tobytes() == b.tobytes()


# ---- the older 15-bit SSAO (ssao15::ssao15), the reference's own tests
# restated (src/ssao15.rs:413-445)

def test_ssao15_arctan_buckets():
    assert O.ssao15_arctan(0, 1) == 16
    assert O.ssao15_arctan(1, 0) == 24
    assert O.ssao15_arctan(0, -1) == 0
    assert O.ssao15_arctan(-1, 0) == 8
    for y, x in [(3, 7), (-5, 2), (-1, -9), (6, -6)]:
        assert 0 <= O.ssao15_arctan(y, x) < 32
    # the buckets go round the circle once, in order, as the angle grows
    prev, turns = None, 0
    for k in range(360):
        a = np.deg2rad(k + 0.5)
        b = O.ssao15_arctan(int(round(1000 * np.sin(a))), int(round(1000 * np.cos(a))))
        if prev is not None and b < prev:
            turns += 1
        prev = b
    assert turns == 1


def test_ssao15_axis_grid():
    v = O.ssao15_axis(50, 100, 12, 2)
    assert v[0] == -12 and v[-1] == 12 and len(v) == 13
    assert O.ssao15_axis(3, 100, 12, 4)[:3] == [-3, 0, 4]
    assert O.ssao15_axis(97, 100, 12, 4)[-1] == 2


def test_ssao15_hole_is_darker_than_plane():
    w = h = 64
    yy, xx = np.mgrid[0:h, 0:w]
    d = np.sqrt((xx - 32.0) ** 2 + (yy - 32.0) ** 2)
    pit = np.where(d < 10.0, 3000.0 * (1.0 - d / 10.0), 0.0)
    g = O.ssao15(_depth_gbuf(w, h, (4_000_000.0 - pit).astype(np.int64)), w, h, 300.0, 0.001)
    center, far = int(g["amb_shadow"][32 * w + 32]), int(g["amb_shadow"][5 * w + 5])
    assert center > far, (center, far)


def test_ssao15_variants_and_background():
    """The t0 variant and the wrap change the occlusion but keep it in
    0..16383; the background keeps its record; the result does not depend
    on the number of threads."""
    w, h = 90, 70
    yy, xx = np.mgrid[0:h, 0:w]
    depth = 4_000_000 - ((xx * 7919 + yy * 104729) % 5000)
    depth[:, :7] = -1  # background columns
    g0 = _depth_gbuf(w, h, depth)
    a = O.ssao15(g0, w, h, 300.0, 0.001, threads=1)
    b = O.ssao15(g0, w, h, 300.0, 0.001, threads=5)
    assert a.tobytes() == b.tobytes()
    bg = (g0["zpos_fine"] >> 16) >= 32768
    assert bg.sum() == 7 * h and np.array_equal(a[bg], g0[bg])
    for kw in ({"t0": True}, {"wrap_x": True}, {"threshold": 0.5}):
        c = O.ssao15(g0, w, h, 300.0, 0.001, **kw)
        assert c["amb_shadow"].max() <= 16383 and not np.array_equal(c["amb_shadow"], a["amb_shadow"]), kw
    # pictures below 4 x 4 stay as they are
    small = _depth_gbuf(3, 3, np.full((3, 3), 4_000_000))
    assert O.ssao15(small, 3, 3, 300.0, 0.001).tobytes() == small.tobytes()


# ---- the interpolation hybrid, the reference's own test restated
# (tests/render.rs:179-214, interpolation_hybrid_blends_two_formulas)

def test_interpolation_hybrid_blends_two_formulas():
    """Weights 1 : 0 give the first formula alone, for the gradient DE
    (Integer Power) and the analytic one (Amazing Box): the same iteration
    counts and DEs within 1e-9; a real blend is finite and renders."""
    for a, b in (("Integer Power", "Real Power"), ("Amazing Box", "Integer Power")):
        single = scenes.preset(a, 96, 72)
        ip = scenes.interpolated(a, b, (2.0, 0.0), 96, 72)
        pos = np.array([[0.3, 0.2, -2.0], [0.7, -0.4, 0.5], [0.0, 1.5, -6.0]])
        d1, i1 = O.de_at(single, pos)
        d2, i2 = O.de_at(ip, pos)
        assert np.array_equal(i1, i2), (a, i1, i2)
        assert np.all(np.abs(d1 - d2) <= 1e-9 * np.maximum(np.abs(d1), 1e-3)), (a, d1, d2)
        blend = scenes.interpolated(a, b, (0.5, 0.5), 96, 72)
        d3, _ = O.de_at(blend, pos[1:2])
        assert np.isfinite(d3).all()
        g = O.march(blend, mb3dcu.SILIGHT)
        assert (~mb3dcu.is_background(g)).mean() > 0.01, a


def test_interpolation_needs_two_formulas_and_valid_options():
    ip = scenes.interpolated("Integer Power", "Amazing Box", (0.6, 0.4), 32, 24)
    ip.n_slots = 1
    with pytest.raises(RuntimeError):
        O.march(ip, mb3dcu.SILIGHT)


def test_quaternion_4d_rotation_turns_the_set():
    """The 4D hybrid's rotation (BuildSMatrix4, src/math.rs:176-206): zero
    angles leave the preset as it is; turning the XW plane changes it; the
    rotation matrix is orthonormal to single precision."""
    a = scenes.preset("Quaternion", 96, 72)
    g0 = O.march(a, mb3dcu.SILIGHT)
    b = scenes.preset("Quaternion", 96, 72)
    b.rot_4d[0] = 0.3
    g1 = O.march(b, mb3dcu.SILIGHT)
    assert (g0 != g1).mean() > 0.05
    c = scenes.preset("Quaternion", 96, 72)
    c.rot_4d[0] = 2 * math.pi
    assert O.march(c, mb3dcu.SILIGHT)["zpos_fine"].tobytes() == g0["zpos_fine"].tobytes() or \
        (O.march(c, mb3dcu.SILIGHT)["zpos_fine"] == g0["zpos_fine"]).mean() > 0.99


def test_interpolation_4d_with_weights_one_and_zero_is_the_first_formula():
    """doInterpolHybridPas4D (src/iteration.rs:457-464) as the reference's
    interpolation test asks of the 3D one: weights 1 : 0 of two Quaternions
    give the first alone (the 4D preset)."""
    one = scenes.interpolated("Quaternion", "Quaternion", (2.0, 0.0), 96, 72)
    one.slots[1].options[1] = 0.3
    pos = np.array([[0.3, 0.2, -0.5], [0.1, -0.4, 0.2], [0.5, 0.5, 0.5]])
    d1, i1 = O.de_at(scenes.preset("Quaternion", 96, 72), pos)
    d2, i2 = O.de_at(one, pos)
    assert np.array_equal(i1, i2)
    assert np.all(np.abs(d1 - d2) <= 1e-9 * np.maximum(np.abs(d1), 1e-3)), (d1, d2)


def test_aexion_c_matches_pascal_reference():
    """src/formulas.rs:878-911: Aexion C with its defaults (power 8, z_mul 1,
    rotate C, conditional phi, power C 8, Cz 1, mode 0) against the
    spherical reference formula, for Z and for the turned C."""
    opts = [8.0, 1.0, 1.0, 1.0, 8.0, 1.0, 0.0, 0.0]
    for x, y, z, cx, cy, cz in ((0.3, -0.4, 0.5, 0.2, 0.1, -0.3), (-0.7, 0.2, 0.1, -0.5, 0.4, 0.6),
                                (0.05, 0.9, -0.2, 0.3, -0.8, 0.1)):
        v, j = O.formula_iterate(mb3dcu.F_AEXIONC, opts, [x, y, z, 0.0], [cx, cy, cz, 0.0])
        p = 8.0
        r1 = (x * x + y * y + z * z) ** (p * 0.5)
        th = math.atan2(math.sqrt(x * x + z * z), y) * p
        ph = math.atan2(z, x) * p
        xn, yn, zn = math.cos(th) * math.cos(ph) * r1 + cx, math.cos(th) * math.sin(ph) * r1 + cy, r1 * math.sin(th) + cz
        r = math.sqrt(cx * cx + cy * cy + cz * cz)
        th2 = math.atan2(math.sqrt(cx * cx + cz * cz), cy) * 8.0
        ph2 = math.atan2(cz, cx) * 8.0
        if xn > 0.0:
            ph2 = -ph2
        jr = [math.cos(th2) * math.cos(ph2) * r, math.cos(th2) * math.sin(ph2) * r, r * math.sin(th2)]
        assert np.allclose(v[:3], [xn, yn, zn], atol=1e-9), (v, [xn, yn, zn])
        assert np.allclose(j[:3], jr, atol=1e-9), (j, jr)


# ---- DE combinations (CalcDEfull with FormulaType > 0, src/calc.rs:1365-1455)

def _grid():
    i = np.arange(8000)
    return np.stack([(i % 20) * 0.25 - 1.3, ((i // 20) % 20) * 0.14 - 1.3, (i // 400) * 0.14 - 1.3], 1)


def test_de_combination_grid_reaches_both_parts():
    """tests/render.rs:345-382 (both_parts_of_a_de_combination_use_their_
    compiled_loops): on the scene of two objects, a grid over both (the box
    stands at x = 3.2, size 0.4) has more than 1000 points near part 2, and
    more than 100 points on each side iterate 10 times or more."""
    c = _grid()
    _, its = O.de_at(scenes.two_objects("min"), c)
    far = c[:, 0] > 2.5
    assert far.sum() > 1000
    assert ((its >= 10) & ~far).sum() > 100 and ((its >= 10) & far).sum() > 100


def test_de_combination_min_and_max_are_the_two_parts():
    """min and max of one pair of parts hold the two parts' distances (each
    at least a quarter of the DE stop, calc_de_part): min + max = part 1 +
    part 2, with part 1 the bulb alone; the smooth minima lie below the min
    (src/calc.rs:1398-1430)."""
    c = _grid()[::7]
    d_min, _ = O.de_at(scenes.two_objects("min", place=False), c)
    d_max, _ = O.de_at(scenes.two_objects("max", place=False), c)
    alone = scenes.two_objects("min", place=False)
    alone.decomb = 0
    scenes.set_slots(alone, [scenes.intpow(8, -1.0)])
    alone.rstop = 1024.0  # (the combination's bailout: the largest of its formulas')
    d1, _ = O.de_at(alone, c)
    assert np.all(d_min <= d_max)
    assert np.all((np.abs(d_min - d1) <= 1e-12 * d1) | (np.abs(d_max - d1) <= 1e-12 * d1))
    d2 = d_min + d_max - d1
    assert np.all(d2 >= d_min - 1e-12) and (d2 > d1).any() and (d2 < d1).any()
    for kind in ("smooth_linear", "smooth"):
        d_s, _ = O.de_at(scenes.two_objects(kind, place=False), c)
        assert np.all(d_s <= d_min + 1e-12), kind
        assert (d_s < d_min - 1e-9).any(), kind


def test_de_combination_inverted_max_cuts_the_box_out():
    """max with the inverted part 2 (kind 3, calc_de_part's `invert`): the
    box's inside counts as outside, so the bulb's points inside the box are
    away from the surface and its points outside keep the bulb's distance."""
    c = _grid()[::5]
    d_inv, _ = O.de_at(scenes.two_objects("max_inverted", place=False), c)
    alone = scenes.two_objects("min", place=False)
    alone.decomb = 0
    scenes.set_slots(alone, [scenes.intpow(8, -1.0)])
    alone.rstop = 1024.0  # (the combination's bailout: the largest of its formulas')
    d1, _ = O.de_at(alone, c)
    assert np.all(d_inv >= d1 - 1e-12 * d1)
    assert (d_inv > d1 * 1.5).any() and (np.abs(d_inv - d1) <= 1e-12 * d1).mean() > 0.3


def test_de_combination_checks_and_interpolation_wins():
    """The checks of the second part (src/calc.rs:491-520): 'mix' needs a
    dIFS part 2, a kind beyond 6 is refused; in an interpolation hybrid the
    combination is ignored (src/calc.rs:421)."""
    bad = scenes.two_objects("min")
    bad.decomb = 6
    with pytest.raises(Exception):
        O.de_at(bad, np.zeros((1, 3)))
    bad.decomb = 7
    with pytest.raises(Exception):
        O.de_at(bad, np.zeros((1, 3)))
    ip = scenes.interpolated("Integer Power", "Amazing Box", (0.6, 0.4), 32, 24)
    c = _grid()[::40]
    d0, i0 = O.de_at(ip, c)
    ip.decomb, ip.decomb_end1, ip.decomb_start2, ip.decomb_end2 = 1, 0, 1, 1
    d1, i1 = O.de_at(ip, c)
    assert np.array_equal(d0, d1) and np.array_equal(i0, i1)
