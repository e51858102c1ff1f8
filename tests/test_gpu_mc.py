"""The Monte Carlo tracer on the card against the Monte Carlo oracle.

mb3d_cu_mc_batch is the drop-in for gpu::mc_batch (src/gpu.rs:3022): the
marches of McMarch::run.  In double precision its results agree with the
oracle's up to the last bits of the device's log/sin/cos and of fused
multiply-adds; a march whose step lands a last-bit differently may end a
step apart, so the tests hold the share of identical outcomes, not all.

mb3d_cu_mc_render traces Tracer::ray whole on the card.  In double
precision each ray follows the oracle's ray (the same random numbers), so
most pixels carry the oracle's light to single precision; a few rays part
on a grazing step and take another path, which moves their pixel by up to
that ray's share.  The mixed mode (single precision DE) is an unbiased
variant of the same estimator: held to the oracle by the picture's mean
and by its noise.
"""
import ctypes
import os  # noqa: F401

import numpy as np
import pytest

import mb3dcu
import oracle_py as O
import scenes

pytestmark = pytest.mark.gpu


def _primary_requests(sc, n, seed=7):
    """Primary rays of random pixels as McReq (kind 0, probe) and the
    shadow requests toward the first light from their surfaces."""
    rng = np.random.default_rng(seed)
    p = O.params(sc)
    sw = p[9]
    reqs = (mb3dcu.McReq * n)()
    xs = rng.integers(0, sc.width, n)
    ys = rng.integers(0, sc.height, n)
    # the camera: the view vector of the pixel centre, as the march's
    vg = np.array(sc.vgrads)
    vg = vg / np.linalg.norm(vg, axis=1, keepdims=True) * sw
    ystart = np.array(p[10:13])
    fov = np.deg2rad(sc.fov_y)
    for i in range(n):
        x, y = int(xs[i]), int(ys[i])
        cafy = (y / sc.height - 0.5) * fov
        cafx = (p[21] - (x + 1.0)) * p[22]
        v = np.array([-np.sin(cafx), np.sin(cafy), np.cos(cafy) * np.cos(cafx)])
        v /= np.linalg.norm(v)
        d = v @ vg
        pos = ystart + vg[1] * y + vg[0] * x
        r = reqs[i]
        r.pos[:] = pos
        r.dir[:] = d
        r.zz, r.zz2, r.zzplus, r.len = 0.0, 0.0, 1.0, p[8]
        r.seed = int(rng.integers(-2 ** 31, 2 ** 31))
        r.kind, r.probe = 0, 1
    return reqs


def _arr(res):
    return {k: np.array([getattr(r, k) if not hasattr(getattr(r, k), "__len__") else list(getattr(r, k)) for r in res])
            for k in ("pos", "normals", "zz", "zz2", "len", "seed", "si_grad", "kind", "de_limited", "ms_de_stop")}


def test_mc_batch_fp64_matches_oracle(card):
    sc = scenes.scaled(scenes.c2_hybrid(), 320, 180)
    reqs = _primary_requests(sc, 4000)
    for secant in (True, False):
        a = _arr(O.mc_batch(sc, reqs, secant=secant))
        b = _arr(card.mc_batch(sc, reqs, mb3dcu.FP64, secant=secant))
        assert (a["kind"] == b["kind"]).mean() >= 0.999, secant
        hit = (a["kind"] == 1) & (b["kind"] == 1)
        assert hit.sum() > 500
        same = np.all(np.abs(a["pos"] - b["pos"]) <= 1e-9 * np.abs(a["pos"]).max(), axis=1)
        assert same[hit].mean() >= 0.99, (secant, same[hit].mean())
        assert (a["seed"] == b["seed"]).mean() >= 0.99
        assert (np.abs(a["si_grad"].astype(int) - b["si_grad"].astype(int)) <= 1)[hit].mean() >= 0.99
        cos = np.sum(a["normals"] * b["normals"], axis=1)
        assert (cos > 0.9999)[hit].mean() >= 0.98, np.mean(cos[hit])
    # shadow marches toward the light from the surfaces just found
    lv = mb3dcu.mc_light_default(sc)
    p = O.params(sc)
    sw = p[9]
    hits = [i for i in range(len(reqs)) if a["kind"][i] == 1][:1500]
    sreq = (mb3dcu.McReq * len(hits))()
    ln = np.array(lv.ln[0], dtype=np.float64)
    vg = np.array(sc.vgrads)
    vg = vg / np.linalg.norm(vg, axis=1, keepdims=True)
    toward = -(-ln / np.linalg.norm(ln) * sw) @ vg
    for j, i in enumerate(hits):
        r = sreq[j]
        r.pos[:] = a["pos"][i]
        r.dir[:] = toward
        r.zz, r.zz2, r.zzplus, r.len = abs(a["zz"][i]), a["zz"][i], 0.5, 2000.0
        r.seed, r.kind = 12345, 1
    a2 = _arr(O.mc_batch(sc, sreq))
    for prec in (mb3dcu.FP64, mb3dcu.FP32_FP64):
        b2 = _arr(card.mc_batch(sc, sreq, prec))
        lit_a, lit_b = a2["len"] <= 0.01, b2["len"] <= 0.01
        agree = (lit_a == lit_b).mean()
        assert agree >= (0.995 if prec == mb3dcu.FP64 else 0.98), (prec, agree)
        if prec == mb3dcu.FP64:
            rel = np.abs(a2["len"] - b2["len"]) / np.maximum(np.abs(a2["len"]), 1.0)
            assert (rel < 1e-6).mean() >= 0.99


def test_mc_render_fp64_matches_oracle(card):
    sc = scenes.scaled(scenes.c2_hybrid(), 160, 90)
    lv = mb3dcu.mc_light_default(sc)
    opts = mb3dcu.mc_opts(8, depth=3)
    ref = O.mc_render(sc, lv, opts)
    got = card.mc_render(sc, opts, lv, mb3dcu.FP64)
    assert ref["inside"] == 0 and card.stats()["mc_inside_rays"] == 0
    assert (ref["hit"] == got["hit"]).mean() >= 0.999
    a, b = ref["radiance"], got["radiance"].astype(np.float64)
    scale = a.max()
    close = np.all(np.abs(a - b) <= 1e-5 * scale, axis=2)
    assert close.mean() >= 0.97, close.mean()
    # a parted ray moves its pixel by at most its share of the light
    assert np.abs(a - b).max() <= 400.0 / 8 + 1e-6
    assert abs(a.mean() - b.mean()) <= 2e-3 * a.mean()
    hit = (ref["depth"] > 0) & (got["depth"] > 0)
    assert hit.mean() > 0.1
    assert (np.abs(ref["depth"] - got["depth"]) <= 1e-6 * np.abs(ref["depth"]).max())[hit].mean() >= 0.99
    assert (np.abs(ref["albedo"] - got["albedo"]).max(axis=2) <= 1e-6)[hit].mean() >= 0.99
    assert (np.sum(ref["normal"] * got["normal"], axis=2) > 0.9999)[hit].mean() >= 0.98


def test_mc_render_mixed_is_the_same_estimator(card):
    sc = scenes.scaled(scenes.c2_hybrid(), 160, 90)
    lv = mb3dcu.mc_light_default(sc)
    opts = mb3dcu.mc_opts(32, depth=3)
    a = card.mc_render(sc, opts, lv, mb3dcu.FP64)["radiance"].astype(np.float64)
    b = card.mc_render(sc, opts, lv, mb3dcu.FP32_FP64)["radiance"].astype(np.float64)
    # the same picture up to noise: the means agree, and the difference is
    # far below the picture's own contrast
    assert abs(a.mean() - b.mean()) <= 0.01 * a.mean()
    mse = np.mean((a - b) ** 2)
    psnr = 10 * np.log10(a.max() ** 2 / mse)
    assert psnr > 30.0, psnr


def test_mc_render_is_deterministic_and_splits(card):
    import torch
    sc = scenes.scaled(scenes.c2_hybrid(), 128, 72)
    lv = mb3dcu.mc_light_default(sc)
    whole = card.mc_render(sc, mb3dcu.mc_opts(8), lv)
    again = card.mc_render(sc, mb3dcu.mc_opts(8), lv)
    assert whole["radiance"].tobytes() == again["radiance"].tobytes()
    h1 = card.mc_render(sc, mb3dcu.mc_opts(4, ray0=0), lv)["radiance"].astype(np.float64)
    h2 = card.mc_render(sc, mb3dcu.mc_opts(4, ray0=4), lv)["radiance"].astype(np.float64)
    assert np.abs((h1 + h2) / 2 - whole["radiance"]).max() <= 1e-5 * whole["radiance"].max()
    # a rectangle equals that part of the whole picture
    part = card.mc_render(sc, mb3dcu.mc_opts(8, rect=(16, 8, 40, 24)), lv)
    assert part["radiance"].tobytes() == whole["radiance"][8:32, 16:56].copy().tobytes()
    # device buffers give the host buffers' values
    dev = {"radiance": torch.zeros((72, 128, 3), dtype=torch.float32, device="cuda"),
           "hit": torch.zeros((72, 128), dtype=torch.uint8, device="cuda")}
    got = card.mc_render(sc, mb3dcu.mc_opts(8), lv, out=dev)
    torch.cuda.synchronize()
    assert got["radiance"].cpu().numpy().tobytes() == whole["radiance"].tobytes()
    assert np.array_equal(got["hit"].cpu().numpy(), whole["hit"])


def test_mc_errors(card):
    sc = scenes.scaled(scenes.c2_hybrid(), 64, 36)
    lv = mb3dcu.mc_light_default(sc)
    with pytest.raises(mb3dcu.CardError) as e:
        card.mc_render(sc, mb3dcu.mc_opts(0), lv)
    assert e.value.status == mb3dcu.EINVAL
    with pytest.raises(mb3dcu.CardError) as e:
        card.mc_render(sc, mb3dcu.mc_opts(2, rect=(60, 0, 10, 10)), lv)
    assert e.value.status == mb3dcu.EINVAL
    reqs = (mb3dcu.McReq * 1)()
    reqs[0].kind = 2
    with pytest.raises(mb3dcu.CardError) as e:
        card.mc_batch(sc, reqs)
    assert e.value.status == mb3dcu.ENOTSUP
    flag = ctypes.c_int(1)
    with pytest.raises(mb3dcu.CardError) as e:
        card.mc_render(sc, mb3dcu.mc_opts(2), lv, cancel=flag)
    assert e.value.status == mb3dcu.ECANCELED


def test_mc_paint_matches_oracle(card):
    """paint_recs on the card against the oracle's: HDR and negative colours,
    the soft clip, both gamma curves, saturation, pixels without rays, host
    and device buffers.  The same single precision arithmetic, unfused on
    both sides; cube roots may differ in the last bit, which moves a byte by
    at most one."""
    import torch
    rng = np.random.default_rng(21)
    c = np.concatenate([rng.uniform(-0.3, 1.5, (30000, 3)), rng.gamma(0.7, 3.0, (10000, 3))]).astype(np.float32)
    rays = (rng.uniform(size=len(c)) > 0.05).astype(np.uint8)
    settings = []
    for contrast, sat, options, gamma in ((128, 32, 2, 32.0), (200, 40, 3, 32.0), (128, 32, 2, 63.0),
                                          (90, 32, 2, 0.0), (128, 64, 1, 50.0)):
        o = mb3dcu.mc_paint_default()
        o.contrast, o.saturation, o.options, o.gamma = contrast, sat, options, gamma
        settings.append(o)
    for o in settings:
        want = O.mc_paint(c, o, rays).astype(int)
        got = card.mc_paint(c, o, rays).astype(int)
        assert np.abs(got - want).max() <= 1, (o.contrast, o.options, o.gamma)
        assert (got == want).mean() >= 0.999, (o.contrast, o.options, o.gamma)
    # device buffers (torch), no ray mask
    o = settings[1]
    dc = torch.from_numpy(c).cuda()
    dout = torch.zeros((len(c), 3), dtype=torch.uint8, device="cuda")
    card.mc_paint(dc, o, None, out=dout)
    want = O.mc_paint(c, o).astype(int)
    assert np.abs(dout.cpu().numpy().astype(int) - want).max() <= 1


def test_split_render_equals_one_kernel_render(card, monkeypatch):
    """The split render (logic kernel + list-fed march kernel, the default)
    traces the same rays as the one-kernel form: in double precision the
    same records.  In the mixed mode the single precision DE is compiled
    into two different kernels, where the code generator may fuse its
    multiplies and adds differently: the last bits of a ray's positions,
    and with them of most pixels' light, differ (as they do against the
    oracle), and a grazing ray can part.  There the two are held to the same
    picture."""
    sc = scenes.scaled(scenes.c2_hybrid(), 160, 90)
    lv = mb3dcu.mc_light_default(sc)
    for prec in (mb3dcu.FP64, mb3dcu.FP32_FP64):
        split = card.mc_render(sc, mb3dcu.mc_opts(8, depth=4), lv, prec)
        monkeypatch.setenv("MB3D_CU_MC_MEGA", "1")
        one = card.mc_render(sc, mb3dcu.mc_opts(8, depth=4), lv, prec)
        monkeypatch.delenv("MB3D_CU_MC_MEGA")
        if prec == mb3dcu.FP64:
            for k in ("radiance", "albedo", "normal", "depth", "hit"):
                assert split[k].tobytes() == one[k].tobytes(), (prec, k)
        else:
            assert (split["hit"] == one["hit"]).mean() >= 0.999
            a = split["radiance"].astype(np.float64)
            b = one["radiance"].astype(np.float64)
            assert abs(a.mean() - b.mean()) <= 0.01 * a.mean()
            psnr = 10 * np.log10(a.max() ** 2 / max(float(np.mean((a - b) ** 2)), 1e-30))
            assert psnr > 30.0, psnr


def test_adaptive_pass_fp64_matches_oracle(card):
    """mb3d_cu_mc_pass (mc::pass with calc_n and the per-pixel rounds)
    against the oracle's pass on the same records: the first pass gives every
    pixel 4 rays; the second, from the same records on both sides, the same
    ray counts (calc_n and the rounds' noise test decide alike) and the same
    records up to the rays that part on a grazing step."""
    sc = scenes.scaled(scenes.c2_hybrid(), 96, 54)
    lv = mb3dcu.mc_light_default(sc)
    opts = mb3dcu.mc_opts(1, depth=3)
    n = sc.width * sc.height
    a = card.mc_pass(sc, opts, np.zeros(n, mb3dcu.MC_RECORD), 0, lv, mb3dcu.FP64)
    b = O.mc_pass(sc, lv, opts, 0, np.zeros(n, mb3dcu.MC_RECORD))
    assert (a["ray_count"] == 4).all() and (b["ray_count"] == 4).all()
    assert (a["hit"] == b["hit"]).mean() >= 0.99
    scale = float(np.abs(b["col"]).max())
    close = np.all(np.abs(a["col"] - b["col"]) <= 1e-5 * scale, axis=1)
    assert close.mean() >= 0.97, close.mean()
    # the second pass from the oracle's records on both sides
    a2 = card.mc_pass(sc, opts, b.copy(), 1, lv, mb3dcu.FP64)
    b2 = O.mc_pass(sc, lv, opts, 1, b.copy())
    assert b2["ray_count"].mean() > 4.5
    same = (a2["ray_count"] == b2["ray_count"]).mean()
    assert same >= 0.97, same
    close = np.all(np.abs(a2["col"] - b2["col"]) <= 1e-4 * scale, axis=1)
    assert close.mean() >= 0.95, close.mean()
    assert abs(float(a2["ray_count"].sum()) - float(b2["ray_count"].sum())) <= 0.01 * float(b2["ray_count"].sum())


def test_adaptive_passes_converge_on_the_card(card):
    """The reference's passes_converge (src/mc.rs:4197-4221) on the card in
    the mixed mode, with the records in device memory for the later passes."""
    import torch
    sc = scenes.preset("Integer Power", 48, 36)
    lv = mb3dcu.mc_light_default(sc)
    opts = mb3dcu.mc_opts(1, depth=3)
    recs = card.mc_pass(sc, opts, np.zeros(48 * 36, mb3dcu.MC_RECORD), 0, lv)
    assert (recs["ray_count"] == 4).all()
    assert 200 < int(recs["hit"].sum()) < 48 * 36
    avg1 = recs["ray_count"].mean()
    dev = torch.from_numpy(recs.view(np.uint8).copy()).cuda()
    for k in (1, 2):
        card.mc_pass(sc, opts, dev, k, lv)
    torch.cuda.synchronize()
    out = np.frombuffer(dev.cpu().numpy().tobytes(), dtype=mb3dcu.MC_RECORD)
    assert out["ray_count"].mean() > avg1
    host = recs.copy()
    for k in (1, 2):
        card.mc_pass(sc, opts, host, k, lv)
    assert host.tobytes() == out.tobytes()  # (device and host records: the same passes)
