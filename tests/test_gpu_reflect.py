"""The reflection pass's rays on the card (mb3d_cu_reflect_batch, the
counterpart of gpu::reflect_batch, src/gpu.rs:2521) against the oracle's
SrTracer::march_ray (src/reflect.rs:1464-1675) with calc_hs and deao_1pos.

The first bounce of every object pixel of the hybrid frame (the oracle's
restatement of start_pixel and step's mirror ray) and the second bounce
from those hits, marched on the card in double precision: hits, depths,
normals, colours, shadow bits and ambient occlusion against the oracle's,
per ray (the records bit for bit but for the occlusion, which takes the
card's acos and sincos in its turn to the normal).  The card's FP64 arithmetic may fuse a multiply and an add where
the oracle does not, so a ray that grazes a surface may land elsewhere; the
bounds below allow for that on a small share of rays."""
import numpy as np
import pytest

import mb3dcu
import oracle_py as O
import scenes

pytestmark = pytest.mark.gpu


def _agree(got, want):
    h_g, h_w = got["hit"] == 1, want["hit"] == 1
    both = h_g & h_w
    sg, sw = got["si"][both], want["si"][both]
    same = np.ones(len(sg), bool)
    for f in ("normal", "zpos_fine", "shadow", "si_gradient", "otrap"):
        same &= (sg[f] == sw[f]).reshape(len(sg), -1).all(axis=1)
    # (the ambient occlusion apart: its turn to the normal takes the card's acos and sincos)
    r = {"hit_agree": float((h_g == h_w).mean()), "both": int(both.sum()), "exact_si": float(same.mean())}
    zg, zw = got["zz2"][both], want["zz2"][both]
    rel = np.abs(zg - zw) / np.maximum(np.abs(zw), 1e-30)
    r["zz2_rel_median"] = float(np.median(rel))
    r["zz2_rel_p99"] = float(np.quantile(rel, 0.99))
    r["shadow_agree"] = float(((got["si"]["shadow"][both] >> 10) == (want["si"]["shadow"][both] >> 10)).mean())
    da = np.abs(got["si"]["amb_shadow"][both].astype(np.int64) - want["si"]["amb_shadow"][both].astype(np.int64))
    r["amb_within_8"] = float((da <= 8).mean())
    miss = ~h_g & ~h_w
    r["miss_steps_agree"] = float(((got["si"]["shadow"][miss] & 0x3FF) == (want["si"]["shadow"][miss] & 0x3FF)).mean())
    return r


def _check(r):
    t = str(r)
    assert r["hit_agree"] >= 0.98, t
    assert r["exact_si"] >= 0.9, t
    assert r["zz2_rel_median"] < 1e-9 and r["zz2_rel_p99"] < 1e-4, t
    assert r["shadow_agree"] >= 0.97, t
    assert r["amb_within_8"] >= 0.95, t
    assert r["miss_steps_agree"] >= 0.97, t


@pytest.fixture(scope="module")
def c2_first():
    sc = scenes.scaled(scenes.c2_hybrid(), 240, 135)
    g = O.march(sc, mb3dcu.SILIGHT)
    rays = O.reflect_first_rays(sc, g)
    assert len(rays) > 0.2 * sc.width * sc.height
    return sc, rays


def test_first_bounce_matches_oracle(card, c2_first):
    sc, rays = c2_first
    want = O.reflect_batch(sc, rays)
    got = card.reflect_batch(sc, rays)
    assert 0.2 < want["hit"].mean() < 0.95  # (both hits and open air)
    _check(_agree(got, want))


def test_second_bounce_and_far_fog(card, c2_first):
    sc, rays = c2_first
    first = O.reflect_batch(sc, rays)
    idx = np.nonzero(first["hit"] == 1)[0]
    vg = np.ctypeslib.as_array(sc.vgrads).astype(np.float64).reshape(3, 3)
    nrm = first["si"]["normal"][idx].astype(np.float64) / 32767.0 @ vg
    d = rays["dir"][idx]
    k = 2.0 * (nrm * d).sum(1) / np.maximum((nrm * nrm).sum(1), 1e-300)
    r2 = np.zeros(len(idx), mb3dcu.REFLECT_RAY)
    r2["origin"] = first["pos"][idx]
    r2["dir"] = d - nrm * k[:, None]
    r2["zz"] = first["zz"][idx]
    r2["pixel"] = rays["pixel"][idx]
    r2["rit"] = 2
    for far_fog in (False, True):
        want = O.reflect_batch(sc, r2, far_fog=far_fog)
        got = card.reflect_batch(sc, r2, far_fog=far_fog)
        _check(_agree(got, want))
    # a limited march length ends rays in the open air
    r3 = r2.copy()
    r3["max_len"] = 2.0
    want, got = O.reflect_batch(sc, r3), card.reflect_batch(sc, r3)
    assert want["hit"].mean() < O.reflect_batch(sc, r2)["hit"].mean()
    _check(_agree(got, want))


def test_soft_shadow_and_no_occlusion(card, c2_first):
    sc, rays = c2_first
    soft = scenes.scene_copy(sc)
    soft.shadow_soft, soft.soft_radius = 1, 2.0
    soft.deao_quality = -1
    want, got = O.reflect_batch(soft, rays), card.reflect_batch(soft, rays)
    _check(_agree(got, want))
    hit = want["hit"] == 1
    assert np.all(want["si"]["amb_shadow"][hit] == 5000) and np.all(got["si"]["amb_shadow"][got["hit"] == 1] == 5000)
    # the soft shadow's 6 bits take more than two values
    assert len(np.unique(want["si"]["shadow"][hit] >> 10)) > 4


def test_device_buffers_and_refusals(card, c2_first):
    import torch
    sc, rays = c2_first
    host = card.reflect_batch(sc, rays[:500])
    dr = torch.from_numpy(rays[:500].view(np.uint8).copy()).cuda()
    dh = torch.zeros(500 * mb3dcu.REFLECT_HIT.itemsize, dtype=torch.uint8, device="cuda")
    card.reflect_batch(sc, dr, out=dh)
    torch.cuda.synchronize()
    assert dh.cpu().numpy().tobytes() == host.tobytes()
    bad = rays[:4].copy()
    bad["pixel"][2] = sc.width * sc.height
    with pytest.raises(mb3dcu.CardError) as e:
        card.reflect_batch(sc, bad)
    assert e.value.status == mb3dcu.EINVAL
    rnd = scenes.scene_copy(sc)
    rnd.deao_first_step_random = 1
    with pytest.raises(mb3dcu.CardError) as e:
        card.reflect_batch(rnd, rays[:4])
    assert e.value.status == mb3dcu.ENOTSUP
    assert len(card.reflect_batch(sc, rays[:0])) == 0


def test_first_rays_on_the_card(card, c2_first):
    """mb3d_cu_reflect_first_rays against the oracle's start_pixel + mirror
    ray: the same pixels send rays (in pixel order), their origins and
    directions agree to the FP64 surface search's last bits, and the card's
    batch over the card's rays agrees with the oracle's over the oracle's."""
    import torch
    sc, want = c2_first
    g = O.march(sc, mb3dcu.SILIGHT)
    got = card.reflect_first_rays(sc, g)
    common = np.intersect1d(got["pixel"], want["pixel"])
    assert len(common) >= 0.999 * max(len(got), len(want)), (len(got), len(want), len(common))
    assert np.all(np.diff(got["pixel"].astype(np.int64)) > 0)
    a = got[np.isin(got["pixel"], common)]
    b = want[np.isin(want["pixel"], common)]
    rel = np.abs(a["zz"] - b["zz"]) / np.maximum(np.abs(b["zz"]), 1e-30)
    assert np.median(rel) < 1e-12 and np.quantile(rel, 0.99) < 1e-6, (np.median(rel), np.quantile(rel, 0.99))
    assert np.abs(a["dir"] - b["dir"]).max() < 1e-6 * np.abs(b["dir"]).max()
    _check(_agree(card.reflect_batch(sc, a), O.reflect_batch(sc, b)))
    # device buffers
    gd = torch.from_numpy(g.view(np.uint8).copy()).cuda()
    out = torch.zeros(sc.width * sc.height * mb3dcu.REFLECT_RAY.itemsize, dtype=torch.uint8, device="cuda")
    out, n = card.reflect_first_rays(sc, gd, out=out)
    torch.cuda.synchronize()
    assert n == len(got) and out[:n * mb3dcu.REFLECT_RAY.itemsize].cpu().numpy().tobytes() == got.tobytes()
