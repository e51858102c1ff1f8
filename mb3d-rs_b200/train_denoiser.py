"""Trains the Monte Carlo denoiser on pictures the card's path tracer renders
and evaluates it on the 1920x1080 Monte Carlo workload.

    python mb3d-rs_b200/train_denoiser.py train --crops 2000 --steps 6000
    python mb3d-rs_b200/train_denoiser.py eval

Training data: `--crops` seeded random scenes (scenes.random_training_scene)
rendered at 256x256: the 4- and 16-ray pictures (rays 0..15) with their
first surfaces' albedo, normal and depth, and an independent target of
`--target-rays` rays (rays 16..); all kept in device memory.  Training:
Adam on random 128x128 pieces (flipped and turned at random), the input
taken at 4 or 16 rays, the loss `--loss` (mb3d_cu_dn_set_loss: the L1 loss
in log space, the squared error of x / (1 + x), or that plus the squared
error of the colour clamped to 0..1 that the default painter shows;
mb3d_cu_dn_train_step: forward and backward on the card's own BF16
convolution kernels), a cosine learning rate.  Of several learning rates and
losses the network with the best held-out PSNR of the clamped colour is
kept.  The weights go to weights/denoiser.f32 (FP32, little endian, the
library's parameter order).
"""
import argparse
import json
import math
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import mb3dcu  # noqa: E402
import scenes  # noqa: E402

WEIGHTS = os.path.join(HERE, "weights", "denoiser.f32")


def _torch():
    import torch
    return torch


def render_set(card, sc, rays, ray0, depth, torch, with_aov, rect=None):
    """mc_render into device tensors."""
    w, h = (rect[2], rect[3]) if rect else (sc.width, sc.height)
    out = {"radiance": torch.zeros((h, w, 3), dtype=torch.float32, device="cuda"),
           "hit": torch.zeros((h, w), dtype=torch.uint8, device="cuda")}
    if with_aov:
        for k, shp in (("albedo", (h, w, 3)), ("normal", (h, w, 3)), ("depth", (h, w))):
            out[k] = torch.zeros(shp, dtype=torch.float32, device="cuda")
    else:
        out["albedo"] = out["normal"] = out["depth"] = None
    lv = mb3dcu.mc_light_default(sc)
    card.mc_render(sc, mb3dcu.mc_opts(rays, depth=depth, ray0=ray0, rect=rect), lv, mb3dcu.FP32_FP64, out=out)
    return out


def make_dataset(card, n_crops, target_rays, depth, size=256, seed=scenes.TRAIN_SEED, log=print):
    torch = _torch()
    data = {k: torch.zeros((n_crops, size, size, c), dtype=torch.float32, device="cuda")
            for k, c in (("r4", 3), ("r16", 3), ("alb", 3), ("nrm", 3), ("dep", 1), ("tgt", 3))}
    t0 = time.time()
    s = seed
    i = 0
    skipped = 0
    while i < n_crops:
        s += 1
        sc = scenes.random_training_scene(s, size, size)
        a = render_set(card, sc, 4, 0, depth, torch, True)
        hit = a["hit"].float().mean().item()
        if hit < 0.03 or card.stats()["mc_inside_rays"] > 0.01 * size * size * 4:
            skipped += 1
            continue
        b = render_set(card, sc, 12, 4, depth, torch, False)
        t = render_set(card, sc, target_rays, 16, depth, torch, False)
        data["r4"][i] = a["radiance"]
        data["r16"][i] = (a["radiance"] * 4 + b["radiance"] * 12) / 16
        data["alb"][i] = torch.nan_to_num(a["albedo"], 0.0, 0.0, 0.0)
        data["nrm"][i] = torch.nan_to_num(a["normal"], 0.0, 0.0, 0.0)
        d = torch.nan_to_num(a["depth"], 0.0, 0.0, 0.0)
        dmax = d.max()
        data["dep"][i, ..., 0] = d / dmax if dmax > 0 else d
        data["tgt"][i] = t["radiance"]
        i += 1
        if i % 200 == 0:
            log(f"  {i} crops, {time.time() - t0:.0f} s, skipped {skipped}", flush=True)
    torch.cuda.synchronize()
    return data, time.time() - t0, skipped


LOSSES = {"l1": mb3dcu.Denoiser.LOSS_L1_LOG, "tone": mb3dcu.Denoiser.LOSS_TONE_MSE,
          "display": mb3dcu.Denoiser.LOSS_TONE_DISPLAY}


def train(card, data, steps, batch=8, piece=128, lr_max=2e-3, seed=1, loss="l1", log=print):
    torch = _torch()
    dn = mb3dcu.Denoiser(card, seed=seed)
    dn.set_loss(LOSSES[loss])
    g = torch.Generator(device="cuda")
    g.manual_seed(seed)
    n, size = data["r4"].shape[0], data["r4"].shape[1]
    t0 = time.time()
    losses = []
    for step in range(steps):
        idx = torch.randint(0, n, (batch,), device="cuda", generator=g)
        oy, ox = (int(v) for v in torch.randint(0, size - piece + 1, (2,), generator=g, device="cuda"))
        sel = lambda k: data[k][idx, oy:oy + piece, ox:ox + piece]
        use16 = (torch.rand((batch, 1, 1, 1), device="cuda", generator=g) < 0.5).float()
        rad = sel("r4") * (1 - use16) + sel("r16") * use16
        alb, nrm, dep, tgt = sel("alb"), sel("nrm"), sel("dep"), sel("tgt")
        flip = int(torch.randint(0, 8, (1,), generator=g, device="cuda"))

        def aug(t):
            if flip & 1:
                t = t.flip(1)
            if flip & 2:
                t = t.flip(2)
            if flip & 4:
                t = t.transpose(1, 2)
            return t.contiguous()

        rad, alb, nrm, dep, tgt = (aug(t) for t in (rad, alb, nrm, dep, tgt))
        warm = min(1.0, (step + 1) / 200)
        lr = lr_max * warm * 0.5 * (1 + math.cos(math.pi * step / steps))
        loss = dn.train_step(rad, tgt, alb, nrm, dep[..., 0].contiguous(), depth_scale=1.0, lr=max(lr, 1e-6))
        losses.append(loss)
        if (step + 1) % 500 == 0:
            log(f"  step {step + 1}: loss {np.mean(losses[-500:]):.5f} ({time.time() - t0:.0f} s)", flush=True)
    torch.cuda.synchronize()
    return dn, time.time() - t0, losses


def val_scores(dn, data, lo, hi):
    """The denoised held-out pictures (4 and 16 rays) against their targets:
    the L1 loss in log space, and the PSNRs of x / (1 + x) and of the colour
    clamped to 0..1, per ray count."""
    torch = _torch()
    l1, se = [], {k: [[], []] for k in ("r4", "r16")}
    for i in range(lo, hi, 8):
        j = min(i + 8, hi)
        tgt = data["tgt"][i:j].clamp(min=0)
        for k in ("r4", "r16"):
            den = dn.denoise(data[k][i:j].contiguous(), data["alb"][i:j].contiguous(), data["nrm"][i:j].contiguous(),
                             data["dep"][i:j, ..., 0].contiguous(), depth_scale=1.0)
            l1.append(float((torch.log1p(den) - torch.log1p(tgt)).abs().mean()))
            se[k][0].append(float(((den / (1 + den) - tgt / (1 + tgt)) ** 2).mean()))
            se[k][1].append(float(((den.clamp(max=1) - tgt.clamp(max=1)) ** 2).mean()))
    out = {"l1_log": float(np.mean(l1))}
    for k in se:
        out[f"psnr_tone_{k}"] = 10 * math.log10(1 / max(np.mean(se[k][0]), 1e-20))
        out[f"psnr_clamp_{k}"] = 10 * math.log10(1 / max(np.mean(se[k][1]), 1e-20))
    out["psnr_clamp"] = 0.5 * (out["psnr_clamp_r4"] + out["psnr_clamp_r16"])
    return out


def tonemap(x):
    return x / (1.0 + x)


def psnr(a, ref):
    """PSNR of two radiance pictures after x / (1 + x) (both in 0..1)."""
    mse = float(np.mean((tonemap(np.maximum(a, 0)) - tonemap(np.maximum(ref, 0))) ** 2))
    return 10.0 * math.log10(1.0 / max(mse, 1e-20))


def evaluate(card, dn, rect=None, ref_rays=1024, levels=(4, 8, 16, 32, 64), log=print):
    """The 1920x1080 Monte Carlo workload (the whole frame, or a rectangle
    (x, y, w, h)): the plain trace at ref_rays, and per ray count the method:
    two traces of half the rays each (their mean is the plain trace of all
    the rays), the denoised picture of their mean, the plain trace kept where
    the denoised picture leaves it (mb3d_cu_dn_fallback, 16x16 pieces, 3
    sigma); times on the card.  PSNRs of the tone-mapped linear records
    (psnr_*) and of the 8-bit pictures the reference's painter makes of them
    (psnr8_*, paint_recs with the default display settings, on the card)."""
    torch = _torch()
    sc = scenes.c5_mc()
    lv = mb3dcu.mc_light_default(sc)

    def trace(rays, ray0=0):
        o = mb3dcu.mc_opts(rays, depth=scenes.C5_DEPTH, ray0=ray0, rect=rect)
        r = card.mc_render(sc, o, lv, mb3dcu.FP32_FP64)
        return r, card.stats()["ms_total"]

    ref, ms_ref = trace(ref_rays, ray0=4096)  # (rays of their own, each with its own Halton record (< 65536))
    st = card.stats()
    area = list(rect) if rect else [0, 0, sc.width, sc.height]
    res = {"rect": area, "ref_rays": ref_rays, "ms_ref": ms_ref,
           "mpaths_per_s": area[2] * area[3] * ref_rays / ms_ref / 1e3, "de_evals_per_s": st["de_evals"] / ms_ref * 1e3,
           "levels": []}
    paint_opts = mb3dcu.mc_paint_default()
    ref8 = card.mc_paint(ref["radiance"], paint_opts).astype(np.float64)

    def psnr8(x):
        mse = float(np.mean((card.mc_paint(x, paint_opts).astype(np.float64) - ref8) ** 2))
        return 10.0 * math.log10(255.0 ** 2 / max(mse, 1e-12))

    for rays in levels:
        half = rays // 2
        ha, ms_a = trace(half, 0)
        hb, ms_b = trace(half, half)
        dmax = float(ha["depth"].max()) or 1.0
        a, b = (torch.from_numpy(v["radiance"]).cuda() for v in (ha, hb))
        alb = torch.from_numpy(ha["albedo"]).cuda()[None]
        nrm = torch.from_numpy(ha["normal"]).cuda()[None]
        dp = torch.from_numpy(ha["depth"]).cuda()[None]
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        for it in range(2):  # (the first round warms)
            ev[0].record()
            noisy = 0.5 * (a + b)
            den = dn.denoise(noisy[None], alb, nrm, dp, depth_scale=1.0 / dmax)[0]
            ev[1].record()
            comp, fb = dn.fallback(a, b, den, tile=16, k=3.0)
            ev[2].record()
            torch.cuda.synchronize()
        ms_dn, ms_fb = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
        noisy, den, comp = (v.cpu().numpy() for v in (noisy, den, comp))
        ms = ms_a + ms_b
        lvl = {"rays": rays, "ms_trace": ms, "ms_denoise": ms_dn, "ms_fallback": ms_fb,
               "psnr_noisy": psnr(noisy, ref["radiance"]), "psnr_denoised": psnr(den, ref["radiance"]),
               "psnr_with_fallback": psnr(comp, ref["radiance"]), "fallback_rate": fb, "psnr8_noisy": psnr8(noisy),
               "psnr8_denoised": psnr8(den), "psnr8_with_fallback": psnr8(comp)}
        res["levels"].append(lvl)
        log(f"  {rays} rays: trace {ms:.1f} ms, denoise {ms_dn:.2f} ms, fallback {ms_fb:.2f} ms, PSNR noisy "
            f"{lvl['psnr_noisy']:.2f} denoised {lvl['psnr_denoised']:.2f} (fallback {fb:.3f}: "
            f"{lvl['psnr_with_fallback']:.2f}); 8-bit noisy {lvl['psnr8_noisy']:.2f} denoised "
            f"{lvl['psnr8_denoised']:.2f} (with fallback {lvl['psnr8_with_fallback']:.2f})", flush=True)
    for lv_ in res["levels"]:
        lv_["ms_method"] = lv_["ms_trace"] + lv_["ms_denoise"] + lv_["ms_fallback"]
        lv_["time_ratio_vs_ref"] = lv_["ms_method"] / ms_ref
    ok = [lv_ for lv_ in res["levels"] if lv_["psnr_with_fallback"] >= 35.0]
    if ok:
        best = min(ok, key=lambda l: l["ms_method"])
        res["time_to_35db_ms"] = best["ms_method"]
        res["time_to_35db_rays"] = best["rays"]
        res["time_ratio_vs_ref"] = best["ms_method"] / ms_ref
    plain = [lv_ for lv_ in res["levels"] if lv_["psnr_noisy"] >= 35.0]
    if plain:
        res["plain_to_35db_rays"] = min(l["rays"] for l in plain)
    ok8 = [lv_ for lv_ in res["levels"] if lv_["psnr8_with_fallback"] >= 35.0]
    if ok8:
        best = min(ok8, key=lambda l: l["ms_method"])
        res["time_to_35db_8bit_ms"] = best["ms_method"]
        res["time_to_35db_8bit_rays"] = best["rays"]
        res["time_ratio_8bit_vs_ref"] = best["ms_method"] / ms_ref
    plain8 = [lv_ for lv_ in res["levels"] if lv_["psnr8_noisy"] >= 35.0]
    if plain8:
        res["plain_to_35db_8bit_rays"] = min(l["rays"] for l in plain8)
    return res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("what", choices=["train", "eval"])
    ap.add_argument("--crops", type=int, default=2000)
    ap.add_argument("--target-rays", type=int, default=64)
    ap.add_argument("--steps", type=int, default=6000)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, nargs="+", default=[2e-3])
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--report", default=None)
    ap.add_argument("--ref-rays", type=int, default=1024)
    ap.add_argument("--loss", nargs="+", choices=sorted(LOSSES), default=["display"])
    ap.add_argument("--rect", type=int, nargs=4, default=None, help="x y w h (default: the whole frame)")
    a = ap.parse_args()
    card = mb3dcu.Card(0)
    report = {}
    if a.what == "train":
        n_val = max(8, a.crops // 25)
        data, t_data, skipped = make_dataset(card, a.crops + n_val, a.target_rays, scenes.C5_DEPTH)
        print(f"dataset: {a.crops} + {n_val} held-out crops in {t_data:.0f} s ({skipped} empty scenes skipped)",
              flush=True)
        train_part = {k: v[:a.crops] for k, v in data.items()}
        best = None
        runs = []
        if os.path.exists(a.out):
            # the weights there now stay unless a new network beats them on the held-out pictures
            prev = mb3dcu.Denoiser(card)
            prev.set_params(np.fromfile(a.out, "<f4"))
            report["previous_weights_held_out"] = vs = val_scores(prev, data, a.crops, a.crops + n_val)
            print(f"previous weights: held-out {json.dumps(vs)}", flush=True)
            best = (vs["psnr_clamp"], prev)
        for loss in a.loss:
            for lr in a.lr:
                dn, t_train, losses = train(card, train_part, a.steps, batch=a.batch, lr_max=lr, loss=loss)
                vs = val_scores(dn, data, a.crops, a.crops + n_val)
                print(f"{loss} lr {lr}: {a.steps} steps in {t_train:.0f} s, loss {np.mean(losses[:100]):.4f} -> "
                      f"{np.mean(losses[-200:]):.4f}, held-out {json.dumps(vs)}", flush=True)
                runs.append(dict(loss=loss, lr=lr, s_train=t_train, loss_first=float(np.mean(losses[:100])),
                                 loss_last=float(np.mean(losses[-200:])), held_out=vs))
                if best is None or vs["psnr_clamp"] > best[0]:
                    if best is not None:
                        best[1].close()
                    best = (vs["psnr_clamp"], dn)
                else:
                    dn.close()
        dn = best[1]
        report["kept"] = "previous" if "previous_weights_held_out" in report and \
            best[0] == report["previous_weights_held_out"]["psnr_clamp"] else "new"
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        dn.get_params().astype("<f4").tofile(a.out)
        report.update(crops=a.crops, held_out=n_val, target_rays=a.target_rays, steps=a.steps, batch=a.batch,
                      s_data=t_data, runs=runs)
        del data, train_part
    else:
        dn = mb3dcu.Denoiser(card)
        dn.set_params(np.fromfile(a.out, "<f4"))
    report["eval"] = evaluate(card, dn, rect=tuple(a.rect) if a.rect else None, ref_rays=a.ref_rays)
    print(json.dumps(report))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
