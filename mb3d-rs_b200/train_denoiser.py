"""Trains the Monte Carlo denoiser on pictures the card's path tracer renders
and evaluates it on the 1920x1080 Monte Carlo workload.

    python mb3d-rs_b200/train_denoiser.py train --crops 2000 --steps 6000
    python mb3d-rs_b200/train_denoiser.py eval

Training data: `--crops` seeded random scenes (scenes.random_training_scene)
rendered at 256x256: the 4- and 16-ray pictures (rays 0..15) with their
first surfaces' albedo, normal and depth, and an independent target of
`--target-rays` rays (rays 16..); all kept in device memory.  Training:
Adam on random 128x128 pieces (flipped and turned at random), the input
taken at 4 or 16 rays, the L1 loss of the network in log space
(mb3d_cu_dn_train_step: forward and backward on the card's own BF16
convolution kernels), a cosine learning rate.  The weights go to
weights/denoiser.f32 (FP32, little endian, the library's parameter order).
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


def train(card, data, steps, batch=8, piece=128, lr_max=2e-3, seed=1, log=print):
    torch = _torch()
    dn = mb3dcu.Denoiser(card, seed=seed)
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


def val_loss(dn, data, lo, hi):
    """The L1 loss in log space of the denoised held-out pictures (4 and 16
    rays) against their targets."""
    torch = _torch()
    tot = []
    for i in range(lo, hi, 8):
        j = min(i + 8, hi)
        for k in ("r4", "r16"):
            den = dn.denoise(data[k][i:j].contiguous(), data["alb"][i:j].contiguous(), data["nrm"][i:j].contiguous(),
                             data["dep"][i:j, ..., 0].contiguous(), depth_scale=1.0)
            tot.append(float((torch.log1p(den) - torch.log1p(data["tgt"][i:j].clamp(min=0))).abs().mean()))
    return float(np.mean(tot))


def tonemap(x):
    return x / (1.0 + x)


def psnr(a, ref):
    """PSNR of two radiance pictures after x / (1 + x) (both in 0..1)."""
    mse = float(np.mean((tonemap(np.maximum(a, 0)) - tonemap(np.maximum(ref, 0))) ** 2))
    return 10.0 * math.log10(1.0 / max(mse, 1e-20))


def fallback_tiles(noisy_a, noisy_b, den, tile=16, k=3.0):
    """The tiles where the denoised picture leaves the noisy one by more than
    k times the noise the two independent halves of the rays show: there the
    plain trace is kept.  Returns the composite and the share of such tiles."""
    h, w, _ = den.shape
    noisy = 0.5 * (noisy_a + noisy_b)
    out = den.copy()
    n = bad = 0
    for y in range(0, h - tile + 1, tile):
        for x in range(0, w - tile + 1, tile):
            sl = (slice(y, y + tile), slice(x, x + tile))
            a, b, d, m = (tonemap(v[sl]) for v in (noisy_a, noisy_b, den, noisy))
            sigma = np.sqrt(np.mean((a - b) ** 2) / 4.0 / (tile * tile * 3)) + 1e-3
            n += 1
            if abs(float(np.mean(d - m))) > k * sigma:
                bad += 1
                out[sl] = noisy[sl]
    return out, bad / max(n, 1)


def evaluate(card, dn, rect=(720, 405, 480, 270), ref_rays=1024, log=print):
    """The 1920x1080 workload on a rectangle: the plain trace at ref_rays,
    the 4..64-ray traces and their denoised pictures; times on the card.
    PSNRs of the tone-mapped linear records (psnr_*) and of the 8-bit
    pictures the reference's painter makes of them (psnr8_*, paint_recs with
    the default display settings, on the card)."""
    torch = _torch()
    sc = scenes.c5_mc()
    lv = mb3dcu.mc_light_default(sc)

    def trace(rays, ray0=0):
        o = mb3dcu.mc_opts(rays, depth=scenes.C5_DEPTH, ray0=ray0, rect=rect)
        r = card.mc_render(sc, o, lv, mb3dcu.FP32_FP64)
        return r, card.stats()["ms_total"]

    ref, ms_ref = trace(ref_rays, ray0=4096)  # (rays of their own, each with its own Halton record (< 65536))
    res = {"rect": list(rect), "ref_rays": ref_rays, "ms_ref": ms_ref, "levels": []}
    paint_opts = mb3dcu.mc_paint_default()
    ref8 = card.mc_paint(ref["radiance"], paint_opts).astype(np.float64)

    def psnr8(x):
        mse = float(np.mean((card.mc_paint(x, paint_opts).astype(np.float64) - ref8) ** 2))
        return 10.0 * math.log10(255.0 ** 2 / max(mse, 1e-12))

    for rays in (4, 8, 16, 32, 64):
        r, ms = trace(rays)
        dmax = float(r["depth"].max()) or 1.0
        rad = torch.from_numpy(r["radiance"]).cuda()[None]
        alb = torch.from_numpy(r["albedo"]).cuda()[None]
        nrm = torch.from_numpy(r["normal"]).cuda()[None]
        dp = torch.from_numpy(r["depth"]).cuda()[None]
        dn.denoise(rad, alb, nrm, dp, depth_scale=1.0 / dmax)  # (warm)
        ev = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev[0].record()
        den = dn.denoise(rad, alb, nrm, dp, depth_scale=1.0 / dmax)
        ev[1].record()
        torch.cuda.synchronize()
        ms_dn = ev[0].elapsed_time(ev[1])
        den = den[0].cpu().numpy()
        half = max(rays // 2, 1)
        ha, _ = trace(half, 0)
        hb, _ = trace(half, half)
        comp, fb = fallback_tiles(ha["radiance"], hb["radiance"], den)
        lvl = {"rays": rays, "ms_trace": ms, "ms_denoise": ms_dn, "psnr_noisy": psnr(r["radiance"], ref["radiance"]),
               "psnr_denoised": psnr(den, ref["radiance"]), "psnr_with_fallback": psnr(comp, ref["radiance"]),
               "fallback_rate": fb, "psnr8_noisy": psnr8(r["radiance"]), "psnr8_denoised": psnr8(den),
               "psnr8_with_fallback": psnr8(comp)}
        res["levels"].append(lvl)
        log(f"  {rays} rays: trace {ms:.1f} ms, denoise {ms_dn:.2f} ms, PSNR noisy {lvl['psnr_noisy']:.2f} "
            f"denoised {lvl['psnr_denoised']:.2f} (fallback {fb:.3f}: {lvl['psnr_with_fallback']:.2f}); 8-bit "
            f"noisy {lvl['psnr8_noisy']:.2f} denoised {lvl['psnr8_denoised']:.2f}", flush=True)
    ok = [lv_ for lv_ in res["levels"] if lv_["psnr_denoised"] >= 35.0]
    if ok:
        best = min(ok, key=lambda l: l["ms_trace"] + l["ms_denoise"])
        res["time_to_35db_ms"] = best["ms_trace"] + best["ms_denoise"]
        res["time_to_35db_rays"] = best["rays"]
        res["time_ratio_vs_ref"] = res["time_to_35db_ms"] / ms_ref
    plain = [lv_ for lv_ in res["levels"] if lv_["psnr_noisy"] >= 35.0]
    if plain:
        res["plain_to_35db_rays"] = min(l["rays"] for l in plain)
    ok8 = [lv_ for lv_ in res["levels"] if lv_["psnr8_denoised"] >= 35.0]
    if ok8:
        best = min(ok8, key=lambda l: l["ms_trace"] + l["ms_denoise"])
        res["time_to_35db_8bit_ms"] = best["ms_trace"] + best["ms_denoise"]
        res["time_to_35db_8bit_rays"] = best["rays"]
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
        for lr in a.lr:
            dn, t_train, losses = train(card, train_part, a.steps, batch=a.batch, lr_max=lr)
            vl = val_loss(dn, data, a.crops, a.crops + n_val)
            print(f"lr {lr}: {a.steps} steps in {t_train:.0f} s, loss {np.mean(losses[:100]):.4f} -> "
                  f"{np.mean(losses[-200:]):.4f}, held-out {vl:.4f}", flush=True)
            runs.append(dict(lr=lr, s_train=t_train, loss_first=float(np.mean(losses[:100])),
                             loss_last=float(np.mean(losses[-200:])), val_loss=vl))
            if best is None or vl < best[0]:
                if best is not None:
                    best[1].close()
                best = (vl, dn)
            else:
                dn.close()
        dn = best[1]
        os.makedirs(os.path.dirname(os.path.abspath(a.out)), exist_ok=True)
        dn.get_params().astype("<f4").tofile(a.out)
        report.update(crops=a.crops, held_out=n_val, target_rays=a.target_rays, steps=a.steps, batch=a.batch,
                      s_data=t_data, runs=runs)
        del data, train_part
    else:
        dn = mb3dcu.Denoiser(card)
        dn.set_params(np.fromfile(a.out, "<f4"))
    report["eval"] = evaluate(card, dn, ref_rays=a.ref_rays)
    print(json.dumps(report))
    if a.report:
        with open(a.report, "w") as f:
            json.dump(report, f, indent=1)


if __name__ == "__main__":
    main()
