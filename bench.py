#!/usr/bin/env python3
"""Benchmark of the DE ray march with its post passes on B200.

A step is one whole "Calculate 3D" frame of the hybrid workload: 2 Amazing
Box (scale -1.5) + 1 Integer Power 8 iterations, repeating, 30 iterations,
1920x1080, a seeded camera on the r=3 sphere, hard shadows from one light
and DE ambient occlusion with 17 rays: the primary march (single precision
bulk, double precision origin, ray parameter and finish), the shadow pass
and the DE AO pass, into a device-resident G-buffer.  The metric is primary
rays per second (Mrays/s) of the whole frame.  With N GPUs every rank
renders its own frame (its own camera seed) and the frames' G-buffers are
all-gathered over NCCL inside the step: weak scaling; the time is the max
over ranks.

  value   device-resident G-buffer, kernels timed with CUDA events
  e2e     the same through the C ABI with a pinned host G-buffer (the copy
          back inside the call), timed on the host around each call
  --impl reference   the reference's CPU renderer (its C++ restatement, all
          host cores) on a bounded sample of rows of the same frame

Between timed steps a 512 MiB buffer is written to flush L2 (outside the
events of the step).
"""
import argparse
import ctypes
import datetime
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, "mb3d-rs_b200")]

import numpy as np  # noqa: E402

import mb3dcu  # noqa: E402
import scenes  # noqa: E402

METRIC = "Mrays/s (primary rays, whole frame: march + hard shadows + 17-ray DE AO)"
WORKLOAD = "c2-hybrid-1920x1080: AmazingBox(-1.5,0.5,1)x2 + IntPow8x1, 30 its, hard shadows, DE AO 17 rays"

# algorithmic FP32 operations per formula iteration (adds, multiplies,
# divisions and square roots counted once), from the formula code
FLOPS_PER_IT = {mb3dcu.F_INTPOW: 61, mb3dcu.F_AMAZINGBOX: 30, mb3dcu.F_MENGERIFS: 16, mb3dcu.F_REALPOWER: 30,
                mb3dcu.F_TRICORN: 14, mb3dcu.F_BULBOX: 40, mb3dcu.F_FOLDINGINTPOW: 73}
FLOPS_PER_DE = 40  # the DE's set-up and final formula (numerical gradient)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--scale", type=float, default=1.0, help="picture size factor (profiling runs)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample size")
    ap.add_argument("--no-mc", action="store_true", help="skip the Monte Carlo / denoiser figures")
    ap.add_argument("--mc-ref-rays", type=int, default=1024)
    ap.add_argument("--no-configs", action="store_true", help="skip the plain bulb, deep zoom and flight figures")
    ap.add_argument("--case", default=None, choices=sorted(CASES),
                    help="run one small fixed workload for a profiler instead of the benchmark")
    return ap.parse_args()


def max_over_ranks(x, world, device):
    """The largest value of x over the ranks (the step time of a weak-scaled
    run is its slowest rank's)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def frame(rank, scale):
    sc = scenes.c2_hybrid(scenes.C2_SEED + rank)
    if scale != 1.0:
        sc = scenes.scaled(sc, max(16, int(1920 * scale)), max(16, int(1080 * scale)))
    return sc


# ---------------------------------------------------------------------------
class Clocks:
    """nvidia-smi samples during the timed region (SM clock, throttle reasons)."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = max(mx, float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        os.unlink(self.f.name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def _oracle():
    """The oracle (CPU-baseline leg and reference arm only)."""
    p = os.path.join(ROOT, "oracle")
    if p not in sys.path:
        sys.path.insert(0, p)
    import oracle_py
    return oracle_py


def cpu_rows(sc, seconds, timer_rows=16):
    """Evenly spaced rows whose CPU render takes about `seconds`."""
    O = _oracle()
    h = sc.height
    probe = np.linspace(0, h - 1, timer_rows).round().astype(np.int32)
    t = time.perf_counter()
    O.render_rows(sc, mb3dcu.SILIGHT, probe)
    dt = max(time.perf_counter() - t, 1e-3)
    n = int(min(h, max(timer_rows, timer_rows * seconds / dt)))
    return np.linspace(0, h - 1, n).round().astype(np.int32)


def cpu_baseline(sc, seconds):
    """The oracle (C++ restatement of the reference CPU renderer) on a row
    sample; returns the figure, the rows and the oracle's records of them
    (the checker of the card's frame)."""
    O = _oracle()
    rows = cpu_rows(sc, seconds)
    t = time.perf_counter()
    recs = O.render_rows(sc, mb3dcu.SILIGHT, rows)
    dt = time.perf_counter() - t
    rays = len(rows) * sc.width
    fig = {"value": rays / dt / 1e6, "unit": "Mrays/s", "cores": os.cpu_count(), "kind": "port",
           "sample": f"{len(rows)} evenly spaced rows of the {sc.width}x{sc.height} frame ({rays} primary rays, "
                     f"march + hard shadows + DE AO), {dt:.1f} s, all host threads, C++ restatement of the "
                     f"reference CPU renderer"}
    return fig, rows, recs


def parity_vs_oracle(sc, card_g, rows, ref):
    """The card's G-buffer against the oracle's records of the same rows:
    hit agreement and the per-pixel relative depth error of the pixels both
    call a surface (the painted-picture and record figures are the parity
    tests' business)."""
    g = card_g.reshape(sc.height, sc.width)[rows].reshape(-1)
    r = parity_vs_fp64(sc, g, ref)
    r["pixels"] = int(len(g))
    return r


def run_reference(args):
    sc = frame(0, args.scale)
    rows = cpu_rows(sc, 6.0)
    O = _oracle()
    for _ in range(args.warmup):
        O.render_rows(sc, mb3dcu.SILIGHT, rows[: max(1, len(rows) // 8)])
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        O.render_rows(sc, mb3dcu.SILIGHT, rows)
        times.append(time.perf_counter() - t)
    rays = len(rows) * sc.width
    ms = 1000.0 * statistics.mean(times)
    v = rays / (ms / 1000.0) / 1e6
    sample = (f"{len(rows)} evenly spaced rows of the {sc.width}x{sc.height} frame per step ({rays} primary rays, "
              f"march + hard shadows + DE AO), C++ restatement of the reference CPU renderer (the Rust "
              f"reference cannot be built here), all host threads")
    out = {"metric": METRIC, "value": v, "unit": "Mrays/s", "n_gpus": args.gpus, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": WORKLOAD, "width": sc.width, "height": sc.height, "seed": scenes.C2_SEED},
           "impl": "reference",
           "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": os.cpu_count(), "kind": "port",
                            "sample": sample},
           "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def march_flops(sc, st):
    its = st["orbit_its"]
    f = 0
    for k in range(sc.n_slots):
        f += its[k] * FLOPS_PER_IT.get(sc.slots[k].formula, 30)
    return f + st["de_evals"] * FLOPS_PER_DE


def depth_of(g, sc):
    """mzz (depth in step widths) of G-buffer records from their zpos
    (CalcPPZvals, src/calc.rs:673-676, inverted)."""
    sw = 2.1345 / (sc.zoom * sc.width)
    zcorr = np.sin(max(np.deg2rad(sc.fov_y), 1.0) / sc.height)
    zc_mul = 32767.0 * 256.0 / (np.sqrt((sc.z_end - sc.z_start) * zcorr / sw + 1.0) - 0.999999999)
    zf = (g["zpos_fine"] >> 8).astype(np.float64)
    return (((8388352.0 - zf) / zc_mul + 1.0) ** 2 - 1.0) / zcorr


def parity_vs_fp64(sc, mixed, fp64):
    """The mixed march's G-buffer against the plain FP64 march's (the drop-in,
    itself held to the FP64 oracle by the parity tests)."""
    a, b = mixed, fp64
    ha, hb = mb3dcu.hit_mask(a), mb3dcu.hit_mask(b)
    both = ha & hb
    da, db = depth_of(a[both], sc), depth_of(b[both], sc)
    rel = np.abs(da - db) / np.maximum(np.abs(db), 1e-30)
    return {"hit_agree": float((ha == hb).mean()), "depth_rel_median": float(np.median(rel)),
            "depth_rel_p99": float(np.percentile(rel, 99)), "depth_within_1e-4": float((rel <= 1e-4).mean()),
            "pixels_both_hit": int(both.sum())}


def mc_figures(card, ref_rays):
    """The Monte Carlo workload (the hybrid scene at 1920x1080, 4 ambient
    bounces), the whole frame: the 4- and 16-ray method (two half traces,
    denoised, the plain trace kept where the denoised picture leaves it)
    against an independent plain trace of ref_rays rays."""
    import torch
    import train_denoiser as T
    if not os.path.exists(T.WEIGHTS):
        return {"unavailable": "no trained weights (mb3d-rs_b200/weights/denoiser.f32)"}
    card.set_stream(torch.cuda.current_stream().cuda_stream)  # (the denoiser between the timing events)
    dn = mb3dcu.Denoiser(card)
    dn.set_params(np.fromfile(T.WEIGHTS, "<f4"))
    out = T.evaluate(card, dn, rect=None, ref_rays=ref_rays, levels=(4, 16), log=lambda *a, **k: None)
    out["workload"] = "c5: hybrid scene 1920x1080, MCDepth 4, light 1 + sky; the whole frame"
    l16 = out["levels"][1]
    out["time_ratio_16_denoised_vs_ref"] = l16["time_ratio_vs_ref"]
    out["psnr_metric"] = ("psnr_*: PSNR of x/(1+x) tone-mapped linear records against the plain trace of ref_rays "
                          "rays; psnr8_*: PSNR of the 8-bit pictures paint_recs makes of both (default display "
                          "settings), on the card; ms_method: both half traces + denoiser + fallback")
    dn.close()
    card.set_stream(None)
    return out


def _timed_render(card, sc, prec, gbuf, flush, stream, reps):
    import torch
    card.render(sc, prec, out=gbuf)
    ms = []
    for _ in range(reps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        card.render(sc, prec, out=gbuf)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    return statistics.mean(ms)


def paint_figures(card, sc, gbuf, g_a, g_b, flush, stream, reps=5):
    """render::paint on the card (default lighting) of the frame's records
    resident on the device: its time, and the PSNR of the 8-bit pictures of
    the two precisions' G-buffers (g_a, g_b: host copies of both)."""
    import torch
    rgb = torch.empty((sc.height, sc.width, 3), dtype=torch.uint8, device="cuda")
    card.paint(sc, gbuf, out=rgb)
    ms = []
    for _ in range(reps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        card.paint(sc, gbuf, out=rgb)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    m = statistics.mean(ms)
    npix = sc.width * sc.height
    pa = card.paint(sc, g_a).astype(np.float64)
    pb = card.paint(sc, g_b).astype(np.float64)
    mse = float(np.mean((pa - pb) ** 2))
    return {"ms": m, "mpixels_s": npix / (m / 1000.0) / 1e6, "gbs": npix * 23 / (m / 1000.0) / 1e9,
            "psnr_8bit_mixed_vs_fp64": 10 * np.log10(255.0 ** 2 / max(mse, 1e-12)),
            "note": "k_paint: render::paint with the default lighting, 20 bytes in and 3 out per pixel"}


def reflect_figures(card, sc, gbuf, flush, stream, reps=3):
    """The reflection pass's first bounce of the frame on the card
    (mb3d_cu_reflect_first_rays, then mb3d_cu_reflect_batch: the FP64 march
    of every object pixel's mirror ray with its hit's normal, colour, depth,
    shadow and DE AO), device-resident; times from CUDA events."""
    import torch
    npix = sc.width * sc.height
    rays = torch.empty(npix * mb3dcu.REFLECT_RAY.itemsize, dtype=torch.uint8, device="cuda")
    hits = torch.empty(npix * mb3dcu.REFLECT_HIT.itemsize, dtype=torch.uint8, device="cuda")
    _, n = card.reflect_first_rays(sc, gbuf, out=rays)
    rb, hb = n * mb3dcu.REFLECT_RAY.itemsize, n * mb3dcu.REFLECT_HIT.itemsize
    card.reflect_batch(sc, rays[:rb], out=hits[:hb])
    t_first, t_batch = [], []
    for _ in range(reps):
        flush.zero_()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        ev[0].record(stream)
        card.reflect_first_rays(sc, gbuf, out=rays)
        ev[1].record(stream)
        card.reflect_batch(sc, rays[:rb], out=hits[:hb])
        ev[2].record(stream)
        ev[2].synchronize()
        t_first.append(ev[0].elapsed_time(ev[1]))
        t_batch.append(ev[1].elapsed_time(ev[2]))
    h = np.frombuffer(hits[:hb].cpu().numpy().tobytes(), dtype=mb3dcu.REFLECT_HIT)
    mb = statistics.mean(t_batch)
    return {"rays": int(n), "ms_first_rays": statistics.mean(t_first), "ms_batch": mb,
            "mrays_s": n / (mb / 1000.0) / 1e6, "hit_share": float((h["hit"] == 1).mean()) if n else 0.0,
            "note": "the first bounce of every object pixel of the frame: k_reflect_first + compaction, then "
                    "k_reflect (FP64, one thread per ray, with the hit's shadow and DE AO)"}


def config_figures(card, flush, stream, peak32=None, reps=3):
    """The other workloads, one GPU, device-resident outputs: the plain
    Mandelbulb (640x480) and the deep zoom (1920x1080) in both precisions
    with the mixed march's agreement with the FP64 one; the 240-frame
    1280x720 Menger/Amazing Box flight through one CUDA graph with the
    launch settings the autotuner picked on 8 sample frames."""
    import torch
    card.set_stream(stream.cuda_stream)
    out = {}
    for name, sc in (("c1_plain_bulb_640x480", scenes.c1_plain_bulb()), ("c3_deep_zoom_1920x1080", scenes.c3())):
        npix = sc.width * sc.height
        gbuf = torch.empty(npix * 20, dtype=torch.uint8, device="cuda")
        ms_m = _timed_render(card, sc, mb3dcu.FP32_FP64, gbuf, flush, stream, reps)
        g_m = np.frombuffer(gbuf.cpu().numpy().tobytes(), dtype=mb3dcu.SILIGHT).copy()
        fp64_pix = card.stats()["fp64_pixels"]
        ms_d = _timed_render(card, sc, mb3dcu.FP64, gbuf, flush, stream, reps)
        g_d = np.frombuffer(gbuf.cpu().numpy().tobytes(), dtype=mb3dcu.SILIGHT).copy()
        out[name] = {"mixed_mrays_s": npix / (ms_m / 1000.0) / 1e6, "mixed_ms": ms_m,
                     "fp64_mrays_s": npix / (ms_d / 1000.0) / 1e6, "fp64_ms": ms_d, "mixed_over_fp64": ms_d / ms_m,
                     "mixed_fp64_fallback_pixels": fp64_pix, "parity_vs_fp64": parity_vs_fp64(sc, g_m, g_d)}
        del gbuf
    frames = scenes.c4_frames(240)
    npix = frames[0].width * frames[0].height
    gbuf = torch.empty(len(frames) * npix * 20, dtype=torch.uint8, device="cuda")
    t0 = time.perf_counter()
    tune = card.autotune(frames, 8)
    tune_s = time.perf_counter() - t0
    card.render_frames(frames, mb3dcu.FP32_FP64, tune, out=gbuf)
    ms = []
    for _ in range(reps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        card.render_frames(frames, mb3dcu.FP32_FP64, tune, out=gbuf)
        e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    st = card.stats()
    m = statistics.mean(ms)
    out["c4_flight_240x1280x720"] = {
        "mrays_s": len(frames) * npix / (m / 1000.0) / 1e6, "ms_all_frames": m, "ms_per_frame": m / len(frames),
        "tune": {"blocks_per_sm": tune.blocks_per_sm, "refill_min": tune.refill_min, "streams": tune.streams},
        "autotune_s": tune_s, "launches_per_call": st["launches"]}
    del gbuf
    # the flight's FP32 march kernel against the FP32 peak: the counted
    # formula iterations and DEs of one frame over its mean launch time
    f = frames[37]
    g1 = torch.empty(npix * 20, dtype=torch.uint8, device="cuda")
    card.set_counting(True)
    card.render(f, mb3dcu.FP32_FP64, out=g1)
    cst = card.stats()
    card.set_counting(False)
    kms = []
    for _ in range(reps):
        card.render(f, mb3dcu.FP32_FP64, out=g1)
        s1 = card.stats()
        kms.append(s1["ms_march"] - s1["ms_finish"])
    k = statistics.mean(kms)
    fl = march_flops(f, cst)
    out["c4_flight_240x1280x720"]["roofline_frame37"] = {
        "kernel": "k_march (FP32 bulk march)", "bound": "fp32-alu", "flops_per_launch": fl, "ms_per_launch": k,
        "achieved": fl / (k / 1000.0) / 1e12, "peak": peak32, "unit": "TFLOP/s",
        "frac": fl / (k / 1000.0) / 1e12 / peak32 if peak32 else None}
    del g1
    card.set_stream(None)
    return out


def load_traffic():
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


# ---------------------------------------------------------------------------
# small fixed workloads for profiler runs (ncu), one per hot kernel family;
# `python bench.py --case NAME` runs one and prints a line of its timings

def case_mc():
    """Monte Carlo: the hybrid scene at 480x270, 4 rays, MCDepth 4, mixed."""
    card = mb3dcu.Card(0)
    sc = scenes.scaled(scenes.c2_hybrid(), 480, 270)
    lv = mb3dcu.mc_light_default(sc)
    card.mc_render(sc, mb3dcu.mc_opts(4, depth=4), lv, mb3dcu.FP32_FP64)
    st = card.stats()
    print("ok mc", st["ms_total"], st["de_evals"])


def case_denoise():
    """The denoiser on one 1920x1080 picture (6 passes)."""
    import torch
    card = mb3dcu.Card(0)
    dn = mb3dcu.Denoiser(card)
    h, w = 1080, 1920
    rng = np.random.default_rng(0)
    rad = torch.from_numpy(rng.gamma(1.0, 0.4, (1, h, w, 3)).astype(np.float32)).cuda()
    alb = torch.rand((1, h, w, 3), device="cuda")
    nrm = torch.rand((1, h, w, 3), device="cuda")
    dep = torch.rand((1, h, w), device="cuda")
    out = dn.denoise(rad, alb, nrm, dep, depth_scale=1.0)
    torch.cuda.synchronize()
    card.set_stream(torch.cuda.current_stream().cuda_stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(5):
        dn.denoise(rad, alb, nrm, dep, depth_scale=1.0, out=out)
    e1.record()
    torch.cuda.synchronize()
    print("ok denoise 1920x1080 ms", e0.elapsed_time(e1) / 5)


def case_train():
    """20 denoiser training steps of batch 16 of 128x128 (after 3)."""
    import torch
    card = mb3dcu.Card(0)
    dn = mb3dcu.Denoiser(card)
    n, h, w = 16, 128, 128
    g = torch.Generator(device="cuda").manual_seed(0)
    rad = torch.rand((n, h, w, 3), device="cuda", generator=g) * 2.0
    tgt = rad * 0.9
    alb = torch.rand((n, h, w, 3), device="cuda", generator=g)
    nrm = torch.rand((n, h, w, 3), device="cuda", generator=g)
    dep = torch.rand((n, h, w), device="cuda", generator=g)
    card.set_stream(torch.cuda.current_stream().cuda_stream)
    for _ in range(3):
        dn.train_step(rad, tgt, alb, nrm, dep, depth_scale=1.0, lr=1e-3)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(20):
        loss = dn.train_step(rad, tgt, alb, nrm, dep, depth_scale=1.0, lr=1e-3)
    e1.record()
    torch.cuda.synchronize()
    print("ok train step (16 x 128 x 128) ms", e0.elapsed_time(e1) / 20, "loss", loss)


def case_ssao():
    """The 24-bit SSAO of the 1920x1080 hybrid frame's G-buffer."""
    import torch
    card = mb3dcu.Card(0)
    sc = scenes.c2_hybrid()
    npix = sc.width * sc.height
    g = torch.empty(npix * 20, dtype=torch.uint8, device="cuda")
    card.render(sc, mb3dcu.FP32_FP64, out=g)
    for _ in range(3):
        card.ssao24(sc, g)
    ms = []
    for _ in range(5):
        card.ssao24(sc, g)
        ms.append(card.stats()["ms_total"])
    print("ok ssao24 1920x1080 ms", sum(ms) / len(ms), "Mpixels/s", npix / (sum(ms) / len(ms)) / 1e3)


def _case_both(sc):
    card = mb3dcu.Card(0)
    for prec in (mb3dcu.FP32_FP64, mb3dcu.FP64):
        card.render(sc, prec)
        st = card.stats()
        print("ok", prec, "ms", st["ms_total"], "finish", st["ms_finish"], "fp64 pixels", st["fp64_pixels"])


def case_c1():
    """The plain bulb 640x480: one mixed, one FP64 render."""
    _case_both(scenes.c1_plain_bulb())


def case_c2small():
    """The hybrid frame at 480x270 (march, shadows, DE AO): one mixed, one FP64 render."""
    _case_both(scenes.scaled(scenes.c2_hybrid(), 480, 270))


def case_c4():
    """Frame 37 of the 240-frame flight: one mixed, one FP64 render."""
    _case_both(scenes.c4_frames(240)[37])


CASES = {"mc": case_mc, "denoise": case_denoise, "train": case_train, "ssao": case_ssao, "c1": case_c1,
         "c2small": case_c2small, "c4": case_c4}


def main():
    args = parse()
    if args.case:
        CASES[args.case]()
        return
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                device_id=torch.device("cuda", local))
    prec = mb3dcu.FP32_FP64 if args.precision == "mixed" else mb3dcu.FP64
    card = mb3dcu.Card(local)
    stream = torch.cuda.current_stream()
    card.set_stream(stream.cuda_stream)
    sc = frame(rank, args.scale)
    npix = sc.width * sc.height
    gbuf = torch.empty(npix * 20, dtype=torch.uint8, device="cuda")
    flush = torch.empty(512 << 20, dtype=torch.uint8, device="cuda")

    for _ in range(max(3, args.warmup)):
        card.render(sc, prec, out=gbuf)
    # algorithmic work of the march kernel (a counting pass, not timed)
    card.set_counting(True)
    card.render(sc, prec, out=gbuf)
    counted = card.stats()
    card.set_counting(False)
    peak32 = card.fma_peak(False)
    peak64 = card.fma_peak(True)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    barrier()
    clk = Clocks(local)
    clk.start()
    step_ms, kern = [], []
    launches = 0
    import cards
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        card.render(sc, prec, out=gbuf)
        if world > 1:
            # the frames of all ranks on every rank: one NCCL all_gather (NVLink)
            cards.gather(gbuf, [npix] * world, 20)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        st = card.stats()
        kern.append(st)
        launches += st["launches"]
    barrier()
    clocks = clk.stop()
    ms = max_over_ranks(statistics.mean(step_ms), world, "cuda")
    value = world * npix / (ms / 1000.0) / 1e6

    # end to end: the C ABI with a pinned host G-buffer (copy back inside the call)
    host = torch.empty(npix * 20, dtype=torch.uint8, pin_memory=True)
    hnp = host.numpy()
    card.set_stream(None)
    card.render(sc, prec, out=hnp)
    barrier()
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        t = time.perf_counter()
        card.render(sc, prec, out=hnp)
        e2e_ms.append(1000.0 * (time.perf_counter() - t))
    barrier()
    e2e = max_over_ranks(statistics.mean(e2e_ms), world, "cuda")

    # roofline of the march kernel (single precision bulk): counted flops per
    # launch over its mean launch time, against the measured FP32 FMA peak
    k_ms = statistics.mean(k["ms_march"] - k["ms_finish"] for k in kern)
    stage = {"k_march": k_ms, "k_finish64": statistics.mean(k["ms_finish"] for k in kern),
             "k_shadow": statistics.mean(k["ms_shadow"] for k in kern),
             "k_deao": statistics.mean(k["ms_deao"] for k in kern)}
    flops = march_flops(sc, counted)
    achieved = flops / (k_ms / 1000.0) / 1e12
    traffic = load_traffic().get("k_march")
    roof = {"kernel": "k_march (FP32 bulk march)", "bound": "fp32-alu", "achieved": achieved, "peak": peak32,
            "unit": "TFLOP/s", "frac": achieved / peak32 if peak32 else None,
            "peak_source": "measured FP32 FMA chain on this GPU (MEASURED_PEAKS.json has no FP32 figure)",
            "traffic": traffic, "flops_per_launch": flops, "ms_per_launch": k_ms}
    out = {"metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32+f64" if prec == mb3dcu.FP32_FP64 else "f64", "data": "synthetic",
           "config": {"workload": WORKLOAD, "width": sc.width, "height": sc.height, "seed": scenes.C2_SEED,
                      "precision": args.precision,
                      "parallelism": f"frame per rank x{world}" + (", G-buffers all-gathered in the step" if world > 1 else ""),
                      "l2": "512 MiB buffer written between timed steps (outside the step events)"},
           "e2e": {"value": world * npix / (e2e / 1000.0) / 1e6, "unit": "Mrays/s",
                   "h2d_bytes_per_step": ctypes.sizeof(mb3dcu.Scene), "d2h_bytes_per_step": npix * 20},
           "gpu_launches": launches, "roofline": roof, "stages_ms": stage,
           "peaks": {"fp32_fma_tflops": peak32, "fp64_fma_tflops": peak64},
           "counted": {"de_evals": counted["de_evals"], "orbit_its": counted["orbit_its"],
                       "march_de_evals_per_s": counted["de_evals"] / (k_ms / 1000.0),
                       "march_iteration_lane_use": counted["march_lane_its"] / max(32 * counted["march_warp_its"], 1),
                       "march_busy_lane_use": counted["march_busy_lanes"] / max(32 * counted["march_trips"], 1),
                       "march_warp_trips": counted["march_trips"]},
           "clocks": clocks}
    if rank == 0:
        # the plain FP64 march (the drop-in) on the same frame, and the mixed
        # march's agreement with it
        mixed_g = np.frombuffer(gbuf.cpu().numpy().tobytes(), dtype=mb3dcu.SILIGHT).copy()
        card.set_stream(stream.cuda_stream)
        other = mb3dcu.FP64 if prec == mb3dcu.FP32_FP64 else mb3dcu.FP32_FP64
        card.render(sc, other, out=gbuf)
        o_ms = []
        for _ in range(max(3, args.steps // 2)):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            card.render(sc, other, out=gbuf)
            e1.record(stream)
            e1.synchronize()
            o_ms.append(e0.elapsed_time(e1))
        other_g = np.frombuffer(gbuf.cpu().numpy().tobytes(), dtype=mb3dcu.SILIGHT).copy()
        om = statistics.mean(o_ms)
        if prec == mb3dcu.FP32_FP64:
            out["fp64_march"] = {"value": npix / (om / 1000.0) / 1e6, "unit": "Mrays/s", "ms_per_step": om,
                                 "mixed_over_fp64": om / ms}
            out["parity_vs_fp64"] = parity_vs_fp64(sc, mixed_g, other_g)
        out["paint"] = paint_figures(card, sc, gbuf, mixed_g, other_g, flush, stream)
        if args.scale == 1.0:
            try:
                out["reflect"] = reflect_figures(card, sc, gbuf, flush, stream)
            except Exception as e:  # (a figure beside the headline: its failure is reported, not fatal)
                out["reflect"] = {"error": str(e)[:300]}
        card.set_stream(None)
        if not args.no_configs and args.scale == 1.0:
            out["configs"] = config_figures(card, flush, stream, peak32)
        if not args.no_mc and args.scale == 1.0:
            out["mc"] = mc_figures(card, args.mc_ref_rays)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        fig, rows, ref = cpu_baseline(frame(0, args.scale), args.cpu_seconds)
        out["cpu_baseline"] = fig
        # both card modes against the oracle on the rows the baseline rendered
        if prec == mb3dcu.FP32_FP64:
            out["parity_vs_oracle"] = {"mixed": parity_vs_oracle(sc, mixed_g, rows, ref),
                                       "fp64": parity_vs_oracle(sc, other_g, rows, ref)}
    if rank == 0:
        print(json.dumps(out), flush=True)
    card.close()
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
