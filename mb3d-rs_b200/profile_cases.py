"""Small fixed workloads for profiling runs (ncu), one per hot kernel family.

    python mb3d-rs_b200/profile_cases.py mc        # Monte Carlo: C2 scene 480x270, 4 rays, MCDepth 4, mixed
    python mb3d-rs_b200/profile_cases.py denoise   # the denoiser on one 1920x1080 picture (6 passes)
    python mb3d-rs_b200/profile_cases.py c1        # the plain bulb 640x480: one mixed, one FP64 render
    python mb3d-rs_b200/profile_cases.py c4        # frame 37 of the 240-frame flight: one mixed, one FP64 render
    python mb3d-rs_b200/profile_cases.py de        # single precision DEs of the C2 scene at 3, 6 and 30 iterations
    python mb3d-rs_b200/profile_cases.py train     # 20 denoiser training steps, batch 16 of 128x128 (after 3)
    python mb3d-rs_b200/profile_cases.py ssao      # the 24-bit SSAO of the 1920x1080 hybrid frame's G-buffer

The Calculate 3D kernels are profiled through bench.py (--scale 0.25).
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import numpy as np  # noqa: E402

import mb3dcu  # noqa: E402
import scenes  # noqa: E402


def mc():
    card = mb3dcu.Card(0)
    sc = scenes.scaled(scenes.c2_hybrid(), 480, 270)
    lv = mb3dcu.mc_light_default(sc)
    card.mc_render(sc, mb3dcu.mc_opts(4, depth=4), lv, mb3dcu.FP32_FP64)
    st = card.stats()
    print("ok", st["ms_total"], st["de_evals"])


def denoise():
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


def train():
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


def ssao():
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


def _both(sc):
    card = mb3dcu.Card(0)
    for prec in (mb3dcu.FP32_FP64, mb3dcu.FP64):
        card.render(sc, prec)
        st = card.stats()
        print("ok", prec, "ms", st["ms_total"], "finish", st["ms_finish"], "fp64 pixels", st["fp64_pixels"])


def c1():
    _both(scenes.c1_plain_bulb())


def c4():
    _both(scenes.c4_frames(240)[37])


def de():
    """The instruction cost of one DE: 16 M seeded points of the C2 scene
    probed once in double precision (one launch), then three launches of
    32768 points in single precision whose double precision iteration
    count is 3, 6 and 30 (every lane of a warp at the same count)."""
    card = mb3dcu.Card(0)
    sc = scenes.c2_hybrid()
    pts = np.random.default_rng(5).uniform(-2.0, 2.0, size=(16_000_000, 3))
    _, its = card.de_probe(sc, pts, mb3dcu.FP64)
    for n in (3, 6, 30):
        sel = pts[its == n][:32768]
        _, i = card.de_probe(sc, sel, mb3dcu.FP32_FP64)
        print("ok", n, len(sel), "mean iterations", float(i.mean()))


if __name__ == "__main__":
    {"mc": mc, "denoise": denoise, "c1": c1, "c4": c4, "de": de, "train": train, "ssao": ssao}[sys.argv[1]]()
