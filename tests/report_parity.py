"""Prints the parity figures behind the GPU tests' thresholds (a report, not
a test): the card's FP64 drop-in march and the mixed march against the
oracle on the workloads (and the PSNR of the oracle's painter applied to
both G-buffers), the whole C2 frame painted, the Monte Carlo render
against its oracle.

    python tests/report_parity.py > parity.json      (on a B200)
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path[:0] = [HERE, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "mb3d-rs_b200")]

import numpy as np  # noqa: E402

import mb3dcu  # noqa: E402
import oracle_py as O  # noqa: E402
import scenes  # noqa: E402
from gbcompare import compare  # noqa: E402


def zc(sc):
    p = O.params(sc)
    return p[7], p[6]


def painted_psnr(sc, a, b):
    """PSNR of the oracle's painter (render::paint) applied to two G-buffers."""
    pa, pb = O.paint(sc, a).astype(np.float64), O.paint(sc, b).astype(np.float64)
    mse = float(np.mean((pa - pb) ** 2))
    return float(10 * np.log10(255.0 ** 2 / max(mse, 1e-12)))


def main():
    card = mb3dcu.Card(0)
    out = {}
    f = json.load(open(os.path.join(HERE, "golden", "c3_point.json")))
    cases = {"c1_plain_bulb_640x480": scenes.c1_plain_bulb(),
             "c2_hybrid_480x270": scenes.scaled(scenes.c2_hybrid(), 480, 270),
             "c3_deep_zoom_480x270": scenes.c3_deep_zoom(f["point"], f["view_dir"], 480, 270),
             "c4_menger_box_frame0_320x180": scenes.scaled(scenes.c4_frames(8)[0], 320, 180)}
    for name, sc in cases.items():
        ref = O.march(sc, mb3dcu.SILIGHT)
        row = {}
        for prec, pn in ((mb3dcu.FP64, "fp64"), (mb3dcu.FP32_FP64, "mixed")):
            g = card.march(sc, prec)
            row[pn] = compare(g, ref, *zc(sc))
            row[pn]["fp64_pixels"] = card.stats()["fp64_pixels"]
            row[pn]["painted_psnr"] = painted_psnr(sc, g, ref)
        out[name] = row
        print(name, json.dumps(row), file=sys.stderr, flush=True)
    # the whole C2 frame (march, hard shadows, DE AO) painted
    sc = scenes.scaled(scenes.c2_hybrid(), 480, 270)
    ref = O.deao(sc, O.shadows(sc, O.march(sc, mb3dcu.SILIGHT), per_pixel=True))
    row = {}
    for prec, pn in ((mb3dcu.FP64, "fp64"), (mb3dcu.FP32_FP64, "mixed")):
        row[pn] = {"painted_psnr": painted_psnr(sc, card.render(sc, prec), ref)}
    out["c2_hybrid_480x270_render"] = row
    print("c2_hybrid_480x270_render", json.dumps(row), file=sys.stderr, flush=True)
    sc = scenes.scaled(scenes.c2_hybrid(), 160, 90)
    lv = mb3dcu.mc_light_default(sc)
    opts = mb3dcu.mc_opts(8, depth=4)
    ref = O.mc_render(sc, lv, opts)
    for prec, pn in ((mb3dcu.FP64, "fp64"), (mb3dcu.FP32_FP64, "mixed")):
        got = card.mc_render(sc, opts, lv, prec)
        a, b = ref["radiance"], got["radiance"].astype(np.float64)
        close = np.all(np.abs(a - b) <= 1e-5 * a.max(), axis=2)
        out[f"mc_c2_160x90_8rays_{pn}"] = {"pixels_within_1e-5": float(close.mean()),
                                           "mean_rel_diff": float(abs(a.mean() - b.mean()) / a.mean()),
                                           "hit_agree": float((ref["hit"] == got["hit"]).mean())}
    print(json.dumps(out, indent=1))
    card.close()


if __name__ == "__main__":
    main()
