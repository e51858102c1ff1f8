"""The other workloads through the C ABI: the deep zoom (double precision
where single precision cannot resolve the DE offset), the batched animation
(all frames in one CUDA graph over several streams) and its autotuner."""
import json
import os

import numpy as np
import pytest

import mb3dcu
import oracle_py as O
import scenes
from gbcompare import compare

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def zc(sc):
    p = O.params(sc)
    return p[7], p[6]


def c3_scene(w, h):
    f = json.load(open(os.path.join(HERE, "golden", "c3_point.json")))
    return scenes.c3_deep_zoom(f["point"], f["view_dir"], w, h)


def test_deep_zoom_matches_oracle(card):
    sc = c3_scene(192, 108)
    ref = O.march(sc, mb3dcu.SILIGHT)
    assert mb3dcu.hit_mask(ref).mean() > 0.5
    g64 = card.march(sc, mb3dcu.FP64)
    r = compare(g64, ref, *zc(sc))
    assert r["hit_agree"] >= 0.999 and r["depth_rel_median"] <= 1e-9, r
    # the mixed mode keeps double precision here (the offset is under 3 single steps)
    g = card.march(sc, mb3dcu.FP32_FP64)
    st = card.stats()
    assert st["fp64_pixels"] == sc.width * sc.height
    assert g.tobytes() == g64.tobytes()


def test_frames_in_one_graph_equal_single_renders(card):
    frames = [scenes.scaled(f, 320, 180) for f in scenes.c4_frames(6)]
    batch = card.render_frames(frames, mb3dcu.FP32_FP64, mb3dcu.Tune(3, 16, 3, 0))
    npix = 320 * 180
    for k, f in enumerate(frames):
        one = card.render(f, mb3dcu.FP32_FP64)
        assert batch[k * npix:(k + 1) * npix].tobytes() == one.tobytes(), k
    ref = O.march(frames[0], mb3dcu.SILIGHT)
    r = compare(batch[:npix], ref, *zc(frames[0]))
    assert r["hit_agree"] >= 0.99, r


def test_autotune_picks_valid_settings(card):
    frames = [scenes.scaled(f, 256, 144) for f in scenes.c4_frames(8)]
    t = card.autotune(frames, sample=4)
    assert 1 <= t.blocks_per_sm <= 16 and 1 <= t.refill_min <= 32 and 1 <= t.streams <= 8
    a = card.render_frames(frames, mb3dcu.FP32_FP64, t)
    b = card.render_frames(frames, mb3dcu.FP32_FP64, None)
    assert a.tobytes() == b.tobytes()
