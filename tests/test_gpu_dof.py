"""Depth of field on the card (mb3d_cu_dof) against the oracle's
restatement of dof::apply (src/dof.rs:81-122).

Every output pixel blends the reference's sources in the reference's order
(the sorted variant back to front, the forward one in pixel order) with the
same single precision arithmetic, so the 8-bit pictures agree byte for
byte; the tests allow one pixel in a thousand a step of one (a last-bit tie
in the rounding to 8 bits)."""
import numpy as np
import pytest

import mb3dcu
import oracle_py as O
import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c2_picture():
    sc = scenes.scaled(scenes.c2_hybrid(), 480, 270)
    g = O.deao(sc, O.shadows(sc, O.march(sc, mb3dcu.SILIGHT), per_pixel=True))
    return sc, g, O.paint(sc, g)


@pytest.mark.parametrize("forward", [0, 1])
@pytest.mark.parametrize("passes", [1, 3])
def test_dof_matches_oracle(card, c2_picture, forward, passes):
    sc, g, rgb = c2_picture
    o = mb3dcu.dof_default()
    o.forward, o.passes = forward, passes
    o.z_sharp = o.z_sharp2 = 2.2  # (the focus inside the object's depth range)
    o.aperture = 0.3
    want = O.dof(sc, g, rgb, o)
    got = card.dof(sc, g, rgb, o)
    assert (want != rgb).mean() > 0.3  # (the picture is blurred)
    d = np.abs(got.astype(np.int64) - want.astype(np.int64))
    assert (d == 0).mean() >= 0.999 and d.max() <= 1, ((d == 0).mean(), d.max())


def test_dof_device_buffers_equal_host(card, c2_picture):
    import torch
    sc, g, rgb = c2_picture
    o = mb3dcu.dof_default()
    host = card.dof(sc, g, rgb, o)
    gd = torch.from_numpy(g.view(np.uint8).copy()).cuda()
    rd = torch.from_numpy(rgb.copy()).cuda()
    card.dof(sc, gd, rd, o)
    torch.cuda.synchronize()
    assert rd.cpu().numpy().tobytes() == host.tobytes()


def test_dof_two_depth_checker_matches_oracle(card):
    """The G-buffer of dof.rs's own test scene (src/dof.rs:671-685: left half
    near, right half far, a checker pattern) through the card, both
    variants, against the oracle (the scene's depth constants are the
    hybrid frame's, so the focus lands elsewhere than in the reference's
    test, which the oracle's CPU test restates)."""
    w, h = 64, 32
    rgb = np.zeros((h, w, 3), np.uint8)
    g = np.zeros(w * h, mb3dcu.SILIGHT)
    for y in range(h):
        for x in range(w):
            rgb[y, x] = 255 if (x // 2 + y // 2) % 2 == 0 else 0
            g[y * w + x]["zpos_fine"] = (8_000_000 if x < w // 2 else 6_000_000) << 8
    sc = scenes.scaled(scenes.c2_hybrid(), w, h)
    for forward in (0, 1):
        o = mb3dcu.dof_default()
        o.forward, o.aperture, o.clip_r = forward, 0.5, 20.0
        want = O.dof(sc, g, rgb, o)
        got = card.dof(sc, g, rgb, o)
        assert got.tobytes() == want.tobytes(), forward
