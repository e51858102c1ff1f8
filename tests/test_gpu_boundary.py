"""The rest of gpu::march's contract through the C ABI (mb3d_cu_march_ex):
progress per band, cancel, the device time budget (MB3D_CU_ETIMEDOUT, and
the call that goes on from where it stopped) and the reference card's
single precision overflow rule (src/gpu.rs:2296-2400)."""
import ctypes

import numpy as np
import pytest

import mb3dcu
import scenes

pytestmark = pytest.mark.gpu


def small_c2():
    return scenes.scaled(scenes.c2_hybrid(), 480, 270)


@pytest.mark.parametrize("prec", [mb3dcu.FP64, mb3dcu.FP32_FP64])
def test_budget_stops_and_the_same_call_goes_on(card, prec):
    sc = small_c2()
    want = card.march(sc, prec)
    out = np.zeros_like(want)
    stops = 0
    for _ in range(100000):
        try:
            card.march_ex(sc, prec, out=out, budget_ms=0.02)
            break
        except mb3dcu.CardError as e:
            assert e.status == mb3dcu.ETIMEDOUT, e
            stops += 1
    else:
        raise AssertionError("the budgeted march never finished")
    assert stops >= 2
    assert out.tobytes() == want.tobytes()


def test_another_call_drops_the_stopped_march(card):
    sc = small_c2()
    want = card.march(sc, mb3dcu.FP32_FP64)
    out = np.zeros_like(want)
    with pytest.raises(mb3dcu.CardError) as e:
        card.march_ex(sc, mb3dcu.FP32_FP64, out=out, budget_ms=0.001)
    assert e.value.status == mb3dcu.ETIMEDOUT
    card.march(scenes.preset("Amazing Box", 96, 72), mb3dcu.FP32_FP64)  # reuses the scratch
    out[:] = 0
    card.march_ex(sc, mb3dcu.FP32_FP64, out=out)  # starts over, no budget
    assert out.tobytes() == want.tobytes()


def test_bands_progress_and_device_buffer(card):
    import torch
    sc = small_c2()
    want = card.march(sc, mb3dcu.FP64)
    seen = []
    out = card.march_ex(sc, mb3dcu.FP64, band_rows=64, progress=lambda d, t: seen.append((d, t)) and False)
    assert seen == [(64, 270), (128, 270), (192, 270), (256, 270), (270, 270)]
    assert out.tobytes() == want.tobytes()
    dev = torch.zeros(sc.width * sc.height * 20, dtype=torch.uint8, device="cuda")
    card.march_ex(sc, mb3dcu.FP64, out=dev, band_rows=100)
    torch.cuda.synchronize()
    assert dev.cpu().numpy().tobytes() == want.tobytes()


def test_progress_cancels(card):
    sc = small_c2()
    calls = []
    with pytest.raises(mb3dcu.CardError) as e:
        card.march_ex(sc, mb3dcu.FP64, band_rows=32, progress=lambda d, t: calls.append(d) or len(calls) >= 2)
    assert e.value.status == mb3dcu.ECANCELED
    assert calls == [32, 64]
    flag = ctypes.c_int(1)
    with pytest.raises(mb3dcu.CardError) as e:
        card.march_ex(sc, mb3dcu.FP64, band_rows=300, cancel=flag)
    assert e.value.status == mb3dcu.ECANCELED


def test_overflow_rule(card):
    """A Mandelbulb with a huge bailout overflows the single precision DE
    in many pixels: by default they are marched in double precision (the
    picture agrees with the FP64 one); with overflow_fail the call gives
    the picture up as the reference's card does."""
    sc = scenes.preset("Integer Power", 160, 120)
    card.march_ex(sc, mb3dcu.FP32_FP64, overflow_fail=True)
    assert card.stats()["fp32_overflow_pixels"] * 500 <= sc.width * sc.height
    sc.rstop = 1e15
    g = card.march_ex(sc, mb3dcu.FP32_FP64)
    n = card.stats()["fp32_overflow_pixels"]
    assert n * 500 > sc.width * sc.height, n
    with pytest.raises(mb3dcu.CardError) as e:
        card.march_ex(sc, mb3dcu.FP32_FP64, overflow_fail=True)
    assert e.value.status == mb3dcu.EOVERFLOW
    g64 = card.march(sc, mb3dcu.FP64)
    assert (mb3dcu.hit_mask(g) == mb3dcu.hit_mask(g64)).mean() >= 0.99
