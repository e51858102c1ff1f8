"""The allocation-free march (mb3d_cu_march_noalloc) against the regular one.

Callers whose GPU memory belongs to another allocator (an engine's fixed
pool, PyTorch's caching allocator), or whose render loop cannot take the
device-wide synchronisation of cudaMalloc/cudaFree, march bands through
this entry point; its scratch is a static device array of the library.
Its records must equal mb3d_cu_march's for the same band, on two calls in a
row (the shared scratch keeps nothing that changes the next call), and a
band over the array's size must be refused.  This file runs last (its name)
and also passes alone in a fresh process.
"""
import numpy as np
import pytest

import mb3dcu
import scenes

pytestmark = pytest.mark.gpu


def _device_band(torch, sc, rows):
    return torch.zeros(rows * sc.width * 20, dtype=torch.uint8, device="cuda")


def _records(torch, t):
    torch.cuda.synchronize()
    return np.frombuffer(t.cpu().numpy().tobytes(), dtype=mb3dcu.SILIGHT)


@pytest.mark.parametrize("prec", [mb3dcu.FP32_FP64, mb3dcu.FP64])
def test_noalloc_equals_regular_march_twice(prec):
    import torch
    card = mb3dcu.Card(0)
    try:
        cases = [(scenes.scaled(scenes.c2_hybrid(), 240, 136), 0, 136),   # whole picture, 32640 pixels
                 (scenes.c1_plain_bulb(), 150, 100)]                    # a band of 64000 pixels
        for sc, row0, rows in cases:
            assert rows * sc.width <= mb3dcu.NOALLOC_MAX_PIXELS
            want = card.march(sc, prec, row0=row0, rows=rows)
            for _ in range(2):
                out = _device_band(torch, sc, rows)
                mb3dcu.march_noalloc(sc, out, prec, row0=row0, rows=rows)
                got = _records(torch, out)
                assert got.tobytes() == want.tobytes()
    finally:
        card.close()


def test_noalloc_refuses_a_band_over_its_limit():
    import torch
    sc = scenes.c1_plain_bulb()
    out = _device_band(torch, sc, 480)
    with pytest.raises(mb3dcu.CardError) as e:
        mb3dcu.march_noalloc(sc, out, mb3dcu.FP32_FP64, row0=0, rows=480)
    assert e.value.status == mb3dcu.EINVAL and "limit" in e.value.text
    # a host buffer is refused too (the entry point copies nothing)
    host = np.zeros(10 * sc.width, dtype=mb3dcu.SILIGHT)
    r = mb3dcu.lib().mb3d_cu_march_noalloc(mb3dcu.ctypes.byref(sc), mb3dcu.FP32_FP64, 0, 10, host.ctypes.data, None)
    assert r == mb3dcu.EINVAL
