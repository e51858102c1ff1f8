"""The C ABI library on the host (no GPU needed): it loads, exports every
entry point include/mb3d_cu.h declares, and its host-side checks
(gpu::unsupported, src/gpu.rs:445) answer without a device."""
import ctypes
import os
import re

import numpy as np

import mb3dcu
import scenes

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    txt = open(os.path.join(ROOT, "include", "mb3d_cu.h")).read()
    return sorted(set(re.findall(r"\b(mb3d_cu_[a-z_0-9]+)\s*\(", txt)))


def test_library_loads_and_exports_every_declared_symbol():
    L = mb3dcu.lib()
    names = declared()
    assert len(names) >= 10
    for n in names:
        assert hasattr(L, n), n
    assert set(names) <= set(mb3dcu.EXPORTED)
    assert b"sm_100a" in L.mb3d_cu_version()


def test_struct_layout_matches_header():
    assert ctypes.sizeof(mb3dcu.Slot) == 8 + 16 * 8
    assert mb3dcu.SILIGHT.itemsize == 20
    assert mb3dcu.Scene.slots.offset % 8 == 0


def test_unsupported_answers_on_the_host():
    assert mb3dcu.unsupported(scenes.c2_hybrid()) is None
    assert mb3dcu.unsupported(scenes.c1_plain_bulb()) is None
    s = scenes.default_scene()
    s.slots[0].formula = 2  # Quaternion: a 4D formula, not on this card
    r = mb3dcu.unsupported(s)
    assert r and "formula" in r
    s.n_slots = 0
    try:
        mb3dcu.unsupported(s)
        assert False, "a bad scene must raise"
    except mb3dcu.CardError as e:
        assert e.status == mb3dcu.EINVAL


def test_init_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        return
    try:
        mb3dcu.Card(0)
        assert False
    except mb3dcu.CardError as e:
        assert e.status in (mb3dcu.ENODEV, mb3dcu.EIO)
