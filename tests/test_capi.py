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
    s.slots[0].formula = 2  # Quaternion: a 4D formula, on this card (the sequential FP64 DE)
    assert mb3dcu.unsupported(s) is None
    s.slots[0].formula = 7  # (no formula 7: not on this card)
    r = mb3dcu.unsupported(s)
    assert r and "formula" in r
    s.n_slots = 0
    try:
        mb3dcu.unsupported(s)
        assert False, "a bad scene must raise"
    except mb3dcu.CardError as e:
        assert e.status == mb3dcu.EINVAL


def test_de_combination_checks_on_the_host():
    """A DE combination (src/calc.rs:421-431,491-520) of kinds 1..5 is on the
    card; 'mix' without a dIFS part 2 and kinds beyond 6 are errors; a 4D
    part is not on the card; a combination whose part 1 ends at the last
    slot is none."""
    for kind in scenes.DECOMB_KINDS:
        assert mb3dcu.unsupported(scenes.two_objects(kind)) is None, kind
    for kind in (6, 7, -1):
        s = scenes.two_objects("min")
        s.decomb = kind
        try:
            mb3dcu.unsupported(s)
            assert False, kind
        except mb3dcu.CardError as e:
            assert e.status == mb3dcu.EINVAL
            if kind == 6:
                assert "dIFS" in str(e)
    s = scenes.two_objects("min")
    s.slots[1].formula = mb3dcu.F_QUATERNION
    r = mb3dcu.unsupported(s)
    assert r and "4D" in r
    s = scenes.two_objects("min")
    s.decomb_end1 = 1  # (part 1 takes every slot: no combination)
    assert mb3dcu.unsupported(s) is None


def test_init_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        return
    try:
        mb3dcu.Card(0)
        assert False
    except mb3dcu.CardError as e:
        assert e.status in (mb3dcu.ENODEV, mb3dcu.EIO)


# the ctypes mirrors of the header's structs (C name, ctypes class)
MIRRORS = [("mb3d_cu_slot", "Slot"), ("mb3d_cu_light", "Light"), ("mb3d_cu_scene", "Scene"),
           ("mb3d_cu_stats", "Stats"), ("mb3d_cu_tune", "Tune"), ("mb3d_cu_mc_req", "McReq"),
           ("mb3d_cu_mc_res", "McRes"), ("mb3d_cu_mc_light", "McLight"), ("mb3d_cu_mc_opts", "McOpts"),
           ("mb3d_cu_mc_out", "McOut"), ("mb3d_cu_mc_paint_opts", "McPaintOpts"), ("mb3d_cu_ssao_opts", "SsaoOpts"),
           ("mb3d_cu_march_opts", "MarchOpts"), ("mb3d_cu_dof_opts", "DofOpts")]


# the numpy record types of the header's records (C name, dtype name)
DTYPES = [("mb3d_cu_silight", "SILIGHT"), ("mb3d_cu_mc_record", "MC_RECORD"), ("mb3d_cu_reflect_ray", "REFLECT_RAY"),
          ("mb3d_cu_reflect_hit", "REFLECT_HIT")]


def test_every_struct_mirror_matches_the_header(tmp_path):
    """Size and every field offset of each ctypes mirror against the C
    compiler's layout of include/mb3d_cu.h (gcc, the host ABI)."""
    import subprocess
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "mb3d_cu.h"', "int main(void) {"]
    for cname, pyname in MIRRORS:
        cls = getattr(mb3dcu, pyname)
        lines.append(f'printf("{pyname} size %zu\\n", sizeof({cname}));')
        for f in cls._fields_:
            lines.append(f'printf("{pyname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    for cname, dname in DTYPES:
        dt = getattr(mb3dcu, dname)
        lines.append(f'printf("{dname} size %zu\\n", sizeof({cname}));')
        for f in dt.names:
            lines.append(f'printf("{dname} {f} %zu\\n", offsetof({cname}, {f}));')
    lines.append("return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    checked = 0
    for line in out:
        if not line:
            continue
        pyname, field, value = line.split()
        cls = getattr(mb3dcu, pyname)
        if isinstance(cls, np.dtype):
            want = cls.itemsize if field == "size" else cls.fields[field][1]
        else:
            want = ctypes.sizeof(cls) if field == "size" else getattr(cls, field).offset
        assert want == int(value), (pyname, field, want, value)
        checked += 1
    assert checked > 100


def test_null_arguments_fail_on_the_host():
    """Every entry point answers a missing context or buffer with EINVAL and
    a reason, before it touches a device (the reference's Err(String))."""
    L = mb3dcu.lib()
    sc = scenes.preset("Integer Power", 64, 48)
    buf = np.zeros(64 * 48, dtype=mb3dcu.SILIGHT)
    rgb = np.zeros((48, 64, 3), np.uint8)
    col = np.zeros((48, 64, 3), np.float32)
    calls = [
        lambda: L.mb3d_cu_march(None, ctypes.byref(sc), mb3dcu.FP64, 0, 48, buf.ctypes.data, None),
        lambda: L.mb3d_cu_post(None, ctypes.byref(sc), mb3dcu.FP64, mb3dcu.POST_SHADOW, 0, 48, buf.ctypes.data, None),
        lambda: L.mb3d_cu_paint(None, ctypes.byref(sc), buf.ctypes.data, 0, 48, rgb.ctypes.data),
        lambda: L.mb3d_cu_mc_paint(None, col.ctypes.data, None, 64 * 48, ctypes.byref(mb3dcu.mc_paint_default()),
                                   rgb.ctypes.data),
        lambda: L.mb3d_cu_ssao24(None, ctypes.byref(sc), ctypes.byref(mb3dcu.ssao_default()), buf.ctypes.data),
        lambda: L.mb3d_cu_ssao15(None, ctypes.byref(sc), ctypes.byref(mb3dcu.ssao_default()), buf.ctypes.data),
        lambda: L.mb3d_cu_reflect_batch(None, ctypes.byref(sc), None, 1, 0, None),
        lambda: L.mb3d_cu_reflect_first_rays(None, ctypes.byref(sc), buf.ctypes.data, None, None),
        lambda: L.mb3d_cu_dn_fallback(None, 48, 64, col.ctypes.data, col.ctypes.data, col.ctypes.data, 16, 3.0,
                                      col.ctypes.data, None),
    ]
    for call in calls:
        assert call() == mb3dcu.EINVAL
        assert L.mb3d_cu_last_error()


def test_display_and_light_defaults_on_the_host():
    o = mb3dcu.mc_paint_default()
    assert (o.contrast, o.saturation, o.options, o.gamma) == (128, 32, 2, 32.0)
    a = mb3dcu.ssao_default()
    assert (a.threshold, a.border_mirror, a.t0, a.wrap_x) == (2.0, 0.0, 0, 0)
    lv = mb3dcu.mc_light_default(scenes.c5_mc())
    assert lv is not None
    bad = scenes.preset("Integer Power", 64, 48)
    bad.width = 0
    try:
        mb3dcu.mc_light_default(bad)
        assert False, "a picture without pixels must raise"
    except mb3dcu.CardError as e:
        assert e.status == mb3dcu.EINVAL
