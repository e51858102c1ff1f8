"""Python host binding of libmb3dcu.so (include/mb3d_cu.h) through ctypes.

The class `Card` mirrors the functions of mb3d-rs's card backend that the
library replaces (src/gpu.rs): `unsupported` (gpu::unsupported, :445),
`march` (gpu::march / march_bands, :2296 / :1586), `post_on_card`
(:1649), `de_probe` (:3193), plus `render` (the march and its post passes,
render::calculate_with, src/render.rs:328).  Errors raise `CardError` with
the library's status and text, the way the reference returns
`Err(String)`; there is no CPU fallback here.

Buffers are numpy arrays (host: copied inside the call) or torch CUDA
tensors (device: used in place), viewed as `SILIGHT` records.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("MB3D_CU_LIB") or os.path.join(HERE, "libmb3dcu.so")

OK, EINVAL, ENOMEM, ENODEV, EIO, ECANCELED, ETIMEDOUT, EOVERFLOW, ENOTSUP = 0, -22, -12, -19, -5, -125, -110, -75, -95

F_INTPOW, F_REALPOWER, F_TRICORN, F_AMAZINGBOX, F_BULBOX, F_FOLDINGINTPOW, F_MENGERIFS = 0, 1, 3, 4, 5, 6, 100
F_QUATERNION, F_AEXIONC = 2, 9
FP64, FP32_FP64 = 0, 1
POST_SHADOW, POST_DEAO = 1, 2


class Slot(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int32), ("formula", ctypes.c_int32), ("options", ctypes.c_double * 16)]


class Light(ctypes.Structure):
    _fields_ = [("on", ctypes.c_int32), ("pad", ctypes.c_int32), ("x_angle", ctypes.c_double),
                ("y_angle", ctypes.c_double)]


class Scene(ctypes.Structure):
    _fields_ = [
        ("width", ctypes.c_int32), ("height", ctypes.c_int32),
        ("iterations", ctypes.c_int32), ("min_iterations", ctypes.c_int32),
        ("rstop", ctypes.c_double), ("zoom", ctypes.c_double),
        ("mid", ctypes.c_double * 3),
        ("z_start", ctypes.c_double), ("z_end", ctypes.c_double),
        ("vgrads", (ctypes.c_double * 3) * 3),
        ("fov_y", ctypes.c_double), ("de_stop", ctypes.c_double), ("z_step_div", ctypes.c_double),
        ("raystep_limiter", ctypes.c_double),
        ("smooth_normals", ctypes.c_int32), ("bin_search_steps", ctypes.c_int32),
        ("first_step_random", ctypes.c_int32), ("step_sub_de_stop", ctypes.c_int32),
        ("vary_de_stop_on_fov", ctypes.c_int32), ("normals_on_de", ctypes.c_int32),
        ("disable_analytic_de", ctypes.c_int32), ("julia", ctypes.c_int32),
        ("julia_c", ctypes.c_double * 4),
        ("color_option", ctypes.c_int32), ("color_on_it", ctypes.c_int32),
        ("color_mul", ctypes.c_double),
        ("dfog_on_it", ctypes.c_int32), ("repeat_from", ctypes.c_int32),
        ("n_slots", ctypes.c_int32), ("pad0", ctypes.c_int32),
        ("slots", Slot * 6),
        ("lights", Light * 6),
        ("shadow_lights", ctypes.c_int32), ("shadow_soft", ctypes.c_int32),
        ("soft_radius", ctypes.c_float), ("hs_max_len_mul", ctypes.c_float),
        ("deao_quality", ctypes.c_int32), ("deao_dither", ctypes.c_int32),
        ("deao_max_len", ctypes.c_float), ("deao_first_step_random", ctypes.c_int32),
        ("interpolation", ctypes.c_int32), ("ipol_weights", ctypes.c_float * 2), ("pad1", ctypes.c_int32),
        ("rot_4d", ctypes.c_double * 3),
        ("decomb", ctypes.c_int32), ("decomb_end1", ctypes.c_int32), ("decomb_start2", ctypes.c_int32),
        ("decomb_end2", ctypes.c_int32), ("decomb_repeat2", ctypes.c_int32), ("decomb_iterations2", ctypes.c_int32),
        ("decomb_smooth", ctypes.c_float), ("decomb_mix_pow", ctypes.c_float), ("decomb_mix_color", ctypes.c_int32),
        ("pad2", ctypes.c_int32), ("part2_offset", ctypes.c_double * 3), ("part2_rotation", ctypes.c_double * 3),
        ("part2_scale", ctypes.c_double),
    ]


class Tune(ctypes.Structure):
    _fields_ = [("blocks_per_sm", ctypes.c_int32), ("refill_min", ctypes.c_int32), ("streams", ctypes.c_int32),
                ("pad", ctypes.c_int32)]


class Stats(ctypes.Structure):
    _fields_ = [("ms_march", ctypes.c_float), ("ms_finish", ctypes.c_float), ("ms_shadow", ctypes.c_float),
                ("ms_deao", ctypes.c_float), ("ms_total", ctypes.c_float), ("launches", ctypes.c_uint32),
                ("fp64_pixels", ctypes.c_uint32), ("de_evals", ctypes.c_uint64), ("orbit_its", ctypes.c_uint64 * 6),
                ("mc_inside_rays", ctypes.c_uint32), ("mc_fp64_rays", ctypes.c_uint32),
                ("march_lane_its", ctypes.c_uint64), ("march_warp_its", ctypes.c_uint64),
                ("march_trips", ctypes.c_uint64), ("march_busy_lanes", ctypes.c_uint64),
                ("fp32_overflow_pixels", ctypes.c_uint32), ("pad_stats", ctypes.c_uint32)]


PROGRESS_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_void_p)


class MarchOpts(ctypes.Structure):
    """mb3d_cu_march_opts: gpu::march's progress and cancel, bands, the
    device time budget and the overflow rule."""
    _fields_ = [("cancel", ctypes.c_void_p), ("progress", PROGRESS_FN), ("user", ctypes.c_void_p),
                ("band_rows", ctypes.c_uint32), ("overflow_fail", ctypes.c_int32), ("budget_ms", ctypes.c_double)]


# ---- the Monte Carlo tracer (src/mc.rs) ----
class McReq(ctypes.Structure):
    """McReq (src/mc.rs:402-437): a march of the Monte Carlo tracer."""
    _fields_ = [("pos", ctypes.c_double * 3), ("dir", ctypes.c_double * 3), ("zz", ctypes.c_double),
                ("zz2", ctypes.c_double), ("zzplus", ctypes.c_double), ("len", ctypes.c_double),
                ("seed", ctypes.c_int32), ("kind", ctypes.c_uint8), ("probe", ctypes.c_uint8),
                ("inside", ctypes.c_uint8), ("pad", ctypes.c_uint8)]


class McRes(ctypes.Structure):
    """McRes (src/mc.rs:439-467): the result of a march."""
    _fields_ = [("pos", ctypes.c_double * 3), ("normals", ctypes.c_double * 3), ("zz", ctypes.c_double),
                ("zz2", ctypes.c_double), ("len", ctypes.c_double), ("dyn_fog", ctypes.c_float),
                ("ms_de_stop", ctypes.c_float), ("seed", ctypes.c_int32), ("si_grad", ctypes.c_uint16),
                ("otrap", ctypes.c_uint16), ("kind", ctypes.c_uint8), ("de_limited", ctypes.c_uint8),
                ("inside", ctypes.c_uint8), ("pad", ctypes.c_uint8), ("pad2", ctypes.c_uint32)]


class McLight(ctypes.Structure):
    """The LightVals part the Monte Carlo shading reads (mb3d_cu_mc_light)."""
    _fields_ = [("n_lights", ctypes.c_int32), ("sqr", ctypes.c_int32),
                ("ln", (ctypes.c_float * 3) * 6), ("col", (ctypes.c_float * 3) * 6),
                ("lmax_l", ctypes.c_float * 6), ("pow_func", ctypes.c_int32 * 6),
                ("amb_col", ctypes.c_float * 3), ("amb_col2", ctypes.c_float * 3),
                ("depth_col", ctypes.c_float * 3), ("depth_col2", ctypes.c_float * 3),
                ("dyn_fog_col", ctypes.c_float * 3), ("dyn_fog_col2", ctypes.c_float * 3),
                ("s_depth", ctypes.c_float), ("s_shad", ctypes.c_float), ("s_shad_gr", ctypes.c_float),
                ("s_shad_zmul", ctypes.c_float), ("s_dyn_fog_mul", ctypes.c_float),
                ("s_diff", ctypes.c_float), ("s_spec", ctypes.c_float), ("s_col_zmul", ctypes.c_float),
                ("s_c_start", ctypes.c_float), ("s_c_mul", ctypes.c_float),
                ("col_cycling", ctypes.c_int32), ("col_on_otrap", ctypes.c_int32), ("far_fog", ctypes.c_int32),
                ("depth_func", ctypes.c_int32), ("no_col_ipol", ctypes.c_int32), ("dfog_options", ctypes.c_int32),
                ("col_pos", ctypes.c_int32 * 10), ("col_dif", (ctypes.c_float * 3) * 10),
                ("col_spe", (ctypes.c_float * 3) * 10), ("col_spe_a", ctypes.c_float * 10),
                ("s_c_div", ctypes.c_float * 10)]


class McOpts(ctypes.Structure):
    _fields_ = [("rays", ctypes.c_int32), ("ray0", ctypes.c_int32), ("depth", ctypes.c_int32),
                ("secant", ctypes.c_int32), ("soft_shadow_radius", ctypes.c_float), ("x0", ctypes.c_int32),
                ("y0", ctypes.c_int32), ("w", ctypes.c_int32), ("h", ctypes.c_int32), ("pad", ctypes.c_int32)]


class McOut(ctypes.Structure):
    _fields_ = [("radiance", ctypes.c_void_p), ("albedo", ctypes.c_void_p), ("normal", ctypes.c_void_p),
                ("depth", ctypes.c_void_p), ("hit", ctypes.c_void_p)]


class McPaintOpts(ctypes.Structure):
    """mb3d_cu_mc_paint_opts: McSettings' contrast, saturation, options and the
    lighting's gamma."""
    _fields_ = [("contrast", ctypes.c_uint8), ("saturation", ctypes.c_uint8), ("options", ctypes.c_uint8),
                ("pad", ctypes.c_uint8), ("gamma", ctypes.c_float)]


class SsaoOpts(ctypes.Structure):
    """mb3d_cu_ssao_opts: SsaoParams (src/ssao.rs:14-33), regular or random sampling."""
    _fields_ = [("threshold", ctypes.c_float), ("border_mirror", ctypes.c_float), ("t0", ctypes.c_uint8),
                ("wrap_x", ctypes.c_uint8), ("random", ctypes.c_uint8), ("pad", ctypes.c_uint8)]


class DofOpts(ctypes.Structure):
    """mb3d_cu_dof_opts: DofParams (src/dof.rs:13-31)."""
    _fields_ = [("z_sharp", ctypes.c_float), ("z_sharp2", ctypes.c_float), ("aperture", ctypes.c_float),
                ("clip_r", ctypes.c_float), ("passes", ctypes.c_uint8), ("forward", ctypes.c_uint8),
                ("pad", ctypes.c_uint8 * 2)]


def dof_default():
    """DofParams::default."""
    o = DofOpts()
    lib().mb3d_cu_dof_default(ctypes.byref(o))
    return o


def ssao_default():
    """SsaoParams::default."""
    o = SsaoOpts()
    lib().mb3d_cu_ssao_default(ctypes.byref(o))
    return o


def mc_paint_default():
    o = McPaintOpts()
    lib().mb3d_cu_mc_paint_default(ctypes.byref(o))
    return o


def mc_opts(rays, depth=3, ray0=0, secant=True, soft_shadow_radius=1.0, rect=None):
    """McSettings' defaults (src/scene.rs:607-624): depth 3, options 2 (secant)."""
    x0, y0, w, h = rect if rect is not None else (0, 0, 0, 0)
    return McOpts(rays, ray0, depth, int(bool(secant)), soft_shadow_radius, x0, y0, w, h, 0)


def mc_light_default(scene):
    """LightVals of MB3D's start-up lighting with the scene's lights."""
    lv = McLight()
    r = lib().mb3d_cu_mc_light_default(ctypes.byref(scene), ctypes.byref(lv))
    if r != 0:
        raise CardError(r, lib().mb3d_cu_last_error().decode())
    return lv


# the G-buffer record (mb3d_cu_silight, 20 bytes)
SILIGHT = np.dtype([("normal", "<i2", (3,)), ("pad", "<u2"), ("zpos_fine", "<u4"), ("shadow", "<u2"),
                    ("amb_shadow", "<u2"), ("si_gradient", "<u2"), ("otrap", "<u2")])
assert SILIGHT.itemsize == 20


# the Monte Carlo record (mb3d_cu_mc_record, McRecord: 24 bytes)
MC_RECORD = np.dtype([("col", "<f4", (3,)), ("ysum", "<f4"), ("ysqr", "<f4"), ("ray_count", "<u2"), ("hit", "u1"),
                      ("pad", "u1")])
assert MC_RECORD.itemsize == 24


# a ray of the reflection pass (mb3d_cu_reflect_ray, RayReq: 72 bytes) and
# its march (mb3d_cu_reflect_hit, RayHit: 72 bytes)
REFLECT_RAY = np.dtype([("origin", "<f8", (3,)), ("dir", "<f8", (3,)), ("zz", "<f8"), ("max_len", "<f8"),
                        ("pixel", "<u4"), ("rit", "<u4")])
assert REFLECT_RAY.itemsize == 72
REFLECT_HIT = np.dtype([("si", SILIGHT), ("hit", "u1"), ("de_limited", "u1"), ("pad", "u1", (2,)),
                        ("pos", "<f8", (3,)), ("zz", "<f8"), ("zz2_paint", "<f8"), ("zz2", "<f8")])
assert REFLECT_HIT.itemsize == 72


class CardError(RuntimeError):
    def __init__(self, status, text):
        super().__init__(f"{text} (status {status})")
        self.status = status
        self.text = text


_lib = None


def lib():
    """The loaded library; fails loudly when it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with `make -C mb3d-rs_b200`")
        L = ctypes.CDLL(LIB_PATH)
        vp, sp = ctypes.c_void_p, ctypes.POINTER(Scene)
        L.mb3d_cu_version.restype = ctypes.c_char_p
        L.mb3d_cu_last_error.restype = ctypes.c_char_p
        L.mb3d_cu_init.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
        L.mb3d_cu_free.argtypes = [vp]
        L.mb3d_cu_free.restype = None
        L.mb3d_cu_set_stream.argtypes = [vp, vp]
        L.mb3d_cu_unsupported.argtypes = [sp, ctypes.c_char_p, ctypes.c_size_t]
        L.mb3d_cu_march.argtypes = [vp, sp, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, vp, vp]
        L.mb3d_cu_march_ex.argtypes = [vp, sp, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, vp,
                                       ctypes.POINTER(MarchOpts)]
        L.mb3d_cu_post.argtypes = [vp, sp, ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, vp, vp]
        L.mb3d_cu_render.argtypes = [vp, sp, ctypes.c_int, vp, vp]
        L.mb3d_cu_de_probe.argtypes = [vp, sp, ctypes.c_int, vp, ctypes.c_uint32, vp, vp]
        L.mb3d_cu_stats_get.argtypes = [vp, ctypes.POINTER(Stats)]
        L.mb3d_cu_set_counting.argtypes = [vp, ctypes.c_int]
        L.mb3d_cu_fma_peak.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
        L.mb3d_cu_render_frames.argtypes = [vp, sp, ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(Tune), vp]
        L.mb3d_cu_autotune.argtypes = [vp, sp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, ctypes.POINTER(Tune)]
        L.mb3d_cu_march_noalloc.argtypes = [sp, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, vp, vp]
        fp = ctypes.POINTER(ctypes.c_float)
        L.mb3d_cu_dn_param_count.restype = ctypes.c_size_t
        L.mb3d_cu_dn_create.argtypes = [vp, ctypes.c_uint64, ctypes.POINTER(vp)]
        L.mb3d_cu_dn_free.argtypes = [vp]
        L.mb3d_cu_dn_free.restype = None
        L.mb3d_cu_dn_get_params.argtypes = [vp, vp]
        L.mb3d_cu_dn_set_params.argtypes = [vp, vp]
        L.mb3d_cu_dn_set_loss.argtypes = [vp, ctypes.c_int]
        L.mb3d_cu_dn_fallback.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, vp, vp, ctypes.c_int, ctypes.c_float, vp,
                                          vp]
        L.mb3d_cu_dn_denoise.argtypes = [vp] + [ctypes.c_int] * 3 + [vp] * 4 + [ctypes.c_float, vp]
        L.mb3d_cu_dn_train_step.argtypes = [vp] + [ctypes.c_int] * 3 + [vp] * 4 + [ctypes.c_float, vp, ctypes.c_float, fp]
        L.mb3d_cu_dn_gradient.argtypes = [vp] + [ctypes.c_int] * 3 + [vp] * 4 + [ctypes.c_float, vp, fp, vp]
        L.mb3d_cu_dn_conv_check.argtypes = [vp] + [ctypes.c_int] * 5 + [vp] * 8
        L.mb3d_cu_dn_wait_check.argtypes = [vp, ctypes.c_double, ctypes.c_int]
        L.mb3d_cu_mc_light_default.argtypes = [sp, ctypes.POINTER(McLight)]
        L.mb3d_cu_mc_batch.argtypes = [vp, sp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_uint32, vp]
        L.mb3d_cu_mc_render.argtypes = [vp, sp, ctypes.POINTER(McLight), ctypes.POINTER(McOpts), ctypes.c_int,
                                        ctypes.POINTER(McOut), vp]
        L.mb3d_cu_mc_pass.argtypes = [vp, sp, ctypes.POINTER(McLight), ctypes.POINTER(McOpts), ctypes.c_int,
                                      ctypes.c_uint32, vp, vp]
        L.mb3d_cu_mc_paint_default.argtypes = [ctypes.POINTER(McPaintOpts)]
        L.mb3d_cu_mc_paint_default.restype = None
        L.mb3d_cu_mc_paint.argtypes = [vp, vp, vp, ctypes.c_uint32, ctypes.POINTER(McPaintOpts), vp]
        L.mb3d_cu_paint.argtypes = [vp, sp, vp, ctypes.c_uint32, ctypes.c_uint32, vp]
        L.mb3d_cu_dof_default.argtypes = [ctypes.POINTER(DofOpts)]
        L.mb3d_cu_dof_default.restype = None
        L.mb3d_cu_dof.argtypes = [vp, sp, ctypes.POINTER(DofOpts), vp, vp]
        L.mb3d_cu_ssao_default.argtypes = [ctypes.POINTER(SsaoOpts)]
        L.mb3d_cu_ssao_default.restype = None
        L.mb3d_cu_ssao24.argtypes = [vp, sp, ctypes.POINTER(SsaoOpts), vp]
        L.mb3d_cu_ssao15.argtypes = [vp, sp, ctypes.POINTER(SsaoOpts), vp]
        L.mb3d_cu_reflect_batch.argtypes = [vp, sp, vp, ctypes.c_uint32, ctypes.c_int, vp]
        L.mb3d_cu_reflect_first_rays.argtypes = [vp, sp, vp, vp, vp]
        _lib = L
    return _lib


EXPORTED = ["mb3d_cu_version", "mb3d_cu_last_error", "mb3d_cu_init", "mb3d_cu_free", "mb3d_cu_set_stream",
            "mb3d_cu_unsupported", "mb3d_cu_march", "mb3d_cu_march_ex", "mb3d_cu_post", "mb3d_cu_render", "mb3d_cu_de_probe",
            "mb3d_cu_stats_get", "mb3d_cu_set_counting", "mb3d_cu_fma_peak", "mb3d_cu_march_noalloc", "mb3d_cu_render_frames",
            "mb3d_cu_autotune", "mb3d_cu_mc_light_default", "mb3d_cu_mc_batch", "mb3d_cu_mc_render", "mb3d_cu_mc_pass",
            "mb3d_cu_mc_paint_default", "mb3d_cu_mc_paint", "mb3d_cu_paint", "mb3d_cu_ssao_default", "mb3d_cu_ssao24", "mb3d_cu_ssao15", "mb3d_cu_reflect_batch", "mb3d_cu_reflect_first_rays", "mb3d_cu_dof_default", "mb3d_cu_dof",
            "mb3d_cu_dn_param_count", "mb3d_cu_dn_create", "mb3d_cu_dn_free", "mb3d_cu_dn_get_params",
            "mb3d_cu_dn_set_params", "mb3d_cu_dn_set_loss", "mb3d_cu_dn_fallback", "mb3d_cu_dn_denoise", "mb3d_cu_dn_train_step", "mb3d_cu_dn_gradient",
            "mb3d_cu_dn_conv_check", "mb3d_cu_dn_wait_check"]

NOALLOC_MAX_PIXELS = 65536


def march_noalloc(scene, out, precision=FP32_FP64, row0=0, rows=None, stream=None):
    """mb3d_cu_march_noalloc: the march into a device buffer `out` (a torch
    CUDA tensor of rows * width * 20 bytes) with no device allocation; the
    work is queued on `stream` (a cudaStream_t handle, None: default)."""
    rows = scene.height - row0 if rows is None else rows
    r = lib().mb3d_cu_march_noalloc(ctypes.byref(scene), precision, row0, rows, out.data_ptr(),
                                    ctypes.c_void_p(stream) if stream else None)
    if r != 0:
        raise CardError(r, lib().mb3d_cu_last_error().decode())
    return out


def _ptr(buf):
    """(pointer, is_torch) of a numpy array or a torch tensor."""
    if isinstance(buf, np.ndarray):
        assert buf.flags["C_CONTIGUOUS"]
        return buf.ctypes.data, False
    return buf.data_ptr(), True


def unsupported(scene):
    """gpu::unsupported: None when the card renders the scene, else the reason."""
    reason = ctypes.create_string_buffer(256)
    r = lib().mb3d_cu_unsupported(ctypes.byref(scene), reason, 256)
    if r < 0:
        raise CardError(r, lib().mb3d_cu_last_error().decode())
    return reason.value.decode() if r == 1 else None


class Card:
    """One device context (its own CUDA stream)."""

    def __init__(self, device=0):
        self._ctx = ctypes.c_void_p()
        self._stream = None
        r = lib().mb3d_cu_init(device, ctypes.byref(self._ctx))
        self._check(r)

    def _order(self, *bufs):
        """Device buffers from torch: the library's stream does not wait for
        torch's, so torch's pending work on them (fills, copies, gathers)
        finishes first, unless the card already runs on torch's stream."""
        if any(b is not None and not isinstance(b, np.ndarray) for b in bufs):
            import torch
            cs = torch.cuda.current_stream()
            if self._stream != cs.cuda_stream:
                cs.synchronize()

    def close(self):
        if self._ctx:
            lib().mb3d_cu_free(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _check(r):
        if r != 0:
            raise CardError(r, lib().mb3d_cu_last_error().decode())

    def set_stream(self, stream_handle):
        self._check(lib().mb3d_cu_set_stream(self._ctx, ctypes.c_void_p(stream_handle or None)))
        self._stream = stream_handle or None

    def march(self, scene, precision=FP32_FP64, row0=0, rows=None, out=None, cancel=None):
        rows = scene.height - row0 if rows is None else rows
        if out is None:
            out = np.zeros(rows * scene.width, dtype=SILIGHT)
        p, _ = _ptr(out)
        self._order(out)
        cp = ctypes.cast(ctypes.byref(cancel), ctypes.c_void_p) if cancel is not None else None
        self._check(lib().mb3d_cu_march(self._ctx, ctypes.byref(scene), precision, row0, rows, p, cp))
        return out

    def march_ex(self, scene, precision=FP32_FP64, row0=0, rows=None, out=None, band_rows=0, budget_ms=0.0,
                 overflow_fail=False, progress=None, cancel=None):
        """gpu::march with progress (a callable (rows_done, rows_total) -> bool,
        True cancels), bands, the device time budget (CardError with status
        ETIMEDOUT when it runs out: the same call again goes on) and the
        reference card's overflow rule."""
        rows = scene.height - row0 if rows is None else rows
        if out is None:
            out = np.zeros(rows * scene.width, dtype=SILIGHT)
        p, _ = _ptr(out)
        self._order(out)
        o = MarchOpts()
        o.band_rows, o.overflow_fail, o.budget_ms = band_rows, int(bool(overflow_fail)), budget_ms
        if cancel is not None:
            o.cancel = ctypes.cast(ctypes.byref(cancel), ctypes.c_void_p)
        cb = None
        if progress is not None:
            cb = PROGRESS_FN(lambda done, total, user: 1 if progress(done, total) else 0)
            o.progress = cb
        self._check(lib().mb3d_cu_march_ex(self._ctx, ctypes.byref(scene), precision, row0, rows, p, ctypes.byref(o)))
        return out

    def post_on_card(self, scene, gbuf, passes=POST_SHADOW | POST_DEAO, precision=FP32_FP64, row0=0, rows=None):
        rows = scene.height - row0 if rows is None else rows
        p, _ = _ptr(gbuf)
        self._order(gbuf)
        self._check(lib().mb3d_cu_post(self._ctx, ctypes.byref(scene), precision, passes, row0, rows, p, None))
        return gbuf

    def render(self, scene, precision=FP32_FP64, out=None):
        if out is None:
            out = np.zeros(scene.height * scene.width, dtype=SILIGHT)
        p, _ = _ptr(out)
        self._order(out)
        self._check(lib().mb3d_cu_render(self._ctx, ctypes.byref(scene), precision, p, None))
        return out

    def de_probe(self, scene, pos, precision=FP64):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        n = len(pos)
        de = np.zeros(n, np.float64)
        its = np.zeros(n, np.int32)
        self._check(lib().mb3d_cu_de_probe(self._ctx, ctypes.byref(scene), precision, pos.ctypes.data, n,
                                           de.ctypes.data, its.ctypes.data))
        return de, its

    def stats(self):
        s = Stats()
        self._check(lib().mb3d_cu_stats_get(self._ctx, ctypes.byref(s)))
        d = {k: getattr(s, k) for k, _ in Stats._fields_}
        d["orbit_its"] = list(s.orbit_its)
        return d

    def render_frames(self, frames, precision=FP32_FP64, tune=None, out=None):
        """All frames (a list of scenes of one size) in one CUDA graph."""
        arr = (Scene * len(frames))(*frames)
        npix = frames[0].width * frames[0].height
        if out is None:
            out = np.zeros(len(frames) * npix, dtype=SILIGHT)
        p, _ = _ptr(out)
        self._order(out)
        self._check(lib().mb3d_cu_render_frames(self._ctx, arr, len(frames), precision,
                                                ctypes.byref(tune) if tune is not None else None, p))
        return out

    def autotune(self, frames, sample=8, precision=FP32_FP64):
        arr = (Scene * len(frames))(*frames)
        t = Tune()
        self._check(lib().mb3d_cu_autotune(self._ctx, arr, len(frames), sample, precision, ctypes.byref(t)))
        return t

    def mc_batch(self, scene, reqs, precision=FP64, secant=True):
        """gpu::mc_batch: the marches `reqs` (a ctypes array of McReq)."""
        n = len(reqs)
        res = (McRes * n)()
        self._check(lib().mb3d_cu_mc_batch(self._ctx, ctypes.byref(scene), precision, int(bool(secant)),
                                           ctypes.addressof(reqs), n, ctypes.addressof(res)))
        return res

    def mc_paint(self, colour, opts=None, rays=None, out=None):
        """paint_recs on the card: colours (..., 3) float32 (numpy, or a torch
        CUDA tensor) to 8-bit RGB (..., 3); `rays` marks pixels with rays."""
        opts = mc_paint_default() if opts is None else opts
        if isinstance(colour, np.ndarray):
            colour = np.ascontiguousarray(colour, dtype=np.float32)
        if out is None:
            out = np.zeros(tuple(colour.shape[:-1]) + (3,), np.uint8)
        if rays is not None and isinstance(rays, np.ndarray):
            rays = np.ascontiguousarray(rays, dtype=np.uint8)
        n = int(np.prod(colour.shape[:-1]))
        self._order(colour, rays, out)
        self._check(lib().mb3d_cu_mc_paint(self._ctx, _ptr(colour)[0], None if rays is None else _ptr(rays)[0], n,
                                           ctypes.byref(opts), _ptr(out)[0]))
        return out

    def paint(self, scene, gbuf, row0=0, out=None):
        """render::paint on the card: 8-bit RGB (rows, width, 3) of G-buffer
        records (numpy SILIGHT array or a torch CUDA byte tensor of rows *
        width records) with the default lighting; `out` may be a torch CUDA
        tensor."""
        if isinstance(gbuf, np.ndarray):
            gbuf = np.ascontiguousarray(gbuf)
            rows = gbuf.size // scene.width
        else:
            rows = gbuf.numel() * gbuf.element_size() // (SILIGHT.itemsize * scene.width)
        if out is None:
            out = np.zeros((rows, scene.width, 3), np.uint8)
        self._order(gbuf, out)
        self._check(lib().mb3d_cu_paint(self._ctx, ctypes.byref(scene), _ptr(gbuf)[0], row0, rows, _ptr(out)[0]))
        return out

    def dof(self, scene, gbuf, rgb, opts=None):
        """dof::apply on the card: the depth of field of an 8-bit picture
        (h, w, 3) of the G-buffer gbuf.  A numpy picture is returned as a new
        array; a torch CUDA tensor is changed in place (and returned)."""
        opts = dof_default() if opts is None else opts
        if isinstance(rgb, np.ndarray):
            rgb = np.ascontiguousarray(rgb, dtype=np.uint8).copy()
        if isinstance(gbuf, np.ndarray):
            gbuf = np.ascontiguousarray(gbuf)
        self._order(gbuf, rgb)
        self._check(lib().mb3d_cu_dof(self._ctx, ctypes.byref(scene), ctypes.byref(opts), _ptr(gbuf)[0], _ptr(rgb)[0]))
        return rgb

    def ssao24(self, scene, gbuf, opts=None):
        """gpu::ssao24 on the card: the G-buffer's amb_shadow from its depth
        buffer.  A numpy G-buffer is returned as a new array; a torch CUDA
        byte tensor is changed in place (and returned)."""
        opts = ssao_default() if opts is None else opts
        if isinstance(gbuf, np.ndarray):
            gbuf = np.ascontiguousarray(gbuf).copy()
        self._order(gbuf)
        self._check(lib().mb3d_cu_ssao24(self._ctx, ctypes.byref(scene), ctypes.byref(opts), _ptr(gbuf)[0]))
        return gbuf

    def reflect_batch(self, scene, rays, far_fog=False, out=None):
        """gpu::reflect_batch on the card: every ray of `rays` (REFLECT_RAY,
        numpy or a torch CUDA byte tensor) marched to its hit with the hit's
        normal, colour, depth, shadows and DE ambient occlusion; returns the
        hits (REFLECT_HIT; `out` may give a device buffer)."""
        n = len(rays) if isinstance(rays, np.ndarray) else rays.numel() // REFLECT_RAY.itemsize
        if isinstance(rays, np.ndarray):
            rays = np.ascontiguousarray(rays, REFLECT_RAY)
        if out is None:
            out = np.zeros(n, REFLECT_HIT)
        self._order(rays, out)
        self._check(lib().mb3d_cu_reflect_batch(self._ctx, ctypes.byref(scene), _ptr(rays)[0], n, int(far_fog),
                                                _ptr(out)[0]))
        return out

    def reflect_first_rays(self, scene, gbuf, out=None):
        """mb3d_cu_reflect_first_rays: the first bounce of every object pixel
        (REFLECT_RAY, pixel order).  A numpy G-buffer gives a numpy array of
        the rays; with device buffers (`out`: a torch CUDA byte tensor with
        room for width * height rays) returns (out, count)."""
        n = ctypes.c_uint32()
        if out is None:
            buf = np.zeros(scene.width * scene.height, REFLECT_RAY)
            if not isinstance(gbuf, np.ndarray):
                raise ValueError("device G-buffer: give `out`")
            g = np.ascontiguousarray(gbuf)
            self._check(lib().mb3d_cu_reflect_first_rays(self._ctx, ctypes.byref(scene), _ptr(g)[0], _ptr(buf)[0],
                                                         ctypes.byref(n)))
            return buf[:n.value].copy()
        self._order(gbuf, out)
        self._check(lib().mb3d_cu_reflect_first_rays(self._ctx, ctypes.byref(scene), _ptr(gbuf)[0], _ptr(out)[0],
                                                     ctypes.byref(n)))
        return out, n.value

    def ssao15(self, scene, gbuf, opts=None):
        """gpu::ssao15 on the card: the older 15-bit ambient occlusion
        (threshold, t0 and wrap_x of opts); a numpy G-buffer is returned as a
        new array, a torch CUDA byte tensor is changed in place."""
        opts = ssao_default() if opts is None else opts
        if isinstance(gbuf, np.ndarray):
            gbuf = np.ascontiguousarray(gbuf).copy()
        self._order(gbuf)
        self._check(lib().mb3d_cu_ssao15(self._ctx, ctypes.byref(scene), ctypes.byref(opts), _ptr(gbuf)[0]))
        return gbuf

    def mc_render(self, scene, opts, light=None, precision=FP32_FP64, out=None, cancel=None):
        """The Monte Carlo rays of opts on the card: a dict of radiance, albedo,
        normal (h, w, 3), depth (h, w) and hit (h, w); `out` may give torch CUDA
        tensors (float32; hit uint8) for any of them, used in place."""
        light = mc_light_default(scene) if light is None else light
        w, h = (opts.w, opts.h) if opts.w else (scene.width, scene.height)
        res = dict(out or {})
        for k, shape, dt in (("radiance", (h, w, 3), np.float32), ("albedo", (h, w, 3), np.float32),
                             ("normal", (h, w, 3), np.float32), ("depth", (h, w), np.float32),
                             ("hit", (h, w), np.uint8)):
            if k not in res:
                res[k] = np.zeros(shape, dt)
        ptrs = McOut(*[_ptr(res[k])[0] if res[k] is not None else None
                       for k in ("radiance", "albedo", "normal", "depth", "hit")])
        self._order(*res.values())
        cp = ctypes.cast(ctypes.byref(cancel), ctypes.c_void_p) if cancel is not None else None
        self._check(lib().mb3d_cu_mc_render(self._ctx, ctypes.byref(scene), ctypes.byref(light), ctypes.byref(opts),
                                            precision, ctypes.byref(ptrs), cp))
        return res

    def mc_pass(self, scene, opts, recs, pass_nr, light=None, precision=FP32_FP64, cancel=None):
        """mc::pass: one adaptive pass over the picture; recs (width * height
        MC_RECORD, numpy or a torch CUDA byte tensor) is updated in place."""
        light = mc_light_default(scene) if light is None else light
        if isinstance(recs, np.ndarray):
            assert recs.dtype == MC_RECORD and recs.flags["C_CONTIGUOUS"] and recs.size == scene.width * scene.height
        self._order(recs)
        cp = ctypes.cast(ctypes.byref(cancel), ctypes.c_void_p) if cancel is not None else None
        self._check(lib().mb3d_cu_mc_pass(self._ctx, ctypes.byref(scene), ctypes.byref(light), ctypes.byref(opts),
                                          precision, pass_nr, _ptr(recs)[0], cp))
        return recs

    def set_counting(self, on):
        self._check(lib().mb3d_cu_set_counting(self._ctx, int(on)))

    def fma_peak(self, fp64=False):
        t = ctypes.c_double()
        self._check(lib().mb3d_cu_fma_peak(self._ctx, int(fp64), ctypes.byref(t)))
        return t.value


def is_background(g):
    return (g["zpos_fine"] >> 16) >= 32768


def hit_mask(g):
    """Pixels with a surface (not background, not the start-inside cut)."""
    return ((g["zpos_fine"] >> 16) < 32768) & (g["si_gradient"] < 32768)


def depth_steps(g, scene_params):
    """mzz (depth in step widths) of each record from its zpos (src/calc.rs:2166-2167)."""
    zf = (g["zpos_fine"] >> 8).astype(np.float64)
    zc_mul, zcorr = scene_params
    return (((8388351.5 - zf) / zc_mul + 1.0) ** 2 - 1.0) / zcorr


def _fptr(a):
    """A float32 buffer's pointer (numpy array or torch CUDA tensor), or None."""
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
        return a.ctypes.data
    assert a.is_contiguous()
    return a.data_ptr()


class Denoiser:
    """The Monte Carlo pictures' denoiser (mb3d_cu_dn_*): a BF16 U-Net on the
    card, the counterpart of mb3d-rs's Open Image Denoise call
    (denoise_mc, src/oidn.rs:262-277).  Arrays are (n, h, w, 3) float32 (depth
    (n, h, w)), numpy or torch CUDA tensors."""

    def __init__(self, card, seed=1):
        self.card = card
        self._d = ctypes.c_void_p()
        card._check(lib().mb3d_cu_dn_create(card._ctx, seed, ctypes.byref(self._d)))
        self.n_params = lib().mb3d_cu_dn_param_count()

    def close(self):
        if self._d:
            lib().mb3d_cu_dn_free(self._d)
            self._d = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self):
        p = np.zeros(self.n_params, np.float32)
        self.card._check(lib().mb3d_cu_dn_get_params(self._d, p.ctypes.data))
        return p

    LOSS_L1_LOG, LOSS_TONE_MSE, LOSS_TONE_DISPLAY = 0, 1, 2

    def set_loss(self, kind):
        """The training loss: LOSS_L1_LOG (default), LOSS_TONE_MSE or
        LOSS_TONE_DISPLAY."""
        self.card._check(lib().mb3d_cu_dn_set_loss(self._d, kind))

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.size == self.n_params
        self.card._check(lib().mb3d_cu_dn_set_params(self._d, p.ctypes.data))

    @staticmethod
    def _shape(radiance):
        s = tuple(radiance.shape)
        return (1,) + s[:2] if len(s) == 3 else s[:3]

    def denoise(self, radiance, albedo=None, normal=None, depth=None, depth_scale=None, out=None):
        n, h, w = self._shape(radiance)
        if depth_scale is None:
            depth_scale = _depth_scale(depth)
        if out is None:
            out = np.zeros((n, h, w, 3), np.float32) if isinstance(radiance, np.ndarray) else radiance.new_zeros((n, h, w, 3))
        self.card._order(radiance, albedo, normal, depth, out)
        self.card._check(lib().mb3d_cu_dn_denoise(self._d, n, h, w, _fptr(radiance), _fptr(albedo), _fptr(normal),
                                                  _fptr(depth), depth_scale, _fptr(out)))
        return out

    def fallback(self, half_a, half_b, den, tile=16, k=3.0, out=None):
        """mb3d_cu_dn_fallback: the pieces of den whose mean leaves the plain
        trace's ((half_a + half_b) / 2, two traces from disjoint halves of
        the rays) by more than k times its noise keep the plain trace.
        Pictures (h, w, 3) float32, numpy or torch CUDA tensors.  Returns
        (picture, share of the pieces that keep the plain trace)."""
        h, w = int(den.shape[0]), int(den.shape[1])
        if isinstance(den, np.ndarray):
            half_a, half_b, den = (np.ascontiguousarray(a, np.float32) for a in (half_a, half_b, den))
        if out is None:
            out = np.zeros((h, w, 3), np.float32) if isinstance(den, np.ndarray) else den.new_zeros((h, w, 3))
        share = ctypes.c_float()
        self.card._order(half_a, half_b, den, out)
        self.card._check(lib().mb3d_cu_dn_fallback(self._d, h, w, _fptr(half_a), _fptr(half_b), _fptr(den), tile, k,
                                                   _fptr(out), ctypes.byref(share)))
        return out, share.value

    def train_step(self, radiance, target, albedo=None, normal=None, depth=None, depth_scale=None, lr=1e-3):
        n, h, w = self._shape(radiance)
        if depth_scale is None:
            depth_scale = _depth_scale(depth)
        loss = ctypes.c_float()
        self.card._order(radiance, target, albedo, normal, depth)
        self.card._check(lib().mb3d_cu_dn_train_step(self._d, n, h, w, _fptr(radiance), _fptr(albedo), _fptr(normal),
                                                     _fptr(depth), depth_scale, _fptr(target), lr, ctypes.byref(loss)))
        return loss.value

    def gradient(self, radiance, target, albedo=None, normal=None, depth=None, depth_scale=1.0):
        n, h, w = self._shape(radiance)
        loss = ctypes.c_float()
        g = np.zeros(self.n_params, np.float32)
        self.card._order(radiance, target, albedo, normal, depth)
        self.card._check(lib().mb3d_cu_dn_gradient(self._d, n, h, w, _fptr(radiance), _fptr(albedo), _fptr(normal),
                                                   _fptr(depth), depth_scale, _fptr(target), ctypes.byref(loss),
                                                   g.ctypes.data))
        return loss.value, g


def _depth_scale(depth):
    """1 / the largest depth (the guides' depth about 0..1)."""
    if depth is None:
        return 1.0
    m = float(depth.max())
    return 1.0 / m if m > 0 else 1.0


def conv_check(card, x, w, b, dy):
    """mb3d_cu_dn_conv_check: y, dx, dw, db of one 3x3 convolution."""
    n, h, ww, cin = x.shape
    cout = w.shape[0]
    x, w, b, dy = (np.ascontiguousarray(a, np.float32) for a in (x, w, b, dy))
    y = np.zeros((n, h, ww, cout), np.float32)
    dx = np.zeros_like(x)
    dw = np.zeros_like(w)
    db = np.zeros_like(b)
    card._check(lib().mb3d_cu_dn_conv_check(card._ctx, n, h, ww, cin, cout, x.ctypes.data, w.ctypes.data, b.ctypes.data,
                                            dy.ctypes.data, y.ctypes.data, dx.ctypes.data, dw.ctypes.data,
                                            db.ctypes.data))
    return y, dx, dw, db
