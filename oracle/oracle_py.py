"""TEST INFRASTRUCTURE: ctypes binding of the parity oracle (liboracle.so,
the C++ restatement of mb3d-rs's CPU march).  Only the tests, the smoke
check and the benchmark's CPU-baseline leg load it; the product never does.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = ctypes.CDLL(LIB)
        vp = ctypes.c_void_p
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_params.argtypes = [vp, vp, ctypes.c_int]
        L.oracle_pixel_seed.argtypes = [ctypes.c_int64, ctypes.c_int64]
        L.oracle_pixel_seed.restype = ctypes.c_int32
        L.oracle_formula_iterate.argtypes = [ctypes.c_int, vp, vp, vp, ctypes.c_double, ctypes.c_int]
        L.oracle_de_at.argtypes = [vp, vp, ctypes.c_int, vp, vp]
        L.oracle_march.argtypes = [vp, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int, vp]
        L.oracle_march_pixels.argtypes = [vp, vp, ctypes.c_int, vp, ctypes.c_int]
        L.oracle_shadows.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int]
        L.oracle_deao.argtypes = [vp, vp, ctypes.c_int]
        L.oracle_ao_rays.argtypes = [ctypes.c_int, vp, ctypes.c_int]
        L.oracle_render_rows.argtypes = [vp, vp, ctypes.c_int, vp, ctypes.c_int]
        L.oracle_mc_render.argtypes = [vp, vp, vp, vp, vp, vp, vp, vp, vp, ctypes.c_int]
        L.oracle_mc_batch.argtypes = [vp, ctypes.c_int, vp, ctypes.c_uint32, vp, ctypes.c_int]
        L.oracle_mc_pass.argtypes = [vp, vp, vp, ctypes.c_uint32, vp, ctypes.c_int]
        L.oracle_dof.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_double, vp, ctypes.c_int]
        L.oracle_mc_halton.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, vp]
        L.oracle_mc_halton.restype = None
        L.oracle_mc_seed_of.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_uint32]
        L.oracle_mc_seed_of.restype = ctypes.c_int32
        L.oracle_mc_paint.argtypes = [vp, vp, ctypes.c_size_t, vp, vp]
        L.oracle_mc_paint.restype = None
        L.oracle_paint.argtypes = [vp, vp, ctypes.c_int, ctypes.c_int, vp]
        L.oracle_ssao24.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_reflect_batch.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_int, vp, ctypes.c_int]
        L.oracle_reflect_first_rays.argtypes = [vp, vp, vp, ctypes.c_uint32]
        L.oracle_ssao15.argtypes = [vp, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_float,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.oracle_ssao15_arctan.argtypes = [ctypes.c_int, ctypes.c_int]
        L.oracle_ssao15_axis.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, vp, ctypes.c_int]
        L.oracle_ssao_levels.argtypes = [ctypes.c_int, ctypes.c_int]
        L.oracle_ssao_rne.argtypes = [ctypes.c_float]
        L.oracle_ssao_rne.restype = ctypes.c_float
        _lib = L
    return _lib


def _chk(r):
    if r < 0:
        raise RuntimeError(lib().oracle_last_error().decode())
    return r


def params(scene):
    out = np.zeros(64, np.float64)
    n = _chk(lib().oracle_params(ctypes.addressof(scene), out.ctypes.data, 64))
    return out[:n]


def pixel_seed(y, x):
    return lib().oracle_pixel_seed(y, x)


def formula_iterate(formula, options, v, j, rout=0.0, ade=False):
    o = np.zeros(16, np.float64)
    o[: len(options)] = options
    v = np.array(v, np.float64)
    j = np.array(j, np.float64)
    _chk(lib().oracle_formula_iterate(formula, o.ctypes.data, v.ctypes.data, j.ctypes.data, rout, int(ade)))
    return v, j


def de_at(scene, pos):
    pos = np.ascontiguousarray(pos, np.float64).reshape(-1, 3)
    de = np.zeros(len(pos), np.float64)
    its = np.zeros(len(pos), np.int32)
    _chk(lib().oracle_de_at(ctypes.addressof(scene), pos.ctypes.data, len(pos), de.ctypes.data, its.ctypes.data))
    return de, its


def march(scene, dtype, row0=0, rows=None, threads=0, count=False):
    rows = scene.height - row0 if rows is None else rows
    out = np.zeros(rows * scene.width, dtype=dtype)
    cnt = np.zeros(1, np.uint64)
    _chk(lib().oracle_march(ctypes.addressof(scene), row0, rows, out.ctypes.data, threads,
                            cnt.ctypes.data if count else None))
    return (out, int(cnt[0])) if count else out


def march_pixels(scene, dtype, xy, threads=0):
    xy = np.ascontiguousarray(xy, np.int32).reshape(-1, 2)
    out = np.zeros(len(xy), dtype=dtype)
    _chk(lib().oracle_march_pixels(ctypes.addressof(scene), xy.ctypes.data, len(xy), out.ctypes.data, threads))
    return out


def shadows(scene, gbuf, threads=0, per_pixel=True):
    _chk(lib().oracle_shadows(ctypes.addressof(scene), gbuf.ctypes.data, threads, int(per_pixel)))
    return gbuf


def deao(scene, gbuf, threads=0):
    _chk(lib().oracle_deao(ctypes.addressof(scene), gbuf.ctypes.data, threads))
    return gbuf


def ao_rays(quality):
    d = np.zeros((64, 3), np.float32)
    n = lib().oracle_ao_rays(quality, d.ctypes.data, 64)
    return d[:n]


def render_rows(scene, dtype, rows, threads=0):
    """March + shadows + DE AO of the listed rows (the reference CPU path)."""
    rows = np.ascontiguousarray(rows, np.int32)
    out = np.zeros(len(rows) * scene.width, dtype=dtype)
    _chk(lib().oracle_render_rows(ctypes.addressof(scene), rows.ctypes.data, len(rows), out.ctypes.data, threads))
    return out


def mc_render(scene, light, opts, threads=0):
    """The Monte Carlo oracle (oracle/mc.cpp): radiance, albedo, normal
    (h, w, 3), depth, hit (h, w) and the count of rays that started inside."""
    w, h = (opts.w, opts.h) if opts.w else (scene.width, scene.height)
    rad = np.zeros((h, w, 3))
    alb = np.zeros((h, w, 3))
    nrm = np.zeros((h, w, 3))
    dep = np.zeros((h, w))
    hit = np.zeros((h, w), np.uint8)
    inside = ctypes.c_uint64()
    _chk(lib().oracle_mc_render(ctypes.addressof(scene), ctypes.addressof(light), ctypes.addressof(opts),
                                rad.ctypes.data, alb.ctypes.data, nrm.ctypes.data, dep.ctypes.data, hit.ctypes.data,
                                ctypes.byref(inside), threads))
    return dict(radiance=rad, albedo=alb, normal=nrm, depth=dep, hit=hit, inside=inside.value)


def mc_pass(scene, light, opts, pass_nr, recs, threads=0):
    """One adaptive Monte Carlo pass (mc::pass, src/mc.rs:3110-3300) over
    the whole picture: recs (a numpy array of mb3dcu.MC_RECORD, width*height)
    is updated in place and returned."""
    assert recs.flags["C_CONTIGUOUS"] and recs.size == scene.width * scene.height
    _chk(lib().oracle_mc_pass(ctypes.addressof(scene), ctypes.addressof(light), ctypes.addressof(opts), pass_nr,
                              recs.ctypes.data, threads))
    return recs


def dof_raw(gbuf, rgb, width, height, zc_mul, zcorr, fov_y, opts, threads=0):
    """dof::apply (src/dof.rs:81-122) on an 8-bit picture (h, w, 3) with the
    depth constants given: a new picture; opts is an mb3dcu.DofOpts."""
    out = np.ascontiguousarray(rgb, dtype=np.uint8).copy()
    g = np.ascontiguousarray(gbuf)
    _chk(lib().oracle_dof(out.ctypes.data, g.ctypes.data, width, height, zc_mul, zcorr, fov_y,
                          ctypes.addressof(opts), threads))
    return out


def dof(scene, gbuf, rgb, opts, threads=0):
    """dof::apply with the scene's depth constants (CalcPPZvals)."""
    p = params(scene)
    return dof_raw(gbuf, rgb, scene.width, scene.height, p[7], p[6], scene.fov_y, opts, threads)


def mc_batch(scene, reqs, secant=True, threads=0):
    """McMarch::run on the requests (a ctypes array of mb3dcu.McReq)."""
    import mb3dcu
    res = (mb3dcu.McRes * len(reqs))()
    _chk(lib().oracle_mc_batch(ctypes.addressof(scene), int(bool(secant)), ctypes.addressof(reqs), len(reqs),
                               ctypes.addressof(res), threads))
    return res


def mc_halton(i, x1, y):
    rec = (ctypes.c_uint16 * 4)()
    sh = (ctypes.c_float * 2)()
    lib().oracle_mc_halton(i, x1, y, rec, sh)
    return list(rec), list(sh)


def mc_seed_of(x, y, b):
    return lib().oracle_mc_seed_of(x, y, b)


def mc_paint(colour, opts, rays=None):
    """paint_recs (src/mc.rs:3957-4005): float colours (..., 3) -> uint8 RGB;
    opts is an mb3d_cu_mc_paint_opts (mb3dcu.McPaintOpts)."""
    col = np.ascontiguousarray(colour, dtype=np.float32)
    n = col.size // 3
    out = np.zeros(col.shape[:-1] + (3,), np.uint8)
    r = None if rays is None else np.ascontiguousarray(rays, dtype=np.uint8)
    lib().oracle_mc_paint(col.ctypes.data, None if r is None else r.ctypes.data, n, ctypes.addressof(opts),
                          out.ctypes.data)
    return out


def paint(sc, gbuf, row0=0):
    """render::paint (src/render.rs:2499): 8-bit RGB (rows, width, 3) of G-buffer
    records (a structured array of the card's record layout, rows * width)."""
    g = np.ascontiguousarray(gbuf)
    rows = g.size // sc.width
    out = np.zeros((rows, sc.width, 3), np.uint8)
    _chk(lib().oracle_paint(ctypes.addressof(sc), g.ctypes.data, row0, rows, out.ctypes.data))
    return out


def ssao24(gbuf, w, h, zc_mul, zcorr, threshold=2.0, border_mirror=0.0, t0=False, wrap_x=False, random=0):
    """ssao::ssao24 (src/ssao.rs:129-335), regular sampling or `random`
    passes of random sampling: a copy of the w x h G-buffer records with
    amb_shadow of the object pixels set."""
    g = np.ascontiguousarray(gbuf).copy()
    assert g.size == w * h
    _chk(lib().oracle_ssao24(g.ctypes.data, w, h, zc_mul, zcorr, threshold, border_mirror, int(t0), int(wrap_x),
                             int(random)))
    return g


def ssao15(gbuf, w, h, zc_mul, zcorr, threshold=2.0, t0=False, wrap_x=False, threads=0):
    """ssao15::ssao15 (src/ssao15.rs:282-411): a copy of the G-buffer with
    the 15-bit SSAO's amb_shadow on its object pixels."""
    g = np.ascontiguousarray(gbuf).copy()
    _chk(lib().oracle_ssao15(g.ctypes.data, w, h, zc_mul, zcorr, threshold, int(t0), int(wrap_x), threads))
    return g


def reflect_batch(scene, rays, far_fog=False, threads=0):
    """SrTracer::march_ray (src/reflect.rs:1464-1675) with calc_hs and
    deao_1pos for every ray (an mb3dcu.REFLECT_RAY array): the hits
    (mb3dcu.REFLECT_HIT)."""
    import mb3dcu
    r = np.ascontiguousarray(rays, mb3dcu.REFLECT_RAY)
    out = np.zeros(len(r), mb3dcu.REFLECT_HIT)
    _chk(lib().oracle_reflect_batch(ctypes.addressof(scene), r.ctypes.data, len(r), int(far_fog), out.ctypes.data,
                                    threads))
    return out


def reflect_first_rays(scene, gbuf):
    """The first bounce of every object pixel (start_pixel and step's mirror
    ray, src/reflect.rs:1686-1838, 1286-1311): an mb3dcu.REFLECT_RAY array."""
    import mb3dcu
    g = np.ascontiguousarray(gbuf)
    out = np.zeros(len(g), mb3dcu.REFLECT_RAY)
    n = _chk(lib().oracle_reflect_first_rays(ctypes.addressof(scene), g.ctypes.data, out.ctypes.data, len(out)))
    return out[:n].copy()


def ssao15_arctan(y, x):
    """fastIntArcTan2 (src/ssao15.rs:22-50)."""
    return lib().oracle_ssao15_arctan(y, x)


def ssao15_axis(pos, size, max_rad, step):
    """axis_samples (src/ssao15.rs:193-231)."""
    out = np.zeros(4096, np.int32)
    n = lib().oracle_ssao15_axis(pos, size, max_rad, step, out.ctypes.data, out.size)
    return [int(v) for v in out[:n]]


def ssao_levels(w, h):
    return lib().oracle_ssao_levels(w, h)


def ssao_rne(x):
    return lib().oracle_ssao_rne(x)
