"""Scenes for the card: mb3d-rs's defaults and presets, and the synthetic
benchmark workloads (their sizes and parameters; no reference data files).

`default_scene` restates Scene::default (src/scene.rs:628-697) with the
start-up light preset (src/lighting.rs:290-330); `preset` restates
Scene::preset (src/scene.rs:811-836).
"""
import math

import numpy as np

from mb3dcu import Scene, Slot, Light, F_INTPOW, F_AMAZINGBOX, F_MENGERIFS, F_REALPOWER, F_TRICORN, F_BULBOX, \
    F_FOLDINGINTPOW, F_QUATERNION, F_AEXIONC

PI = math.pi


def slot(formula, iterations, *options):
    s = Slot()
    s.formula = formula
    s.iterations = iterations
    for k, v in enumerate(options):
        s.options[k] = v
    return s


def intpow(power=8, z_mul=-1.0, iterations=1):
    return slot(F_INTPOW, iterations, power, z_mul)


def amazing_box(scale=2.0, min_r=0.5, fold=1.0, iterations=1):
    return slot(F_AMAZINGBOX, iterations, scale, min_r, fold)


def menger_ifs(scale=3.0, cx=1.0, cy=1.0, cz=0.5, iterations=1):
    return slot(F_MENGERIFS, iterations, scale, cx, cy, cz)


def vgrads_from_angles(ax, ay, az):
    """CalcVGradsFromHeader8rots (src/math.rs:101-124)."""
    s1, c1 = math.sin(ax), math.cos(ax)
    s2, c2 = math.sin(ay), math.cos(ay)
    s3, c3 = math.sin(az), math.cos(az)
    m = []
    for i in range(3):
        x1, y1, z1 = (1.0, 0.0, 0.0) if i == 0 else ((0.0, 1.0, 0.0) if i == 1 else (0.0, 0.0, 1.0))
        x2 = x1
        y2 = c1 * y1 + s1 * z1
        z2 = c1 * z1 - s1 * y1
        x1 = c2 * x2 + s2 * z2
        y1 = y2
        z1 = c2 * z2 - s2 * x2
        m.append([c3 * x1 + s3 * y1, c3 * y1 - s3 * x1, z1])
    return m


def set_slots(sc, slots, repeat_from=0):
    for i in range(6):
        sc.slots[i] = Slot()
    for i, s in enumerate(slots):
        sc.slots[i] = s
    sc.n_slots = len(slots)
    sc.repeat_from = repeat_from


def set_vgrads(sc, m):
    for i in range(3):
        for k in range(3):
            sc.vgrads[i][k] = m[i][k]


def default_scene():
    sc = Scene()
    sc.width, sc.height = 800, 600
    sc.iterations, sc.min_iterations = 60, 1
    sc.rstop = 0.0
    sc.zoom = 1.0
    sc.mid[0] = sc.mid[1] = sc.mid[2] = 0.0
    sc.z_start, sc.z_end = -2.0, 30.0
    set_vgrads(sc, [[1, 0, 0], [0, 1, 0], [0, 0, 1]])
    sc.fov_y = 30.0
    sc.de_stop, sc.z_step_div, sc.raystep_limiter = 1.0, 0.5, 1.0
    sc.smooth_normals, sc.bin_search_steps = 0, 8
    sc.first_step_random, sc.step_sub_de_stop, sc.vary_de_stop_on_fov = 1, 0, 1
    sc.normals_on_de, sc.disable_analytic_de, sc.julia = 1, 0, 0
    sc.color_option, sc.color_on_it, sc.color_mul, sc.dfog_on_it = 0, 0, 1.0, 0
    set_slots(sc, [intpow()])
    # the start-up lights: light 1 on, light 2 off
    sc.lights[0] = Light(1, 0, 1500.0 * PI / 16384.0, 5200.0 * PI / 16384.0)
    sc.lights[1] = Light(0, 0, -2822.0 * PI / 16384.0, -7737.0 * PI / 16384.0)
    sc.shadow_lights, sc.shadow_soft, sc.soft_radius, sc.hs_max_len_mul = 0, 0, 1.0, 1.0
    sc.deao_quality, sc.deao_dither, sc.deao_max_len, sc.deao_first_step_random = -1, 0, 1.0, 0
    return sc


def preset(name, width=None, height=None):
    """Scene::preset: one formula with a camera that shows it."""
    sc = default_scene()
    n = name.lower()
    if n == "amazing box":
        f, zs, zoom, its, rot = amazing_box(), -14.0, 0.18, 20, (0.35, -0.6)
    elif n == "bulbox":
        f, zs, zoom, its, rot = slot(F_BULBOX, 1, 2.0, 0.5, 1.0, 1.0, 2.0, 2.0), -14.0, 0.18, 20, (0.35, -0.6)
    elif n == "folding int pow":
        f, zs, zoom, its, rot = slot(F_FOLDINGINTPOW, 1, 2, -1.0, 2.0), -20.0, 0.15, 20, (0.5, 0.4)
    elif n == "tricorn":
        f, zs, zoom, its, rot = slot(F_TRICORN, 1, -2.0, 1.0), -3.0, 0.6, 12, (0.6, 0.2)
    elif n == "real power":
        f, zs, zoom, its, rot = slot(F_REALPOWER, 1, 8.0, -1.0), -2.5, 0.8, 12, (-0.55, 0.45)
    elif n == "aexion c":
        f, zs, zoom, its, rot = slot(F_AEXIONC, 1, 8.0, 1.0, 1.0, 1.0, 8.0, 1.0, 0.0, 0.0), -3.0, 0.65, 10, (0.45, 0.3)
    elif n == "quaternion":
        f, zs, zoom, its, rot = slot(F_QUATERNION, 1, -1.0, 0.0), -3.0, 0.8, 12, (0.4, 0.3)
        sc.julia = 1
        for k, v in enumerate((-0.2, 0.6, 0.2, 0.0)):
            sc.julia_c[k] = v
    else:  # Integer Power
        f, zs, zoom, its, rot = intpow(), -2.5, 0.8, 12, (-0.55, 0.45)
    sc.z_start, sc.zoom, sc.iterations = zs, zoom, its
    set_vgrads(sc, vgrads_from_angles(rot[0], rot[1], 0.0))
    set_slots(sc, [f])
    if width:
        sc.width, sc.height = width, height
    return sc


PRESETS = ["Integer Power", "Real Power", "Quaternion", "Tricorn", "Amazing Box", "Bulbox", "Folding Int Pow",
           "Aexion C"]


def interpolated(first, second, weights, width=None, height=None):
    """An interpolation hybrid (Scene::interpolation): preset `first`'s
    camera and formula, blended in every iteration with preset `second`'s
    formula by `weights` (normalised by the library)."""
    sc = preset(first, width, height)
    a, b = sc.slots[0], preset(second).slots[0]
    a, b = (slot(s.formula, 1, *list(s.options)) for s in (a, b))
    set_slots(sc, [a, b])
    sc.interpolation = 1
    sc.ipol_weights[0], sc.ipol_weights[1] = weights
    return sc


DECOMB_KINDS = {"min": 1, "max": 2, "max_inverted": 3, "smooth_linear": 4, "smooth": 5}


def two_objects(kind="min", width=160, height=120, place=True, smooth=0.5):
    """A DE combination (Scene::decomb): a Mandelbulb (Integer Power 8) as
    part 1 and an Amazing Box as part 2, the box moved to x = 3.2, turned by
    20 and 30 degrees and scaled to 0.4, with the camera on both -- the
    reference's own scene of two objects (tests/data/two_objects.m3s:
    de_combination, decomb_*, part2_*, mid, zoom, z_start, rotation, de_stop,
    raystep, smooth_normals, bin_search).  `place` False leaves the box at
    the origin over the bulb, scaled to 0.12 (about the bulb's size), with
    the camera closer: the scene for the combinations that need both objects
    in one place."""
    sc = default_scene()
    sc.width, sc.height = width, height
    sc.iterations = 30
    sc.zoom, sc.z_start, sc.z_end = (0.55 if place else 1.2), -10.0, 30.0
    sc.mid[0], sc.mid[1], sc.mid[2] = (1.6 if place else 0.0), 0.0, 0.0
    set_vgrads(sc, vgrads_from_angles(math.radians(-30.0), math.radians(20.0), 0.0))
    sc.de_stop, sc.z_step_div = 0.8, 0.4
    sc.smooth_normals, sc.bin_search_steps = 3, 8
    set_slots(sc, [intpow(8, -1.0), amazing_box(2.0, 0.5, 1.0)])
    sc.decomb = DECOMB_KINDS[kind]
    sc.decomb_end1, sc.decomb_start2, sc.decomb_end2, sc.decomb_repeat2 = 0, 1, 1, 1
    sc.decomb_iterations2 = 30
    sc.decomb_smooth, sc.decomb_mix_pow = smooth, 2.0
    if place:
        for k, v in enumerate((3.2, 0.0, 0.0)):
            sc.part2_offset[k] = v
        for k, v in enumerate((20.0, 30.0, 0.0)):
            sc.part2_rotation[k] = v
        sc.part2_scale = 0.4
    else:
        sc.part2_scale = 0.12
    return sc


def splitmix64(state):
    state = (state + 0x9E3779B97F4A7C15) & 0xFFFFFFFFFFFFFFFF
    z = state
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & 0xFFFFFFFFFFFFFFFF
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & 0xFFFFFFFFFFFFFFFF
    return state, z ^ (z >> 31)


def sphere_point(seed, radius):
    """A point drawn uniformly on the sphere of `radius` from a 64-bit seed."""
    st, a = splitmix64(seed)
    st, b = splitmix64(st)
    u, v = a / 2.0 ** 64, b / 2.0 ** 64
    z = 2.0 * u - 1.0
    phi = 2.0 * PI * v
    r = math.sqrt(max(0.0, 1.0 - z * z))
    return [radius * r * math.cos(phi), radius * r * math.sin(phi), radius * z]


def look_at_origin(cam):
    """Camera rows (screen x, screen y, view axis) looking from cam at the origin."""
    d = math.sqrt(sum(c * c for c in cam))
    z = [-c / d for c in cam]
    up = [0.0, 1.0, 0.0] if abs(z[1]) < 0.99 else [1.0, 0.0, 0.0]
    x = [up[1] * z[2] - up[2] * z[1], up[2] * z[0] - up[0] * z[2], up[0] * z[1] - up[1] * z[0]]
    xl = math.sqrt(sum(c * c for c in x))
    x = [c / xl for c in x]
    y = [z[1] * x[2] - z[2] * x[1], z[2] * x[0] - z[0] * x[2], z[0] * x[1] - z[1] * x[0]]
    return [x, y, z]


def place_camera(sc, cam):
    """The start plane's middle at cam, looking at the origin (mid = 0)."""
    set_vgrads(sc, look_at_origin(cam))
    sc.mid[0] = sc.mid[1] = sc.mid[2] = 0.0
    sc.z_start = -math.sqrt(sum(c * c for c in cam))


def c1_plain_bulb():
    """Mandelbulb (Integer Power 8), 60 iterations, bailout 16, raystep 0.5,
    DE stop 1 px, 640x480, camera at (0, 0, -2.6) looking at the origin,
    30 degree field of view, no shadows or AO."""
    sc = default_scene()
    sc.width, sc.height = 640, 480
    sc.iterations = 60
    sc.rstop = 16.0
    sc.z_step_div, sc.de_stop = 0.5, 1.0
    sc.z_start, sc.z_end = -2.6, 30.0
    set_slots(sc, [intpow(8, -1.0, 1)])
    return sc


C2_SEED = 0x5EED0002


def c2_hybrid(seed=C2_SEED, width=1920, height=1080):
    """2 Amazing Box (scale -1.5, min R 0.5, fold 1) then 1 Integer Power 8,
    repeating; 30 iterations; 1920x1080; camera on the r=3 sphere (seeded)
    looking at the origin; hard shadows from light 1; DE AO with 17 rays
    (quality 2, the reference's level nearest to 15 rays)."""
    sc = default_scene()
    sc.width, sc.height = width, height
    sc.iterations = 30
    set_slots(sc, [amazing_box(-1.5, 0.5, 1.0, 2), intpow(8, -1.0, 1)], repeat_from=0)
    place_camera(sc, sphere_point(seed, 3.0))
    sc.shadow_lights = 1
    sc.deao_quality = 2
    return sc


# the surface point of the deep zoom: where the FP64 march of the middle ray
# from the seeded camera met the Mandelbulb (tests/golden/make_fixtures.py)
C3_SEED = 0x5EED0003
# (tests/golden/c3_point.json, made by tests/golden/make_fixtures.py)
C3_POINT = [-0.8697553607530222, 0.22843892661237097, 0.3317609632059464]
C3_VIEW = [0.9074121027226582, -0.2383293694925562, -0.34612481487134783]


def c3_deep_zoom(point, view_dir, width=1920, height=1080):
    """Integer Power 8, 200 iterations, DE stop 0.5 px; the camera 1e-5 in
    front of `point` along `view_dir`, view width 1e-6 (zoom 2.1345e6)."""
    sc = default_scene()
    sc.width, sc.height = width, height
    sc.iterations = 200
    sc.de_stop = 0.5
    sc.zoom = 2.1345 / 1e-6
    set_slots(sc, [intpow(8, -1.0, 1)])
    d = math.sqrt(sum(c * c for c in view_dir))
    z = [c / d for c in view_dir]
    cam = [-c for c in z]
    set_vgrads(sc, look_at_origin(cam))  # rows with z as the view axis
    for k in range(3):
        sc.mid[k] = point[k]
    sc.z_start = point[2] - 1e-5
    sc.z_end = sc.z_start + 1e-3
    return sc


def c3(width=1920, height=1080):
    """The deep zoom workload at the committed surface point."""
    return c3_deep_zoom(C3_POINT, C3_VIEW, width, height)


C4_SEED = 0x5EED0004


def catmull_rom_weights(t):
    """src/anim.rs:692-700."""
    t2, t3 = t * t, t * t * t
    return [0.5 * (-t3 + 2.0 * t2 - t), 0.5 * (3.0 * t3 - 5.0 * t2 + 2.0), 0.5 * (-3.0 * t3 + 4.0 * t2 + t),
            0.5 * (t3 - t2)]


def c4_control_points(seed=C4_SEED, n=8):
    pts = []
    st = seed
    for i in range(n):
        st, a = splitmix64(st)
        r = 1.5 + 2.5 * (a / 2.0 ** 64)
        st, b = splitmix64(st)
        pts.append(sphere_point(b, r))
    return pts


def c4_frames(n_frames=240, width=1280, height=720, seed=C4_SEED):
    """Menger IFS (scale 3, CScale 1/1/0.5) and Amazing Box (scale 2), 12
    iterations, hard shadows; the camera flies a closed Catmull-Rom curve
    through 8 seeded points 1.5..4 from the origin, looking at it."""
    pts = c4_control_points(seed)
    n = len(pts)
    frames = []
    for f in range(n_frames):
        u = f * n / n_frames
        i = int(u)
        t = u - i
        w = catmull_rom_weights(t)
        cam = [0.0, 0.0, 0.0]
        for k, wk in enumerate(w):
            p = pts[(i - 1 + k) % n]
            for c in range(3):
                cam[c] += wk * p[c]
        sc = default_scene()
        sc.width, sc.height = width, height
        sc.iterations = 12
        set_slots(sc, [menger_ifs(3.0, 1.0, 1.0, 0.5, 1), amazing_box(2.0, 0.5, 1.0, 1)])
        place_camera(sc, cam)
        sc.shadow_lights = 1
        frames.append(sc)
    return frames


def scene_copy(sc):
    n = Scene()
    import ctypes
    ctypes.memmove(ctypes.byref(n), ctypes.byref(sc), ctypes.sizeof(Scene))
    return n


def scaled(sc, width, height):
    """The scene at another picture size with its look (Scene::scale_image:
    the DE stop is in pixels)."""
    n = scene_copy(sc)
    f = width / sc.width
    n.width, n.height = width, height
    n.de_stop = max(sc.de_stop * f, 0.001)
    return n


def c5_mc(width=1920, height=1080):
    """The Monte Carlo workload: the C2 hybrid scene, 1920x1080, up to 4
    ambient bounces (MCDepth 4), light 1 plus the ambient sky."""
    return c2_hybrid(width=width, height=height)


C5_DEPTH = 4
TRAIN_SEED = 0x5EED0005


def random_training_scene(seed, width=256, height=256):
    """A seeded scene for the denoiser's training pictures: one of four
    formula families with random parameters (box/bulb hybrid, bulb, box,
    Menger/box), a random camera on a sphere around the origin looking at
    it, a random zoom and a random light direction."""
    st = seed & 0xFFFFFFFFFFFFFFFF
    u = []
    for _ in range(12):
        st, v = splitmix64(st)
        u.append(v / 2.0 ** 64)
    sc = default_scene()
    sc.width, sc.height = width, height
    fam = int(u[0] * 4)
    power = 3 + int(u[1] * 6)
    bscale = (1.3 + 1.2 * u[2]) * (-1.0 if u[3] < 0.6 else 1.0)
    min_r, fold = 0.25 + 0.5 * u[4], 0.8 + 0.4 * u[5]
    if fam == 0:
        set_slots(sc, [amazing_box(bscale, min_r, fold, 1 + int(u[6] * 2)), intpow(power, -1.0, 1)])
        radius = 2.6 + 1.2 * u[7]
    elif fam == 1:
        set_slots(sc, [intpow(power, -1.0, 1)])
        radius = 2.0 + 1.0 * u[7]
    elif fam == 2:
        set_slots(sc, [amazing_box(bscale, min_r, fold, 1)])
        radius = 3.0 + 3.0 * u[7] if bscale < 0 else 5.0 + 3.0 * u[7]
    else:
        set_slots(sc, [menger_ifs(3.0, 1.0, 1.0, 0.5, 1), amazing_box(2.0, 0.5, 1.0, 1)])
        radius = 1.8 + 2.2 * u[7]
    sc.iterations = 12 + int(u[8] * 19)
    place_camera(sc, sphere_point(st, radius))
    sc.zoom = 1.0 + 1.5 * u[9]
    sc.lights[0].x_angle = (u[10] - 0.5) * PI
    sc.lights[0].y_angle = (u[11] - 0.5) * PI * 0.66
    return sc
