"""Generates the committed fixtures of the tests (run from the repository
root: python tests/golden/make_fixtures.py).

c3_point.json: the deep-zoom workload's surface point, found by a seeded
FP64 march of the oracle along the middle ray of a camera drawn on the r=3
sphere (Integer Power 8, 200 iterations): steps of half the oracle's
distance estimate until a sample is inside (all iterations used, or the
estimate under 1e-9), then 80 bisections between the last outside and the
first inside sample -- the camera of that workload sits 1e-5 in front of
the point, outside the set.
"""
import json
import math
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [os.path.join(ROOT, "mb3d-rs_b200"), os.path.join(ROOT, "oracle")]

import oracle_py as O  # noqa: E402
import scenes  # noqa: E402


def c3_point(seed=scenes.C3_SEED):
    cam = scenes.sphere_point(seed, 3.0)
    d = [-c / 3.0 for c in cam]
    probe = scenes.c3_deep_zoom([0.0, 0.0, 0.0], d)
    def inside(t):
        de, its = O.de_at(probe, [[cam[k] + t * d[k] for k in range(3)]])
        return its[0] >= probe.iterations or de[0] < 1e-9, de[0]

    t, t_out = 0.0, 0.0
    for _ in range(100000):
        ins, de = inside(t)
        if ins:
            break
        t_out = t
        t += 0.5 * de
    lo, hi = t_out, t
    for _ in range(80):
        mid = 0.5 * (lo + hi)
        if inside(mid)[0]:
            hi = mid
        else:
            lo = mid
    p = [cam[k] + lo * d[k] for k in range(3)]
    de, its = O.de_at(probe, [p])
    cam_in, _ = inside(lo - 1e-5)
    return {"seed": seed, "camera": cam, "view_dir": d, "point": p, "t": lo, "de": float(de[0]),
            "its": int(its[0]), "camera_outside": not cam_in}


if __name__ == "__main__":
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "c3_point.json")
    r = c3_point()
    with open(out, "w") as f:
        json.dump(r, f, indent=1)
    print(json.dumps(r))
