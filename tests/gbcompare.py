"""G-buffer comparison for the parity tests (hit agreement, depth error,
normal cosine), the measures of mb3d-rs's own card-vs-CPU check
(gbuffer_matches_cpu, src/gpu.rs:4177-4248)."""
import numpy as np

import mb3dcu


def depth(g, zc_mul, zcorr):
    zf = (g["zpos_fine"] >> 8).astype(np.float64)
    return (((8388351.5 - zf) / zc_mul + 1.0) ** 2 - 1.0) / zcorr


def compare(a, b, zc_mul=None, zcorr=None):
    ha, hb = mb3dcu.hit_mask(a), mb3dcu.hit_mask(b)
    bga, bgb = mb3dcu.is_background(a), mb3dcu.is_background(b)
    r = {"n": int(len(a)), "hit_agree": float((ha == hb).mean()), "bg_agree": float((bga == bgb).mean()),
         "exact": float((a == b).mean())}
    both = ha & hb
    r["both_hit"] = int(both.sum())
    if both.any():
        na = a["normal"][both].astype(np.float64) / 32767.0
        nb = b["normal"][both].astype(np.float64) / 32767.0
        cos = (na * nb).sum(1) / np.maximum(np.linalg.norm(na, axis=1) * np.linalg.norm(nb, axis=1), 1e-30)
        r["normal_cos_mean"] = float(cos.mean())
        r["normal_off25"] = float((cos < np.cos(np.radians(25))).mean())
        if zc_mul is not None:
            da, db = depth(a[both], zc_mul, zcorr), depth(b[both], zc_mul, zcorr)
            rel = np.abs(da - db) / np.maximum(np.abs(db), 1e-30)
            r["depth_rel_median"] = float(np.median(rel))
            r["depth_rel_p99"] = float(np.quantile(rel, 0.99))
            r["depth_rel_max"] = float(rel.max())
            r["depth_rel_1e4"] = float((rel <= 1e-4).mean())
        zd = np.abs((a["zpos_fine"][both] >> 16).astype(np.int64) - (b["zpos_fine"][both] >> 16).astype(np.int64))
        r["zpos_diff_mean"] = float(zd.mean())
    return r
