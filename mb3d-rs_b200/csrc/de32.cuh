// The single precision distance estimate of the mixed-precision march.
//
// Numerical DE (MB3D DE option 0, src/calc.rs:1515-1543): the reference runs
// the hybrid at c, then three more times at c + offset on each axis with the
// centre's iteration count as the limit, and takes
//     DE = R ln R * s / (sqrt(sum (R - R_k)^2) + o006).
// Here the four orbits run in lock-step in one loop (same slot sequence,
// four independent dependency chains for the pipelines), and the form is
// the one that stays accurate in single precision:
//     d_k = (v - v_k).(v + v_k) / R,   DE = ln R * s / (sqrt(sum d_k^2) + o006 / R).
// Each offset point is rounded to single precision; the offset it actually
// got (h_k, exact in double) rescales its difference to the reference's
// offset, so the rounding of the coordinates does not bias the gradient.
//
// Analytic DE (options 2 / 11, src/iteration.rs:539-574): one orbit with the
// running derivative in w.
//
// The caller's position is double precision; only the iteration is single.
#pragma once
#include "devparams.h"
#include "formulas.cuh"

namespace mb3dcu {

struct DE32 {
    float de;
    int it;
    bool need64;  // single precision cannot resolve the offset here
};

__device__ __forceinline__ float fast_sqrtf(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }

__device__ __forceinline__ DE32 de32(const DevParams &p, const double c[3], float ms_de_stop) {
    DE32 out;
    out.need64 = false;
    const int max_it = p.max_it;
    if (p.is_custom_de) {
        float v[4], j[3];
        v[0] = (float)c[0];
        v[1] = (float)c[1];
        v[2] = (float)c[2];
        if (p.do_julia) {
            j[0] = p.ju_f[0]; j[1] = p.ju_f[1]; j[2] = p.ju_f[2];
        } else {
            j[0] = v[0]; j[1] = v[1]; j[2] = v[2];
        }
        float rout = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        v[3] = ((p.de_option & 0x38) == 16) ? rout : 1.0f;
        int n = 0, btmp = p.slots[0].iterations, it = 0;
        unsigned int unc = 0;
        for (;;) {
            int guard = 0;
            while (btmp <= 0) {
                n += 1;
                if (n > p.end_to) n = p.repeat_from;
                btmp = p.slots[n].iterations;
                if (++guard > 64) goto done_a;
            }
            {
                const DevSlot &s = p.slots[n];
                formula_iterate<float>(s, v, j, rout);
                if (s.julia_add) {
                    v[0] += j[0]; v[1] += j[1]; v[2] += j[2];
                }
                btmp -= 1;
                if (s.uncounted) {
                    if (++unc > 100000u) goto done_a;
                    continue;
                }
            }
            it += 1;
            rout = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            if (it >= max_it || rout > p.d_rstop_f) break;
        }
    done_a:
        float r;
        if ((p.de_option & 7) == 4) r = __fdividef(fabsf(v[1]) * __logf(fabsf(v[1])), v[3]);
        else r = __fdividef(fast_sqrtf(rout), fabsf(v[3]));
        out.de = r * p.d_de_scale;
        out.it = it;
    } else {
        // four orbits: 0 = centre, 1..3 = the offsets on x, y, z
        float v[4][4], j[4][3], rout[4];
        float corr[3];
        const double off = (double)p.de_offset;
        float cf[3] = {(float)c[0], (float)c[1], (float)c[2]};
#pragma unroll
        for (int k = 0; k < 3; k++) {
            float o = (float)(c[k] + off);
            double h = (double)o - (double)cf[k];
            if (h <= 0.0) out.need64 = true;
            corr[k] = (float)(off / fmax(h, 1e-300));
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
            v[q][0] = cf[0]; v[q][1] = cf[1]; v[q][2] = cf[2]; v[q][3] = 0.0f;
            if (q > 0) v[q][q - 1] = (float)(c[q - 1] + off);
            if (p.do_julia) {
                j[q][0] = p.ju_f[0]; j[q][1] = p.ju_f[1]; j[q][2] = p.ju_f[2];
            } else {
                j[q][0] = v[q][0]; j[q][1] = v[q][1]; j[q][2] = v[q][2];
            }
            rout[q] = v[q][0] * v[q][0] + v[q][1] * v[q][1] + v[q][2] * v[q][2];
        }
        bool live1 = true, live2 = true, live3 = true;
        int n = 0, btmp = p.slots[0].iterations, it = 0;
        unsigned int unc = 0;
        for (;;) {
            int guard = 0;
            while (btmp <= 0) {
                n += 1;
                if (n > p.end_to) n = p.repeat_from;
                btmp = p.slots[n].iterations;
                if (++guard > 64) goto done_n;
            }
            {
                const DevSlot &s = p.slots[n];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    formula_iterate<float>(s, v[q], j[q], rout[q]);
                    if (s.julia_add) {
                        v[q][0] += j[q][0]; v[q][1] += j[q][1]; v[q][2] += j[q][2];
                    }
                }
                btmp -= 1;
                if (s.uncounted) {
                    if (++unc > 100000u) goto done_n;
                    continue;
                }
            }
            it += 1;
            rout[0] = v[0][0] * v[0][0] + v[0][1] * v[0][1] + v[0][2] * v[0][2];
            // an offset orbit stops at its own bailout (RStop3D), its state kept
            if (live1) {
                float r = v[1][0] * v[1][0] + v[1][1] * v[1][1] + v[1][2] * v[1][2];
                rout[1] = r;
                if (r > p.rstop3d_f) live1 = false;
            }
            if (live2) {
                float r = v[2][0] * v[2][0] + v[2][1] * v[2][1] + v[2][2] * v[2][2];
                rout[2] = r;
                if (r > p.rstop3d_f) live2 = false;
            }
            if (live3) {
                float r = v[3][0] * v[3][0] + v[3][1] * v[3][1] + v[3][2] * v[3][2];
                rout[3] = r;
                if (r > p.rstop3d_f) live3 = false;
            }
            if (it >= max_it || rout[0] > p.d_rstop_f) break;
            // (a frozen orbit keeps being iterated in the lock-step; its
            // values are not used, its length is kept)
        }
    done_n:
        float R = rout[0];
        float r;
        if (!(R > 0.0f)) {
            r = 0.0f;
        } else {
            float lr = __logf(R);
            float g = 0.0f;
#pragma unroll
            for (int q = 1; q < 4; q++) {
                float d;
                if (R < 1e30f && rout[q] < 1e30f) {
                    // frozen orbits: their difference from the lengths alone
                    bool live = q == 1 ? live1 : (q == 2 ? live2 : live3);
                    if (live) {
                        d = (v[0][0] - v[q][0]) * (v[0][0] + v[q][0]) + (v[0][1] - v[q][1]) * (v[0][1] + v[q][1]) +
                            (v[0][2] - v[q][2]) * (v[0][2] + v[q][2]);
                        d = __fdividef(d, R);
                    } else {
                        d = __fdividef(R - rout[q], R);
                    }
                } else {
                    d = 1.0f - __expf(__logf(rout[q]) - lr);
                }
                d *= corr[q - 1];
                g += d * d;
            }
            r = __fdividef(lr * p.d_de_scale, fast_sqrtf(g) + __fdividef(p.de_offset006, R));
        }
        out.de = r;
        out.it = it;
    }
    float mn = ms_de_stop * 0.25f;
    if (!(out.de >= mn)) out.de = mn;  // (NaN too)
    return out;
}

}  // namespace mb3dcu
