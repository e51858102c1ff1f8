// TEST INFRASTRUCTURE: the older "15 bit" screen space ambient occlusion of
// the reference (ssao15::ssao15, src/ssao15.rs:282-411; MB3D's
// AmbShadowCalcThreadN) on the CPU, for the parity of the card's pass.
//   levels    the depth buffer of the object pixels scaled to 0..128
//             (build_levels, :92-176), single peaks lowered to their
//             highest neighbour + 1 (3x3), then "a trous" levels: a
//             horizontal and a vertical average with the neighbours step
//             away, step 1, 2, 4, ... (rounded averages of 16-bit values)
//   rings     per level a ring of sample offsets on a grid of the level's
//             step (axis_samples :193-231, rings :257-297), each sample
//             with 1/radius and the 1/32-circle buckets it updates
//   sampling  per object pixel the steepest slope per bucket (the
//             threshold clamps it, or the t0 variant fades it out), the
//             four overflow buckets merged, the arctangents of the 32
//             slopes summed into amb_shadow (:317-408)
// Single precision, unfused (-ffp-contract=off), as the reference; the
// arctangent is the C library's atanf, as the reference's f32::atan.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <thread>
#include <vector>

#include "../include/mb3d_cu.h"

namespace {

inline uint16_t avg16(uint16_t a, uint16_t b) { return (uint16_t)(((uint32_t)a + b + 1u) >> 1); }

inline uint32_t zpos16(const mb3d_cu_silight &s) { return s.zpos_fine >> 16; }

// fastIntArcTan2 (src/ssao15.rs:22-50): the direction (x, y) as a bucket
// 0..31 of the circle; integer divisions truncate toward zero
int arctan32(int32_t y, int32_t x) {
    int r;
    if (x == 0) {
        r = (y >= 0 ? 16 : 0) + 8;
    } else if (y == 0) {
        r = x >= 0 ? 16 : 0;
    } else if (y < 0) {
        if (x < 0)
            r = x >= y ? 7 - (x * 4) / y : (y * 4) / x;
        else
            r = -y < x ? 15 + (y * 4) / x : 8 - (x * 4) / y;
    } else if (x >= 0) {
        r = x > y ? 16 + (y * 4) / x : 23 - (x * 4) / y;
    } else {
        r = y < -x ? 31 + (y * 4) / x : 24 - (x * 4) / y;
    }
    return r & 31;
}

struct Levels {
    int count;
    float corr_mul;
    int64_t zsub;
    std::vector<std::vector<uint16_t>> lev;
    // Levels::zp_of (:63-69): the scaled depth of a pixel, 32768 for the background
    int32_t zp_of(const mb3d_cu_silight &s) const {
        if (zpos16(s) >= 32768u) return 32768;
        return (int32_t)std::nearbyint((double)((int64_t)(s.zpos_fine >> 8) - zsub) * (double)corr_mul);
    }
};

// build_levels (:92-176)
Levels build_levels(const mb3d_cu_silight *g, size_t w, size_t h, bool wrap) {
    Levels L;
    int count = 1;
    for (size_t x = w / 16;;) {
        count++;
        x >>= 1;
        if (count == 8 || x < 4) break;
    }
    L.count = count;
    uint32_t zmin = 32767, zmax = 0;
    const size_t n = w * h;
    for (size_t i = 0; i < n; i++) {
        const uint32_t z = zpos16(g[i]);
        if (z < 32768u) {
            zmax = std::max(zmax, z);
            zmin = std::min(zmin, z);
        }
    }
    uint32_t za = 0, zp = 32768;
    if (zmax >= zmin) {
        za = zmin;
        zp = zmax + 1;
    }
    L.corr_mul = 128.0f / (float)(zp - za);
    L.zsub = (int64_t)za << 8;
    std::vector<uint16_t> l1(n);
    for (size_t i = 0; i < n; i++)
        l1[i] = zpos16(g[i]) < 32768u
                    ? (uint16_t)std::nearbyint((double)((int64_t)(g[i].zpos_fine >> 8) - L.zsub) * (double)L.corr_mul)
                    : 0;
    // single peaks (all eight neighbours lower, not all of them 0) come down
    // to their highest neighbour + 1, in place in pixel order
    if (w >= 3 && h >= 3) {
        const long wi = (long)w;
        const long offs[8] = {-wi - 1, -wi, -wi + 1, -1, 1, wi - 1, wi, wi + 1};
        for (size_t y = 1; y + 1 < h; y++)
            for (size_t x = 1; x + 1 < w; x++) {
                const size_t i = y * w + x;
                const uint16_t c = l1[i];
                uint16_t m = 0;
                for (long o : offs) {
                    const uint16_t v = l1[(size_t)((long)i + o)];
                    if (v >= c) {
                        m = 0;
                        break;
                    }
                    m = std::max(m, v);
                }
                if (m > 0) l1[i] = (uint16_t)(m + 1);
            }
    }
    L.lev.push_back(l1);
    std::vector<uint16_t> tmp(n);
    size_t step = 1;
    for (int k = 2; k <= count; k++) {
        const std::vector<uint16_t> &src = L.lev.back();
        const long s = (long)step;
        for (size_t y = 0; y < h; y++) {
            const uint16_t *r = &src[y * w];
            uint16_t *d = &tmp[y * w];
            auto at = [&](long i) { return r[std::clamp(i, 0L, (long)w - 1)]; };
            for (size_t i = 0; i < w; i++) {
                const long ii = (long)i;
                if (wrap) {
                    const long wl = (long)w;
                    d[i] = avg16(r[i], avg16(r[((ii - s) % wl + wl) % wl], r[((ii + s) % wl + wl) % wl]));
                } else if (i < step) {
                    d[i] = avg16(r[i], avg16(r[0], at(ii + s)));
                } else if (i + step < w) {
                    d[i] = avg16(r[i], avg16(at(ii - s), at(ii + s)));
                } else {
                    d[i] = (uint16_t)(((uint32_t)r[i] + 1u + (((uint32_t)at(ii - s) + r[w - 1]) >> 1)) >> 1);
                }
            }
        }
        std::vector<uint16_t> dst(n);
        for (size_t x = 0; x < w; x++) {
            auto at = [&](long j) { return tmp[(size_t)std::clamp(j, 0L, (long)h - 1) * w + x]; };
            for (size_t j = 0; j < h; j++) {
                const long jj = (long)j;
                const uint16_t c = tmp[j * w + x];
                if (j < step)
                    dst[j * w + x] = avg16(avg16(at(jj + s), tmp[x]), c);
                else if (j + step < h)
                    dst[j * w + x] = avg16(avg16(at(jj - s), at(jj + s)), c);
                else
                    dst[j * w + x] = avg16(avg16(at(jj - s), tmp[(h - 1) * w + x]), c);
            }
        }
        L.lev.push_back(std::move(dst));
        step *= 2;
    }
    return L;
}

// sampling_constants (:73-89): (szrt, smul, st2)
void sampling_constants(const Levels &L, double zc_mul, double zcorr, float threshold, bool t0, float &szrt,
                        float &smul, float &st2) {
    const float n = (float)L.count;
    const float thr = std::max(threshold, 0.01f);
    const double q = 256.0 / zc_mul + 1.0;
    const float zscale = (float)((q * q - 1.0) / zcorr);
    st2 = zscale / (L.corr_mul * 256.0f);
    const float pi = 3.14159265358979323846f;
    if (t0) {
        szrt = std::max(thr * 2.0f / st2, 0.01f);
        smul = 1.35f * 32767.0f / (pi * 32.0f * std::pow(std::atan(thr * 0.8f * std::sqrt(std::sqrt(n))), 0.9f));
    } else {
        szrt = thr / st2;
        smul = 1.35f * 32767.0f / (pi * 32.0f * std::pow(std::atan(thr * std::sqrt(std::sqrt(n))), 0.8f));
    }
}

// axis_samples (:193-231): the sample positions of one axis around pos,
// the clipped border first, then the step grid, the last snapped to the
// border
void axis_samples(int32_t pos, int32_t size, int32_t max_rad, int32_t step, std::vector<int32_t> &out) {
    out.clear();
    int32_t a = -max_rad, a2 = INT32_MAX;
    if (a + pos < 0) {
        a2 = a;
        while (a2 + pos < 0) a2 += step;
        if (a2 + pos >= size) a2 = size - pos - 1;
        a = -pos;
        if (a == a2) a2 = INT32_MAX;
    }
    const int32_t e = pos + max_rad >= size ? size - pos - 1 : max_rad;
    int32_t v = a;
    for (;;) {
        if (v > a2) {
            v = a2;
            a2 = INT32_MAX;
        }
        out.push_back(v);
        const int32_t vt = v;
        v += step;
        if (v > e && vt < e) v = e;
        if (v > e) break;
    }
}

struct Sample {
    long off;
    float r1d;
    int lo, hi;
};

struct Ring {
    int32_t max_rad, min_rad, step;
    float rm, zrt;
    bool multi;
    std::vector<Sample> samples;
};

// the buckets a sample updates: its own, or with `multi` a run of
// rne(rm / radius) buckets centred on it (:272-279)
inline void buckets(bool multi, float rm, float r1d, int c, int &lo, int &hi) {
    if (multi) {
        const int ic = (int)std::nearbyint(rm * r1d);
        const int start = (c - (ic >> 1)) & 31;
        lo = start;
        hi = std::min(start + ic, 39);
    } else {
        lo = hi = c;
    }
}

// rings (:257-297)
std::vector<Ring> make_rings(const Levels &L, size_t w, float szrt) {
    const float n = (float)L.count;
    int32_t max_rad = 0, min_rad = 0;
    std::vector<Ring> out;
    std::vector<int32_t> axis;
    for (int atl = 1; atl <= L.count; atl++) {
        Ring R;
        R.step = 1 << (atl - 1);
        R.rm = std::sqrt((float)R.step) * 5.0f;
        max_rad += 4 * R.step;
        R.multi = std::nearbyint(R.rm / (float)(min_rad + 1)) > 0.0f;
        R.zrt = szrt * std::sqrt(std::sqrt(n / (float)atl));
        R.max_rad = max_rad;
        R.min_rad = min_rad;
        axis_samples(max_rad, 2 * max_rad + 1, max_rad, R.step, axis);
        const int32_t maxs = max_rad * max_rad, mins = min_rad * min_rad;
        for (int32_t y2 : axis)
            for (int32_t x2 : axis) {
                const int32_t rads = y2 * y2 + x2 * x2;
                if (rads <= mins || rads > maxs) continue;
                Sample s;
                s.r1d = 1.0f / std::sqrt((float)rads);
                buckets(R.multi, R.rm, s.r1d, arctan32(y2, x2), s.lo, s.hi);
                s.off = (long)y2 * (long)w + x2;
                R.samples.push_back(s);
            }
        out.push_back(std::move(R));
        min_rad = max_rad;
    }
    return out;
}

// the steepest slope per bucket, kept where larger (:324-341)
inline void update(float *ang, float st, float zrt, int lo, int hi, bool t0) {
    if (t0) {
        if (st >= zrt) return;
        const float s3 = st / zrt;
        st *= 1.0f - s3 * s3 * s3;
    } else if (st > zrt) {
        st = zrt;
    }
    for (int k = lo; k <= hi; k++)
        if (ang[k] < st) ang[k] = st;
}

}  // namespace

extern "C" {

int oracle_ssao15_arctan(int y, int x) { return arctan32(y, x); }

/* axis_samples into out (cap entries at most); returns the count */
int oracle_ssao15_axis(int pos, int size, int max_rad, int step, int *out, int cap) {
    std::vector<int32_t> v;
    axis_samples(pos, size, max_rad, step, v);
    const int n = (int)std::min<size_t>(v.size(), (size_t)cap);
    for (int i = 0; i < n; i++) out[i] = v[i];
    return (int)v.size();
}

/* ssao15::ssao15 (src/ssao15.rs:282-411) on the whole G-buffer: amb_shadow
 * of the object pixels; pictures below 4 x 4 stay as they are. */
int oracle_ssao15(mb3d_cu_silight *gbuf, int w_, int h_, double zc_mul, double zcorr, float threshold, int t0_,
                  int wrap_, int threads) {
    if (!gbuf || w_ < 0 || h_ < 0) return -1;
    if (w_ < 4 || h_ < 4) return 0;
    const size_t w = (size_t)w_, h = (size_t)h_;
    const bool t0 = t0_ != 0, wrap = wrap_ != 0;
    const Levels L = build_levels(gbuf, w, h, wrap);
    float szrt, smul, st2;
    sampling_constants(L, zc_mul, zcorr, threshold, t0, szrt, smul, st2);
    const std::vector<Ring> rings = make_rings(L, w, szrt);
    std::vector<int32_t> zps(w * h);
    for (size_t i = 0; i < w * h; i++) zps[i] = L.zp_of(gbuf[i]);
    int nt = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    nt = std::min<int>(nt, (int)h);
    auto rows = [&](int t) {
        std::vector<int32_t> ys, xs;
        for (size_t y = (size_t)t; y < h; y += (size_t)nt)
            for (size_t x = 0; x < w; x++) {
                mb3d_cu_silight &si = gbuf[y * w + x];
                if (zpos16(si) >= 32768u) continue;
                const int32_t zp = zps[y * w + x];
                float ang[40];
                for (float &a : ang) a = -1e10f;
                const int32_t xi = (int32_t)x, yi = (int32_t)y;
                for (size_t ri = 0; ri < rings.size(); ri++) {
                    const Ring &R = rings[ri];
                    const uint16_t *l = L.lev[ri].data();
                    const int32_t r = R.max_rad;
                    if (xi >= r && xi + r < (int32_t)w && yi >= r && yi + r < (int32_t)h) {
                        const long base = (long)(y * w + x);
                        for (const Sample &s : R.samples) {
                            const float st = (float)((int32_t)l[base + s.off] - zp) * s.r1d;
                            update(ang, st, R.zrt, s.lo, s.hi, t0);
                        }
                        continue;
                    }
                    // near the borders: the clipped grid (with the wrap: x on the other side)
                    const int32_t maxs = r * r, mins = R.min_rad * R.min_rad;
                    axis_samples(yi, (int32_t)h, r, R.step, ys);
                    if (wrap)
                        axis_samples(r, 2 * r + 1, r, R.step, xs);
                    else
                        axis_samples(xi, (int32_t)w, r, R.step, xs);
                    for (int32_t y2 : ys) {
                        const size_t rowi = (size_t)(yi + y2) * w;
                        for (int32_t x2 : xs) {
                            const int32_t rads = y2 * y2 + x2 * x2;
                            if (rads <= mins || rads > maxs) continue;
                            const float r1d = 1.0f / std::sqrt((float)rads);
                            const int32_t wi = (int32_t)w;
                            const size_t xx = (size_t)(((xi + x2) % wi + wi) % wi);
                            const float st = (float)((int32_t)l[rowi + xx] - zp) * r1d;
                            int lo, hi;
                            buckets(R.multi, R.rm, r1d, arctan32(y2, x2), lo, hi);
                            update(ang, st, R.zrt, lo, hi, t0);
                        }
                    }
                }
                for (int k = 0; k < 4; k++)
                    if (ang[k + 32] > ang[k]) ang[k] = ang[k + 32];
                float s = 0.0f;
                for (int k = 0; k < 32; k++)
                    if (ang[k] > -1e9f) s += std::atan(ang[k] * st2);
                const float v = std::min(std::max(std::nearbyint(s * smul), 0.0f), 16383.0f);
                si.amb_shadow = (uint16_t)v;
            }
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(rows, t);
    rows(0);
    for (auto &th : pool) th.join();
    return 0;
}

}  // extern "C"
