// TEST INFRASTRUCTURE: the screen space ambient occlusion of the reference
// ("24 bit" SSAO, ssao::ssao24, src/ssao.rs:129-335) on the CPU, for the
// parity of the card's SSAO pass: per object pixel the largest elevation
// angle of the depth buffer in 32 directions, on levels of an ever smoother
// depth buffer (NextATlevelHiQ, src/ssao.rs:86-110) with the sampling radius
// doubling per level, the angles' arctangents summed on the last level into
// amb_shadow.  Regular sampling and random sampling (SsaoParams::random
// passes, TAmbHiQCalcR: each sample jittered inside its step cell by a
// per-row LCG chain), the threshold, the "down to 0" variant (t0), the
// mirrored border and the panorama's wrap.
// Single precision, unfused, as the reference.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../include/mb3d_cu.h"

namespace {

// round half to even of a float (src/ssao.rs:42-49): |x| < 2^23 by adding
// and subtracting 2^23, larger values are integers already
float rne(float x) {
    const float M = 8388608.0f;
    float a = std::fabs(x);
    if (a < M) return std::copysign((a + M) - M, x);
    return x;
}

// SmoothH / SmoothV on a line (src/ssao.rs:59-69)
void smooth_line(uint32_t *dst, const uint32_t *src, size_t n, size_t step, bool wrap) {
    if (n == 0) return;
    const size_t last = n - 1;
    for (size_t x = 0; x < n; x++) {
        size_t a, b;
        if (wrap) {
            a = (x + n - step % n) % n;
            b = (x + step) % n;
        } else {
            a = x >= step ? x - step : 0;
            b = x + step < last ? x + step : last;
        }
        dst[x] = (uint32_t)(((uint64_t)dst[x] + (((uint64_t)src[a] + (uint64_t)src[b]) >> 1)) >> 1);
    }
}

// NextATlevelHiQ (src/ssao.rs:86-110): rows, then columns
void next_level(std::vector<uint32_t> &pia, size_t w, size_t h, size_t step, bool wrap) {
    std::vector<uint32_t> sa(w);
    for (size_t y = 0; y < h; y++) {
        uint32_t *row = &pia[y * w];
        std::memcpy(sa.data(), row, w * 4);
        smooth_line(row, sa.data(), w, step, wrap);
    }
    const std::vector<uint32_t> src = pia;
    for (size_t y = 0; y < h; y++) {
        const uint32_t *a = &src[(y >= step ? y - step : 0) * w];
        const uint32_t *b = &src[(y + step < h - 1 ? y + step : h - 1) * w];
        uint32_t *row = &pia[y * w];
        for (size_t x = 0; x < w; x++)
            row[x] = (uint32_t)(((uint64_t)row[x] + (((uint64_t)a[x] + (uint64_t)b[x]) >> 1)) >> 1);
    }
}

}  // namespace

extern "C" {

// aATlevelCount (src/ssao.rs:113-125)
int oracle_ssao_levels(int w, int h) {
    const int64_t ymin = (int64_t)std::nearbyint(std::sqrt((double)((size_t)w * w + (size_t)h * h)) * 0.5);
    int y = 1;
    int64_t x = 5;
    for (;;) {
        y += 1;
        x <<= 1;
        if (y == 15 || x > ymin) break;
    }
    return y;
}

// rne of the reference, for its known-answer test
float oracle_ssao_rne(float x) { return rne(x); }

/* ssao24 on the w x h G-buffer gbuf (in place: amb_shadow of the object
 * pixels); zc_mul, zcorr are the scene's z-buffer constants. */
int oracle_ssao24(mb3d_cu_silight *gbuf, int w_, int h_, double zc_mul, double zcorr, float threshold,
                  float border_mirror, int t0, int wrap_x, int random) {
    if (w_ <= 0 || h_ <= 0) return 0;
    const size_t w = (size_t)w_, h = (size_t)h_, npix = w * h;
    const int levels = oracle_ssao_levels(w_, h_);
    const double z_scale = (std::pow(256.0 / zc_mul + 1.0, 2) - 1.0) / zcorr;
    const float thr = std::fmax(threshold, 0.01f);
    const int64_t wlo = (int64_t)std::nearbyint((float)w * border_mirror), whi = (int64_t)w - 1 - wlo;
    const int64_t hlo = (int64_t)std::nearbyint((float)h * border_mirror), hhi = (int64_t)h - 1 - hlo;
    const int64_t mw2 = 2 * ((int64_t)w - 1), mh2 = 2 * ((int64_t)h - 1);
    float dx[32], dy[32];
    for (int i = 0; i < 32; i++) {
        const double a = (double)i * M_PI / 16.0;
        dx[i] = (float)std::sin(a);
        dy[i] = (float)std::cos(a);
    }
    std::vector<uint8_t> object(npix);
    std::vector<uint32_t> pia(npix);
    std::vector<uint32_t> zfine(npix);
    for (size_t i = 0; i < npix; i++) zfine[i] = (gbuf[i].zpos_fine & 0xFFFFFF00u) >> 1;
    for (size_t i = 0; i < npix; i++) object[i] = (gbuf[i].zpos_fine >> 16) < 32768;
    std::vector<int16_t> ang(npix * 32);
    const int passes = random > 0 ? random : 1;
    const bool rnd = random > 0;
    std::vector<uint32_t> acc(npix, 0u);
    for (int pass = 0; pass < passes; pass++) {
    for (size_t i = 0; i < npix; i++) pia[i] = object[i] ? zfine[i] : 0u;
    std::fill(ang.begin(), ang.end(), (int16_t)-32768);
    for (int level = 1; level <= levels; level++) {
        const bool sum_up = level == levels;
        float sit = (float)(z_scale / 22000.0 * 4096.0);
        float szrt = thr * (t0 ? 1.0f : 0.7f) * 4096.0f / sit * std::sqrt(std::sqrt((float)levels / (float)level));
        if (t0) szrt *= szrt;
        const float at = rnd ? std::atan(thr * (t0 ? 0.64f : 0.65f) * std::sqrt(std::sqrt((float)levels)))
                             : std::atan(thr * 0.6f * std::sqrt(std::sqrt((float)levels)));
        const float smul = 1.5f * 32767.0f / ((float)M_PI * 32.0f * (t0 ? at : std::pow(at, 0.9f))) / (float)passes;
        const int imin = 16383 / passes;
        const int64_t iand = ((int64_t)1 << (level - 1)) - 1;
        const float ssub = (float)iand * 0.5f;
        const int64_t istep = (int64_t)1 << (level - 1);
        const float smin_rad = istep < 2 ? 1.0f : 3.25f * (float)istep;
        const int step_count = istep < 2 ? 5 : 3;
        float rma[5];
        for (int k = 0; k < step_count; k++) rma[k] = 1.0f / (smin_rad + (float)((int64_t)k * istep) + 0.1f);
        // the random mode's cell corners (src/ssao.rs:188-203)
        int64_t cells[32][5][2];
        for (int d = 0; d < 32; d++) {
            float ox = dx[d] * smin_rad - ssub, oy = dy[d] * smin_rad - ssub;
            for (int k = 0; k < step_count; k++) {
                cells[d][k][0] = (int64_t)rne(ox);
                cells[d][k][1] = (int64_t)rne(oy);
                ox += dx[d] * (float)istep;
                oy += dy[d] * (float)istep;
            }
        }
        sit *= szrt;
        for (size_t y = 0; y < h; y++) {
            int32_t seed = (int32_t)(0x24563487LL + ((int64_t)y + 1) * 0x324594A1LL + (int64_t)pass * 0x5851F42DLL);
            for (size_t x = 0; x < w; x++) {
                const size_t i = y * w + x;
                if (!object[i]) continue;
                const int64_t zp = (int64_t)zfine[i];
                int16_t *am = &ang[i * 32];
                for (int d = 0; d < 32; d++) {
                    float sx = (float)x + dx[d] * smin_rad;
                    float sy = (float)y + dy[d] * smin_rad;
                    for (int k = 0; k < step_count; k++) {
                        float r = rma[k];
                        int64_t x2, y2;
                        if (rnd) {
                            // TAmbHiQCalcR: a jittered sample inside the step's cell
                            seed = (int32_t)((uint32_t)seed * 214013u + 2531011u);
                            const int64_t jx = cells[d][k][0] + ((int64_t)((uint32_t)seed >> 16) & iand);
                            const int64_t jy = cells[d][k][1] + ((int64_t)((uint32_t)seed >> 10) & iand);
                            const float dd = (float)(jx * jx + jy * jy);
                            if (dd == 0.0f) {
                                sx += dx[d] * (float)istep;
                                sy += dy[d] * (float)istep;
                                continue;
                            }
                            r = 1.0f / std::sqrt(dd);
                            x2 = (int64_t)x + jx;
                            y2 = (int64_t)y + jy;
                        } else {
                            x2 = (int64_t)rne(sx);
                            y2 = (int64_t)rne(sy);
                        }
                        if (wrap_x) {
                            x2 = ((x2 % (int64_t)w) + (int64_t)w) % (int64_t)w;
                        } else if (x2 < 0) {
                            x2 = -x2;
                            if (x2 >= wlo) break;
                        } else if (x2 >= (int64_t)w) {
                            x2 = mw2 - x2;
                            if (x2 < whi) break;
                        }
                        if (y2 < 0) {
                            y2 = -y2;
                            if (y2 >= hlo) break;
                        } else if (y2 >= (int64_t)h) {
                            y2 = mh2 - y2;
                            if (y2 < hhi) break;
                        }
                        const float st = (float)((int64_t)pia[(size_t)y2 * w + (size_t)x2] - zp) * r;
                        float it = rne(t0 ? st * sit / (st * st + szrt) : st * sit / (szrt + std::fabs(st)));
                        if (std::isnan(it)) it = -32768.0f;
                        const int16_t iv = it >= 32767.0f ? (int16_t)32767 : it <= -32768.0f ? (int16_t)-32768 : (int16_t)it;
                        if (iv > am[d]) am[d] = iv;
                        sx += dx[d] * (float)istep;
                        sy += dy[d] * (float)istep;
                    }
                }
                if (sum_up) {
                    float s = 0.0f;
                    for (int d = 0; d < 32; d++)
                        if (am[d] > -32768) s += std::atan((float)am[d] * 0.0002441406f);
                    const float q = rne(s * smul);
                    int v = q >= 2147483647.0f ? 2147483647 : q <= -2147483648.0f ? (-2147483647 - 1) : (int)q;
                    v = v < 0 ? 0 : v > imin ? imin : v;
                    acc[i] += (uint32_t)v;
                }
            }
        }
        if (level < levels) next_level(pia, w, h, (size_t)1 << level, wrap_x != 0);
    }
    }
    for (size_t i = 0; i < npix; i++)
        if (object[i]) gbuf[i].amb_shadow = (uint16_t)(acc[i] > 16383u ? 16383u : acc[i]);
    return 0;
}
}
