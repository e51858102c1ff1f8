// The 24-bit screen space ambient occlusion on the card: gpu::ssao24
// (src/gpu.rs:3503) / ssao::ssao24 (src/ssao.rs:129-335) with regular
// sampling.  Per object pixel the largest elevation angle of the depth
// buffer in 32 directions, on levels of an ever smoother depth buffer
// (NextATlevelHiQ: a horizontal, then a vertical pass of
// (p + (p[-step] + p[+step]) / 2) / 2 on 32-bit depths, exact integers) with
// the sampling radius doubling per level; the directions' arctangents summed
// into amb_shadow.
//   k_ssao_first   the first level of the depth pyramid
//   k_ssao_h / _v  the next level's smoothing passes (the whole pyramid is
//                  kept: levels x 4 bytes per pixel)
//   k_ssao_warp    a warp per object pixel, a lane per direction: every
//                  level's 3 or 5 samples with the running maximum in a
//                  register, then the 32 arctangents summed in the
//                  directions' order through shuffles
// The constants of the levels are made on the host by the reference's
// expressions; the samples' arithmetic is single precision, unfused (this
// file is built with -fmad=false), as the reference's CPU pass, so that the
// angles are the reference's bit for bit; the sum's arctangent is the card's
// atanf.
#include <cuda_runtime.h>
#include <stdint.h>
#include <cmath>
#include "kernels.h"

namespace mb3dcu {

namespace {

constexpr int SSAO_MAX_LEVELS = 15;

struct SsaoConsts {
    float dx[32], dy[32];
    float rma[SSAO_MAX_LEVELS][5];
    float smin_rad[SSAO_MAX_LEVELS], istep_f[SSAO_MAX_LEVELS], sit[SSAO_MAX_LEVELS], szrt[SSAO_MAX_LEVELS];
    int step_count[SSAO_MAX_LEVELS];
    int64_t wlo, whi, hlo, hhi, mw2, mh2;
    float smul;
    int levels, t0, wrap, w, h;
};

__device__ __forceinline__ float rne_d(float x) {
    const float M = 8388608.0f;
    const float a = fabsf(x);
    return a < M ? copysignf(__fsub_rn(__fadd_rn(a, M), M), x) : x;
}

__global__ void k_ssao_first(const mb3d_cu_silight *gbuf, uint32_t npix, uint32_t *pia) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        const uint32_t zf = gbuf[i].zpos_fine;
        pia[i] = (zf >> 16) < 32768u ? (zf & 0xFFFFFF00u) >> 1 : 0u;
    }
}

__global__ void k_ssao_warp(const __grid_constant__ SsaoConsts C, mb3d_cu_silight *gbuf, const uint32_t *pyr,
                            uint32_t npix) {
    const int d = (int)(threadIdx.x & 31);
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; i < npix; i += warps) {
        const uint32_t zf = gbuf[i].zpos_fine;
        if ((zf >> 16) >= 32768u) continue;  // (the whole warp: one pixel)
        const int64_t zp = (int64_t)((zf & 0xFFFFFF00u) >> 1);
        const int x = (int)(i % (uint32_t)C.w), y = (int)(i / (uint32_t)C.w);
        const float dx = C.dx[d], dy = C.dy[d];
        int am = -32768;
        for (int l = 0; l < C.levels; l++) {
            const uint32_t *pia = pyr + (size_t)l * npix;
            const float smin_rad = C.smin_rad[l], istep_f = C.istep_f[l], sit = C.sit[l], szrt = C.szrt[l];
            float sx = __fadd_rn((float)x, __fmul_rn(dx, smin_rad));
            float sy = __fadd_rn((float)y, __fmul_rn(dy, smin_rad));
            for (int k = 0; k < C.step_count[l]; k++) {
                const float r = C.rma[l][k];
                int64_t x2 = (int64_t)rne_d(sx), y2 = (int64_t)rne_d(sy);
                if (C.wrap) {
                    x2 = ((x2 % (int64_t)C.w) + (int64_t)C.w) % (int64_t)C.w;
                } else if (x2 < 0) {
                    x2 = -x2;
                    if (x2 >= C.wlo) break;
                } else if (x2 >= (int64_t)C.w) {
                    x2 = C.mw2 - x2;
                    if (x2 < C.whi) break;
                }
                if (y2 < 0) {
                    y2 = -y2;
                    if (y2 >= C.hlo) break;
                } else if (y2 >= (int64_t)C.h) {
                    y2 = C.mh2 - y2;
                    if (y2 < C.hhi) break;
                }
                // (the mirrored index lies in the picture: the border test
                // above stops a sample that would leave it)
                if (x2 < 0 || x2 >= (int64_t)C.w || y2 < 0 || y2 >= (int64_t)C.h) break;
                const float st = __fmul_rn((float)((int64_t)pia[(size_t)y2 * (size_t)C.w + (size_t)x2] - zp), r);
                const float q = C.t0 ? __fdiv_rn(__fmul_rn(st, sit), __fadd_rn(__fmul_rn(st, st), szrt))
                                     : __fdiv_rn(__fmul_rn(st, sit), __fadd_rn(szrt, fabsf(st)));
                float it = rne_d(q);
                if (isnan(it)) it = -32768.0f;
                const int iv = it >= 32767.0f ? 32767 : it <= -32768.0f ? -32768 : (int)it;
                am = iv > am ? iv : am;
                sx = __fadd_rn(sx, __fmul_rn(dx, istep_f));
                sy = __fadd_rn(sy, __fmul_rn(dy, istep_f));
            }
        }
        // the sum of the arctangents in the directions' order (as the
        // reference's loop): every lane adds the 32 lanes' terms in turn
        const bool valid = am > -32768;
        const float at = valid ? atanf(__fmul_rn((float)am, 0.0002441406f)) : 0.0f;
        float s = 0.0f;
#pragma unroll
        for (int k = 0; k < 32; k++) {
            const float v = __shfl_sync(0xffffffffu, at, k);
            const int f = __shfl_sync(0xffffffffu, valid ? 1 : 0, k);
            if (f) s = __fadd_rn(s, v);
        }
        if (d == 0) {
            const float q = rne_d(__fmul_rn(s, C.smul));
            int v = q >= 2147483647.0f ? 2147483647 : q <= -2147483648.0f ? (-2147483647 - 1) : (int)q;
            v = v < 0 ? 0 : v > 16383 ? 16383 : v;
            gbuf[i].amb_shadow = (uint16_t)v;
        }
    }
}

// ---------------------------------------------------------------------------
// random sampling (TAmbHiQCalcR, src/ssao.rs:207-247): every sample jittered
// inside its step cell by an LCG whose chain runs, per pass, level and row,
// through the row's object pixels in order, their directions in order and
// the directions' steps; a direction that leaves the picture stops early and
// draws fewer numbers.  A warp walks one row (a lane per direction), so the
// chain is kept exactly: where no sample of the pixel can leave the picture
// every direction draws step_count numbers and lane d starts d * step_count
// numbers on (a jump ahead of the chain); elsewhere the lanes guess those
// starts, count what they drew, and take the counts' prefix sum as the next
// guess until it holds (each round fixes at least one more direction).

struct SsaoRnd {
    uint32_t ja[161], jc[161];  // the chain's jump by n numbers: s -> ja[n] s + jc[n]
    int32_t cxmin[SSAO_MAX_LEVELS], cxmax[SSAO_MAX_LEVELS], cymin[SSAO_MAX_LEVELS], cymax[SSAO_MAX_LEVELS];
    int32_t iand[SSAO_MAX_LEVELS];
    float ssub[SSAO_MAX_LEVELS];
    int pass, imin;
};

__device__ __forceinline__ uint32_t jump(const SsaoRnd &R, uint32_t s, int n) { return R.ja[n] * s + R.jc[n]; }

// one direction's samples of a pixel from the chain state s (before its
// first number): the numbers it drew and its largest angle
__device__ __forceinline__ int rnd_dir(const SsaoConsts &C, const SsaoRnd &R, int l, int d, uint32_t s, int x, int y,
                                       int64_t zp, const uint32_t *pia, int am_in, int &am_out) {
    const float dx = C.dx[d], dy = C.dy[d], smin_rad = C.smin_rad[l], istep_f = C.istep_f[l];
    const float sit = C.sit[l], szrt = C.szrt[l], ssub = R.ssub[l];
    const int64_t iand = R.iand[l];
    float ox = __fsub_rn(__fmul_rn(dx, smin_rad), ssub), oy = __fsub_rn(__fmul_rn(dy, smin_rad), ssub);
    int am = am_in, drawn = 0;
    for (int k = 0; k < C.step_count[l]; k++) {
        const int64_t cx = (int64_t)rne_d(ox), cy = (int64_t)rne_d(oy);
        ox = __fadd_rn(ox, __fmul_rn(dx, istep_f));
        oy = __fadd_rn(oy, __fmul_rn(dy, istep_f));
        s = s * 214013u + 2531011u;
        drawn++;
        const int64_t jx = cx + ((int64_t)(s >> 16) & iand), jy = cy + ((int64_t)(s >> 10) & iand);
        const float dd = (float)(jx * jx + jy * jy);
        if (dd == 0.0f) continue;
        const float r = __fdiv_rn(1.0f, __fsqrt_rn(dd));
        int64_t x2 = (int64_t)x + jx, y2 = (int64_t)y + jy;
        if (C.wrap) {
            x2 = ((x2 % (int64_t)C.w) + (int64_t)C.w) % (int64_t)C.w;
        } else if (x2 < 0) {
            x2 = -x2;
            if (x2 >= C.wlo) break;
        } else if (x2 >= (int64_t)C.w) {
            x2 = C.mw2 - x2;
            if (x2 < C.whi) break;
        }
        if (y2 < 0) {
            y2 = -y2;
            if (y2 >= C.hlo) break;
        } else if (y2 >= (int64_t)C.h) {
            y2 = C.mh2 - y2;
            if (y2 < C.hhi) break;
        }
        if (x2 < 0 || x2 >= (int64_t)C.w || y2 < 0 || y2 >= (int64_t)C.h) break;
        const float st = __fmul_rn((float)((int64_t)pia[(size_t)y2 * (size_t)C.w + (size_t)x2] - zp), r);
        const float q = C.t0 ? __fdiv_rn(__fmul_rn(st, sit), __fadd_rn(__fmul_rn(st, st), szrt))
                             : __fdiv_rn(__fmul_rn(st, sit), __fadd_rn(szrt, fabsf(st)));
        float it = rne_d(q);
        if (isnan(it)) it = -32768.0f;
        const int iv = it >= 32767.0f ? 32767 : it <= -32768.0f ? -32768 : (int)it;
        am = iv > am ? iv : am;
    }
    am_out = am;
    return drawn;
}

// one pass: a warp per row; ang holds each pixel's 32 largest angles + 32768
// (0: none yet), acc the passes' sums
__global__ void k_ssao_rnd(const __grid_constant__ SsaoConsts C, const __grid_constant__ SsaoRnd R,
                           const mb3d_cu_silight *gbuf, const uint32_t *pyr, uint16_t *ang, uint32_t *acc,
                           uint32_t npix) {
    const int d = (int)(threadIdx.x & 31);
    const int warps = (int)((gridDim.x * blockDim.x) >> 5);
    for (int y = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5); y < C.h; y += warps) {
        for (int l = 0; l < C.levels; l++) {
            const uint32_t *pia = pyr + (size_t)l * npix;
            const int sc = C.step_count[l];
            const bool last = l == C.levels - 1;
            uint32_t s = (uint32_t)(int32_t)(0x24563487LL + ((int64_t)y + 1) * 0x324594A1LL + (int64_t)R.pass * 0x5851F42DLL);
            const bool safe_y = y + R.cymin[l] >= 0 && y + R.cymax[l] + R.iand[l] < C.h;
            for (int x = 0; x < C.w; x++) {
                const size_t i = (size_t)y * C.w + x;
                const uint32_t zf = gbuf[i].zpos_fine;
                if ((zf >> 16) >= 32768u) continue;  // (the whole warp: one pixel)
                const int64_t zp = (int64_t)((zf & 0xFFFFFF00u) >> 1);
                const int am_in = (int)ang[i * 32 + d] - 32768;
                const bool safe = safe_y && (C.wrap || (x + R.cxmin[l] >= 0 && x + R.cxmax[l] + R.iand[l] < C.w));
                int off = d * sc, am = am_in, total = 32 * sc;
                for (int round = 0; round < 40; round++) {
                    const int drawn = rnd_dir(C, R, l, d, jump(R, s, off), x, y, zp, pia, am_in, am);
                    if (safe) break;  // (every direction drew step_count numbers)
                    int incl = drawn;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        const int v = __shfl_up_sync(0xffffffffu, incl, o);
                        if (d >= o) incl += v;
                    }
                    const int next = incl - drawn;
                    total = __shfl_sync(0xffffffffu, incl, 31);
                    if (__all_sync(0xffffffffu, next == off)) break;
                    off = next;
                }
                ang[i * 32 + d] = (uint16_t)(am + 32768);
                if (last) {
                    const bool valid = am > -32768;
                    const float at = valid ? atanf(__fmul_rn((float)am, 0.0002441406f)) : 0.0f;
                    float sum = 0.0f;
#pragma unroll
                    for (int k = 0; k < 32; k++) {
                        const float v = __shfl_sync(0xffffffffu, at, k);
                        const int f = __shfl_sync(0xffffffffu, valid ? 1 : 0, k);
                        if (f) sum = __fadd_rn(sum, v);
                    }
                    if (d == 0) {
                        const float q = rne_d(__fmul_rn(sum, C.smul));
                        int v = q >= 2147483647.0f ? 2147483647 : q <= -2147483648.0f ? (-2147483647 - 1) : (int)q;
                        v = v < 0 ? 0 : v > R.imin ? R.imin : v;
                        acc[i] += (uint32_t)v;
                    }
                }
                s = jump(R, s, total);
            }
        }
    }
}

__global__ void k_ssao_acc(const uint32_t *acc, mb3d_cu_silight *gbuf, uint32_t npix) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x)
        if ((gbuf[i].zpos_fine >> 16) < 32768u) gbuf[i].amb_shadow = (uint16_t)(acc[i] > 16383u ? 16383u : acc[i]);
}

__global__ void k_ssao_h(const uint32_t *src, uint32_t *dst, int w, int h, int step, int wrap) {
    const size_t n = (size_t)w * h;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % (size_t)w);
        const size_t row = i - (size_t)x;
        int a, b;
        if (wrap) {
            a = (int)(((size_t)x + (size_t)w - (size_t)step % (size_t)w) % (size_t)w);
            b = (int)(((size_t)x + (size_t)step) % (size_t)w);
        } else {
            a = x >= step ? x - step : 0;
            b = x + step < w - 1 ? x + step : w - 1;
        }
        dst[i] = (uint32_t)(((uint64_t)src[i] + (((uint64_t)src[row + a] + (uint64_t)src[row + b]) >> 1)) >> 1);
    }
}

__global__ void k_ssao_v(const uint32_t *src, uint32_t *dst, int w, int h, int step) {
    const size_t n = (size_t)w * h;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int y = (int)(i / (size_t)w), x = (int)(i % (size_t)w);
        const int ya = y >= step ? y - step : 0, yb = y + step < h - 1 ? y + step : h - 1;
        dst[i] = (uint32_t)(((uint64_t)src[i] + (((uint64_t)src[(size_t)ya * w + x] + (uint64_t)src[(size_t)yb * w + x]) >> 1)) >> 1);
    }
}

// aATlevelCount (src/ssao.rs:113-125)
int level_count(int w, int h) {
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

int grid_of(size_t n, int sms) {
    size_t b = (n + 255) / 256;
    const size_t cap = (size_t)sms * 16;
    return (int)(b < 1 ? 1 : b > cap ? cap : b);
}

}  // namespace

// the scratch: the depth pyramid (a level per 4 bytes x pixels) and one
// level of the smoothing's intermediate
size_t ssao_scratch_bytes(int w, int h, int random) {
    const size_t npix = (size_t)w * h;
    const size_t pyr = ((size_t)level_count(w, h) + 1) * npix * sizeof(uint32_t);
    return random > 0 ? pyr + npix * 32 * sizeof(uint16_t) + npix * sizeof(uint32_t) : pyr;
}

void ssao24_launch(mb3d_cu_silight *gbuf, int w, int h, double zc_mul, double zcorr, const mb3d_cu_ssao_opts &o,
                   void *scratch, int sms, cudaStream_t s) {
    const uint32_t npix = (uint32_t)((size_t)w * h);
    const int levels = level_count(w, h);
    uint32_t *pyr = reinterpret_cast<uint32_t *>(scratch), *tmp = pyr + (size_t)levels * npix;
    const double z_scale = (std::pow(256.0 / zc_mul + 1.0, 2) - 1.0) / zcorr;
    const float thr = std::fmax(o.threshold, 0.01f);
    SsaoConsts C;
    for (int i = 0; i < 32; i++) {
        const double a = (double)i * M_PI / 16.0;
        C.dx[i] = (float)std::sin(a);
        C.dy[i] = (float)std::cos(a);
    }
    C.wlo = (int64_t)std::nearbyint((float)w * o.border_mirror);
    C.whi = (int64_t)w - 1 - C.wlo;
    C.hlo = (int64_t)std::nearbyint((float)h * o.border_mirror);
    C.hhi = (int64_t)h - 1 - C.hlo;
    C.mw2 = 2 * ((int64_t)w - 1);
    C.mh2 = 2 * ((int64_t)h - 1);
    C.t0 = o.t0 ? 1 : 0;
    C.wrap = o.wrap_x ? 1 : 0;
    C.w = w;
    C.h = h;
    C.levels = levels;
    const bool t0 = o.t0 != 0;
    const int passes = o.random > 0 ? o.random : 1;
    const bool rnd = o.random > 0;
    for (int level = 1; level <= levels; level++) {
        const int l = level - 1;
        float sit = (float)(z_scale / 22000.0 * 4096.0);
        float szrt = thr * (t0 ? 1.0f : 0.7f) * 4096.0f / sit * std::sqrt(std::sqrt((float)levels / (float)level));
        if (t0) szrt *= szrt;
        const float at = rnd ? std::atan(thr * (t0 ? 0.64f : 0.65f) * std::sqrt(std::sqrt((float)levels)))
                             : std::atan(thr * 0.6f * std::sqrt(std::sqrt((float)levels)));
        C.smul = 1.5f * 32767.0f / ((float)M_PI * 32.0f * (t0 ? at : std::pow(at, 0.9f))) / (float)passes;
        const int64_t istep = (int64_t)1 << (level - 1);
        C.smin_rad[l] = istep < 2 ? 1.0f : 3.25f * (float)istep;
        C.step_count[l] = istep < 2 ? 5 : 3;
        for (int k = 0; k < 5; k++)
            C.rma[l][k] = k < C.step_count[l] ? 1.0f / (C.smin_rad[l] + (float)((int64_t)k * istep) + 0.1f) : 0.0f;
        C.istep_f[l] = (float)istep;
        sit *= szrt;
        C.sit[l] = sit;
        C.szrt[l] = szrt;
    }
    // the pyramid: level 1 from the depths, level l + 1 from level l
    k_ssao_first<<<grid_of(npix, sms), 256, 0, s>>>(gbuf, npix, pyr);
    for (int level = 1; level < levels; level++) {
        const int step = 1 << level;
        k_ssao_h<<<grid_of(npix, sms), 256, 0, s>>>(pyr + (size_t)(level - 1) * npix, tmp, w, h, step, C.wrap);
        k_ssao_v<<<grid_of(npix, sms), 256, 0, s>>>(tmp, pyr + (size_t)level * npix, w, h, step);
    }
    if (!rnd) {
        k_ssao_warp<<<grid_of((size_t)npix * 32, sms), 256, 0, s>>>(C, gbuf, pyr, npix);
        return;
    }
    // random sampling: the chain's jumps and each level's cells' reach
    SsaoRnd R;
    R.ja[0] = 1u;
    R.jc[0] = 0u;
    for (int n = 1; n <= 160; n++) {
        R.ja[n] = R.ja[n - 1] * 214013u;
        R.jc[n] = R.jc[n - 1] * 214013u + 2531011u;
    }
    for (int level = 1; level <= levels; level++) {
        const int l = level - 1;
        const int64_t istep = (int64_t)1 << (level - 1);
        R.iand[l] = (int32_t)(istep - 1);
        R.ssub[l] = (float)(istep - 1) * 0.5f;
        int64_t xmin = 0, xmax = 0, ymin = 0, ymax = 0;
        for (int d = 0; d < 32; d++) {
            float ox = C.dx[d] * C.smin_rad[l] - R.ssub[l], oy = C.dy[d] * C.smin_rad[l] - R.ssub[l];
            for (int k = 0; k < C.step_count[l]; k++) {
                const int64_t cx = (int64_t)std::nearbyint(ox), cy = (int64_t)std::nearbyint(oy);
                xmin = std::min(xmin, cx - 1);
                xmax = std::max(xmax, cx + 1);
                ymin = std::min(ymin, cy - 1);
                ymax = std::max(ymax, cy + 1);
                ox += C.dx[d] * C.istep_f[l];
                oy += C.dy[d] * C.istep_f[l];
            }
        }
        // (one more pixel each way than the cells: a safe bound on the rounding)
        R.cxmin[l] = (int32_t)xmin;
        R.cxmax[l] = (int32_t)xmax;
        R.cymin[l] = (int32_t)ymin;
        R.cymax[l] = (int32_t)ymax;
    }
    R.imin = 16383 / passes;
    uint16_t *ang = reinterpret_cast<uint16_t *>(tmp + npix);
    uint32_t *acc = reinterpret_cast<uint32_t *>(ang + (size_t)npix * 32);
    cudaMemsetAsync(acc, 0, (size_t)npix * sizeof(uint32_t), s);
    const int row_blocks = (h * 32 + 255) / 256;
    for (int pass = 0; pass < passes; pass++) {
        R.pass = pass;
        cudaMemsetAsync(ang, 0, (size_t)npix * 32 * sizeof(uint16_t), s);
        k_ssao_rnd<<<row_blocks, 256, 0, s>>>(C, R, gbuf, pyr, ang, acc, npix);
    }
    k_ssao_acc<<<grid_of(npix, sms), 256, 0, s>>>(acc, gbuf, npix);
}

}  // namespace mb3dcu
