// The 24-bit screen space ambient occlusion on the card: gpu::ssao24
// (src/gpu.rs:3503) / ssao::ssao24 (src/ssao.rs:129-335) with regular
// sampling.  Per object pixel the largest elevation angle of the depth
// buffer in 32 directions, on levels of an ever smoother depth buffer
// (NextATlevelHiQ: a horizontal, then a vertical pass of
// (p + (p[-step] + p[+step]) / 2) / 2 on 32-bit depths, exact integers) with
// the sampling radius doubling per level; on the last level the directions'
// arctangents are summed into amb_shadow.
//   k_ssao_first   the first level and the angles' start (-32768)
//   k_ssao_angles  one thread per (object pixel, direction): the level's
//                  3 or 5 samples, the running maximum per direction
//   k_ssao_h / _v  the next level's smoothing passes
//   k_ssao_sum     per object pixel the sum of the 32 arctangents
// The constants of a level are made on the host by the reference's
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

struct SsaoLevel {
    float dx[32], dy[32];
    float rma[5];
    float smin_rad, istep_f, sit, szrt;
    int64_t wlo, whi, hlo, hhi, mw2, mh2;
    int step_count, t0, wrap, w, h;
};

__device__ __forceinline__ float rne_d(float x) {
    const float M = 8388608.0f;
    const float a = fabsf(x);
    return a < M ? copysignf(__fsub_rn(__fadd_rn(a, M), M), x) : x;
}

__global__ void k_ssao_first(const mb3d_cu_silight *gbuf, uint32_t npix, uint32_t *pia, int16_t *ang) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        const uint32_t zf = gbuf[i].zpos_fine;
        pia[i] = (zf >> 16) < 32768u ? (zf & 0xFFFFFF00u) >> 1 : 0u;
        int4 *a = reinterpret_cast<int4 *>(ang + (size_t)i * 32);
        const int v = (int)0x80008000u;  // two int16 of -32768
#pragma unroll
        for (int k = 0; k < 4; k++) a[k] = make_int4(v, v, v, v);
    }
}

__global__ void k_ssao_angles(const __grid_constant__ SsaoLevel L, const mb3d_cu_silight *gbuf, const uint32_t *pia,
                              int16_t *ang, uint32_t npix) {
    const size_t n = (size_t)npix * 32;
    for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n; t += (size_t)gridDim.x * blockDim.x) {
        const uint32_t i = (uint32_t)(t >> 5);
        const int d = (int)(t & 31);
        const uint32_t zf = gbuf[i].zpos_fine;
        if ((zf >> 16) >= 32768u) continue;
        const int64_t zp = (int64_t)((zf & 0xFFFFFF00u) >> 1);
        const int x = (int)(i % (uint32_t)L.w), y = (int)(i / (uint32_t)L.w);
        const float dx = L.dx[d], dy = L.dy[d];
        float sx = __fadd_rn((float)x, __fmul_rn(dx, L.smin_rad));
        float sy = __fadd_rn((float)y, __fmul_rn(dy, L.smin_rad));
        int am = ang[t];
        for (int k = 0; k < L.step_count; k++) {
            const float r = L.rma[k];
            int64_t x2 = (int64_t)rne_d(sx), y2 = (int64_t)rne_d(sy);
            if (L.wrap) {
                x2 = ((x2 % (int64_t)L.w) + (int64_t)L.w) % (int64_t)L.w;
            } else if (x2 < 0) {
                x2 = -x2;
                if (x2 >= L.wlo) break;
            } else if (x2 >= (int64_t)L.w) {
                x2 = L.mw2 - x2;
                if (x2 < L.whi) break;
            }
            if (y2 < 0) {
                y2 = -y2;
                if (y2 >= L.hlo) break;
            } else if (y2 >= (int64_t)L.h) {
                y2 = L.mh2 - y2;
                if (y2 < L.hhi) break;
            }
            // (the mirrored index lies in the picture: the border test above
            // stops a sample that would leave it)
            if (x2 < 0 || x2 >= (int64_t)L.w || y2 < 0 || y2 >= (int64_t)L.h) break;
            const float st = __fmul_rn((float)((int64_t)pia[(size_t)y2 * (size_t)L.w + (size_t)x2] - zp), r);
            const float q = L.t0 ? __fdiv_rn(__fmul_rn(st, L.sit), __fadd_rn(__fmul_rn(st, st), L.szrt))
                                 : __fdiv_rn(__fmul_rn(st, L.sit), __fadd_rn(L.szrt, fabsf(st)));
            float it = rne_d(q);
            if (isnan(it)) it = -32768.0f;
            const int iv = it >= 32767.0f ? 32767 : it <= -32768.0f ? -32768 : (int)it;
            am = iv > am ? iv : am;
            sx = __fadd_rn(sx, __fmul_rn(dx, L.istep_f));
            sy = __fadd_rn(sy, __fmul_rn(dy, L.istep_f));
        }
        ang[t] = (int16_t)am;
    }
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

__global__ void k_ssao_sum(mb3d_cu_silight *gbuf, const int16_t *ang, uint32_t npix, float smul, int imin) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        if ((gbuf[i].zpos_fine >> 16) >= 32768u) continue;
        float s = 0.0f;
        for (int d = 0; d < 32; d++) {
            const int v = ang[(size_t)i * 32 + d];
            if (v > -32768) s = __fadd_rn(s, atanf(__fmul_rn((float)v, 0.0002441406f)));
        }
        const float q = rne_d(__fmul_rn(s, smul));
        int v = q >= 2147483647.0f ? 2147483647 : q <= -2147483648.0f ? (-2147483647 - 1) : (int)q;
        v = v < 0 ? 0 : v > imin ? imin : v;
        gbuf[i].amb_shadow = (uint16_t)(v > 16383 ? 16383 : v);
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

// the scratch: two depth levels (ping-pong), then the angles at a 256-byte
// boundary (their 16-byte stores)
static size_t ang_offset(size_t npix) { return (2 * npix * sizeof(uint32_t) + 255) & ~(size_t)255; }

size_t ssao_scratch_bytes(int w, int h) {
    const size_t npix = (size_t)w * h;
    return ang_offset(npix) + npix * 32 * sizeof(int16_t);
}

void ssao24_launch(mb3d_cu_silight *gbuf, int w, int h, double zc_mul, double zcorr, const mb3d_cu_ssao_opts &o,
                   void *scratch, int sms, cudaStream_t s) {
    const uint32_t npix = (uint32_t)((size_t)w * h);
    uint32_t *pa = reinterpret_cast<uint32_t *>(scratch), *pb = pa + npix;
    int16_t *ang = reinterpret_cast<int16_t *>(reinterpret_cast<unsigned char *>(scratch) + ang_offset(npix));
    const int levels = level_count(w, h);
    const double z_scale = (std::pow(256.0 / zc_mul + 1.0, 2) - 1.0) / zcorr;
    const float thr = std::fmax(o.threshold, 0.01f);
    SsaoLevel L;
    for (int i = 0; i < 32; i++) {
        const double a = (double)i * M_PI / 16.0;
        L.dx[i] = (float)std::sin(a);
        L.dy[i] = (float)std::cos(a);
    }
    L.wlo = (int64_t)std::nearbyint((float)w * o.border_mirror);
    L.whi = (int64_t)w - 1 - L.wlo;
    L.hlo = (int64_t)std::nearbyint((float)h * o.border_mirror);
    L.hhi = (int64_t)h - 1 - L.hlo;
    L.mw2 = 2 * ((int64_t)w - 1);
    L.mh2 = 2 * ((int64_t)h - 1);
    L.t0 = o.t0 ? 1 : 0;
    L.wrap = o.wrap_x ? 1 : 0;
    L.w = w;
    L.h = h;
    const bool t0 = o.t0 != 0;
    k_ssao_first<<<grid_of(npix, sms), 256, 0, s>>>(gbuf, npix, pa, ang);
    float smul = 0.0f;
    for (int level = 1; level <= levels; level++) {
        float sit = (float)(z_scale / 22000.0 * 4096.0);
        float szrt = thr * (t0 ? 1.0f : 0.7f) * 4096.0f / sit * std::sqrt(std::sqrt((float)levels / (float)level));
        if (t0) szrt *= szrt;
        const float at = std::atan(thr * 0.6f * std::sqrt(std::sqrt((float)levels)));
        smul = 1.5f * 32767.0f / ((float)M_PI * 32.0f * (t0 ? at : std::pow(at, 0.9f))) / 1.0f;
        const int64_t istep = (int64_t)1 << (level - 1);
        L.smin_rad = istep < 2 ? 1.0f : 3.25f * (float)istep;
        L.step_count = istep < 2 ? 5 : 3;
        for (int k = 0; k < 5; k++) L.rma[k] = k < L.step_count ? 1.0f / (L.smin_rad + (float)((int64_t)k * istep) + 0.1f) : 0.0f;
        L.istep_f = (float)istep;
        sit *= szrt;
        L.sit = sit;
        L.szrt = szrt;
        k_ssao_angles<<<grid_of((size_t)npix * 32, sms), 256, 0, s>>>(L, gbuf, pa, ang, npix);
        if (level < levels) {
            const int step = 1 << level;
            k_ssao_h<<<grid_of(npix, sms), 256, 0, s>>>(pa, pb, w, h, step, L.wrap);
            k_ssao_v<<<grid_of(npix, sms), 256, 0, s>>>(pb, pa, w, h, step);
        }
    }
    k_ssao_sum<<<grid_of(npix, sms), 256, 0, s>>>(gbuf, ang, npix, smul, 16383);
}

}  // namespace mb3dcu
