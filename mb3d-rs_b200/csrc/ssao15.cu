// The older "15 bit" screen space ambient occlusion on the card:
// gpu::ssao15 (src/gpu.rs:3726) / ssao15::ssao15 (src/ssao15.rs:282-411),
// MB3D's AmbShadowCalcThreadN.  The whole pass runs here (the reference
// builds its depth levels on the CPU and samples on the card):
//   k15_zrange   the object pixels' nearest and farthest coarse depth
//   k15_level1   the depth buffer scaled to 0..128 (build_levels :109-122)
//   k15_peaks    single peaks lowered to their highest neighbour + 1: the
//                reference does it in place in pixel order, which gives
//                what this out-of-place pass gives, since a peak's
//                neighbours are all lower and so none of them is a peak
//                (a pixel's decision never sees a changed value)
//   k15_h/_v     the next "a trous" level: a horizontal then a vertical
//                rounded average with the neighbours step away (:147-175)
//   k15_sample   a warp per object pixel: per level its ring of samples (a
//                table made on the host for pixels whose ring lies inside
//                the picture; the clipped grid of axis_samples near the
//                borders), the lanes taking the samples, the steepest slope
//                per 1/32-circle bucket kept by shared-memory atomic maxima
//                (the reference notes the samples' order does not matter),
//                then the 32 arctangents summed in the buckets' order
// Single precision, unfused (built with -fmad=false), as the reference's
// CPU pass, so that the slopes are the reference's bit for bit; the
// arctangent is the card's atanf.
#include <cuda_runtime.h>
#include <stdint.h>
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include "kernels.h"

namespace mb3dcu {

namespace {

constexpr int MAX_RINGS = 8;
constexpr int AXIS_MAX = 24;  // (an axis of a ring has at most 2 * 8 + 3 samples)

struct Ring15 {
    int max_rad, min_rad, step, multi;
    float rm, zrt;
    int first, count;  // its interior samples in the table
};

struct Sample15 {
    int16_t dx, dy;
    float r1d;
    uint8_t lo, hi, pad[2];
};

struct Ssao15Consts {
    Ring15 ring[MAX_RINGS];
    int rings, w, h, t0, wrap;
    float st2, smul;
    int64_t zsub;
    float corr_mul;
    size_t stride;  // the levels' distance in elements
};

__device__ __forceinline__ uint16_t avg16(uint32_t a, uint32_t b) { return (uint16_t)((a + b + 1u) >> 1); }

// a float's bits as an unsigned integer of the same order
__device__ __forceinline__ unsigned int ord(float f) {
    const unsigned int b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float unord(unsigned int u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

// fastIntArcTan2 (src/ssao15.rs:22-50)
__host__ __device__ inline int arctan32(int y, int x) {
    int r;
    if (x == 0)
        r = (y >= 0 ? 16 : 0) + 8;
    else if (y == 0)
        r = x >= 0 ? 16 : 0;
    else if (y < 0)
        r = x < 0 ? (x >= y ? 7 - (x * 4) / y : (y * 4) / x) : (-y < x ? 15 + (y * 4) / x : 8 - (x * 4) / y);
    else if (x >= 0)
        r = x > y ? 16 + (y * 4) / x : 23 - (x * 4) / y;
    else
        r = y < -x ? 31 + (y * 4) / x : 24 - (x * 4) / y;
    return r & 31;
}

// axis_samples (src/ssao15.rs:193-231); returns the count (out: AXIS_MAX)
__host__ __device__ inline int axis_samples(int pos, int size, int max_rad, int step, int *out) {
    int n = 0;
    int a = -max_rad, a2 = INT_MAX;
    if (a + pos < 0) {
        a2 = a;
        while (a2 + pos < 0) a2 += step;
        if (a2 + pos >= size) a2 = size - pos - 1;
        a = -pos;
        if (a == a2) a2 = INT_MAX;
    }
    const int e = pos + max_rad >= size ? size - pos - 1 : max_rad;
    int v = a;
    for (;;) {
        if (v > a2) {
            v = a2;
            a2 = INT_MAX;
        }
        if (n < AXIS_MAX) out[n] = v;
        n++;
        const int vt = v;
        v += step;
        if (v > e && vt < e) v = e;
        if (v > e) break;
    }
    return n;
}

__global__ void k15_zrange(const mb3d_cu_silight *g, size_t n, unsigned int *zr) {
    unsigned int lo = 32767u, hi = 0u;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const unsigned int z = g[i].zpos_fine >> 16;
        if (z < 32768u) {
            lo = min(lo, z);
            hi = max(hi, z);
        }
    }
    lo = __reduce_min_sync(0xffffffffu, lo);
    hi = __reduce_max_sync(0xffffffffu, hi);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&zr[0], lo);
        atomicMax(&zr[1], hi);
    }
}

__global__ void k15_level1(const mb3d_cu_silight *g, size_t n, int64_t zsub, float s1, uint16_t *l) {
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t zf = g[i].zpos_fine;
        l[i] = (zf >> 16) < 32768u ? (uint16_t)rint((double)((int64_t)(zf >> 8) - zsub) * (double)s1) : (uint16_t)0;
    }
}

__global__ void k15_peaks(const uint16_t *src, int w, int h, uint16_t *dst) {
    const size_t n = (size_t)w * h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % (size_t)w), y = (int)(i / (size_t)w);
        const uint16_t c = src[i];
        uint16_t out = c;
        if (w >= 3 && h >= 3 && x >= 1 && x + 1 < w && y >= 1 && y + 1 < h) {
            uint16_t m = 0;
            bool peak = true;
            for (int dy = -1; dy <= 1 && peak; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    if (dx == 0 && dy == 0) continue;
                    const uint16_t v = src[i + (ptrdiff_t)dy * w + dx];
                    if (v >= c) {
                        peak = false;
                        break;
                    }
                    m = max(m, v);
                }
            if (peak && m > 0) out = (uint16_t)(m + 1);
        }
        dst[i] = out;
    }
}

__global__ void k15_h(const uint16_t *src, int w, int h, int step, int wrap, uint16_t *dst) {
    const size_t n = (size_t)w * h;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(k % (size_t)w);
        const uint16_t *r = src + (k - i);
        auto at = [&](int j) { return (uint32_t)r[min(max(j, 0), w - 1)]; };
        uint16_t v;
        if (wrap)
            v = avg16(r[i], avg16(r[((i - step) % w + w) % w], r[((i + step) % w + w) % w]));
        else if (i < step)
            v = avg16(r[i], avg16(r[0], at(i + step)));
        else if (i + step < w)
            v = avg16(r[i], avg16(at(i - step), at(i + step)));
        else
            v = (uint16_t)(((uint32_t)r[i] + 1u + ((at(i - step) + r[w - 1]) >> 1)) >> 1);
        dst[k] = v;
    }
}

__global__ void k15_v(const uint16_t *src, int w, int h, int step, uint16_t *dst) {
    const size_t n = (size_t)w * h;
    for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
        const int x = (int)(k % (size_t)w), j = (int)(k / (size_t)w);
        auto at = [&](int jj) { return (uint32_t)src[(size_t)min(max(jj, 0), h - 1) * w + x]; };
        const uint32_t c = src[k];
        uint16_t v;
        if (j < step)
            v = avg16(avg16(at(j + step), src[x]), c);
        else if (j + step < h)
            v = avg16(avg16(at(j - step), at(j + step)), c);
        else
            v = avg16(avg16(at(j - step), src[(size_t)(h - 1) * w + x]), c);
        dst[k] = v;
    }
}

constexpr int WARPS15 = 8;

__global__ void __launch_bounds__(WARPS15 * 32) k15_sample(const __grid_constant__ Ssao15Consts C,
                                                           mb3d_cu_silight *g, const uint16_t *lev,
                                                           const Sample15 *tab) {
    __shared__ unsigned int ang[WARPS15][40];
    __shared__ int axis[WARPS15][2][AXIS_MAX];
    __shared__ int axis_n[WARPS15][2];
    const int wid = (int)(threadIdx.x >> 5), lane = (int)(threadIdx.x & 31);
    const size_t npix = (size_t)C.w * C.h;
    const size_t warps = (size_t)gridDim.x * WARPS15;
    for (size_t i = (size_t)blockIdx.x * WARPS15 + wid; i < npix; i += warps) {
        const uint32_t zf = g[i].zpos_fine;
        if ((zf >> 16) >= 32768u) continue;
        // Levels::zp_of (src/ssao15.rs:63-69)
        const int zp = (int)rint((double)((int64_t)(zf >> 8) - C.zsub) * (double)C.corr_mul);
        const int xi = (int)(i % (size_t)C.w), yi = (int)(i / (size_t)C.w);
        for (int k = lane; k < 40; k += 32) ang[wid][k] = ord(-1e10f);
        __syncwarp();
        for (int ri = 0; ri < C.rings; ri++) {
            const Ring15 &R = C.ring[ri];
            const uint16_t *l = lev + (size_t)ri * C.stride;
            const int r = R.max_rad;
            auto update = [&](float st, int lo, int hi) {
                if (C.t0) {
                    if (st >= R.zrt) return;
                    const float s3 = st / R.zrt;
                    st *= 1.0f - s3 * s3 * s3;
                } else if (st > R.zrt) {
                    st = R.zrt;
                }
                const unsigned int u = ord(st);
                for (int b = lo; b <= hi; b++) atomicMax(&ang[wid][b], u);
            };
            if (xi >= r && xi + r < C.w && yi >= r && yi + r < C.h) {
                for (int k = lane; k < R.count; k += 32) {
                    const Sample15 s = tab[R.first + k];
                    const float st = (float)((int)l[(size_t)(yi + s.dy) * C.w + (xi + s.dx)] - zp) * s.r1d;
                    update(st, s.lo, s.hi);
                }
                continue;
            }
            // near the borders: the clipped grid (with the wrap: x on the other side)
            if (lane == 0) axis_n[wid][0] = axis_samples(yi, C.h, r, R.step, axis[wid][0]);
            if (lane == 1)
                axis_n[wid][1] = C.wrap ? axis_samples(r, 2 * r + 1, r, R.step, axis[wid][1])
                                        : axis_samples(xi, C.w, r, R.step, axis[wid][1]);
            __syncwarp();
            const int ny = min(axis_n[wid][0], AXIS_MAX), nx = min(axis_n[wid][1], AXIS_MAX);
            const int maxs = r * r, mins = R.min_rad * R.min_rad;
            for (int k = lane; k < ny * nx; k += 32) {
                const int y2 = axis[wid][0][k / nx], x2 = axis[wid][1][k % nx];
                const int rads = y2 * y2 + x2 * x2;
                if (rads <= mins || rads > maxs) continue;
                const float r1d = 1.0f / sqrtf((float)rads);
                const int xx = ((xi + x2) % C.w + C.w) % C.w;
                const float st = (float)((int)l[(size_t)(yi + y2) * C.w + xx] - zp) * r1d;
                const int c = arctan32(y2, x2);
                if (R.multi) {
                    const int ic = (int)rintf(R.rm * r1d);
                    const int start = (c - (ic >> 1)) & 31;
                    update(st, start, min(start + ic, 39));
                } else {
                    update(st, c, c);
                }
            }
            __syncwarp();
        }
        __syncwarp();
        float a = unord(ang[wid][lane]);
        if (lane < 4) {
            const float o = unord(ang[wid][lane + 32]);
            if (o > a) a = o;
        }
        const float t = a > -1e9f ? atanf(a * C.st2) : 0.0f;
        float s = 0.0f;
        for (int k = 0; k < 32; k++) {
            const float tk = __shfl_sync(0xffffffffu, t, k);
            const float ak = __shfl_sync(0xffffffffu, a, k);
            if (ak > -1e9f) s += tk;
        }
        if (lane == 0) {
            const float v = fminf(fmaxf(rintf(s * C.smul), 0.0f), 16383.0f);
            g[i].amb_shadow = (uint16_t)v;
        }
        __syncwarp();
    }
}

}  // namespace

size_t ssao15_scratch_bytes(int w, int h) {
    const size_t plane = ((size_t)w * h * sizeof(uint16_t) + 255) & ~(size_t)255;
    return 256 + (size_t)(MAX_RINGS + 1) * plane + (size_t)MAX_RINGS * 17 * 17 * sizeof(Sample15) + 256;
}

int ssao15_run(mb3d_cu_silight *g, int w, int h, double zc_mul, double zcorr, const mb3d_cu_ssao_opts &o,
               unsigned char *scratch, int sms, cudaStream_t s, uint32_t *launches) {
    *launches = 0;
    if (w < 4 || h < 4) return 0;
    const size_t n = (size_t)w * h;
    const size_t plane = (n * sizeof(uint16_t) + 255) & ~(size_t)255;
    unsigned int *zr = (unsigned int *)scratch;
    uint16_t *lev = (uint16_t *)(scratch + 256);
    uint16_t *tmp = (uint16_t *)(scratch + 256 + (size_t)MAX_RINGS * plane);
    Sample15 *tab = (Sample15 *)(scratch + 256 + (size_t)(MAX_RINGS + 1) * plane);
    const int blocks = sms * 8;
    // build_levels (src/ssao15.rs:92-176): the level count, the depth range
    int count = 1;
    for (size_t x = (size_t)w / 16;;) {
        count++;
        x >>= 1;
        if (count == 8 || x < 4) break;
    }
    unsigned int hz[2] = {32767u, 0u};
    if (cudaMemcpyAsync(zr, hz, 8, cudaMemcpyHostToDevice, s) != cudaSuccess) return -1;
    k15_zrange<<<blocks, 256, 0, s>>>(g, n, zr);
    if (cudaMemcpyAsync(hz, zr, 8, cudaMemcpyDeviceToHost, s) != cudaSuccess) return -1;
    if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
    uint32_t za = 0, zp = 32768;
    if (hz[1] >= hz[0]) {
        za = hz[0];
        zp = hz[1] + 1;
    }
    const float s1 = 128.0f / (float)(zp - za);
    const int64_t zsub = (int64_t)za << 8;
    k15_level1<<<blocks, 256, 0, s>>>(g, n, zsub, s1, tmp);
    k15_peaks<<<blocks, 256, 0, s>>>(tmp, w, h, lev);
    *launches += 3;
    int step = 1;
    for (int k = 2; k <= count; k++) {
        k15_h<<<blocks, 256, 0, s>>>(lev + (size_t)(k - 2) * (plane / 2), w, h, step, o.wrap_x ? 1 : 0, tmp);
        k15_v<<<blocks, 256, 0, s>>>(tmp, w, h, step, lev + (size_t)(k - 1) * (plane / 2));
        *launches += 2;
        step *= 2;
    }
    // sampling_constants (src/ssao15.rs:73-89), in the reference's single precision order
    Ssao15Consts C;
    std::memset(&C, 0, sizeof(C));
    const float nl = (float)count;
    const float thr = std::max(o.threshold, 0.01f);
    const double q = 256.0 / zc_mul + 1.0;
    const float zscale = (float)((q * q - 1.0) / zcorr);
    const float st2 = zscale / (s1 * 256.0f);
    const float pi = 3.14159265358979323846f;
    float szrt, smul;
    if (o.t0) {
        szrt = std::max(thr * 2.0f / st2, 0.01f);
        smul = 1.35f * 32767.0f / (pi * 32.0f * std::pow(std::atan(thr * 0.8f * std::sqrt(std::sqrt(nl))), 0.9f));
    } else {
        szrt = thr / st2;
        smul = 1.35f * 32767.0f / (pi * 32.0f * std::pow(std::atan(thr * std::sqrt(std::sqrt(nl))), 0.8f));
    }
    C.rings = count;
    C.w = w;
    C.h = h;
    C.t0 = o.t0 ? 1 : 0;
    C.wrap = o.wrap_x ? 1 : 0;
    C.st2 = st2;
    C.smul = smul;
    C.zsub = zsub;
    C.corr_mul = s1;
    C.stride = plane / sizeof(uint16_t);
    // rings (src/ssao15.rs:257-297): the interior samples of every level
    std::vector<Sample15> samples;
    int max_rad = 0, min_rad = 0;
    int ax[AXIS_MAX];
    for (int atl = 1; atl <= count; atl++) {
        Ring15 &R = C.ring[atl - 1];
        R.step = 1 << (atl - 1);
        R.rm = std::sqrt((float)R.step) * 5.0f;
        max_rad += 4 * R.step;
        R.multi = std::nearbyint(R.rm / (float)(min_rad + 1)) > 0.0f ? 1 : 0;
        R.zrt = szrt * std::sqrt(std::sqrt(nl / (float)atl));
        R.max_rad = max_rad;
        R.min_rad = min_rad;
        R.first = (int)samples.size();
        const int na = axis_samples(max_rad, 2 * max_rad + 1, max_rad, R.step, ax);
        if (na > AXIS_MAX) return -2;
        const int maxs = max_rad * max_rad, mins = min_rad * min_rad;
        for (int iy = 0; iy < na; iy++)
            for (int ix = 0; ix < na; ix++) {
                const int y2 = ax[iy], x2 = ax[ix];
                const int rads = y2 * y2 + x2 * x2;
                if (rads <= mins || rads > maxs) continue;
                Sample15 t;
                std::memset(&t, 0, sizeof(t));
                t.dx = (int16_t)x2;
                t.dy = (int16_t)y2;
                t.r1d = 1.0f / std::sqrt((float)rads);
                const int c = arctan32(y2, x2);
                if (R.multi) {
                    const int ic = (int)std::nearbyint(R.rm * t.r1d);
                    const int start = (c - (ic >> 1)) & 31;
                    t.lo = (uint8_t)start;
                    t.hi = (uint8_t)std::min(start + ic, 39);
                } else {
                    t.lo = t.hi = (uint8_t)c;
                }
                samples.push_back(t);
            }
        R.count = (int)samples.size() - R.first;
        min_rad = max_rad;
    }
    if (samples.size() > (size_t)MAX_RINGS * 17 * 17) return -2;
    if (cudaMemcpyAsync(tab, samples.data(), samples.size() * sizeof(Sample15), cudaMemcpyHostToDevice, s) !=
        cudaSuccess)
        return -1;
    k15_sample<<<sms * 16, WARPS15 * 32, 0, s>>>(C, g, lev, tab);
    *launches += 1;
    // (the table's host copy must outlive the copy)
    if (cudaStreamSynchronize(s) != cudaSuccess) return -1;
    return 0;
}

}  // namespace mb3dcu
