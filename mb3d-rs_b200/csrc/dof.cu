// Depth of field on the card (dof::apply, src/dof.rs:81-122): every pixel
// of the painted picture spread over a disk whose radius grows with its
// distance from the focus, in one to four passes.
//
// The reference spreads (scatters) each source pixel over its disk; a
// destination pixel's sums therefore receive its sources in the order the
// sources are walked: pixel order in the forward variant, back to front by
// fine depth (ties in pixel order) in the sorted one, whose blending is not
// a plain sum.  Here every destination gathers: per 16 x 16 tile of the
// picture one block lists the sources whose disk can reach the tile (from
// the window of the tile widened by the largest radius), sorts the list in
// shared memory by the reference's order (a bitonic sort of 64-bit keys),
// and then every thread walks the list for its own pixel.  Each pixel so
// blends the reference's contributions in the reference's order, in the same
// single precision arithmetic (built with -fmad=false).
//
//   k_dof_zrange   the nearest and farthest object depths (the sorted pass's
//                  largest radius, src/dof.rs:274-287)
//   k_dof_src      per source pixel: its radius and weights (sorted_src,
//                  :231-252; the forward pass's :142-153) and its sort key
//   k_dof_tiles    per tile: the list, its order, the blending (the CPU loops
//                  :368-413 and :188-214), the 8-bit result (from_dof)
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/mb3d_cu.h"
#include "kernels.h"

namespace mb3dcu {

namespace {

constexpr int TILE = 16;

__device__ __forceinline__ float zsteps(double z, double zc_mul_inv, double zcorr_inv) {
    const double a = z * zc_mul_inv + 1.0;
    return (float)((a * a - 1.0) * zcorr_inv);
}

__device__ __forceinline__ int32_t sort_depth(const mb3d_cu_silight &s) {
    const int32_t z = (int32_t)(s.zpos_fine >> 8);
    return (z > 8388352 || (s.zpos_fine >> 16) > 32767) ? -1 : z;
}

__global__ void k_dof_zrange(const mb3d_cu_silight *g, size_t n, unsigned int *zr) {
    unsigned int lo = 32768u, hi = 0u;
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

__global__ void k_dof_src(const DofPass d, const mb3d_cu_silight *g, const uint8_t *rgb, DofSrc *src,
                          unsigned long long *key, unsigned int *max_r_bits) {
    const size_t n = (size_t)d.w * d.h;
    float mr = 0.0f;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const mb3d_cu_silight s = g[i];
        DofSrc o;
        o.c[0] = (float)rgb[3 * i];
        o.c[1] = (float)rgb[3 * i + 1];
        o.c[2] = (float)rgb[3 * i + 2];
        if (d.forward) {
            // src/dof.rs:144-153
            const float w = (s.zpos_fine >> 16) > 32767u ? d.bg
                                                         : zsteps((double)(8388352 - (int64_t)(s.zpos_fine >> 8)),
                                                                  d.zc_mul_inv, d.zcorr_inv);
            float v = (w - d.z_sharp) / (1.0f + w * d.dsf) * d.ap;
            const float sg = signbit(v) ? -1.0f : 1.0f;
            v = fmaxf(fabsf(v) - d.r_sub, 0.0f) * sg;
            if (fabsf(v) > d.clip_r) v = d.clip_r * sg;
            mr = fmaxf(mr, fabsf(v));
            const float a = fabsf(v) + 1.0f;
            o.s_ms = a * a;
            o.sw = 0.5f / o.s_ms;
            o.rr = v;
            o.ims = 0;
            o.r = (int)rintf(fabsf(v) + 0.5f);
            o.flags = 0;
            key[i] = (unsigned long long)i;
        } else {
            // sorted_src (src/dof.rs:231-252)
            const int32_t iz = sort_depth(s);
            const float w = zsteps((double)(8388352 - (int64_t)iz), d.zc_mul_inv, d.zcorr_inv);
            float sr = (w - d.z_sharp) * d.ap / (1.0f + w * d.dsf);
            const bool descale = sr < 0.0f;
            sr = fminf(fmaxf(fabsf(sr) - d.r_sub, 0.0f), d.max_r);
            o.s_ms = sr + 1.0f;
            o.sw = 1.0f / (2.5f * sr * sr + 1.0f);
            o.ims = (int)(o.s_ms * o.s_ms);
            o.r = (int)rintf(fabsf(sr) + 0.5f);
            o.rr = 0.0f;
            o.flags = (descale ? 1u : 0u) | (iz == -1 ? 2u : 0u);
            key[i] = ((unsigned long long)(uint32_t)(iz + 1) << 32) | (unsigned long long)i;
        }
        src[i] = o;
    }
    if (d.forward) {
        // (non-negative: the bits order as the values)
        const unsigned int mb = __reduce_max_sync(0xffffffffu, __float_as_uint(mr));
        if ((threadIdx.x & 31) == 0) atomicMax(max_r_bits, mb);
    }
}

// one block of 256 threads per 16 x 16 tile; dynamic shared memory: cap keys,
// cap a power of two (the sort pads the list to one: a list of at most cap
// keys pads to at most cap)
__global__ void __launch_bounds__(256) k_dof_tiles(const DofPass d, const DofSrc *src, const unsigned long long *key,
                                                   uint8_t *out, int cap, unsigned int *overflow) {
    extern __shared__ unsigned long long keys[];
    __shared__ unsigned int count;
    const int tx0 = (int)blockIdx.x * TILE, ty0 = (int)blockIdx.y * TILE;
    const int tx1 = min(tx0 + TILE, d.w) - 1, ty1 = min(ty0 + TILE, d.h) - 1;
    const int wx0 = max(tx0 - d.rmax, 0), wx1 = min(tx1 + d.rmax, d.w - 1);
    const int wy0 = max(ty0 - d.rmax, 0), wy1 = min(ty1 + d.rmax, d.h - 1);
    const int ww = wx1 - wx0 + 1, wh = wy1 - wy0 + 1;
    if (threadIdx.x == 0) count = 0u;
    __syncthreads();
    // the sources whose disk reaches the tile
    for (int k = threadIdx.x; k < ww * wh; k += blockDim.x) {
        const int x = wx0 + k % ww, y = wy0 + k / ww;
        const size_t i = (size_t)y * d.w + x;
        const int r = src[i].r;
        if (x - r <= tx1 && x + r >= tx0 && y - r <= ty1 && y + r >= ty0) {
            const unsigned int q = atomicAdd(&count, 1u);
            if ((int)q < cap) keys[q] = key[i];
        }
    }
    __syncthreads();
    const int n = (int)count;
    if (n > cap) {
        if (threadIdx.x == 0) atomicAdd(overflow, 1u);
        return;
    }
    // the reference's order: a bitonic sort of the keys (padded to a power of two)
    int np = 1;
    while (np < n) np <<= 1;
    for (int k = n + threadIdx.x; k < np; k += blockDim.x) keys[k] = ~0ull;
    __syncthreads();
    for (int size = 2; size <= np; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int t = threadIdx.x; t < np / 2; t += blockDim.x) {
                const int lo = 2 * t - (t & (stride - 1)), hi = lo + stride;
                const bool up = (lo & size) == 0;
                const unsigned long long a = keys[lo], b = keys[hi];
                if ((a > b) == up) {
                    keys[lo] = b;
                    keys[hi] = a;
                }
            }
            __syncthreads();
        }
    }
    // this thread's pixel
    const int px = tx0 + (int)(threadIdx.x % TILE), py = ty0 + (int)(threadIdx.x / TILE);
    const bool mine = px <= tx1 && py <= ty1;
    float pc[3] = {0.0f, 0.0f, 0.0f}, pt = 0.0f;
    const float rj = mine ? src[(size_t)py * d.w + px].rr : 0.0f;
    for (int k = 0; k < n; k++) {
        const size_t i = (size_t)(keys[k] & 0xFFFFFFFFull);
        const DofSrc s = src[i];
        const int x = (int)(i % (size_t)d.w), y = (int)(i / (size_t)d.w);
        const int xx = px - x, yy = py - y;
        if (!mine || xx < -s.r || xx > s.r || yy < -s.r || yy > s.r) continue;
        if (d.forward) {
            // src/dof.rs:201-212
            float w = __fsub_rn(__fsub_rn(s.s_ms, (float)(xx * xx)), (float)(yy * yy));
            if (w > 0.0f) {
                if (w > 1.0f) w = 1.0f;
                if (rj >= s.rr) w = __fmul_rn(w, s.sw);
                else w = __fmul_rn(w, __fmul_rn(__fmul_rn(s.sw, fabsf(rj)), d.sm));
                pt = __fadd_rn(pt, w);
                for (int c = 0; c < 3; c++) pc[c] = __fadd_rn(pc[c], __fmul_rn(s.c[c], w));
            }
        } else {
            // src/dof.rs:380-411
            const int ii = xx * xx + yy * yy;
            if (ii > s.ims) continue;
            float w = __fsub_rn(s.s_ms, __fsqrt_rn((float)ii));
            float dw = 0.0f;
            const bool descale = (s.flags & 1u) != 0, bg = (s.flags & 2u) != 0;
            if (descale) {
                const float q = __fdiv_rn(__fmul_rn(0.8f, w), s.s_ms);
                dw = __fsub_rn(1.0f, __fmul_rn(q, q));
            }
            w = w > 1.0f ? s.sw : __fmul_rn(w, s.sw);
            if (descale && pt > dw) {
                const float f = __fdiv_rn(dw, pt);
                for (int c = 0; c < 3; c++) pc[c] = __fmul_rn(pc[c], f);
                pt = __fmul_rn(pt, f);
            }
            if (!bg && __fadd_rn(w, pt) > 1.01f) {
                const float st = __fdiv_rn(__fsub_rn(1.01f, w), pt);
                for (int c = 0; c < 3; c++) pc[c] = __fadd_rn(__fmul_rn(pc[c], st), __fmul_rn(s.c[c], w));
                pt = 1.01f;
            } else {
                for (int c = 0; c < 3; c++) pc[c] = __fadd_rn(pc[c], __fmul_rn(s.c[c], w));
                pt = __fadd_rn(pt, w);
            }
        }
    }
    if (mine) {
        const float m = pt < 1e-10f ? 1e10f : __fdiv_rn(1.0f, pt);
        uint8_t *o = out + 3 * ((size_t)py * d.w + px);
        for (int c = 0; c < 3; c++) o[c] = (uint8_t)rintf(fminf(fmaxf(__fmul_rn(pc[c], m), 0.0f), 255.0f));
    }
}

}  // namespace

void dof_zrange(const mb3d_cu_silight *g, size_t n, unsigned int *zr, int sms, cudaStream_t s) {
    k_dof_zrange<<<sms * 4, 256, 0, s>>>(g, n, zr);
}
void dof_src(const DofPass &d, const mb3d_cu_silight *g, const uint8_t *rgb, DofSrc *src, unsigned long long *key,
             unsigned int *max_r_bits, int sms, cudaStream_t s) {
    k_dof_src<<<sms * 8, 256, 0, s>>>(d, g, rgb, src, key, max_r_bits);
}
int dof_tiles(const DofPass &d, const DofSrc *src, const unsigned long long *key, uint8_t *out, int cap,
              unsigned int *overflow, cudaStream_t s) {
    const size_t smem = (size_t)cap * sizeof(unsigned long long);
    if (cudaFuncSetAttribute(k_dof_tiles, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return -1;
    dim3 grid((unsigned)((d.w + TILE - 1) / TILE), (unsigned)((d.h + TILE - 1) / TILE));
    k_dof_tiles<<<grid, 256, smem, s>>>(d, src, key, out, cap, overflow);
    return 0;
}

}  // namespace mb3dcu
