// The adaptive Monte Carlo pass on the card (mc::pass, src/mc.rs:3110-3300,
// with Tracer::pixel :2766-2834 and calc_n :2657-2762).
//
// The reference walks the pixels one by one; each pixel takes its rays in
// rounds until the round's mean luminance agrees with the record.  Pixels
// are independent, so here every round is one step for all pixels at once:
//   k_mcp_start   per pixel, the first round's ray count: 4 for a pixel
//                 without rays, else calc_n from the snapshot of the records
//                 taken at the start of the pass (its random number from the
//                 pixel's seed, as the reference draws it);
//   k_mcp_count   the round's rays per block of 1024 pixels (the host splits
//                 the pixels into chunks of at most a few hundred million rays);
//   k_mcp_items   the round's items of a chunk: (pixel, ray number) with ray
//                 numbers from the record's count up, so every ray has the
//                 reference's seed and Halton place; the pixel's round sums
//                 start at zero;
//   (the tracer's split render over the items: light, luminance and its
//    square of every ray into the pixel's fixed-point sums)
//   k_mcp_update  per pixel of the round: the record's new averages in double
//                 precision as the reference forms them, and the next round's
//                 count where the round's mean left the record's by more than
//                 its noise.
// The sums are fixed point (32.32, and 40.24 for the squares), so their
// result does not depend on the order the rays end in.
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/mb3d_cu.h"
#include "kernels.h"

namespace mb3dcu {

namespace {

__device__ __forceinline__ int32_t seed_of_d(int32_t x, int32_t y, uint32_t b) {  // src/mc.rs:1107-1116
    auto mix = [](uint32_t h) {
        h ^= h >> 16;
        h *= 0x7FEB352Du;
        h ^= h >> 15;
        h *= 0x846CA68Bu;
        return h ^ (h >> 16);
    };
    return (int32_t)mix((uint32_t)x * 0x9E3779B1u ^ mix((uint32_t)y * 0x85EBCA77u ^ mix(b + 0x165667B1u)));
}

__device__ __forceinline__ double rand_d(int32_t &seed) {  // src/mc.rs:1177-1180
    seed = (int32_t)((uint32_t)seed * 0x343FDu + 0x269EC3u);
    return (double)(seed & 0x7FFFFFFF) * (1.0 / 2147483647.0);
}

__device__ __forceinline__ double rec_y(const mb3d_cu_mc_record &r) { return (double)r.ysum; }
__device__ __forceinline__ double rec_noise(const mb3d_cu_mc_record &r) {
    return (double)r.ysqr - rec_y(r) * rec_y(r);
}
__device__ __forceinline__ double sq(double x) { return x * x; }

// calc_n (src/mc.rs:2657-2762); x1, y1 1-based, snap the records at the
// start of the pass
__device__ int calc_n_d(const McPassArgs &a, int x1, int y1, const mb3d_cu_mc_record &rec, int32_t &seed) {
    const int w = a.w, h = a.h;
    auto at = [&](int x, int y) -> const mb3d_cu_mc_record & { return a.snap[(size_t)(y - 1) * w + (x - 1)]; };
    double maxyd = 0, maxyd2 = 0, maxnoise = 0;
    int n = 0, n2 = 0, avg_rc = 0;
    const double dt2 = rec_y(rec);
    if (y1 > 1) {
        const mb3d_cu_mc_record &r = at(x1, y1 - 1);
        const double dt = rec_y(r);
        maxyd = sq(dt - dt2);
        maxnoise = rec_noise(r);
        avg_rc = r.ray_count;
        n += 1;
        if (x1 > 1) {
            const mb3d_cu_mc_record &r3 = at(x1 - 1, y1 - 1);
            const double dt3 = rec_y(r3);
            maxyd += sq(dt2 - dt3);
            maxyd2 = sq(dt - dt3);
            maxnoise = fmax(maxnoise, rec_noise(r3));
            avg_rc += r3.ray_count;
            n += 1;
            n2 += 1;
        }
        if (x1 < w) {
            const mb3d_cu_mc_record &r3 = at(x1 + 1, y1 - 1);
            const double dt3 = rec_y(r3);
            maxyd += sq(dt2 - dt3);
            maxyd2 += sq(dt - dt3);
            maxnoise = fmax(maxnoise, rec_noise(r3));
            avg_rc += r3.ray_count;
            n += 1;
            n2 += 1;
        }
    }
    double dt = 0;
    if (x1 > 1) {
        const mb3d_cu_mc_record &r = at(x1 - 1, y1);
        dt = rec_y(r);
        maxyd += sq(dt - dt2);
        maxnoise = fmax(maxnoise, rec_noise(r));
        avg_rc += r.ray_count;
        n += 1;
    }
    if (x1 < w) {
        const mb3d_cu_mc_record &r = at(x1 + 1, y1);
        const double dt3 = rec_y(r);
        maxyd += sq(dt3 - dt2);
        if (x1 > 1) {
            maxyd2 += sq(dt - dt3);
            n2 += 1;
        }
        maxnoise = fmax(maxnoise, rec_noise(r));
        avg_rc += r.ray_count;
        n += 1;
    }
    if (y1 < h) {
        const mb3d_cu_mc_record &r = at(x1, y1 + 1);
        const double dty = rec_y(r);
        maxyd += sq(dty - dt2);
        maxnoise = fmax(maxnoise, rec_noise(r));
        avg_rc += r.ray_count;
        n += 1;
        if (x1 > 1) {
            const mb3d_cu_mc_record &r3 = at(x1 - 1, y1 + 1);
            const double dt3 = rec_y(r3);
            maxyd += sq(dt2 - dt3);
            maxyd2 += sq(dty - dt3);
            maxnoise = fmax(maxnoise, rec_noise(r3));
            avg_rc += r3.ray_count;
            n += 1;
            n2 += 1;
        }
        if (x1 < w) {
            const mb3d_cu_mc_record &r3 = at(x1 + 1, y1 + 1);
            const double dt3 = rec_y(r3);
            maxyd += sq(dt2 - dt3);
            maxyd2 += sq(dty - dt3);
            maxnoise = fmax(maxnoise, rec_noise(r3));
            avg_rc += r3.ray_count;
            n += 1;
            n2 += 1;
        }
    }
    const double nf = (double)(n > 1 ? n : 1), n2f = (double)(n2 > 1 ? n2 : 1);
    maxyd /= nf;
    maxyd2 /= n2f;
    const double dt3 = ((double)rec.ysqr - dt2 * dt2) / (fmax(dt2, 0.0) + 0.01);
    double dm = 0.0;
    if (rec.hit) {
        const double r = fmin(fmax((double)rec.ray_count - (double)avg_rc / nf, -4.0), 4.0);
        dm = fmax(fmax(maxyd, maxyd2) - 20.0 * a.avrg_vari, 0.0) * r;
    }
    const double q = dt2 / sqrt(1.0 + (dt2 * 0.9) * (dt2 * 0.9));
    const double d = fmax(fmax(dt3, maxnoise) / fmax(q * (double)rec.ray_count, 0.3) - dm, 0.0);
    const double d2 = d * 4.0 / a.avrg_vari;
    if (d2 >= 1.0) return (int)rint(fmin((double)a.avrg_rcount * 0.5 + 8.0, d2));
    if (rand_d(seed) * 1.1 - 0.1 > fmax(d2, 0.0)) return 0;
    return 1;
}

__global__ void k_mcp_start(const McPassArgs a) {
    const size_t npix = (size_t)a.w * a.h;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (size_t)gridDim.x * blockDim.x) {
        const mb3d_cu_mc_record rec = a.recs[i];
        const int x1 = (int)(i % (size_t)a.w) + 1, y = (int)(i / (size_t)a.w);
        int total;
        if (rec.ray_count == 0) {
            total = 4;
        } else if (a.skip_nonzero) {
            total = 0;
        } else {
            int32_t seed = seed_of_d(x1, y, 0x80000000u | a.pass_nr);
            total = calc_n_d(a, x1, y + 1, rec, seed);
        }
        if (total + (int)rec.ray_count > 65535) total = 65535 - (int)rec.ray_count;
        a.total[i] = total > 0 ? total : 0;
    }
}

// the round's rays per block of 1024 pixels
__global__ void __launch_bounds__(1024) k_mcp_count(const McPassArgs a, unsigned int *block_sum) {
    const size_t npix = (size_t)a.w * a.h;
    const size_t i = (size_t)blockIdx.x * 1024 + threadIdx.x;
    unsigned int t = i < npix ? (unsigned int)a.total[i] : 0u;
    t = __reduce_add_sync(0xffffffffu, t);
    __shared__ unsigned int part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x < 32) {
        unsigned int u = part[threadIdx.x];
        u = __reduce_add_sync(0xffffffffu, u);
        if (threadIdx.x == 0) block_sum[blockIdx.x] = u;
    }
}

// the items of blocks [b0, b1): block b's rays start at offset[b - b0];
// the pixels' round sums start at zero
__global__ void __launch_bounds__(1024) k_mcp_items(const McPassArgs a, int b0, const unsigned int *offset,
                                                    unsigned int *fill, uint2 *items, McAcc acc) {
    const size_t npix = (size_t)a.w * a.h;
    const int b = b0 + (int)blockIdx.x;
    const size_t i = (size_t)b * 1024 + threadIdx.x;
    if (i >= npix) return;
    const int t = a.total[i];
    if (t <= 0) return;
    for (int k = 0; k < 3; k++) acc.sum[3 * i + k] = 0ull;
    acc.ysum[2 * i] = 0ull;
    acc.ysum[2 * i + 1] = 0ull;
    acc.hit[i] = 0u;
    const unsigned int base = offset[blockIdx.x] + atomicAdd(&fill[blockIdx.x], (unsigned int)t);
    const unsigned int rc = a.recs[i].ray_count;
    for (int j = 0; j < t; j++) items[base + j] = make_uint2((unsigned int)i, rc + (unsigned int)j);
}

// the record after the round (src/mc.rs:2801-2832) and the next round's count
__global__ void k_mcp_update(const McPassArgs a, McAcc acc, unsigned int *more) {
    const size_t npix = (size_t)a.w * a.h;
    const double MC_MAX = 1096.6331584284585 - 2.718281828459045 + 2.0;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (size_t)gridDim.x * blockDim.x) {
        const int itcount = a.total[i];
        if (itcount <= 0) continue;
        mb3d_cu_mc_record rec = a.recs[i];
        rec.hit = (rec.hit || acc.hit[i]) ? 1 : 0;
        float at[3];
        for (int k = 0; k < 3; k++) at[k] = (float)((double)acc.sum[3 * i + k] * (1.0 / 4294967296.0));
        const double sum = (double)acc.ysum[2 * i] * (1.0 / 4294967296.0);
        const double sqr_sum = (double)acc.ysum[2 * i + 1] * (1.0 / 16777216.0);
        const double dtmp = (double)rec.ysum, zz = (double)rec.ysqr;
        const int itmp = rec.ray_count;
        const double yy = itmp != 0 ? fmax((zz - dtmp * dtmp) * 10.0, 0.03) : 0.0;
        float light[3];
        if (a.sqr) {
            const float inv = __fdiv_rn(1.0f, (float)itcount);
            for (int k = 0; k < 3; k++) {
                const float v = __fmul_rn(at[k], inv);
                light[k] = __fmul_rn(v > 0.0f ? __fsqrt_rn(v) : v, (float)itcount);
            }
        } else {
            for (int k = 0; k < 3; k++) light[k] = at[k];
        }
        const double xx = 1.0 / (double)(itmp + itcount);
        for (int k = 0; k < 3; k++)
            rec.col[k] = (float)fmin(fmax(((double)rec.col[k] * itmp + (double)light[k]) * xx, -1.0), MC_MAX);
        rec.ysum = (float)fmin(fmax((dtmp * itmp + sum) * xx, -1.0), MC_MAX);
        rec.ysqr = (float)fmin(fmax((zz * itmp + sqr_sum) * xx, -1.0), MC_MAX);
        rec.ray_count = (uint16_t)(itmp + itcount);
        const double mean = sum / (double)itcount;
        int next = 0;
        if (itmp != 0 && (int)rec.ray_count < a.max_new && (mean - dtmp) * (mean - dtmp) > yy) {
            const int m = max(min(itmp, itcount), 4);
            next = (int)rint(sqrt((mean - dtmp) * (mean - dtmp) / yy) * (double)m);
            if (next + (int)rec.ray_count > 65535) next = 65535 - (int)rec.ray_count;
            if (next < 0) next = 0;
        }
        a.recs[i] = rec;
        a.total[i] = next;
        if (next > 0) atomicAdd(more, 1u);
    }
}

}  // namespace

void launch_mcp_start(const McPassArgs &a, int sms, cudaStream_t s) { k_mcp_start<<<sms * 8, 256, 0, s>>>(a); }
void launch_mcp_count(const McPassArgs &a, unsigned int *block_sum, cudaStream_t s) {
    const size_t npix = (size_t)a.w * a.h;
    k_mcp_count<<<(unsigned int)((npix + 1023) / 1024), 1024, 0, s>>>(a, block_sum);
}
void launch_mcp_items(const McPassArgs &a, int b0, int b1, const unsigned int *offset, unsigned int *fill, uint2 *items,
                      const McAcc &acc, cudaStream_t s) {
    if (b1 > b0) k_mcp_items<<<b1 - b0, 1024, 0, s>>>(a, b0, offset, fill, items, acc);
}
void launch_mcp_update(const McPassArgs &a, const McAcc &acc, unsigned int *more, int sms, cudaStream_t s) {
    k_mcp_update<<<sms * 8, 256, 0, s>>>(a, acc, more);
}

}  // namespace mb3dcu
