// The launches by formula set, and the FMA throughput kernel of the
// measurement helper.
#include <cuda_runtime.h>
#include "kernels.h"
#include "formulas.cuh"

namespace mb3dcu {

int kernel_set(int fmask) {
    const int sets[3] = {KSET_IP8, KSET_IP8BOX, KSET_MENGERBOX};
    for (int s : sets)
        if ((fmask & ~s) == 0) return s;
    return KSET_ALL;
}

static const LaunchTable &table(int fmask) {
    static const LaunchTable t1 = table_ip8(), t5 = table_ip8box(), t12 = table_mengerbox(), ta = table_all();
    switch (kernel_set(fmask)) {
        case KSET_IP8: return t1;
        case KSET_IP8BOX: return t5;
        case KSET_MENGERBOX: return t12;
        default: return ta;
    }
}

void launch_march(const DevParams &p, bool mixed, int row0, int rows, mb3d_cu_silight *out, Hand *list,
                  unsigned int *counters, unsigned long long *gcount, int blocks, cudaStream_t s) {
    table(p.fmask).march(p, mixed, row0, rows, out, list, counters, gcount, blocks, s);
}
void launch_finish(const DevParams &p, bool mixed, int row0, const Hand *list, unsigned int *counters, Hand *slow,
                   mb3d_cu_silight *out, int blocks, cudaStream_t s) {
    table(p.fmask).finish(p, mixed, row0, list, counters, slow, out, blocks, s);
}
void launch_finish_fast(const DevParams &p, bool mixed, int row0, const Hand *list, unsigned int *counters, Hand *slow,
                        mb3d_cu_silight *out, int blocks, cudaStream_t s) {
    table(p.fmask).finish_fast(p, mixed, row0, list, counters, slow, out, blocks, s);
}
void launch_finish_slow(const DevParams &p, bool mixed, int row0, const Hand *list, unsigned int *counters, Hand *slow,
                        mb3d_cu_silight *out, int blocks, cudaStream_t s) {
    table(p.fmask).finish_slow(p, mixed, row0, list, counters, slow, out, blocks, s);
}
void launch_post_start(const DevParams &p, bool mixed, int row0, int passes, const mb3d_cu_silight *gbuf,
                       const uint32_t *list, const unsigned int *count, unsigned int *queue, PostStart *ps, int blocks,
                       cudaStream_t s) {
    table(p.fmask).post_start(p, mixed, row0, passes, gbuf, list, count, queue, ps, blocks, s);
}
void launch_shadow_rays(const DevParams &p, bool mixed, int row0, const PostStart *ps, const unsigned int *count,
                        mb3d_cu_silight *gbuf, unsigned int *queue, int blocks, cudaStream_t s) {
    table(p.fmask).shadow_rays(p, mixed, row0, ps, count, gbuf, queue, blocks, s);
}
void launch_ao_rays(const DevParams &p, bool mixed, const PostStart *ps, const mb3d_cu_silight *gbuf,
                    const unsigned int *count, float *min_ra, unsigned int *queue, int blocks, cudaStream_t s) {
    table(p.fmask).ao_rays(p, mixed, ps, gbuf, count, min_ra, queue, blocks, s);
}
void launch_mc(const DevParams &p, const McDev &m, bool mixed, bool batch, const McAcc &acc, const mb3d_cu_mc_req *reqs,
               mb3d_cu_mc_res *res, unsigned int *queue, uint32_t n_items, const uint32_t *list, int sms,
               cudaStream_t s) {
    static const McTable t1 = mc_table_ip8(), t5 = mc_table_ip8box(), t12 = mc_table_mengerbox(), ta = mc_table_all();
    const McTable *t = &ta;
    switch (kernel_set(p.fmask)) {
        case KSET_IP8: t = &t1; break;
        case KSET_IP8BOX: t = &t5; break;
        case KSET_MENGERBOX: t = &t12; break;
        default: break;
    }
    t->run(p, m, mixed, batch, acc, reqs, res, queue, n_items, list, sms, s);
}
void launch_reflect(const DevParams &p, const mb3d_cu_reflect_ray *rays, uint32_t n, int far_fog, const ReflAO *tab,
                    mb3d_cu_reflect_hit *hits, int blocks, cudaStream_t s) {
    table(p.fmask).reflect(p, rays, n, far_fog, tab, hits, blocks, s);
}
void launch_reflect_first(const DevParams &p, const mb3d_cu_silight *gbuf, mb3d_cu_reflect_ray *tmp,
                          unsigned char *valid, int blocks, cudaStream_t s) {
    table(p.fmask).reflect_first(p, gbuf, tmp, valid, blocks, s);
}

__global__ void __launch_bounds__(1024) k_flag_count(const unsigned char *valid, size_t n, unsigned int *block_sum) {
    const size_t i = (size_t)blockIdx.x * 1024 + threadIdx.x;
    const unsigned int v = __popc(__ballot_sync(0xffffffffu, i < n && valid[i]));
    __shared__ unsigned int part[32];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x < 32) {
        const unsigned int u = __reduce_add_sync(0xffffffffu, part[threadIdx.x]);
        if (threadIdx.x == 0) block_sum[blockIdx.x] = u;
    }
}

__global__ void __launch_bounds__(1024) k_flag_scatter(const unsigned char *valid, const mb3d_cu_reflect_ray *tmp,
                                                      size_t n, const unsigned int *offset, mb3d_cu_reflect_ray *out) {
    const size_t i = (size_t)blockIdx.x * 1024 + threadIdx.x;
    const int lane = (int)(threadIdx.x & 31), warp = (int)(threadIdx.x >> 5);
    const bool v = i < n && valid[i];
    const unsigned int b = __ballot_sync(0xffffffffu, v);
    __shared__ unsigned int wsum[32];
    if (lane == 0) wsum[warp] = __popc(b);
    __syncthreads();
    if (warp == 0) {
        // exclusive scan of the 32 warps' counts
        const unsigned int c = wsum[lane];
        unsigned int x = c;
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned int y = __shfl_up_sync(0xffffffffu, x, d);
            if (lane >= d) x += y;
        }
        wsum[lane] = x - c;
    }
    __syncthreads();
    if (v) out[offset[blockIdx.x] + wsum[warp] + __popc(b & ((1u << lane) - 1u))] = tmp[i];
}

void flag_count(const unsigned char *valid, size_t n, unsigned int *block_sum, cudaStream_t s) {
    k_flag_count<<<(unsigned)((n + 1023) / 1024), 1024, 0, s>>>(valid, n, block_sum);
}
void flag_scatter(const unsigned char *valid, const mb3d_cu_reflect_ray *tmp, size_t n, const unsigned int *offset,
                  mb3d_cu_reflect_ray *out, cudaStream_t s) {
    k_flag_scatter<<<(unsigned)((n + 1023) / 1024), 1024, 0, s>>>(valid, tmp, n, offset, out);
}

void launch_de_probe(const DevParams &p, const double *pos, int n, double *de, int *its, bool mixed, cudaStream_t s) {
    table(p.fmask).de_probe(p, pos, n, de, its, mixed, s);
}

// FMA throughput: 8 independent chains per thread (the issue peak of the
// FP32 or FP64 pipe); the store keeps the chains alive.
template <typename T>
__global__ void __launch_bounds__(256) k_fma_peak(T *out, int iters, T a, T b) {
    T x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            x0 = x0 * a + b; x1 = x1 * a + b; x2 = x2 * a + b; x3 = x3 * a + b;
            x4 = x4 * a + b; x5 = x5 * a + b; x6 = x6 * a + b; x7 = x7 * a + b;
        }
    }
    T s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
    if (s == (T)-1.2345) out[0] = s;  // (never true: keeps the work)
}

int launch_fma_peak(bool fp64, void *out, int blocks, int iters, cudaStream_t s) {
    if (fp64) k_fma_peak<double><<<blocks, 256, 0, s>>>((double *)out, iters, 0.999999, 1e-7);
    else k_fma_peak<float><<<blocks, 256, 0, s>>>((float *)out, iters, 0.999999f, 1e-7f);
    return 1;
}

}  // namespace mb3dcu
