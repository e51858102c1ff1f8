// The denoiser's 3x3 convolution (stride 1, zero padding 1) on the fifth
// generation tensor cores, as an implicit GEMM:
//   M = 128 output pixels, a box 8 wide and 16 high of one image,
//   N = the output channels (up to 256, one tile),
//   K = 9 taps x cin.
// For each group of 16 input channels the TMA brings the tile's input box
// with its one-pixel halo, 10 x 18 pixels, as two 8-channel halves in shared
// memory ([y][x][8 channels], 16 bytes a pixel; the picture's border is the
// TMA's zero fill).  That is the A operand of all nine taps: for tap (dy, dx)
// the 8 output pixels of a row are 8 consecutive pixels of the box, so the
// tap's operand is the box seen from start ((dy + 1) * 10 + dx + 1) * 16 with
// 8-row groups 160 bytes apart and the two channel halves one box apart, in
// the no-swizzle K-major layout tcgen05.mma reads.  The weights come in the
// matching layout ([group][tap][half][cout][8], made by dn_cast_weights); they
// stay in shared memory for the whole kernel where they fit, else each group's
// block comes with its input box.  Nine tcgen05.mma (M=128, N=BN, K=16,
// BF16 x BF16 -> FP32) per group add into the accumulator in tensor memory.
// The blocks are persistent (one per SM) and take every grid-th tile.  Roles
// in a block of 320 threads: lane 0 of warp 0 issues the TMA loads through a
// ring of stages, lane 0 of warp 1 the MMAs (each group's commit frees its
// stage; tile i accumulates in TMEM buffer i % NBUF -- four buffers where
// they fit in the 512 columns, else two -- so that the epilogues of earlier
// tiles overlap the MMAs of the next), and two groups of four epilogue warps
// (warps 2..5 the even tiles, 6..9 the odd ones) read the accumulator (warp w
// holds TMEM lanes 32 (w % 4) .. + 31, i.e. four rows of the tile's pixels),
// add the bias (kept in shared memory), apply the ReLU and free the buffer.
// The plain store (no mask, no accumulation, cout <= 128) goes through a
// shared memory tile per warp, [4 rows][8 pixels][cout] bf16, that one lane
// writes to the picture with a TMA tensor store (the box clips at the
// picture's edge); the others store 16 bytes per lane.
// Every wait is bounded (about a second of clock cycles); a wait that runs out
// sets the error word and the block stops issuing, and frees its tensor memory.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "dn.h"

namespace mb3dcu {

namespace {

constexpr int TC_M = 128, TILE_W = 8, TILE_H = 16, HALO_W = TILE_W + 2, HALO_H = TILE_H + 2;
// one 8-channel half of an input box: the bytes the TMA brings, and its
// place in shared memory, padded to the 128-byte alignment a TMA destination
// needs
constexpr uint32_t BOX_BYTES = HALO_W * HALO_H * 16;
constexpr uint32_t HALF_BYTES = (BOX_BYTES + 127) / 128 * 128;
constexpr uint32_t A_BYTES = 2 * HALF_BYTES;
constexpr int MAX_STAGES = 16;
constexpr int EPI_WARPS = 8;                            // two groups of four
constexpr int CONV_THREADS = 64 + 32 * EPI_WARPS;
constexpr int TS_MAX_BN = 128;                          // the TMA store epilogue up to this many output channels
constexpr uint32_t SMEM_BUDGET = 200 * 1024;           // the dynamic shared memory a block takes
constexpr uint32_t RESIDENT_MAX = 112 * 1024;          // weights up to this stay in shared memory
constexpr long long TC_WAIT_CYCLES = 2000000000LL;     // ~1 s at 1.9-2 GHz

struct ConvTc {
    const __nv_bfloat16 *wt;
    const float *bias;
    __nv_bfloat16 *out;
    int n, h, w;
    int in_off, cin;
    int out_c, out_off, cout;
    int relu, accumulate;
    const __nv_bfloat16 *mask;
    int mask_c, mask_off;
    int tiles_x, tiles_y;
    int stages, resident;
    uint32_t w_bytes, stage_bytes;
    int *err;
    long long wait_cycles;  // the limit of every wait
    int no_issue;           // (a test of the limit: the TMA and MMA lanes issue nothing)
    int tstore;             // the TMA store epilogue (its staging after the stages)
    uint32_t stage_out;     // bytes of one warp's staging tile (32 pixels x cout bf16)
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// bounded wait for the phase with parity `parity` to complete (the thread
// sleeps in the barrier up to 20 us per try, woken by the phase's completion)
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, const volatile int *abort,
                                          long long limit = TC_WAIT_CYCLES) {
    long long t0 = clock64();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity), "r"(20000)
            : "memory");
        if (ok) return true;
        if (*abort || clock64() - t0 > limit) return false;
    }
}

__device__ __forceinline__ void tma_load_4d(uint32_t dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                            uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];" ::"r"(dst),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
        : "memory");
}
// a contiguous block (16-byte aligned, a multiple of 16 bytes)
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

// a tile of shared memory to the picture (the box of the output map at
// {c0, c1, c2, c3}), in the warp's bulk group; and the waits on the group
__device__ __forceinline__ void tma_store_4d(const CUtensorMap *map, uint32_t src, int c0, int c1, int c2, int c3) {
    asm volatile("cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group [%0, {%2, %3, %4, %5}], [%1];" ::"l"(
                     (uint64_t)map),
                 "r"(src), "r"(c0), "r"(c1), "r"(c2), "r"(c3)
                 : "memory");
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
}
__device__ __forceinline__ void bulk_wait_read() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }

// shared memory descriptor of a K-major operand without swizzle: core
// matrices of 8 rows x 16 bytes (rows 16 bytes apart), `lbo` bytes between the
// two 8-element halves of K, `sbo` bytes between 8-row groups
__device__ __forceinline__ uint64_t desc_plain(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);  // version 1, layout 0 (no swizzle)
}

// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major
template <int BN>
__device__ __forceinline__ uint32_t idesc_bf16() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 16 accumulator columns of one pixel: bias, ReLU, (the old value), (the
// mask), bf16
__device__ __forceinline__ void store16(__nv_bfloat16 *o, const __nv_bfloat16 *mk, int nb, const uint32_t (&r)[16],
                                        const ConvTc &a, const float *sbias) {
    float v[16];
#pragma unroll
    for (int k = 0; k < 16; k++) {
        v[k] = __uint_as_float(r[k]) + sbias[nb + k];
        if (a.relu) v[k] = fmaxf(v[k], 0.0f);
    }
    if (nb + 16 <= a.cout) {
        __align__(16) __nv_bfloat162 p[8];
        uint4 *dst = reinterpret_cast<uint4 *>(o + nb);
        if (a.accumulate) {
            uint4 old0 = dst[0], old1 = dst[1];
            const __nv_bfloat162 *q0 = reinterpret_cast<const __nv_bfloat162 *>(&old0);
            const __nv_bfloat162 *q1 = reinterpret_cast<const __nv_bfloat162 *>(&old1);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                v[2 * k] += __low2float(q0[k]);
                v[2 * k + 1] += __high2float(q0[k]);
                v[8 + 2 * k] += __low2float(q1[k]);
                v[8 + 2 * k + 1] += __high2float(q1[k]);
            }
        }
        if (mk) {
            const uint4 m0 = reinterpret_cast<const uint4 *>(mk + nb)[0], m1 = reinterpret_cast<const uint4 *>(mk + nb)[1];
            const __nv_bfloat162 *q0 = reinterpret_cast<const __nv_bfloat162 *>(&m0);
            const __nv_bfloat162 *q1 = reinterpret_cast<const __nv_bfloat162 *>(&m1);
#pragma unroll
            for (int k = 0; k < 4; k++) {
                if (!(__low2float(q0[k]) > 0.0f)) v[2 * k] = 0.0f;
                if (!(__high2float(q0[k]) > 0.0f)) v[2 * k + 1] = 0.0f;
                if (!(__low2float(q1[k]) > 0.0f)) v[8 + 2 * k] = 0.0f;
                if (!(__high2float(q1[k]) > 0.0f)) v[8 + 2 * k + 1] = 0.0f;
            }
        }
#pragma unroll
        for (int k = 0; k < 8; k++) p[k] = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
        dst[0] = *reinterpret_cast<const uint4 *>(&p[0]);
        dst[1] = *reinterpret_cast<const uint4 *>(&p[4]);
    } else {
        for (int k = 0; k < 16 && nb + k < a.cout; k++) {
            float x = v[k];
            if (a.accumulate) x += __bfloat162float(o[nb + k]);
            if (mk && !(__bfloat162float(mk[nb + k]) > 0.0f)) x = 0.0f;
            o[nb + k] = __float2bfloat16_rn(x);
        }
    }
}

__device__ __forceinline__ void tile_of(const ConvTc &a, int g, int &img, int &x0, int &y0) {
    const int tx = g % a.tiles_x;
    g /= a.tiles_x;
    const int ty = g % a.tiles_y;
    img = g / a.tiles_y;
    x0 = tx * TILE_W;
    y0 = ty * TILE_H;
}

template <int BN>
__global__ void __launch_bounds__(CONV_THREADS, 1) k_conv3x3_tc(const __grid_constant__ CUtensorMap ta,
                                                                const __grid_constant__ CUtensorMap to, const ConvTc a) {
    constexpr uint32_t COLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;  // one accumulator
    constexpr int NBUF = 4 * COLS <= 512 ? 4 : 2;                                     // accumulators in TMEM
    constexpr uint32_t B_TAP = BN * 32;                                               // one tap's weights
    extern __shared__ __align__(1024) uint8_t dyn[];
    __shared__ __align__(8) uint64_t full[MAX_STAGES], empty[MAX_STAGES], acc_full[4], acc_empty[4], wbar;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;
    __shared__ float sbias[256];
    // (the dynamic area is aligned to 1024 bytes by hand): the resident
    // weights, then the stages (input box, and the group's weights when they
    // are not resident), then the epilogue warps' staging tiles
    uint8_t *base = dyn + ((1024u - (smem_addr(dyn) & 1023u)) & 1023u);
    const uint32_t w0 = smem_addr(base), st0 = w0 + (a.resident ? a.w_bytes : 0u);
    const uint32_t out0 = (st0 + (uint32_t)a.stages * a.stage_bytes + 127u) & ~127u;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int groups = a.cin >> 4, ns = a.stages;
    const int total = a.n * a.tiles_y * a.tiles_x;
    const uint32_t grp_bytes = 9 * B_TAP;

    if (tid == 0) {
        for (int s = 0; s < ns; s++) {
            mbar_init(smem_addr(&full[s]), 1);
            mbar_init(smem_addr(&empty[s]), 1);
        }
        for (int b = 0; b < NBUF; b++) {
            mbar_init(smem_addr(&acc_full[b]), 1);
            mbar_init(smem_addr(&acc_empty[b]), 4);
        }
        mbar_init(smem_addr(&wbar), 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int k = tid; k < 256; k += blockDim.x) sbias[k] = (a.bias && k < a.cout) ? a.bias[k] : 0.0f;
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(NBUF * COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == 0) {
        if (lane == 0 && !a.no_issue) {
            // the TMA producer
            if (a.resident) {
                mbar_expect_tx(smem_addr(&wbar), a.w_bytes);
                bulk_load(w0, a.wt, a.w_bytes, smem_addr(&wbar));
            }
            uint32_t q = 0;
            for (int g = blockIdx.x; g < total && !abort_flag; g += gridDim.x) {
                int img, x0, y0;
                tile_of(a, g, img, x0, y0);
                for (int grp = 0; grp < groups; grp++, q++) {
                    const uint32_t s = q % (uint32_t)ns;
                    if (q >= (uint32_t)ns && !mbar_wait(smem_addr(&empty[s]), ((q / ns) - 1) & 1, &abort_flag, a.wait_cycles)) {
                        abort_flag = 1;
                        break;
                    }
                    const uint32_t bar = smem_addr(&full[s]), sa = st0 + s * a.stage_bytes;
                    mbar_expect_tx(bar, 2 * BOX_BYTES + (a.resident ? 0u : grp_bytes));
                    const int c = a.in_off + 16 * grp;
                    tma_load_4d(sa, &ta, c, x0 - 1, y0 - 1, img, bar);
                    tma_load_4d(sa + HALF_BYTES, &ta, c + 8, x0 - 1, y0 - 1, img, bar);
                    if (!a.resident) bulk_load(sa + A_BYTES, a.wt + (size_t)grp * 9 * BN * 16, grp_bytes, bar);
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0 && !a.no_issue) {
            // the MMA issuer: nine taps per group; tile i accumulates in buffer i % NBUF
            const uint32_t idesc = idesc_bf16<BN>();
            if (a.resident && !mbar_wait(smem_addr(&wbar), 0, &abort_flag, a.wait_cycles)) abort_flag = 1;
            uint32_t q = 0;
            int i = 0;
            for (int g = blockIdx.x; g < total && !abort_flag; g += gridDim.x, i++) {
                const int buf = i % NBUF;
                if (i >= NBUF && !mbar_wait(smem_addr(&acc_empty[buf]), ((i / NBUF) - 1) & 1, &abort_flag, a.wait_cycles)) {
                    abort_flag = 1;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)buf * COLS;
                for (int grp = 0; grp < groups; grp++, q++) {
                    const uint32_t s = q % (uint32_t)ns;
                    if (!mbar_wait(smem_addr(&full[s]), (q / ns) & 1, &abort_flag, a.wait_cycles)) {
                        abort_flag = 1;
                        break;
                    }
                    tc_fence_after();
                    const uint32_t sa = st0 + s * a.stage_bytes;
                    const uint32_t sb = a.resident ? w0 + (uint32_t)grp * grp_bytes : sa + A_BYTES;
#pragma unroll
                    for (int tap = 0; tap < 9; tap++) {
                        const int dy = tap / 3, dx = tap % 3;  // (offsets + 1)
                        const uint64_t ad = desc_plain(sa + (uint32_t)(dy * HALO_W + dx) * 16, HALF_BYTES, HALO_W * 16);
                        const uint64_t bd = desc_plain(sb + (uint32_t)tap * B_TAP, BN * 16, 128);
                        const uint32_t acc = (grp | tap) ? 1u : 0u;
                        asm volatile(
                            "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                            " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
                            "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                            : "memory");
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     smem_addr(&empty[s]))
                                 : "memory");
                }
                if (abort_flag) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 smem_addr(&acc_full[buf]))
                             : "memory");
            }
        }
    } else {
        // the epilogue: group e = 0 (warps 2..5) takes the even tiles, e = 1
        // (warps 6..9) the odd ones; warp w reads TMEM lanes 32 (w % 4) .. + 31
        const int ew = warp - 2, e = ew >> 2;
        const int quarter = warp & 3, row = quarter * 32 + lane;
        const uint32_t stg = out0 + (uint32_t)ew * a.stage_out;  // (the TMA store's staging tile)
        bool pending = false;                                    // (lane 0: a store of the warp in flight)
        int i = e;
        for (int g = blockIdx.x + e * gridDim.x; g < total; g += 2 * gridDim.x, i += 2) {
            const int buf = i % NBUF;
            bool ready = mbar_wait(smem_addr(&acc_full[buf]), (i / NBUF) & 1, &abort_flag, a.wait_cycles);
            ready = __all_sync(0xffffffffu, ready);
            if (!ready) {
                abort_flag = 1;
                break;
            }
            tc_fence_after();
            int img, x0, y0;
            tile_of(a, g, img, x0, y0);
            const int px = x0 + row % TILE_W, py = y0 + row / TILE_W;
            const bool valid = px < a.w && py < a.h;
            if (a.tstore) {
                // the staging tile is free once the warp's last store has read it
                if (lane == 0 && pending) bulk_wait_read();
                __syncwarp();
#pragma unroll
                for (int c = 0; c < BN; c += 16) {
                    uint32_t r[16];
                    const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * COLS + c);
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                        "[%16];"
                        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                        : "r"(taddr)
                        : "memory");
                    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                    uint32_t pk[8];
#pragma unroll
                    for (int k = 0; k < 8; k++) {
                        float v0 = __uint_as_float(r[2 * k]) + sbias[c + 2 * k];
                        float v1 = __uint_as_float(r[2 * k + 1]) + sbias[c + 2 * k + 1];
                        if (a.relu) {
                            v0 = fmaxf(v0, 0.0f);
                            v1 = fmaxf(v1, 0.0f);
                        }
                        const __nv_bfloat162 b2 = __floats2bfloat162_rn(v0, v1);
                        pk[k] = *reinterpret_cast<const uint32_t *>(&b2);
                    }
                    // the lane's pixel is entry `lane` of the [4][8] tile
                    const uint32_t sp = stg + (uint32_t)(lane * BN + c) * 2u;
                    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sp), "r"(pk[0]), "r"(pk[1]), "r"(pk[2]),
                                 "r"(pk[3])
                                 : "memory");
                    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(sp + 16u), "r"(pk[4]), "r"(pk[5]),
                                 "r"(pk[6]), "r"(pk[7])
                                 : "memory");
                }
                // (the accumulator is read: free it before the store goes out)
                tc_fence_before();
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                __syncwarp();
                if (lane == 0) {
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&acc_empty[buf])) : "memory");
                    const int ry = y0 + quarter * 4;
                    if (ry < a.h) {
                        tma_store_4d(&to, stg, a.out_off, x0, ry, img);
                        pending = true;
                    } else {
                        pending = false;
                    }
                }
                continue;
            }
            const size_t pix = (size_t)(img * a.h + (valid ? py : 0)) * a.w + (valid ? px : 0);
            __nv_bfloat16 *o = a.out + pix * a.out_c + a.out_off;
            const __nv_bfloat16 *mk = a.mask ? a.mask + pix * a.mask_c + a.mask_off : nullptr;
#pragma unroll
            for (int c = 0; c < BN; c += 16) {
                uint32_t r[16];
                const uint32_t taddr = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * COLS + c);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                    "[%16];"
                    : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                      "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                    : "r"(taddr)
                    : "memory");
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                if (valid && c < a.cout) store16(o, mk, c, r, a, sbias);
            }
            // the accumulator buffer is free for the MMAs of tile i + NBUF
            tc_fence_before();
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&acc_empty[buf])) : "memory");
        }
        // (the warp's last store has left shared memory and reached the picture)
        if (lane == 0 && pending) bulk_wait_all();
        __syncwarp();
    }
    tc_fence_before();
    __syncthreads();
    if (tid == 0 && abort_flag) atomicExch(a.err, 1);
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NBUF * COLS) : "memory");
}

// ---------------------------------------------------------------------------
// The weight gradient on the same tensor cores:
//   dW[co][tap][ci] += sum over the pixels p of dz[p][co] x[p + tap][ci]
// as a GEMM with M = 128 rows of co (cout <= 128; the rows past cout read
// zeros), N = 144 columns (tap, ci) of one group of 16 input channels,
// K = the 128 pixels of a tile (8 x 16), in eight K steps of 16 pixels.
// Both operands are arrays of TMA boxes [16 rows][8 pixels][8 channels]
// (2048 bytes), read in the MN-major layout without swizzle: core matrices
// of 8 pixels x 8 channels, 128 bytes apart along K and one box apart along
// M or N.  A = dz transposed: one box per 8 output channels.  B = the
// tile's input seen from each tap: the TMA brings the tile's input box with
// its one-pixel halo (10 x 18 pixels, zero fill at the picture's border, two
// channel halves), and two warps copy out of it, for tap (dy, dx) and half
// h, the 8 x 16 box shifted by (dx - 1, dy - 1) as box 2 tap + h -- so that
// one MMA of N = 144 takes all nine taps and A is read once per K step,
// while the input crosses L2 once per tile.  A block takes
// one channel group and every (grid / groups)-th tile and accumulates in
// TMEM over all of its tiles; the blocks of group 0 also form the bias
// gradient db[co] = sum over p of dz[p][co], as one more MMA per K step with
// a B operand of ones into 16 more columns.  At the end the four warps read
// the accumulators (warp w: co 32 w .. 32 w + 31) and add them to dW and db
// with FP32 atomics.  Roles: lane 0 of warp 0 issues the TMA loads, lane 0 of
// warp 1 the MMAs, warps 2 and 3 make the shifted boxes; every wait is
// bounded as in the forward kernel.
constexpr uint32_t WG_BOX = TILE_W * TILE_H * 16;    // one box of a tile (2048 bytes)
constexpr uint32_t WG_A_BYTES = 16 * WG_BOX;          // M = 128: 16 boxes of 8 output channels
constexpr uint32_t WG_HALO = 2 * HALF_BYTES;          // the input box with its halo, two channel halves
constexpr uint32_t WG_B_BYTES = 18 * WG_BOX;          // nine taps x two channel halves
constexpr uint32_t WG_STAGE = WG_A_BYTES + WG_HALO + WG_B_BYTES;
constexpr int WG_STAGES = 3;
constexpr uint32_t WG_COLS = 256;                     // 144 columns of (tap, ci), 16 of the bias
constexpr uint32_t WG_ONES = 1024;                    // the ones operand (512 bytes) before the stages

struct WgTc {
    float *dw, *db;
    int n, h, w, cin, cout, dz_off, x_off;
    int tiles_x, tiles_y, groups;
    int *err;
};

__global__ void __launch_bounds__(128, 1) k_wgrad_tc(const __grid_constant__ CUtensorMap tz,
                                                     const __grid_constant__ CUtensorMap tx, const WgTc a) {
    extern __shared__ __align__(1024) uint8_t dyn[];
    __shared__ __align__(8) uint64_t full[WG_STAGES], copied[WG_STAGES], empty[WG_STAGES], done;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;
    uint8_t *base = dyn + ((1024u - (smem_addr(dyn) & 1023u)) & 1023u);
    const uint32_t ones = smem_addr(base), st0 = ones + WG_ONES;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int grp = (int)blockIdx.x % a.groups;
    const bool bias = a.db && grp == 0;
    const int first = (int)blockIdx.x / a.groups, step = (int)gridDim.x / a.groups;
    const int total = a.n * a.tiles_y * a.tiles_x;
    const int cog = a.cout >> 3;  // the dz boxes of a tile
    // the A boxes past cout stay zero (the rows of M that no output channel
    // has); the ones operand
    for (int st = 0; st < WG_STAGES; st++) {
        uint4 *z = reinterpret_cast<uint4 *>(base + WG_ONES + (size_t)st * WG_STAGE + (size_t)cog * WG_BOX);
        const int n16 = (16 - cog) * (int)(WG_BOX / 16);
        for (int i = tid; i < n16; i += blockDim.x) z[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    if (tid < 32) reinterpret_cast<uint4 *>(base)[tid] = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (tid == 0) {
        for (int st = 0; st < WG_STAGES; st++) {
            mbar_init(smem_addr(&full[st]), 1);
            mbar_init(smem_addr(&copied[st]), 2);
            mbar_init(smem_addr(&empty[st]), 1);
        }
        mbar_init(smem_addr(&done), 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(WG_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (warp == 0 && lane == 0) {
        // the TMA producer: one stage per tile
        uint32_t q = 0;
        for (int g = first; g < total && !abort_flag; g += step, q++) {
            const uint32_t st = q % (uint32_t)WG_STAGES;
            if (q >= (uint32_t)WG_STAGES &&
                !mbar_wait(smem_addr(&empty[st]), ((q / WG_STAGES) - 1) & 1, &abort_flag)) {
                abort_flag = 1;
                break;
            }
            const int tx_ = g % a.tiles_x, rest = g / a.tiles_x;
            const int x0 = tx_ * TILE_W, y0 = (rest % a.tiles_y) * TILE_H, img = rest / a.tiles_y;
            const uint32_t bar = smem_addr(&full[st]), sa = st0 + st * WG_STAGE, sh = sa + WG_A_BYTES;
            mbar_expect_tx(bar, (uint32_t)cog * WG_BOX + 2 * BOX_BYTES);
            for (int j = 0; j < cog; j++) tma_load_4d(sa + (uint32_t)j * WG_BOX, &tz, a.dz_off + 8 * j, x0, y0, img, bar);
            const int c = a.x_off + 16 * grp;
            tma_load_4d(sh, &tx, c, x0 - 1, y0 - 1, img, bar);
            tma_load_4d(sh + HALF_BYTES, &tx, c + 8, x0 - 1, y0 - 1, img, bar);
        }
    } else if (warp >= 2) {
        // warps 2 and 3: each tap's shifted 8 x 16 box, two channel halves,
        // copied out of the halo box (16 bytes a pixel) for the B operand
        const int t = tid - 64;
        uint32_t q = 0;
        for (int g = first; g < total && !abort_flag; g += step, q++) {
            const uint32_t st = q % (uint32_t)WG_STAGES;
            bool ready = mbar_wait(smem_addr(&full[st]), (q / WG_STAGES) & 1, &abort_flag);
            ready = __all_sync(0xffffffffu, ready);
            if (!ready) {
                abort_flag = 1;
                break;
            }
            const uint8_t *halo = base + WG_ONES + (size_t)st * WG_STAGE + WG_A_BYTES;
            uint8_t *bbox = base + WG_ONES + (size_t)st * WG_STAGE + WG_A_BYTES + WG_HALO;
            for (int i = t; i < 18 * 128; i += 64) {
                const int box = i >> 7, within = i & 127, r = within >> 3, x = within & 7;
                const int tap = box >> 1, h = box & 1, dy = tap / 3, dx = tap % 3;
                *reinterpret_cast<uint4 *>(bbox + (size_t)box * WG_BOX + (size_t)within * 16) =
                    *reinterpret_cast<const uint4 *>(halo + (size_t)h * HALF_BYTES + (size_t)((r + dy) * HALO_W + x + dx) * 16);
            }
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            __syncwarp();
            if (lane == 0)
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(&copied[st])) : "memory");
        }
    } else if (warp == 1 && lane == 0) {
        // the MMA issuer: per tile eight K steps of one N = 144 MMA (and the
        // bias's N = 16 one); a step's descriptors are the stage's first ones
        // plus the step's 256 bytes in 16-byte units (the address field is
        // their low 14 bits)
        const uint32_t mn = (1u << 4) | (1u << 7) | (1u << 10) | (1u << 15) | (1u << 16) | ((uint32_t)(TC_M >> 4) << 24);
        const uint32_t idesc = mn | ((144u >> 3) << 17), idesc_b = mn | ((16u >> 3) << 17);
        // (FP32 += BF16 x BF16, A and B MN-major, M = 128)
        const uint64_t od = desc_plain(ones, 128u, 256u);
        uint32_t q = 0;
        for (int g = first; g < total && !abort_flag; g += step, q++) {
            const uint32_t st = q % (uint32_t)WG_STAGES;
            if (!mbar_wait(smem_addr(&copied[st]), (q / WG_STAGES) & 1, &abort_flag)) {
                abort_flag = 1;
                break;
            }
            tc_fence_after();
            const uint32_t sa = st0 + st * WG_STAGE;
            const uint64_t ad0 = desc_plain(sa, 128u, WG_BOX), bd0 = desc_plain(sa + WG_A_BYTES + WG_HALO, 128u, WG_BOX);
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const uint32_t acc = (q | (uint32_t)k) ? 1u : 0u;
                asm volatile(
                    "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                    " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                    "l"(ad0 + (uint64_t)(k * 16)), "l"(bd0 + (uint64_t)(k * 16)), "r"(idesc), "r"(acc)
                    : "memory");
                if (bias)
                    asm volatile(
                        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem + 144u),
                        "l"(ad0 + (uint64_t)(k * 16)), "l"(od), "r"(idesc_b), "r"(acc)
                        : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&empty[st]))
                         : "memory");
        }
        // (also after an abort: the MMAs issued so far end before the memory is freed)
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(&done))
                     : "memory");
    }
    __syncwarp();
    // the epilogue: warp w holds TMEM lanes (output channels) 32 w .. 32 w + 31
    bool ok = mbar_wait(smem_addr(&done), 0, &abort_flag);
    ok = __all_sync(0xffffffffu, ok && !abort_flag);
    if (ok && first < total) {
        tc_fence_after();
        const int co = warp * 32 + lane;
        for (int col = 0; col < (bias ? 160 : 144); col += 16) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)col;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "
                "[%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(taddr)
                : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (co < a.cout) {
                if (col == 144) {
                    atomicAdd(a.db + co, __uint_as_float(r[0]));
                } else {
                    const int tap = col >> 4;
                    float4 *d = reinterpret_cast<float4 *>(a.dw + ((size_t)co * 9 + tap) * a.cin + 16 * grp);
#pragma unroll
                    for (int k = 0; k < 4; k++)
                        atomicAdd(d + k, make_float4(__uint_as_float(r[4 * k]), __uint_as_float(r[4 * k + 1]),
                                                     __uint_as_float(r[4 * k + 2]), __uint_as_float(r[4 * k + 3])));
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (tid == 0 && abort_flag) atomicExch(a.err, 1);
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(WG_COLS) : "memory");
}

// cuTensorMapEncodeTiled from the driver, looked up once
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static EncodeTiledFn fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

int *err_word() {
    static int *e = nullptr;
    if (!e && cudaMalloc((void **)&e, sizeof(int)) == cudaSuccess) cudaMemset(e, 0, sizeof(int));
    return e;
}

int sm_count() {
    static int n = 0;
    if (!n) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            n < 1)
            n = 148;
    }
    return n;
}

template <int BN>
void launch_tc(const CUtensorMap &ta, const CUtensorMap &to, ConvTc c, int total, cudaStream_t s) {
    // the weights stay in shared memory where they leave room for 8 stages;
    // the TMA store epilogue's staging tiles (8 warps x 32 pixels x cout
    // bf16) come off the stages' room
    const uint32_t grp_bytes = 9u * BN * 32u;
    c.stage_out = 32u * BN * 2u;
    const uint32_t out_bytes = c.tstore ? (uint32_t)EPI_WARPS * c.stage_out + 128u : 0u;
    const uint32_t budget = SMEM_BUDGET - out_bytes;
    c.w_bytes = (uint32_t)(c.cin / 16) * grp_bytes;
    c.resident = c.w_bytes <= RESIDENT_MAX && c.w_bytes + 8 * A_BYTES <= budget;
    c.stage_bytes = c.resident ? A_BYTES : A_BYTES + grp_bytes;
    const uint32_t room = budget - (c.resident ? c.w_bytes : 0u);
    int st = (int)(room / c.stage_bytes);
    c.stages = st > MAX_STAGES ? MAX_STAGES : st < 2 ? 2 : st;
    const size_t smem = 1024 + (c.resident ? c.w_bytes : 0u) + (size_t)c.stages * c.stage_bytes + out_bytes;
    cudaFuncSetAttribute(k_conv3x3_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    int grid = sm_count();
    if (grid > total) grid = total;
    k_conv3x3_tc<BN><<<grid, CONV_THREADS, smem, s>>>(ta, to, c);
}

}  // namespace

int dn_conv(const ConvArgs &a, cudaStream_t s) {
    if (a.cin % 16 || a.cout % 16 || a.cout > 256 || a.in_c % 8 || a.in_off % 8 || a.out_c % 8 || a.out_off % 8) return -1;
    if (a.mask && (a.mask_c % 8 || a.mask_off % 8 || a.mask_c < a.mask_off + a.cout)) return -1;
    if (a.n < 1 || a.h < 1 || a.w < 1 || a.in_c < a.in_off + a.cin || a.out_c < a.out_off + a.cout) return -1;
    EncodeTiledFn enc = encode_fn();
    int *err = err_word();
    if (!enc || !err) return -1;
    ConvTc c;
    c.wt = a.wt;
    c.bias = a.bias;
    c.out = a.out;
    c.n = a.n;
    c.h = a.h;
    c.w = a.w;
    c.in_off = a.in_off;
    c.cin = a.cin;
    c.out_c = a.out_c;
    c.out_off = a.out_off;
    c.cout = a.cout;
    c.relu = a.relu;
    c.accumulate = a.accumulate;
    c.mask = a.mask;
    c.mask_c = a.mask_c;
    c.mask_off = a.mask_off;
    c.tiles_x = (a.w + TILE_W - 1) / TILE_W;
    c.tiles_y = (a.h + TILE_H - 1) / TILE_H;
    c.err = err;
    c.wait_cycles = a.wait_cycles > 0 ? a.wait_cycles : TC_WAIT_CYCLES;
    c.no_issue = a.no_issue;
    c.stages = 2;
    c.resident = 0;
    c.w_bytes = 0;
    c.stage_bytes = 0;
    // the activations: dims (channels, x, y, image), the box 8 channels x the
    // tile's 10 x 18 pixels with the halo
    CUtensorMap ta;
    cuuint64_t da[4] = {(cuuint64_t)a.in_c, (cuuint64_t)a.w, (cuuint64_t)a.h, (cuuint64_t)a.n};
    cuuint64_t sa[3] = {(cuuint64_t)a.in_c * 2, (cuuint64_t)a.in_c * 2 * a.w, (cuuint64_t)a.in_c * 2 * a.w * a.h};
    cuuint32_t ba[4] = {8, (cuuint32_t)HALO_W, (cuuint32_t)HALO_H, 1};
    cuuint32_t ea[4] = {1, 1, 1, 1};
    if (enc(&ta, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)a.in, da, sa, ba, ea, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return -1;
    // the output, for the TMA store epilogue (no mask, no accumulation, up to
    // TS_MAX_BN channels): dims (channels, x, y, image), the box cout
    // channels x 8 x 4 pixels, one epilogue warp's four rows of a tile
    CUtensorMap to = ta;
    c.tstore = 0;
    if (!a.mask && !a.accumulate && a.cout <= TS_MAX_BN) {
        cuuint64_t dout[4] = {(cuuint64_t)a.out_c, (cuuint64_t)a.w, (cuuint64_t)a.h, (cuuint64_t)a.n};
        cuuint64_t sout[3] = {(cuuint64_t)a.out_c * 2, (cuuint64_t)a.out_c * 2 * a.w, (cuuint64_t)a.out_c * 2 * a.w * a.h};
        cuuint32_t bout[4] = {(cuuint32_t)a.cout, (cuuint32_t)TILE_W, 4, 1};
        if (enc(&to, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)a.out, dout, sout, bout, ea, CU_TENSOR_MAP_INTERLEAVE_NONE,
                CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_NONE, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS)
            c.tstore = 1;
        else
            to = ta;
    }
    const int tiles = a.n * c.tiles_y * c.tiles_x;
    switch (a.cout) {
        case 16: launch_tc<16>(ta, to, c, tiles, s); break;
        case 32: launch_tc<32>(ta, to, c, tiles, s); break;
        case 48: launch_tc<48>(ta, to, c, tiles, s); break;
        case 64: launch_tc<64>(ta, to, c, tiles, s); break;
        case 80: launch_tc<80>(ta, to, c, tiles, s); break;
        case 96: launch_tc<96>(ta, to, c, tiles, s); break;
        case 112: launch_tc<112>(ta, to, c, tiles, s); break;
        case 128: launch_tc<128>(ta, to, c, tiles, s); break;
        case 144: launch_tc<144>(ta, to, c, tiles, s); break;
        case 160: launch_tc<160>(ta, to, c, tiles, s); break;
        case 176: launch_tc<176>(ta, to, c, tiles, s); break;
        case 192: launch_tc<192>(ta, to, c, tiles, s); break;
        case 208: launch_tc<208>(ta, to, c, tiles, s); break;
        case 224: launch_tc<224>(ta, to, c, tiles, s); break;
        case 240: launch_tc<240>(ta, to, c, tiles, s); break;
        default: launch_tc<256>(ta, to, c, tiles, s); break;
    }
    return 0;
}

int dn_wgrad_tc(const WgradArgs &a, float *db, cudaStream_t s) {
    if (a.cin % 16 || a.cout % 16 || a.cout > 128 || a.dz_c % 8 || a.dz_off % 8 || a.x_c % 8 || a.x_off % 8) return -1;
    if (a.n < 1 || a.h < 1 || a.w < 1 || a.dz_c < a.dz_off + a.cout || a.x_c < a.x_off + a.cin) return -1;
    EncodeTiledFn enc = encode_fn();
    int *err = err_word();
    if (!enc || !err) return -1;
    WgTc c;
    c.dw = a.dw;
    c.db = db;
    c.n = a.n;
    c.h = a.h;
    c.w = a.w;
    c.cin = a.cin;
    c.cout = a.cout;
    c.dz_off = a.dz_off;
    c.x_off = a.x_off;
    c.tiles_x = (a.w + TILE_W - 1) / TILE_W;
    c.tiles_y = (a.h + TILE_H - 1) / TILE_H;
    c.groups = a.cin / 16;
    c.err = err;
    // dz and x: dims (channels, x, y, image), one 8-channel box of 8 x 16 pixels
    CUtensorMap tz, tx;
    cuuint64_t dz[4] = {(cuuint64_t)a.dz_c, (cuuint64_t)a.w, (cuuint64_t)a.h, (cuuint64_t)a.n};
    cuuint64_t sz[3] = {(cuuint64_t)a.dz_c * 2, (cuuint64_t)a.dz_c * 2 * a.w, (cuuint64_t)a.dz_c * 2 * a.w * a.h};
    cuuint64_t dx[4] = {(cuuint64_t)a.x_c, (cuuint64_t)a.w, (cuuint64_t)a.h, (cuuint64_t)a.n};
    cuuint64_t sx[3] = {(cuuint64_t)a.x_c * 2, (cuuint64_t)a.x_c * 2 * a.w, (cuuint64_t)a.x_c * 2 * a.w * a.h};
    cuuint32_t box[4] = {8, (cuuint32_t)TILE_W, (cuuint32_t)TILE_H, 1};
    cuuint32_t hbox[4] = {8, (cuuint32_t)HALO_W, (cuuint32_t)HALO_H, 1};
    cuuint32_t e1[4] = {1, 1, 1, 1};
    if (enc(&tz, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)a.dz, dz, sz, box, e1, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS ||
        enc(&tx, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)a.x, dx, sx, hbox, e1, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return -1;
    const int tiles = a.n * c.tiles_y * c.tiles_x;
    // blocks: about one per SM, each with at least 4 tiles (every block adds
    // its sums to dW once)
    int chunks = sm_count() / c.groups;
    if (chunks > tiles / 4) chunks = tiles / 4;
    if (chunks < 1) chunks = 1;
    const size_t smem = 1024 + WG_ONES + (size_t)WG_STAGES * WG_STAGE;
    cudaFuncSetAttribute(k_wgrad_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    k_wgrad_tc<<<c.groups * chunks, 128, smem, s>>>(tz, tx, c);
    return 0;
}

int dn_conv_error(cudaStream_t s) {
    int *e = err_word();
    if (!e) return 0;
    int h = 0;
    if (cudaMemcpyAsync(&h, e, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
        return 1;
    if (h) cudaMemsetAsync(e, 0, sizeof(int), s);
    return h;
}

}  // namespace mb3dcu
