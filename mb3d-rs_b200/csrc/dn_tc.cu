// The denoiser's 3x3 convolution (stride 1, zero padding 1) on the fifth
// generation tensor cores: an implicit GEMM with
//   M = 128 pixels of a bw x bh box of one image (bw * bh = 128),
//   N = the output channels (one tile of up to 256; more in grid.y tiles),
//   K = 9 taps x cin, in chunks of 16 channels of one tap (32 bytes).
// Per chunk one TMA load brings the box's 16 channels at the tap's offset
// (the picture's border comes as the TMA's zero fill) and one the weights'
// 16 K-columns; both land in shared memory in the 32-byte swizzled K-major
// layout that tcgen05.mma reads, and one tcgen05.mma (M=128, N=BN, K=16,
// BF16 x BF16 -> FP32) adds the chunk into the accumulator in tensor memory.
// Roles in the block of 128 threads: thread 0 issues the TMA loads, thread 32
// the MMAs (each MMA's commit frees its stage); then all four warps read the
// accumulator (warp w holds TMEM lanes 32w..32w+31, i.e. pixels), add the
// bias, apply the ReLU and store bf16 NHWC.
// Every wait is bounded (about a second of clock cycles); a wait that runs out
// sets the error word and the block stops issuing, and frees its tensor memory.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "dn.h"

namespace mb3dcu {

namespace {

constexpr int TC_STAGES = 6;
constexpr int TC_M = 128;
constexpr long long TC_WAIT_CYCLES = 2000000000LL;  // ~1 s at 1.9-2 GHz

struct ConvTc {
    const float *bias;
    __nv_bfloat16 *out;
    int n, h, w;
    int in_off, cin;
    int out_c, out_off, cout;
    int relu, accumulate;
    int bw, bh, tiles_x, tiles_y;
    int *err;
};

__device__ __forceinline__ uint32_t smem_addr(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
// bounded wait for the phase with parity `parity` to complete
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity, const volatile int *abort) {
    long long t0 = clock64();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(bar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (*abort || clock64() - t0 > TC_WAIT_CYCLES) return false;
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
__device__ __forceinline__ void tma_load_2d(uint32_t dst, const CUtensorMap *map, int c0, int c1, uint32_t bar) {
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(bar)
        : "memory");
}

// shared memory descriptor of a K-major operand in the 32-byte swizzle:
// rows of 32 bytes (16 bf16), 8-row groups 256 bytes apart
__device__ __forceinline__ uint64_t desc_sw32(uint32_t addr) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16)  // leading byte offset (unused when swizzled)
           | ((uint64_t)(256 >> 4) << 32)                           // stride byte offset: 8 rows x 32 B
           | ((uint64_t)1 << 46)                                    // descriptor version
           | ((uint64_t)6 << 61);                                   // layout: 32-byte swizzle
}

// instruction descriptor: FP32 accumulator, BF16 A and B, both K-major
template <int BN>
__device__ __forceinline__ uint32_t idesc_bf16() {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(TC_M >> 4) << 24);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

template <int BN>
__global__ void __launch_bounds__(128) k_conv3x3_tc(const __grid_constant__ CUtensorMap ta,
                                                   const __grid_constant__ CUtensorMap tb, const ConvTc a) {
    constexpr uint32_t A_BYTES = TC_M * 32, B_BYTES = BN * 32;
    constexpr uint32_t COLS = BN <= 32 ? 32 : BN <= 64 ? 64 : BN <= 128 ? 128 : 256;
    extern __shared__ __align__(1024) uint8_t dyn[];
    __shared__ __align__(8) uint64_t full[TC_STAGES], empty[TC_STAGES], done;
    __shared__ uint32_t tmem_slot;
    __shared__ volatile int abort_flag;
    // (the dynamic area is aligned to 1024 bytes by hand)
    uint8_t *base = dyn + ((1024u - (smem_addr(dyn) & 1023u)) & 1023u);
    const uint32_t sa0 = smem_addr(base), sb0 = sa0 + TC_STAGES * A_BYTES;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    int t = blockIdx.x;
    const int tx = t % a.tiles_x;
    t /= a.tiles_x;
    const int ty = t % a.tiles_y, img = t / a.tiles_y;
    const int x0 = tx * a.bw, y0 = ty * a.bh, n0 = blockIdx.y * BN;
    const int cin16 = a.cin >> 4, kchunks = 9 * cin16;

    if (tid == 0) {
        for (int s = 0; s < TC_STAGES; s++) {
            mbar_init(smem_addr(&full[s]), 1);
            mbar_init(smem_addr(&empty[s]), 1);
        }
        mbar_init(smem_addr(&done), 1);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&tmem_slot)),
                     "r"(COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_slot;

    if (tid == 0) {
        // the TMA producer
        for (int kc = 0; kc < kchunks; kc++) {
            const int s = kc % TC_STAGES;
            if (kc >= TC_STAGES && !mbar_wait(smem_addr(&empty[s]), ((kc / TC_STAGES) - 1) & 1, &abort_flag)) {
                abort_flag = 1;
                break;
            }
            const int tap = kc / cin16, ci0 = (kc - tap * cin16) << 4;
            const int dy = tap / 3 - 1, dx = tap - (tap / 3) * 3 - 1;
            const uint32_t bar = smem_addr(&full[s]);
            mbar_expect_tx(bar, A_BYTES + B_BYTES);
            tma_load_4d(sa0 + s * A_BYTES, &ta, a.in_off + ci0, x0 + dx, y0 + dy, img, bar);
            tma_load_2d(sb0 + s * B_BYTES, &tb, tap * a.cin + ci0, n0, bar);
        }
    } else if (tid == 32) {
        // the MMA issuer
        const uint32_t idesc = idesc_bf16<BN>();
        bool ok = true;
        for (int kc = 0; kc < kchunks; kc++) {
            const int s = kc % TC_STAGES;
            if (!mbar_wait(smem_addr(&full[s]), (kc / TC_STAGES) & 1, &abort_flag)) {
                abort_flag = 1;
                ok = false;
                break;
            }
            tc_fence_after();
            const uint64_t ad = desc_sw32(sa0 + s * A_BYTES), bd = desc_sw32(sb0 + s * B_BYTES);
            const uint32_t acc = kc > 0 ? 1u : 0u;
            asm volatile(
                "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
                " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
                "l"(ad), "l"(bd), "r"(idesc), "r"(acc)
                : "memory");
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&empty[s]))
                         : "memory");
        }
        if (ok)
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&done))
                         : "memory");
    }
    __syncwarp();

    // the epilogue: TMEM -> registers -> bias, ReLU -> bf16 NHWC
    bool ready = mbar_wait(smem_addr(&done), 0, &abort_flag);
    if (!ready) abort_flag = 1;
    ready = __all_sync(0xffffffffu, ready);
    tc_fence_after();
    if (ready) {
        const int row = warp * 32 + lane;
        const int px = x0 + row % a.bw, py = y0 + row / a.bw;
        const bool valid = px < a.w && py < a.h;
        __nv_bfloat16 *o = a.out + ((size_t)(img * a.h + (valid ? py : 0)) * a.w + (valid ? px : 0)) * a.out_c + a.out_off;
#pragma unroll
        for (int c = 0; c < BN; c += 16) {
            uint32_t r[16];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c;
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                : "r"(taddr)
                : "memory");
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const int nb = n0 + c;
            if (valid && nb < a.cout) {
                float v[16];
#pragma unroll
                for (int k = 0; k < 16; k++) {
                    v[k] = __uint_as_float(r[k]);
                    if (a.bias && nb + k < a.cout) v[k] += a.bias[nb + k];
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
#pragma unroll
                    for (int k = 0; k < 8; k++) p[k] = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
                    dst[0] = *reinterpret_cast<const uint4 *>(&p[0]);
                    dst[1] = *reinterpret_cast<const uint4 *>(&p[4]);
                } else {
                    for (int k = 0; k < 16 && nb + k < a.cout; k++) {
                        float x = v[k];
                        if (a.accumulate) x += __bfloat162float(o[nb + k]);
                        o[nb + k] = __float2bfloat16_rn(x);
                    }
                }
            }
        }
    }
    if (tid == 0 && abort_flag) atomicExch(a.err, 1);
    tc_fence_before();
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(COLS) : "memory");
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

template <int BN>
void launch_tc(const CUtensorMap &ta, const CUtensorMap &tb, const ConvTc &c, int tiles, int ntiles, cudaStream_t s) {
    const size_t smem = 1024 + (size_t)TC_STAGES * (TC_M * 32 + BN * 32);
    static bool attr = false;
    if (!attr) {
        cudaFuncSetAttribute(k_conv3x3_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        attr = true;
    }
    k_conv3x3_tc<BN><<<dim3(tiles, ntiles), 128, smem, s>>>(ta, tb, c);
}

}  // namespace

// the picture box of a tile: 128 pixels, as wide as the picture needs (a
// power of two from 8 to 128)
static void tile_box(int w, int &bw, int &bh) {
    bw = 128;
    while (bw > 8 && bw / 2 >= w) bw /= 2;
    bh = TC_M / bw;
}

int dn_conv(const ConvArgs &a, cudaStream_t s) {
    if (a.cin % 16 || a.cout <= 0 || a.in_c % 8 || a.in_off % 8 || a.out_c % 8 || a.out_off % 8) return -1;
    if (a.n < 1 || a.h < 1 || a.w < 1 || a.in_c < a.in_off + a.cin || a.out_c < a.out_off + a.cout) return -1;
    EncodeTiledFn enc = encode_fn();
    int *err = err_word();
    if (!enc || !err) return -1;
    const int bn_max = 256;
    int bn = ((a.cout + 15) / 16) * 16;
    int ntiles = 1;
    if (bn > bn_max) {
        ntiles = (a.cout + bn_max - 1) / bn_max;
        bn = ((a.cout + ntiles * 16 - 1) / (ntiles * 16)) * 16;
    }
    ConvTc c;
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
    tile_box(a.w, c.bw, c.bh);
    c.tiles_x = (a.w + c.bw - 1) / c.bw;
    c.tiles_y = (a.h + c.bh - 1) / c.bh;
    c.err = err;
    // the activations: dims (channels, x, y, image), the box 16 channels x bw x bh
    CUtensorMap ta, tb;
    cuuint64_t da[4] = {(cuuint64_t)a.in_c, (cuuint64_t)a.w, (cuuint64_t)a.h, (cuuint64_t)a.n};
    cuuint64_t sa[3] = {(cuuint64_t)a.in_c * 2, (cuuint64_t)a.in_c * 2 * a.w, (cuuint64_t)a.in_c * 2 * a.w * a.h};
    cuuint32_t ba[4] = {16, (cuuint32_t)c.bw, (cuuint32_t)c.bh, 1};
    cuuint32_t ea[4] = {1, 1, 1, 1};
    if (enc(&ta, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, (void *)a.in, da, sa, ba, ea, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return -1;
    // the weights [cout][9 * cin]: the box 16 K-columns x bn rows
    cuuint64_t dw[2] = {(cuuint64_t)9 * a.cin, (cuuint64_t)a.cout};
    cuuint64_t sw[1] = {(cuuint64_t)9 * a.cin * 2};
    cuuint32_t bw_[2] = {16, (cuuint32_t)bn};
    cuuint32_t ew[2] = {1, 1};
    if (enc(&tb, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, (void *)a.wt, dw, sw, bw_, ew, CU_TENSOR_MAP_INTERLEAVE_NONE,
            CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return -1;
    const int tiles = a.n * c.tiles_y * c.tiles_x;
    switch (bn) {
        case 16: launch_tc<16>(ta, tb, c, tiles, ntiles, s); break;
        case 32: launch_tc<32>(ta, tb, c, tiles, ntiles, s); break;
        case 48: launch_tc<48>(ta, tb, c, tiles, ntiles, s); break;
        case 64: launch_tc<64>(ta, tb, c, tiles, ntiles, s); break;
        case 80: launch_tc<80>(ta, tb, c, tiles, ntiles, s); break;
        case 96: launch_tc<96>(ta, tb, c, tiles, ntiles, s); break;
        case 112: launch_tc<112>(ta, tb, c, tiles, ntiles, s); break;
        case 128: launch_tc<128>(ta, tb, c, tiles, ntiles, s); break;
        case 144: launch_tc<144>(ta, tb, c, tiles, ntiles, s); break;
        case 160: launch_tc<160>(ta, tb, c, tiles, ntiles, s); break;
        case 176: launch_tc<176>(ta, tb, c, tiles, ntiles, s); break;
        case 192: launch_tc<192>(ta, tb, c, tiles, ntiles, s); break;
        case 208: launch_tc<208>(ta, tb, c, tiles, ntiles, s); break;
        case 224: launch_tc<224>(ta, tb, c, tiles, ntiles, s); break;
        case 240: launch_tc<240>(ta, tb, c, tiles, ntiles, s); break;
        default: launch_tc<256>(ta, tb, c, tiles, ntiles, s); break;
    }
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
