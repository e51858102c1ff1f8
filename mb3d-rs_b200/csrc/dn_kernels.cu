// The denoiser's kernels besides the tensor-core convolution, weight and
// bias gradients (dn_tc.cu): the elementwise pieces of the U-Net (pooling,
// upsampling, ReLU masks, input packing, the loss, Adam).
//
// Activations are NHWC bf16 tensors whose channel counts are multiples of
// 16; a convolution reads `cin` channels at offset `in_off` of a tensor of
// `in_c` channels and writes `cout` channels at `out_off` of one of `out_c`
// channels, so the decoder's concatenations are slots of one tensor.
// Weights are [cout][tap][cin] (tap = ky * 3 + kx), bf16.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>
#include "dn.h"

namespace mb3dcu {

// ---------------------------------------------------------------------------
// elementwise pieces (one thread per element or per 2x2 group)

// dz = dy * (y > 0) in place (the ReLU's backward), on a channel slot
__global__ void k_relu_mask(__nv_bfloat16 *d, const __nv_bfloat16 *y, int c_tot, int off, int cn, size_t m) {
    size_t n = m * (size_t)cn;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        size_t p = i / cn, c = i - p * cn;
        size_t k = p * c_tot + off + c;
        if (!(__bfloat162float(y[k]) > 0.0f)) d[k] = __float2bfloat16(0.0f);
    }
}

// 2x2 max pooling: out (h/2, w/2, cn) from a slot of in (h, w); one thread
// per output pixel and 8 channels (16-byte loads and stores; cn, in_c and
// in_off are multiples of 8)
__global__ void k_pool2(const __nv_bfloat16 *in, int in_c, int in_off, int cn, int n, int h, int w, __nv_bfloat16 *out) {
    int h2 = h >> 1, w2 = w >> 1, c8n = cn >> 3;
    size_t total = (size_t)n * h2 * w2 * c8n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int c8 = (int)(i % c8n);
        size_t q = i / c8n;
        int x = (int)(q % w2), y = (int)((q / w2) % h2), b = (int)(q / ((size_t)w2 * h2));
        size_t base = (((size_t)b * h + 2 * y) * w + 2 * x) * in_c + in_off + c8 * 8;
        uint4 v0 = *reinterpret_cast<const uint4 *>(in + base);
        uint4 v1 = *reinterpret_cast<const uint4 *>(in + base + in_c);
        uint4 v2 = *reinterpret_cast<const uint4 *>(in + base + (size_t)w * in_c);
        uint4 v3 = *reinterpret_cast<const uint4 *>(in + base + (size_t)w * in_c + in_c);
        const __nv_bfloat162 *a0 = reinterpret_cast<const __nv_bfloat162 *>(&v0);
        const __nv_bfloat162 *a1 = reinterpret_cast<const __nv_bfloat162 *>(&v1);
        const __nv_bfloat162 *a2 = reinterpret_cast<const __nv_bfloat162 *>(&v2);
        const __nv_bfloat162 *a3 = reinterpret_cast<const __nv_bfloat162 *>(&v3);
        uint4 r;
        __nv_bfloat162 *o = reinterpret_cast<__nv_bfloat162 *>(&r);
#pragma unroll
        for (int k = 0; k < 4; k++) o[k] = __hmax2(__hmax2(a0[k], a1[k]), __hmax2(a2[k], a3[k]));
        *reinterpret_cast<uint4 *>(out + q * cn + c8 * 8) = r;
    }
}

// its backward: the gradient to the first of the four inputs that holds the
// maximum, added to the slot of din
__global__ void k_pool2_bwd(const __nv_bfloat16 *in, int in_c, int in_off, int cn, int n, int h, int w,
                            const __nv_bfloat16 *dout, __nv_bfloat16 *din) {
    int h2 = h >> 1, w2 = w >> 1;
    size_t total = (size_t)n * h2 * w2 * cn;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int c = (int)(i % cn);
        size_t q = i / cn;
        int x = (int)(q % w2), y = (int)((q / w2) % h2), b = (int)(q / ((size_t)w2 * h2));
        size_t base = (((size_t)b * h + 2 * y) * w + 2 * x) * in_c + in_off + c;
        size_t k[4] = {base, base + in_c, base + (size_t)w * in_c, base + (size_t)w * in_c + in_c};
        float best = __bfloat162float(in[k[0]]);
        int arg = 0;
#pragma unroll
        for (int j = 1; j < 4; j++) {
            float v = __bfloat162float(in[k[j]]);
            if (v > best) {
                best = v;
                arg = j;
            }
        }
        float g = __bfloat162float(dout[i]);
        din[k[arg]] = __float2bfloat16(__bfloat162float(din[k[arg]]) + g);
    }
}

// nearest 2x upsampling of in (h/2, w/2, cn) into a slot of out (h, w); one
// thread per input pixel and 8 channels, its 2x2 block of outputs (cn, out_c
// and out_off are multiples of 8)
__global__ void k_up2(const __nv_bfloat16 *in, int cn, int n, int h, int w, __nv_bfloat16 *out, int out_c, int out_off) {
    int h2 = h >> 1, w2 = w >> 1, c8n = cn >> 3;
    size_t total = (size_t)n * h2 * w2 * c8n;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int c8 = (int)(i % c8n);
        size_t q = i / c8n;
        int x = (int)(q % w2), y = (int)((q / w2) % h2), b = (int)(q / ((size_t)w2 * h2));
        uint4 v = *reinterpret_cast<const uint4 *>(in + q * cn + c8 * 8);
        size_t o = (((size_t)b * h + 2 * y) * w + 2 * x) * out_c + out_off + c8 * 8;
        *reinterpret_cast<uint4 *>(out + o) = v;
        *reinterpret_cast<uint4 *>(out + o + out_c) = v;
        *reinterpret_cast<uint4 *>(out + o + (size_t)w * out_c) = v;
        *reinterpret_cast<uint4 *>(out + o + (size_t)w * out_c + out_c) = v;
    }
}

// its backward: the sum of the four gradients
__global__ void k_up2_bwd(const __nv_bfloat16 *dout, int out_c, int out_off, int cn, int n, int h, int w,
                          __nv_bfloat16 *din) {
    int h2 = h >> 1, w2 = w >> 1;
    size_t total = (size_t)n * h2 * w2 * cn;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int c = (int)(i % cn);
        size_t q = i / cn;
        int x = (int)(q % w2), y = (int)((q / w2) % h2), b = (int)(q / ((size_t)w2 * h2));
        size_t base = (((size_t)b * h + 2 * y) * w + 2 * x) * out_c + out_off + c;
        float s = __bfloat162float(dout[base]) + __bfloat162float(dout[base + out_c]) +
                  __bfloat162float(dout[base + (size_t)w * out_c]) + __bfloat162float(dout[base + (size_t)w * out_c + out_c]);
        din[i] = __float2bfloat16(s);
    }
}

// the network's input: log(1 + radiance), albedo, normal, depth / its
// maximum, zero channels 10..15; pixels outside (w_src, h_src) and values
// that are not finite are zero.
// Sources are float (h_src, w_src, 3) per image, images one after another.
__global__ void k_pack_input(const float *rad, const float *alb, const float *nrm, const float *dep, float depth_scale,
                             int n, int h_src, int w_src, int h, int w, __nv_bfloat16 *out) {
    size_t total = (size_t)n * h * w;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int x = (int)(i % w), y = (int)((i / w) % h), b = (int)(i / ((size_t)w * h));
        float v[16];
#pragma unroll
        for (int c = 0; c < 16; c++) v[c] = 0.0f;
        if (y < h_src && x < w_src) {
            size_t s = ((size_t)b * h_src + y) * w_src + x;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                v[c] = log1pf(fmaxf(rad[3 * s + c], 0.0f));
                if (alb) v[3 + c] = alb[3 * s + c];
                if (nrm) v[6 + c] = nrm[3 * s + c];
            }
            if (dep) v[9] = dep[s] * depth_scale;
        }
#pragma unroll
        for (int c = 0; c < 10; c++)
            if (!isfinite(v[c])) v[c] = 0.0f;  // (a non-finite guide would poison the gradients)
        __nv_bfloat16 *o = out + i * 16;
#pragma unroll
        for (int c = 0; c < 16; c += 2) *reinterpret_cast<__nv_bfloat162 *>(o + c) = __floats2bfloat162_rn(v[c], v[c + 1]);
    }
}

// the network's output (log space, 16 channels) as radiance (h_src, w_src, 3)
__global__ void k_unpack_output(const __nv_bfloat16 *pred, int n, int h, int w, int h_src, int w_src, float *out) {
    size_t total = (size_t)n * h_src * w_src;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int x = (int)(i % w_src), y = (int)((i / w_src) % h_src), b = (int)(i / ((size_t)w_src * h_src));
        size_t p = ((size_t)b * h + y) * w + x;
#pragma unroll
        for (int c = 0; c < 3; c++) out[3 * i + c] = fmaxf(expm1f(__bfloat162float(pred[p * 16 + c])), 0.0f);
    }
}

// L1 loss in log space on channels 0..2 of the valid pixels: its sum into
// *loss, its gradient (1/count per element, the sign) into dpred
__global__ void k_l1_loss(const __nv_bfloat16 *pred, const float *target, int n, int h, int w, int h_src, int w_src,
                          float inv_count, __nv_bfloat16 *dpred, float *loss) {
    __shared__ float s[256];
    size_t total = (size_t)n * h * w;
    float acc = 0.0f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int x = (int)(i % w), y = (int)((i / w) % h), b = (int)(i / ((size_t)w * h));
        __nv_bfloat16 *d = dpred + i * 16;
        for (int c = 0; c < 16; c++) d[c] = __float2bfloat16(0.0f);
        if (y < h_src && x < w_src) {
            size_t t = ((size_t)b * h_src + y) * w_src + x;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float e = __bfloat162float(pred[i * 16 + c]) - log1pf(fmaxf(target[3 * t + c], 0.0f));
                acc += fabsf(e);
                d[c] = __float2bfloat16(e > 0.0f ? inv_count : (e < 0.0f ? -inv_count : 0.0f));
            }
        }
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, s[0] * inv_count);
}

// the squared error of the tone-mapped colour x / (1 + x) (the space the
// pictures' PSNR is measured in) on channels 0..2 of the valid pixels: the
// prediction p is log(1 + x), so its tone is 1 - exp(-p) (taken for every p
// above -30, a smooth continuation where the output clamps x at 0; below, as
// at -30); with display set,
// plus the squared error of the colour clamped to 0..1 (what the painter
// makes of a record with its default settings), whose gradient passes the
// clamp wherever the two clamped colours differ (so that a prediction above
// 1 for a target below it is still pulled down); the loss's sum into *loss
// and its gradient into dpred
__global__ void k_tone_loss(const __nv_bfloat16 *pred, const float *target, int n, int h, int w, int h_src, int w_src,
                            float inv_count, int display, __nv_bfloat16 *dpred, float *loss) {
    __shared__ float s[256];
    size_t total = (size_t)n * h * w;
    float acc = 0.0f;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int x = (int)(i % w), y = (int)((i / w) % h), b = (int)(i / ((size_t)w * h));
        __nv_bfloat16 *d = dpred + i * 16;
        for (int c = 0; c < 16; c++) d[c] = __float2bfloat16(0.0f);
        if (y < h_src && x < w_src) {
            size_t t = ((size_t)b * h_src + y) * w_src + x;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float p = __bfloat162float(pred[i * 16 + c]);
                const float q = expf(-fmaxf(p, -30.0f));  // (bounded: an untrained network's outputs run wild)
                const float yv = fmaxf(target[3 * t + c], 0.0f);
                const float e = (1.0f - q) - yv / (1.0f + yv);
                acc += e * e;
                float g = 2.0f * e * q;
                if (display) {
                    const float ed = fminf(fmaxf(expm1f(p), 0.0f), 1.0f) - fminf(yv, 1.0f);
                    acc += ed * ed;
                    g += 2.0f * ed * expf(fminf(p, 0.69314718f));
                }
                d[c] = __float2bfloat16(g * inv_count);
            }
        }
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if ((int)threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, s[0] * inv_count);
}

// The plain trace as the denoiser's fallback and judge, one block per
// tile x tile piece of the picture (the last row and column of pieces
// ragged): the two independent halves a and b of the trace's rays give the
// noise of their mean m = (a + b) / 2 over the piece, and where the mean of
// the denoised piece leaves m's by more than k times that noise (+0.001),
// both in the tone x / (1 + x) of max(x, 0), the piece keeps m; out may be
// den itself.
__device__ __forceinline__ double tone01(float x) {
    const double v = fmax((double)x, 0.0);
    return v / (1.0 + v);
}

__global__ void k_dn_fallback(const float *a, const float *b, const float *den, int h, int w, int tile, float k,
                              float *out, unsigned int *bad) {
    __shared__ double s_ab[256], s_dm[256];
    const int tx = (w + tile - 1) / tile;
    const int x0 = (blockIdx.x % tx) * tile, y0 = (blockIdx.x / tx) * tile;
    const int tw = min(tile, w - x0), th = min(tile, h - y0);
    const int cnt = tw * th * 3;
    double ab = 0.0, dm = 0.0;
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
        const int px = j / 3, c = j % 3;
        const size_t i = ((size_t)(y0 + px / tw) * w + x0 + px % tw) * 3 + c;
        const double ta = tone01(a[i]), tb = tone01(b[i]);
        const double tm = tone01(0.5f * (a[i] + b[i]));
        ab += (ta - tb) * (ta - tb);
        dm += tone01(den[i]) - tm;
    }
    s_ab[threadIdx.x] = ab;
    s_dm[threadIdx.x] = dm;
    __syncthreads();
    for (int r = blockDim.x / 2; r > 0; r >>= 1) {
        if ((int)threadIdx.x < r) {
            s_ab[threadIdx.x] += s_ab[threadIdx.x + r];
            s_dm[threadIdx.x] += s_dm[threadIdx.x + r];
        }
        __syncthreads();
    }
    const double sigma = sqrt(s_ab[0] / cnt / 4.0 / cnt) + 1e-3;
    const bool keep_plain = fabs(s_dm[0] / cnt) > (double)k * sigma;
    if (keep_plain && threadIdx.x == 0) atomicAdd(bad, 1u);
    for (int j = threadIdx.x; j < cnt; j += blockDim.x) {
        const int px = j / 3, c = j % 3;
        const size_t i = ((size_t)(y0 + px / tw) * w + x0 + px % tw) * 3 + c;
        out[i] = keep_plain ? 0.5f * (a[i] + b[i]) : den[i];
    }
}

// Adam on the FP32 master parameters
__global__ void k_adam(float *param, const float *grad, float *m1, float *m2, size_t n, float lr, float b1, float b2,
                       float eps, float c1, float c2) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float g = grad[i];
        float a = b1 * m1[i] + (1.0f - b1) * g;
        float b = b2 * m2[i] + (1.0f - b2) * g * g;
        m1[i] = a;
        m2[i] = b;
        param[i] -= lr * (a * c1) / (sqrtf(b * c2) + eps);
    }
}

// the bf16 weights of a convolution in the layout its kernel reads (dn.h):
// [cin/16][tap][8-channel half][cout][8] for the forward, from w[co][tap][ci];
// the backward to the input (input and output channels swapped, the taps
// mirrored) likewise, [cout/16][tap][half][cin][8]
__global__ void k_cast_weights(const float *w, int cout, int cin, __nv_bfloat16 *wf, __nv_bfloat16 *wb) {
    size_t total = (size_t)cout * 9 * cin;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        int ci = (int)(i % cin), tap = (int)((i / cin) % 9), co = (int)(i / ((size_t)cin * 9));
        __nv_bfloat16 v = __float2bfloat16(w[i]);
        // the forward: input channel ci, output channel co
        wf[((((size_t)(ci >> 4) * 9 + tap) * 2 + ((ci >> 3) & 1)) * cout + co) * 8 + (ci & 7)] = v;
        // the backward to the input: input channel co, output channel ci, the tap mirrored
        if (wb) wb[((((size_t)(co >> 4) * 9 + (8 - tap)) * 2 + ((co >> 3) & 1)) * cin + ci) * 8 + (co & 7)] = v;
    }
}

// ---------------------------------------------------------------------------
// launchers

static int grid_for(size_t n, int per = 256) {
    size_t b = (n + per - 1) / per;
    return (int)(b < 148 * 16 ? (b < 1 ? 1 : b) : 148 * 16);
}

int dn_wgrad(const WgradArgs &a, float *db, cudaStream_t s) { return dn_wgrad_tc(a, db, s) ? -1 : 0; }

void dn_relu_mask(__nv_bfloat16 *d, const __nv_bfloat16 *y, int c_tot, int off, int cn, size_t m, cudaStream_t s) {
    k_relu_mask<<<grid_for(m * cn), 256, 0, s>>>(d, y, c_tot, off, cn, m);
}
void dn_pool2(const __nv_bfloat16 *in, int in_c, int in_off, int cn, int n, int h, int w, __nv_bfloat16 *out,
              cudaStream_t s) {
    k_pool2<<<grid_for((size_t)n * (h / 2) * (w / 2) * (cn / 8)), 256, 0, s>>>(in, in_c, in_off, cn, n, h, w, out);
}
void dn_pool2_bwd(const __nv_bfloat16 *in, int in_c, int in_off, int cn, int n, int h, int w, const __nv_bfloat16 *dout,
                  __nv_bfloat16 *din, cudaStream_t s) {
    k_pool2_bwd<<<grid_for((size_t)n * (h / 2) * (w / 2) * cn), 256, 0, s>>>(in, in_c, in_off, cn, n, h, w, dout, din);
}
void dn_up2(const __nv_bfloat16 *in, int cn, int n, int h, int w, __nv_bfloat16 *out, int out_c, int out_off, cudaStream_t s) {
    k_up2<<<grid_for((size_t)n * (h / 2) * (w / 2) * (cn / 8)), 256, 0, s>>>(in, cn, n, h, w, out, out_c, out_off);
}
void dn_up2_bwd(const __nv_bfloat16 *dout, int out_c, int out_off, int cn, int n, int h, int w, __nv_bfloat16 *din,
                cudaStream_t s) {
    k_up2_bwd<<<grid_for((size_t)n * (h / 2) * (w / 2) * cn), 256, 0, s>>>(dout, out_c, out_off, cn, n, h, w, din);
}
void dn_pack_input(const float *rad, const float *alb, const float *nrm, const float *dep, float depth_scale, int n,
                   int h_src, int w_src, int h, int w, __nv_bfloat16 *out, cudaStream_t s) {
    k_pack_input<<<grid_for((size_t)n * h * w), 256, 0, s>>>(rad, alb, nrm, dep, depth_scale, n, h_src, w_src, h, w, out);
}
void dn_unpack_output(const __nv_bfloat16 *pred, int n, int h, int w, int h_src, int w_src, float *out, cudaStream_t s) {
    k_unpack_output<<<grid_for((size_t)n * h_src * w_src), 256, 0, s>>>(pred, n, h, w, h_src, w_src, out);
}
void dn_l1_loss(const __nv_bfloat16 *pred, const float *target, int n, int h, int w, int h_src, int w_src,
                __nv_bfloat16 *dpred, float *loss, cudaStream_t s) {
    float inv = 1.0f / (float)((size_t)n * h_src * w_src * 3);
    k_l1_loss<<<grid_for((size_t)n * h * w), 256, 0, s>>>(pred, target, n, h, w, h_src, w_src, inv, dpred, loss);
}
void dn_tone_loss(const __nv_bfloat16 *pred, const float *target, int n, int h, int w, int h_src, int w_src,
                  int display, __nv_bfloat16 *dpred, float *loss, cudaStream_t s) {
    float inv = 1.0f / (float)((size_t)n * h_src * w_src * 3);
    k_tone_loss<<<grid_for((size_t)n * h * w), 256, 0, s>>>(pred, target, n, h, w, h_src, w_src, inv, display, dpred,
                                                             loss);
}
void dn_fallback(const float *a, const float *b, const float *den, int h, int w, int tile, float k, float *out,
                 unsigned int *bad, cudaStream_t s) {
    const int tiles = ((w + tile - 1) / tile) * ((h + tile - 1) / tile);
    k_dn_fallback<<<tiles, 256, 0, s>>>(a, b, den, h, w, tile, k, out, bad);
}
void dn_adam(float *param, const float *grad, float *m1, float *m2, size_t n, float lr, int t, cudaStream_t s) {
    const float b1 = 0.9f, b2 = 0.999f;
    float c1 = 1.0f / (1.0f - powf(b1, (float)t)), c2 = 1.0f / (1.0f - powf(b2, (float)t));
    k_adam<<<grid_for(n), 256, 0, s>>>(param, grad, m1, m2, n, lr, b1, b2, 1e-8f, c1, c2);
}
void dn_cast_weights(const float *w, int cout, int cin, __nv_bfloat16 *wf, __nv_bfloat16 *wb, cudaStream_t s) {
    k_cast_weights<<<grid_for((size_t)cout * 9 * cin), 256, 0, s>>>(w, cout, cin, wf, wb);
}

}  // namespace mb3dcu
