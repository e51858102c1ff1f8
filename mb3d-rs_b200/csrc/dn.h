// The denoiser's kernels (dn_kernels.cu) as the host code (dn.cu) calls them.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stddef.h>

namespace mb3dcu {

// a 3x3 convolution: m = n * h * w pixels of NHWC tensors
struct ConvArgs {
    const __nv_bfloat16 *in;  // in_c channels per pixel; cin of them from in_off
    const __nv_bfloat16 *wt;  // [cin/16][9 taps][2 halves][cout][8] (dn_cast_weights)
    const float *bias;        // cout, or null
    __nv_bfloat16 *out;       // out_c channels per pixel; cout of them at out_off
    int n, h, w, m;
    int in_c, in_off, cin;
    int out_c, out_off, cout;
    int relu, accumulate;
    // (or null) the ReLU's backward fused into the store: the outputs whose
    // value in mask (mask_c channels per pixel, cout of them at mask_off) is
    // not positive are zero
    const __nv_bfloat16 *mask = nullptr;
    int mask_c = 0, mask_off = 0;
    // the limit of every wait in the tensor-core pipeline, clock cycles (0:
    // about one second); no_issue (a test of the limit): the TMA and MMA
    // lanes issue nothing, so the epilogue's first wait runs out with no copy
    // or MMA in flight
    long long wait_cycles = 0;
    int no_issue = 0;
};

// its weight gradient: dw[co][tap][ci] += sum_p dz[p][co] x[p + tap][ci]
struct WgradArgs {
    const __nv_bfloat16 *dz;  // dz_c channels per pixel; cout of them from dz_off
    const __nv_bfloat16 *x;   // x_c channels per pixel; cin of them from x_off
    float *dw;
    int n, h, w, m;
    int dz_c, dz_off, cout;
    int x_c, x_off, cin;
};

// (the tensor-core convolution; requires cin and cout multiples of 16, cout
// <= 256, in_c, in_off, out_c and out_off multiples of 8; -1 on bad arguments)
int dn_conv(const ConvArgs &a, cudaStream_t s);
// nonzero (and cleared) when a convolution's pipeline wait ran out since the
// last call; synchronises s
int dn_conv_error(cudaStream_t s);
int dn_wgrad(const WgradArgs &a, float *db, cudaStream_t s);
// (its tensor-core kernel, dn_tc.cu, with the bias gradient db (or null):
// cin and cout multiples of 16, cout <= 128, the channel counts and offsets
// multiples of 8; -1 on bad arguments)
int dn_wgrad_tc(const WgradArgs &a, float *db, cudaStream_t s);
void dn_relu_mask(__nv_bfloat16 *d, const __nv_bfloat16 *y, int c_tot, int off, int cn, size_t m, cudaStream_t s);
void dn_pool2(const __nv_bfloat16 *in, int in_c, int in_off, int cn, int n, int h, int w, __nv_bfloat16 *out,
              cudaStream_t s);
void dn_pool2_bwd(const __nv_bfloat16 *in, int in_c, int in_off, int cn, int n, int h, int w, const __nv_bfloat16 *dout,
                  __nv_bfloat16 *din, cudaStream_t s);
void dn_up2(const __nv_bfloat16 *in, int cn, int n, int h, int w, __nv_bfloat16 *out, int out_c, int out_off, cudaStream_t s);
void dn_up2_bwd(const __nv_bfloat16 *dout, int out_c, int out_off, int cn, int n, int h, int w, __nv_bfloat16 *din,
                cudaStream_t s);
void dn_pack_input(const float *rad, const float *alb, const float *nrm, const float *dep, float depth_scale, int n,
                   int h_src, int w_src, int h, int w, __nv_bfloat16 *out, cudaStream_t s);
void dn_unpack_output(const __nv_bfloat16 *pred, int n, int h, int w, int h_src, int w_src, float *out, cudaStream_t s);
void dn_l1_loss(const __nv_bfloat16 *pred, const float *target, int n, int h, int w, int h_src, int w_src,
                __nv_bfloat16 *dpred, float *loss, cudaStream_t s);
void dn_tone_loss(const __nv_bfloat16 *pred, const float *target, int n, int h, int w, int h_src, int w_src,
                  int display, __nv_bfloat16 *dpred, float *loss, cudaStream_t s);
void dn_fallback(const float *a, const float *b, const float *den, int h, int w, int tile, float k, float *out,
                 unsigned int *bad, cudaStream_t s);
void dn_adam(float *param, const float *grad, float *m1, float *m2, size_t n, float lr, int t, cudaStream_t s);
void dn_cast_weights(const float *w, int cout, int cin, __nv_bfloat16 *wf, __nv_bfloat16 *wb, cudaStream_t s);

}  // namespace mb3dcu
