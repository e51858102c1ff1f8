// The path tracer's learned denoiser: a 5-level U-Net of 3x3 convolutions
// (32/48/64/80/96 channels, ReLU, 2x2 max pooling, nearest upsampling,
// skip concatenation), BF16 weights and activations with FP32 accumulation
// and FP32 master weights, trained with Adam on an L1 loss in log space.
// It takes the place of the Open Image Denoise call of mb3d-rs
// (oidn::Input, src/oidn.rs:170-180; denoise_mc, src/oidn.rs:262-277):
// colour plus the albedo, normal and depth guides in, colour out.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cmath>
#include <cstring>
#include <mutex>
#include <random>
#include <string>
#include <vector>
#include "../../include/mb3d_cu.h"
#include "dn.h"

namespace mb3dcu {
int dn_fail(int code, const std::string &msg);
bool dn_is_device_ptr(const void *p);
cudaStream_t dn_stream(mb3d_cu_ctx *c);
int dn_device(mb3d_cu_ctx *c);
}  // namespace mb3dcu

using namespace mb3dcu;

namespace {

const int CH[5] = {32, 48, 64, 80, 96};
const int IN_C = 16, OUT_C = 16;
enum { ENC_A = 0, ENC_B = 1 };  // layer l*2 + k for the encoder levels 0..3

struct Layer {
    int cin, cout;
    bool relu;
    size_t w_off, b_off;  // in the flat parameter array
    __nv_bfloat16 *wf = nullptr, *wb = nullptr;
};

// the 19 convolutions: enc0a enc0b enc1a enc1b enc2a enc2b enc3a enc3b bota
// botb dec3a dec3b dec2a dec2b dec1a dec1b dec0a dec0b out
std::vector<Layer> make_layers(size_t &count) {
    std::vector<Layer> L;
    auto add = [&](int cin, int cout, bool relu) {
        Layer l;
        l.cin = cin;
        l.cout = cout;
        l.relu = relu;
        L.push_back(l);
    };
    int prev = IN_C;
    for (int l = 0; l < 4; l++) {
        add(prev, CH[l], true);
        add(CH[l], CH[l], true);
        prev = CH[l];
    }
    add(CH[3], CH[4], true);
    add(CH[4], CH[4], true);
    for (int l = 3; l >= 0; l--) {
        add(CH[l + 1] + CH[l], CH[l], true);
        add(CH[l], CH[l], true);
    }
    add(CH[0], OUT_C, false);
    count = 0;
    for (auto &l : L) {
        l.w_off = count;
        count += (size_t)l.cout * 9 * l.cin;
        l.b_off = count;
        count += (size_t)l.cout;
    }
    return L;
}

const int L_BOT_A = 8, L_BOT_B = 9, L_OUT = 18;
int l_enc(int l, int k) { return l * 2 + k; }
int l_dec(int l, int k) { return 10 + (3 - l) * 2 + k; }

typedef __nv_bfloat16 bf16;

struct Acts {
    bf16 *x0 = nullptr, *ea[4] = {}, *cat[4] = {}, *pool[5] = {}, *ba = nullptr, *bb = nullptr, *da[4] = {}, *db[4] = {},
         *pred = nullptr;
};

}  // namespace

struct mb3d_cu_dn {
    mb3d_cu_ctx *ctx;
    std::vector<Layer> layers;
    size_t nparam = 0;
    float *param = nullptr, *grad = nullptr, *m1 = nullptr, *m2 = nullptr;
    bf16 *wbuf = nullptr;
    int step = 0;
    int loss_kind = MB3D_CU_DN_LOSS_L1_LOG;
    // activations (and gradients) for n x h x w
    int n = 0, h = 0, w = 0;
    bool train = false;
    Acts a, g;
    std::vector<void *> allocs;
    float *stage = nullptr;  // host inputs and outputs, loss
    size_t stage_cap = 0;
    unsigned char *fb = nullptr;  // the fallback's host inputs and output, its count
    size_t fb_cap = 0;
    std::mutex mu;
};

namespace {

void free_acts(mb3d_cu_dn *d) {
    for (void *p : d->allocs) cudaFree(p);
    d->allocs.clear();
    d->a = Acts();
    d->g = Acts();
    d->n = d->h = d->w = 0;
}

int alloc_t(mb3d_cu_dn *d, bf16 **p, size_t elems) {
    if (cudaMalloc((void **)p, elems * sizeof(bf16)) != cudaSuccess) return dn_fail(MB3D_CU_ENOMEM, "device memory (denoiser)");
    d->allocs.push_back(*p);
    return 0;
}

int alloc_acts(mb3d_cu_dn *d, Acts &A, int n, int h, int w) {
    size_t M[5];
    for (int l = 0; l < 5; l++) M[l] = (size_t)n * (h >> l) * (w >> l);
    if (int e = alloc_t(d, &A.x0, M[0] * IN_C)) return e;
    for (int l = 0; l < 4; l++) {
        if (int e = alloc_t(d, &A.ea[l], M[l] * CH[l])) return e;
        if (int e = alloc_t(d, &A.cat[l], M[l] * (CH[l + 1] + CH[l]))) return e;
        if (int e = alloc_t(d, &A.pool[l + 1], M[l + 1] * CH[l])) return e;
        if (int e = alloc_t(d, &A.da[l], M[l] * CH[l])) return e;
        if (int e = alloc_t(d, &A.db[l], M[l] * CH[l])) return e;
    }
    if (int e = alloc_t(d, &A.ba, M[4] * CH[4])) return e;
    if (int e = alloc_t(d, &A.bb, M[4] * CH[4])) return e;
    if (int e = alloc_t(d, &A.pred, M[0] * OUT_C)) return e;
    return 0;
}

int ensure(mb3d_cu_dn *d, int n, int h, int w, bool train) {
    if (d->n == n && d->h == h && d->w == w && (d->train || !train)) return 0;
    free_acts(d);
    if (int e = alloc_acts(d, d->a, n, h, w)) return e;
    if (train)
        if (int e = alloc_acts(d, d->g, n, h, w)) return e;
    d->n = n;
    d->h = h;
    d->w = w;
    d->train = train;
    return 0;
}

ConvArgs conv_args(const Layer &L, const bf16 *in, int in_c, int in_off, bf16 *out, int out_c, int out_off, int n, int h,
                   int w, const float *bias) {
    ConvArgs a;
    a.in = in;
    a.wt = L.wf;
    a.bias = bias;
    a.out = out;
    a.n = n;
    a.h = h;
    a.w = w;
    a.m = n * h * w;
    a.in_c = in_c;
    a.in_off = in_off;
    a.cin = L.cin;
    a.out_c = out_c;
    a.out_off = out_off;
    a.cout = L.cout;
    a.relu = L.relu ? 1 : 0;
    a.accumulate = 0;
    return a;
}

#define DN_TRY(x)                                                                   \
    do {                                                                            \
        if ((x) != 0) return dn_fail(MB3D_CU_EINVAL, "denoiser launch arguments"); \
    } while (0)

int forward(mb3d_cu_dn *d, cudaStream_t s) {
    const int n = d->n, h = d->h, w = d->w;
    Acts &A = d->a;
    auto bias = [&](int li) { return d->param + d->layers[li].b_off; };
    for (int l = 0; l < 4; l++) {
        int hl = h >> l, wl = w >> l, cu = CH[l + 1] + CH[l];
        const Layer &La = d->layers[l_enc(l, ENC_A)], &Lb = d->layers[l_enc(l, ENC_B)];
        const bf16 *in = l == 0 ? A.x0 : A.pool[l];
        int inc = l == 0 ? IN_C : CH[l - 1];
        DN_TRY(dn_conv(conv_args(La, in, inc, 0, A.ea[l], CH[l], 0, n, hl, wl, bias(l_enc(l, ENC_A))), s));
        DN_TRY(dn_conv(conv_args(Lb, A.ea[l], CH[l], 0, A.cat[l], cu, CH[l + 1], n, hl, wl, bias(l_enc(l, ENC_B))), s));
        dn_pool2(A.cat[l], cu, CH[l + 1], CH[l], n, hl, wl, A.pool[l + 1], s);
    }
    int h4 = h >> 4, w4 = w >> 4;
    DN_TRY(dn_conv(conv_args(d->layers[L_BOT_A], A.pool[4], CH[3], 0, A.ba, CH[4], 0, n, h4, w4, bias(L_BOT_A)), s));
    DN_TRY(dn_conv(conv_args(d->layers[L_BOT_B], A.ba, CH[4], 0, A.bb, CH[4], 0, n, h4, w4, bias(L_BOT_B)), s));
    for (int l = 3; l >= 0; l--) {
        int hl = h >> l, wl = w >> l, cu = CH[l + 1] + CH[l];
        const bf16 *low = l == 3 ? A.bb : A.db[l + 1];
        dn_up2(low, CH[l + 1], n, hl, wl, A.cat[l], cu, 0, s);
        DN_TRY(dn_conv(conv_args(d->layers[l_dec(l, 0)], A.cat[l], cu, 0, A.da[l], CH[l], 0, n, hl, wl, bias(l_dec(l, 0))), s));
        DN_TRY(dn_conv(conv_args(d->layers[l_dec(l, 1)], A.da[l], CH[l], 0, A.db[l], CH[l], 0, n, hl, wl, bias(l_dec(l, 1))), s));
    }
    DN_TRY(dn_conv(conv_args(d->layers[L_OUT], A.db[0], CH[0], 0, A.pred, OUT_C, 0, n, h, w, bias(L_OUT)), s));
    return 0;
}

// the gradients of layer li: dz (a slot of a tensor, already masked by the
// ReLU) and its input x; dx_out (may be null) receives the input's gradient,
// masked by dx_mask (may be null: the ReLU output the layer's input is, same
// layout as dx)
int layer_bwd(mb3d_cu_dn *d, int li, const bf16 *dz, int dz_c, int dz_off, const bf16 *x, int x_c, int x_off, bf16 *dx,
              int dx_c, int n, int h, int w, cudaStream_t s, const bf16 *dx_mask = nullptr) {
    const Layer &L = d->layers[li];
    WgradArgs wa;
    wa.dz = dz;
    wa.x = x;
    wa.dw = d->grad + L.w_off;
    wa.n = n;
    wa.h = h;
    wa.w = w;
    wa.m = n * h * w;
    wa.dz_c = dz_c;
    wa.dz_off = dz_off;
    wa.cout = L.cout;
    wa.x_c = x_c;
    wa.x_off = x_off;
    wa.cin = L.cin;
    DN_TRY(dn_wgrad(wa, d->grad + L.b_off, s));
    if (dx) {
        ConvArgs a;
        a.in = dz;
        a.wt = L.wb;
        a.bias = nullptr;
        a.out = dx;
        a.n = n;
        a.h = h;
        a.w = w;
        a.m = n * h * w;
        a.in_c = dz_c;
        a.in_off = dz_off;
        a.cin = L.cout;
        a.out_c = dx_c;
        a.out_off = 0;
        a.cout = L.cin;
        a.relu = 0;
        a.accumulate = 0;
        // (the ReLU's backward of the layer below, when its output is x: dx
        // stays where x > 0)
        a.mask = dx_mask;
        a.mask_c = dx_c;
        a.mask_off = 0;
        DN_TRY(dn_conv(a, s));
    }
    return 0;
}

int backward(mb3d_cu_dn *d, cudaStream_t s) {
    const int n = d->n, h = d->h, w = d->w;
    Acts &A = d->a, &G = d->g;
    // the output layer (no ReLU): g.pred holds the loss gradient
    // (the ReLU masks of the gradients that a convolution's input gradient
    // writes whole are fused into that convolution's store)
    if (int e = layer_bwd(d, L_OUT, G.pred, OUT_C, 0, A.db[0], CH[0], 0, G.db[0], CH[0], n, h, w, s, A.db[0])) return e;
    for (int l = 0; l < 4; l++) {
        int hl = h >> l, wl = w >> l, cu = CH[l + 1] + CH[l];
        size_t Ml = (size_t)n * hl * wl;
        if (l > 0) dn_relu_mask(G.db[l], A.db[l], CH[l], 0, CH[l], Ml, s);
        if (int e = layer_bwd(d, l_dec(l, 1), G.db[l], CH[l], 0, A.da[l], CH[l], 0, G.da[l], CH[l], n, hl, wl, s, A.da[l]))
            return e;
        if (int e = layer_bwd(d, l_dec(l, 0), G.da[l], CH[l], 0, A.cat[l], cu, 0, G.cat[l], cu, n, hl, wl, s)) return e;
        bf16 *glow = l == 3 ? G.bb : G.db[l + 1];
        dn_up2_bwd(G.cat[l], cu, 0, CH[l + 1], n, hl, wl, glow, s);
    }
    int h4 = h >> 4, w4 = w >> 4;
    size_t M4 = (size_t)n * h4 * w4;
    dn_relu_mask(G.bb, A.bb, CH[4], 0, CH[4], M4, s);
    if (int e = layer_bwd(d, L_BOT_B, G.bb, CH[4], 0, A.ba, CH[4], 0, G.ba, CH[4], n, h4, w4, s, A.ba)) return e;
    if (int e = layer_bwd(d, L_BOT_A, G.ba, CH[4], 0, A.pool[4], CH[3], 0, G.pool[4], CH[3], n, h4, w4, s)) return e;
    for (int l = 3; l >= 0; l--) {
        int hl = h >> l, wl = w >> l, cu = CH[l + 1] + CH[l];
        size_t Ml = (size_t)n * hl * wl;
        // the skip's gradient: from the decoder (in g.cat) plus the pooling's
        dn_pool2_bwd(A.cat[l], cu, CH[l + 1], CH[l], n, hl, wl, G.pool[l + 1], G.cat[l], s);
        dn_relu_mask(G.cat[l], A.cat[l], cu, CH[l + 1], CH[l], Ml, s);
        if (int e = layer_bwd(d, l_enc(l, ENC_B), G.cat[l], cu, CH[l + 1], A.ea[l], CH[l], 0, G.ea[l], CH[l], n, hl, wl, s,
                              A.ea[l]))
            return e;
        const bf16 *x = l == 0 ? A.x0 : A.pool[l];
        int xc = l == 0 ? IN_C : CH[l - 1];
        if (int e = layer_bwd(d, l_enc(l, ENC_A), G.ea[l], CH[l], 0, x, xc, 0, l == 0 ? nullptr : G.pool[l], xc, n, hl, wl, s))
            return e;
    }
    return 0;
}

void cast_all(mb3d_cu_dn *d, cudaStream_t s) {
    for (auto &L : d->layers) dn_cast_weights(d->param + L.w_off, L.cout, L.cin, L.wf, L.wb, s);
}

// inputs of (n, hs, ws) pixels on the device (copied there when host)
struct Inputs {
    const float *rad, *alb, *nrm, *dep, *tgt;
};

int stage_inputs(mb3d_cu_dn *d, int n, int hs, int ws, const float *rad, const float *alb, const float *nrm,
                 const float *dep, const float *tgt, Inputs &in, cudaStream_t s) {
    size_t px = (size_t)n * hs * ws;
    size_t need = (px * 3 * 3 + px + px * 3 + 16) * sizeof(float);
    if (d->stage_cap < need) {
        cudaFree(d->stage);
        d->stage = nullptr;
        d->stage_cap = 0;
        if (cudaMalloc((void **)&d->stage, need) != cudaSuccess) return dn_fail(MB3D_CU_ENOMEM, "device memory (denoiser)");
        d->stage_cap = need;
    }
    float *p = d->stage + 16;  // (the first 16 floats: the loss)
    auto put = [&](const float *src, size_t count) -> const float * {
        if (!src) return nullptr;
        if (dn_is_device_ptr(src)) return src;
        float *dst = p;
        p += count;
        cudaMemcpyAsync(dst, src, count * sizeof(float), cudaMemcpyHostToDevice, s);
        return dst;
    };
    in.rad = put(rad, px * 3);
    in.alb = put(alb, px * 3);
    in.nrm = put(nrm, px * 3);
    in.dep = put(dep, px);
    in.tgt = tgt ? put(tgt, px * 3) : nullptr;
    return 0;
}

int check(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return dn_fail(MB3D_CU_EIO, std::string(what) + ": " + cudaGetErrorString(e));
    return 0;
}

int sizes(int n, int hs, int ws, int &h, int &w) {
    if (n < 1 || hs < 1 || ws < 1 || hs > 16384 || ws > 16384) return dn_fail(MB3D_CU_EINVAL, "bad picture size");
    h = (hs + 15) & ~15;
    w = (ws + 15) & ~15;
    return 0;
}

// forward, loss and backward into d->grad; *loss on the host
int grad_pass(mb3d_cu_dn *d, int n, int hs, int ws, const float *rad, const float *alb, const float *nrm, const float *dep,
              float depth_scale, const float *target, float *loss) {
    cudaStream_t s = dn_stream(d->ctx);
    int h, w;
    if (int e = sizes(n, hs, ws, h, w)) return e;
    if (int e = ensure(d, n, h, w, true)) return e;
    Inputs in;
    if (int e = stage_inputs(d, n, hs, ws, rad, alb, nrm, dep, target, in, s)) return e;
    dn_pack_input(in.rad, in.alb, in.nrm, in.dep, depth_scale, n, hs, ws, h, w, d->a.x0, s);
    if (int e = forward(d, s)) return e;
    cudaMemsetAsync(d->stage, 0, 16 * sizeof(float), s);
    if (d->loss_kind == MB3D_CU_DN_LOSS_L1_LOG) dn_l1_loss(d->a.pred, in.tgt, n, h, w, hs, ws, d->g.pred, d->stage, s);
    else
        dn_tone_loss(d->a.pred, in.tgt, n, h, w, hs, ws, d->loss_kind == MB3D_CU_DN_LOSS_TONE_DISPLAY, d->g.pred,
                     d->stage, s);
    cudaMemsetAsync(d->grad, 0, d->nparam * sizeof(float), s);
    if (int e = backward(d, s)) return e;
    if (int e = check("denoiser backward")) return e;
    if (loss) {
        cudaMemcpyAsync(loss, d->stage, sizeof(float), cudaMemcpyDeviceToHost, s);
        if (cudaStreamSynchronize(s) != cudaSuccess) return check("denoiser step");
    }
    return 0;
}

}  // namespace

extern "C" {

size_t mb3d_cu_dn_param_count(void) {
    size_t n = 0;
    make_layers(n);
    return n;
}

int mb3d_cu_dn_create(mb3d_cu_ctx *ctx, uint64_t seed, mb3d_cu_dn **out) {
    if (!ctx || !out) return dn_fail(MB3D_CU_EINVAL, "NULL argument");
    *out = nullptr;
    if (cudaSetDevice(dn_device(ctx)) != cudaSuccess) return dn_fail(MB3D_CU_EIO, "cudaSetDevice failed");
    mb3d_cu_dn *d = new mb3d_cu_dn();
    d->ctx = ctx;
    d->layers = make_layers(d->nparam);
    size_t wcount = 0;
    for (auto &L : d->layers) wcount += (size_t)L.cout * 9 * L.cin;
    bool ok = cudaMalloc((void **)&d->param, d->nparam * 4) == cudaSuccess &&
              cudaMalloc((void **)&d->grad, d->nparam * 4) == cudaSuccess &&
              cudaMalloc((void **)&d->m1, d->nparam * 4) == cudaSuccess &&
              cudaMalloc((void **)&d->m2, d->nparam * 4) == cudaSuccess &&
              cudaMalloc((void **)&d->wbuf, 2 * wcount * sizeof(bf16)) == cudaSuccess;
    if (!ok) {
        mb3d_cu_dn_free(d);
        return dn_fail(MB3D_CU_ENOMEM, "device memory (denoiser)");
    }
    size_t o = 0;
    for (auto &L : d->layers) {
        size_t k = (size_t)L.cout * 9 * L.cin;
        L.wf = d->wbuf + o;
        L.wb = d->wbuf + wcount + o;
        o += k;
    }
    // He initialisation from the seed; zero biases; the output layer's
    // channels 3..15 zero
    std::vector<float> h(d->nparam, 0.0f);
    std::mt19937_64 rng(seed);
    for (size_t li = 0; li < d->layers.size(); li++) {
        const Layer &L = d->layers[li];
        std::normal_distribution<float> nd(0.0f, std::sqrt(2.0f / (9.0f * (float)L.cin)));
        for (int co = 0; co < L.cout; co++)
            for (int k = 0; k < 9 * L.cin; k++) {
                float v = nd(rng);
                if ((int)li == L_OUT && co >= 3) v = 0.0f;
                h[L.w_off + (size_t)co * 9 * L.cin + k] = v;
            }
    }
    cudaStream_t s = dn_stream(ctx);
    cudaMemcpyAsync(d->param, h.data(), d->nparam * 4, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(d->m1, 0, d->nparam * 4, s);
    cudaMemsetAsync(d->m2, 0, d->nparam * 4, s);
    cast_all(d, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) {
        mb3d_cu_dn_free(d);
        return check("denoiser init");
    }
    *out = d;
    return 0;
}

void mb3d_cu_dn_free(mb3d_cu_dn *d) {
    if (!d) return;
    cudaSetDevice(dn_device(d->ctx));
    cudaStreamSynchronize(dn_stream(d->ctx));
    free_acts(d);
    cudaFree(d->param);
    cudaFree(d->grad);
    cudaFree(d->m1);
    cudaFree(d->m2);
    cudaFree(d->wbuf);
    cudaFree(d->stage);
    cudaFree(d->fb);
    delete d;
}

int mb3d_cu_dn_get_params(mb3d_cu_dn *d, float *params) {
    if (!d || !params) return dn_fail(MB3D_CU_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(d->mu);
    cudaStream_t s = dn_stream(d->ctx);
    cudaMemcpyAsync(params, d->param, d->nparam * 4, cudaMemcpyDefault, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return check("denoiser get_params");
    return 0;
}

int mb3d_cu_dn_set_params(mb3d_cu_dn *d, const float *params) {
    if (!d || !params) return dn_fail(MB3D_CU_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(d->mu);
    cudaStream_t s = dn_stream(d->ctx);
    cudaMemcpyAsync(d->param, params, d->nparam * 4, cudaMemcpyDefault, s);
    cudaMemsetAsync(d->m1, 0, d->nparam * 4, s);
    cudaMemsetAsync(d->m2, 0, d->nparam * 4, s);
    d->step = 0;
    cast_all(d, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return check("denoiser set_params");
    return 0;
}

int mb3d_cu_dn_denoise(mb3d_cu_dn *d, int n, int hs, int ws, const float *rad, const float *alb, const float *nrm,
                       const float *dep, float depth_scale, float *out) {
    if (!d || !rad || !out) return dn_fail(MB3D_CU_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(d->mu);
    if (cudaSetDevice(dn_device(d->ctx)) != cudaSuccess) return dn_fail(MB3D_CU_EIO, "cudaSetDevice failed");
    cudaStream_t s = dn_stream(d->ctx);
    int h, w;
    if (int e = sizes(n, hs, ws, h, w)) return e;
    if (int e = ensure(d, n, h, w, d->train && d->n == n && d->h == h && d->w == w)) return e;
    Inputs in;
    if (int e = stage_inputs(d, n, hs, ws, rad, alb, nrm, dep, nullptr, in, s)) return e;
    dn_pack_input(in.rad, in.alb, in.nrm, in.dep, depth_scale, n, hs, ws, h, w, d->a.x0, s);
    if (int e = forward(d, s)) return e;
    size_t px = (size_t)n * hs * ws;
    bool dev = dn_is_device_ptr(out);
    float *o = out;
    if (!dev) {
        // (the staging after the inputs: they are consumed by now in stream order)
        o = d->stage + 16;
    }
    dn_unpack_output(d->a.pred, n, h, w, hs, ws, o, s);
    if (!dev) cudaMemcpyAsync(out, o, px * 3 * sizeof(float), cudaMemcpyDeviceToHost, s);
    if (int e = check("denoiser forward")) return e;
    if (cudaStreamSynchronize(s) != cudaSuccess) return check("denoiser forward");
    if (dn_conv_error(s)) return dn_fail(MB3D_CU_EIO, "denoiser forward: a convolution's pipeline wait ran out");
    return 0;
}

int mb3d_cu_dn_fallback(mb3d_cu_dn *d, int h, int w, const float *half_a, const float *half_b, const float *den,
                        int tile, float k, float *out, float *plain_share) {
    if (!d || !half_a || !half_b || !den || !out) return dn_fail(MB3D_CU_EINVAL, "NULL argument");
    if (h < 1 || w < 1 || h > 16384 || w > 16384) return dn_fail(MB3D_CU_EINVAL, "bad picture size");
    if (tile < 1 || tile > 1024 || !(k >= 0.0f) || !std::isfinite(k)) return dn_fail(MB3D_CU_EINVAL, "bad tile or k");
    std::lock_guard<std::mutex> lk(d->mu);
    if (cudaSetDevice(dn_device(d->ctx)) != cudaSuccess) return dn_fail(MB3D_CU_EIO, "cudaSetDevice failed");
    cudaStream_t s = dn_stream(d->ctx);
    const size_t bytes = (size_t)h * w * 3 * sizeof(float);
    const float *src[3] = {half_a, half_b, den};
    bool dev[3], dev_out = dn_is_device_ptr(out);
    size_t need = 256;  // (the count of pieces that keep the plain trace)
    for (int i = 0; i < 3; i++) {
        dev[i] = dn_is_device_ptr(src[i]);
        if (!dev[i]) need += bytes;
    }
    if (!dev_out) need += bytes;
    if (need > d->fb_cap) {
        cudaFree(d->fb);
        d->fb = nullptr;
        d->fb_cap = 0;
        if (cudaMalloc((void **)&d->fb, need) != cudaSuccess) return dn_fail(MB3D_CU_ENOMEM, "device memory (denoiser)");
        d->fb_cap = need;
    }
    unsigned int *bad = (unsigned int *)d->fb;
    unsigned char *q = d->fb + 256;
    const float *dsrc[3];
    for (int i = 0; i < 3; i++) {
        dsrc[i] = src[i];
        if (!dev[i]) {
            cudaMemcpyAsync(q, src[i], bytes, cudaMemcpyHostToDevice, s);
            dsrc[i] = (const float *)q;
            q += bytes;
        }
    }
    float *dout = dev_out ? out : (float *)q;
    cudaMemsetAsync(bad, 0, sizeof(unsigned int), s);
    dn_fallback(dsrc[0], dsrc[1], dsrc[2], h, w, tile, k, dout, bad, s);
    if (!dev_out) cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, s);
    unsigned int nbad = 0;
    cudaMemcpyAsync(&nbad, bad, sizeof(nbad), cudaMemcpyDeviceToHost, s);
    if (int e = check("denoiser fallback")) return e;
    if (cudaStreamSynchronize(s) != cudaSuccess) return check("denoiser fallback");
    const double pieces = (double)((w + tile - 1) / tile) * ((h + tile - 1) / tile);
    if (plain_share) *plain_share = (float)(nbad / pieces);
    return 0;
}

int mb3d_cu_dn_gradient(mb3d_cu_dn *d, int n, int hs, int ws, const float *rad, const float *alb, const float *nrm,
                        const float *dep, float depth_scale, const float *target, float *loss, float *grad) {
    if (!d || !rad || !target || !grad) return dn_fail(MB3D_CU_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(d->mu);
    if (cudaSetDevice(dn_device(d->ctx)) != cudaSuccess) return dn_fail(MB3D_CU_EIO, "cudaSetDevice failed");
    if (int e = grad_pass(d, n, hs, ws, rad, alb, nrm, dep, depth_scale, target, loss)) return e;
    cudaStream_t s = dn_stream(d->ctx);
    cudaMemcpyAsync(grad, d->grad, d->nparam * 4, cudaMemcpyDefault, s);
    if (cudaStreamSynchronize(s) != cudaSuccess) return check("denoiser gradient");
    if (dn_conv_error(s)) return dn_fail(MB3D_CU_EIO, "denoiser gradient: a convolution's pipeline wait ran out");
    return 0;
}

int mb3d_cu_dn_set_loss(mb3d_cu_dn *d, int kind) {
    if (!d) return dn_fail(MB3D_CU_EINVAL, "NULL argument");
    if (kind < MB3D_CU_DN_LOSS_L1_LOG || kind > MB3D_CU_DN_LOSS_TONE_DISPLAY) return dn_fail(MB3D_CU_EINVAL, "unknown loss");
    std::lock_guard<std::mutex> lk(d->mu);
    d->loss_kind = kind;
    return 0;
}

int mb3d_cu_dn_train_step(mb3d_cu_dn *d, int n, int hs, int ws, const float *rad, const float *alb, const float *nrm,
                          const float *dep, float depth_scale, const float *target, float lr, float *loss) {
    if (!d || !rad || !target) return dn_fail(MB3D_CU_EINVAL, "NULL argument");
    std::lock_guard<std::mutex> lk(d->mu);
    if (cudaSetDevice(dn_device(d->ctx)) != cudaSuccess) return dn_fail(MB3D_CU_EIO, "cudaSetDevice failed");
    if (int e = grad_pass(d, n, hs, ws, rad, alb, nrm, dep, depth_scale, target, loss)) return e;
    cudaStream_t s = dn_stream(d->ctx);
    d->step += 1;
    dn_adam(d->param, d->grad, d->m1, d->m2, d->nparam, lr, d->step, s);
    cast_all(d, s);
    if (int e = check("denoiser update")) return e;
    if (!loss && cudaStreamSynchronize(s) != cudaSuccess) return check("denoiser update");
    if (dn_conv_error(s)) return dn_fail(MB3D_CU_EIO, "denoiser update: a convolution's pipeline wait ran out");
    return 0;
}

// one convolution and its two gradients on float data (bf16 inside)
int mb3d_cu_dn_conv_check(mb3d_cu_ctx *ctx, int n, int h, int w, int cin, int cout, const float *x, const float *wt,
                          const float *b, const float *dy, float *y, float *dx, float *dw, float *db) {
    if (!ctx || !x || !wt || !b || !dy || !y || !dx || !dw || !db) return dn_fail(MB3D_CU_EINVAL, "NULL argument");
    if (cin % 16 || cout % 16 || cout > 128 || n < 1 || h < 1 || w < 1) return dn_fail(MB3D_CU_EINVAL, "bad shape");
    if (cudaSetDevice(dn_device(ctx)) != cudaSuccess) return dn_fail(MB3D_CU_EIO, "cudaSetDevice failed");
    cudaStream_t s = dn_stream(ctx);
    size_t m = (size_t)n * h * w, nw = (size_t)cout * 9 * cin;
    std::vector<bf16> hx(m * cin), hdy(m * cout);
    for (size_t i = 0; i < hx.size(); i++) hx[i] = __float2bfloat16(x[i]);
    for (size_t i = 0; i < hdy.size(); i++) hdy[i] = __float2bfloat16(dy[i]);
    bf16 *dxin, *ddy, *dyo, *ddx, *dwf, *dwb;
    float *dwt, *dbias, *ddw, *ddb;
    bool ok = cudaMalloc((void **)&dxin, m * cin * 2) == cudaSuccess && cudaMalloc((void **)&ddy, m * cout * 2) == cudaSuccess &&
              cudaMalloc((void **)&dyo, m * cout * 2) == cudaSuccess && cudaMalloc((void **)&ddx, m * cin * 2) == cudaSuccess &&
              cudaMalloc((void **)&dwf, nw * 2) == cudaSuccess && cudaMalloc((void **)&dwb, nw * 2) == cudaSuccess &&
              cudaMalloc((void **)&dwt, nw * 4) == cudaSuccess && cudaMalloc((void **)&dbias, cout * 4) == cudaSuccess &&
              cudaMalloc((void **)&ddw, nw * 4) == cudaSuccess && cudaMalloc((void **)&ddb, cout * 4) == cudaSuccess;
    if (!ok) return dn_fail(MB3D_CU_ENOMEM, "device memory");
    cudaMemcpyAsync(dxin, hx.data(), m * cin * 2, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(ddy, hdy.data(), m * cout * 2, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dwt, wt, nw * 4, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(dbias, b, cout * 4, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(ddw, 0, nw * 4, s);
    cudaMemsetAsync(ddb, 0, cout * 4, s);
    dn_cast_weights(dwt, cout, cin, dwf, dwb, s);
    ConvArgs a;
    a.in = dxin; a.wt = dwf; a.bias = dbias; a.out = dyo;
    a.n = n; a.h = h; a.w = w; a.m = (int)m;
    a.in_c = cin; a.in_off = 0; a.cin = cin;
    a.out_c = cout; a.out_off = 0; a.cout = cout;
    a.relu = 0; a.accumulate = 0;
    int r = dn_conv(a, s);
    ConvArgs bd = a;
    bd.in = ddy; bd.wt = dwb; bd.bias = nullptr; bd.out = ddx;
    bd.in_c = cout; bd.cin = cout; bd.out_c = cin; bd.cout = cin;
    r |= dn_conv(bd, s);
    WgradArgs wa;
    wa.dz = ddy; wa.x = dxin; wa.dw = ddw;
    wa.n = n; wa.h = h; wa.w = w; wa.m = (int)m;
    wa.dz_c = cout; wa.dz_off = 0; wa.cout = cout;
    wa.x_c = cin; wa.x_off = 0; wa.cin = cin;
    r |= dn_wgrad(wa, ddb, s);
    std::vector<bf16> hy(m * cout), hdx(m * cin);
    cudaMemcpyAsync(hy.data(), dyo, m * cout * 2, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(hdx.data(), ddx, m * cin * 2, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(dw, ddw, nw * 4, cudaMemcpyDeviceToHost, s);
    cudaMemcpyAsync(db, ddb, cout * 4, cudaMemcpyDeviceToHost, s);
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFree(dxin); cudaFree(ddy); cudaFree(dyo); cudaFree(ddx); cudaFree(dwf); cudaFree(dwb);
    cudaFree(dwt); cudaFree(dbias); cudaFree(ddw); cudaFree(ddb);
    if (r) return dn_fail(MB3D_CU_EINVAL, "convolution launch arguments");
    if (e != cudaSuccess) return dn_fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    if (dn_conv_error(s)) return dn_fail(MB3D_CU_EIO, "convolution: a pipeline wait ran out");
    for (size_t i = 0; i < hy.size(); i++) y[i] = __bfloat162float(hy[i]);
    for (size_t i = 0; i < hdx.size(); i++) dx[i] = __bfloat162float(hdx[i]);
    return 0;
}

int mb3d_cu_dn_wait_check(mb3d_cu_ctx *ctx, double wait_us, int no_issue) {
    if (!ctx) return dn_fail(MB3D_CU_EINVAL, "NULL argument");
    if (!(wait_us >= 1.0 && wait_us <= 2e6)) return dn_fail(MB3D_CU_EINVAL, "wait_us outside 1 .. 2e6");
    if (cudaSetDevice(dn_device(ctx)) != cudaSuccess) return dn_fail(MB3D_CU_EIO, "cudaSetDevice failed");
    int khz = 0;
    if (cudaDeviceGetAttribute(&khz, cudaDevAttrClockRate, dn_device(ctx)) != cudaSuccess || khz <= 0) khz = 2000000;
    cudaStream_t s = dn_stream(ctx);
    const int n = 1, h = 16, w = 16, c = 16;
    const size_t m = (size_t)n * h * w, nw = (size_t)c * 9 * c;
    bf16 *din = nullptr, *dout = nullptr, *dwf = nullptr, *dwb = nullptr;
    float *dwt = nullptr;
    bool ok = cudaMalloc((void **)&din, m * c * 2) == cudaSuccess && cudaMalloc((void **)&dout, m * c * 2) == cudaSuccess &&
              cudaMalloc((void **)&dwf, nw * 2) == cudaSuccess && cudaMalloc((void **)&dwb, nw * 2) == cudaSuccess &&
              cudaMalloc((void **)&dwt, nw * 4) == cudaSuccess;
    if (ok) {
        cudaMemsetAsync(din, 0, m * c * 2, s);
        cudaMemsetAsync(dwt, 0, nw * 4, s);
        dn_cast_weights(dwt, c, c, dwf, dwb, s);
    }
    int r = -1;
    if (ok) {
        ConvArgs a;
        a.in = din; a.wt = dwf; a.bias = nullptr; a.out = dout;
        a.n = n; a.h = h; a.w = w; a.m = (int)m;
        a.in_c = c; a.in_off = 0; a.cin = c;
        a.out_c = c; a.out_off = 0; a.cout = c;
        a.relu = 0; a.accumulate = 0;
        a.wait_cycles = (long long)(wait_us * (double)khz * 1e-3);
        a.no_issue = no_issue ? 1 : 0;
        r = dn_conv(a, s);
    }
    cudaError_t e = cudaStreamSynchronize(s);
    cudaFree(din); cudaFree(dout); cudaFree(dwf); cudaFree(dwb); cudaFree(dwt);
    if (!ok) return dn_fail(MB3D_CU_ENOMEM, "device memory");
    if (r) return dn_fail(MB3D_CU_EINVAL, "convolution launch arguments");
    if (e != cudaSuccess) return dn_fail(MB3D_CU_EIO, std::string("device: ") + cudaGetErrorString(e));
    if (dn_conv_error(s)) return dn_fail(MB3D_CU_EIO, "convolution: a pipeline wait ran out");
    return 0;
}

}  // extern "C"
