// paint_recs (src/mc.rs:3957-4005) on the card: the Monte Carlo records'
// colours to 8-bit RGB.  Built with -fmad=false: the reference's single
// precision arithmetic is unfused.
#include <cuda_runtime.h>
#include <stdint.h>
#include "kernels.h"

namespace mb3dcu {

namespace {

struct PaintK {
    float contrast, saturation, sgamma;
    int gmode, soft_clip;
};

// SVecRGB2Lab (src/mc.rs:3906-3919)
__device__ __forceinline__ void rgb_to_lab(const float v[3], float o[3]) {
    const float sftc = 216.0f / (29.0f * 29.0f * 29.0f), s4d29 = 4.0f / 29.0f, smul = 29.0f * 29.0f / 108.0f;
    float x[3] = {(0.412453f * v[0] + 0.35758f * v[1] + 0.180423f * v[2]) * 1.052111f,
                  0.212671f * v[0] + 0.71516f * v[1] + 0.072169f * v[2],
                  (0.019334f * v[0] + 0.119193f * v[1] + 0.950227f * v[2]) * 0.918417f};
#pragma unroll
    for (int k = 0; k < 3; k++) x[k] = x[k] > sftc ? cbrtf(x[k]) : smul * x[k] + s4d29;
    o[0] = 1.16f * x[1] - 0.16f;
    o[1] = x[0] - x[1];
    o[2] = x[1] - x[2];
}

// SVecLab2RGB (src/mc.rs:3922-3938)
__device__ __forceinline__ void lab_to_rgb(const float v[3], float o[3]) {
    const float sftc = 6.0f / 29.0f, s4d29 = 4.0f / 29.0f, smul = 108.0f / 841.0f;
    float y = (v[0] + 0.16f) / 1.16f;
    float x[3] = {y + v[1], y, y - v[2]};
#pragma unroll
    for (int k = 0; k < 3; k++) x[k] = x[k] > sftc ? x[k] * x[k] * x[k] : (x[k] - s4d29) * smul;
    x[0] *= 0.95047f;
    x[2] *= 1.08883f;
    o[0] = 3.240479f * x[0] - 1.537150f * x[1] - 0.498535f * x[2];
    o[1] = -0.969256f * x[0] + 1.875992f * x[1] + 0.041556f * x[2];
    o[2] = 0.055648f * x[0] - 0.204043f * x[1] + 1.057311f * x[2];
}

__global__ void k_mc_paint(const float *col, const uint8_t *rays, uint32_t n, PaintK k, uint8_t *out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint8_t o[3] = {0, 0, 0};
        if (!rays || rays[i]) {
            float v[3];
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float x = fmaxf(col[3 * i + c] * k.contrast, 0.0f);
                v[c] = x * x;
            }
            float lab[3];
            rgb_to_lab(v, lab);
            float scol = k.saturation;
            if (lab[0] > 0.0f) {
                if (k.gmode != 0) {
                    float s2 = lab[0];
                    float s = k.gmode > 0 ? sqrtf(lab[0]) : lab[0] * lab[0];
                    lab[0] += (s - lab[0]) * k.sgamma;
                    if (k.gmode > 0 && s2 > 1.0f) scol *= lab[0] / s2;
                }
                if (k.soft_clip) {
                    float s = lab[0];
                    float x2 = s * s;
                    float q = x2 * 0.9f;
                    lab[0] = sqrtf(x2 / sqrtf(q * q + 1.0f));
                    scol *= lab[0] / s;
                }
            }
            lab[1] *= scol;
            lab[2] *= scol;
            float rgb[3];
            lab_to_rgb(lab, rgb);
#pragma unroll
            for (int c = 0; c < 3; c++) {
                float x = sqrtf(fmaxf(rgb[c], 0.0f));
                x = fminf(fmaxf(x, 0.0f), 1.0f) * 255.0f;
                o[c] = (uint8_t)roundf(x);
            }
        }
        out[3 * i] = o[0];
        out[3 * i + 1] = o[1];
        out[3 * i + 2] = o[2];
    }
}

}  // namespace

// the constants of paint_recs from the settings, then the kernel
void mc_paint_launch(const float *col, const uint8_t *rays, uint32_t n, const mb3d_cu_mc_paint_opts &mc, uint8_t *out,
                     int blocks, cudaStream_t s) {
    PaintK k;
    float c = (float)mc.contrast / 256.0f + 0.5f;
    k.contrast = c * c;
    k.soft_clip = (mc.options & 1) != 0;
    k.saturation = (float)(mc.saturation & 0x7F) / 32.0f;
    // (gamma.round() as i32).clamp(0, 63): the cast saturates, NaN gives 0
    float gr = roundf(mc.gamma);
    int ig = gr != gr ? 0 : gr < 0.0f ? 0 : gr > 63.0f ? 63 : (int)gr;
    int igamma = (ig << 2) & 0xFC;
    if (k.soft_clip) {
        igamma = igamma - 20 > 0 ? igamma - 20 : 0;
        k.contrast *= 1.1f;
    }
    if (igamma > 128) {
        k.gmode = 1;
        k.sgamma = (float)(igamma - 128) / 127.0f;
    } else if (igamma < 128) {
        k.gmode = -1;
        k.sgamma = 1.0f - (float)igamma / 128.0f;
    } else {
        k.gmode = 0;
        k.sgamma = 1.0f;
    }
    k_mc_paint<<<blocks, 256, 0, s>>>(col, rays, n, k, out);
}

}  // namespace mb3dcu
