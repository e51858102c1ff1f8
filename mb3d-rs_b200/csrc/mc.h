// The Monte Carlo tracer's launch parameters, shared by the host code and
// the kernels (mc.cuh).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "../../include/mb3d_cu.h"

namespace mb3dcu {

// the render constants of CalcMCT (src/mc.rs:3120-3237) the card needs
struct McDev {
    mb3d_cu_mc_light lv;
    double hs_vecs[6][3];  // HSvecs: -step width x the light direction, world
    double amb_max_l, zz_stmit_dif;
    float fovy1d, soft_shadow_radius, hs_max_lmul, pad;
    int32_t max_amb_depth, secant, rays, ray0;
    int32_t x0, y0, w, h;
    uint32_t npad, tiles_x;  // the rectangle's pixels in 8x4 tiles (npad = tiles x 32)
    const uint2 *halton;     // halton_seq (src/mc.rs:117-128): (hrx | hry << 16, hdx | hdy << 16)
    // (or null) the items of an adaptive pass: item i is ray items[i].y of
    // pixel items[i].x of the rectangle (no first-surface outputs)
    const uint2 *items;
};

// per pixel accumulators of a render
struct McAcc {
    unsigned long long *sum;  // 3 per pixel, light in 32.32 fixed point
    unsigned int *hit;        // 1 per pixel
    float *albedo, *normal, *depth;  // the first surface of ray ray0 (device, may be null)
    unsigned long long *counters;    // [0] DE evaluations, [1] centre iterations, [2] inside starts, [3] FP64 fallbacks
    // (or null) 2 per pixel: the rays' luminance (YofSVec of the clamped
    // light) in 32.32 fixed point and its square in 40.24 fixed point
    unsigned long long *ysum = nullptr;
};

// an adaptive Monte Carlo pass over the whole picture (mc_pass.cu)
struct McPassArgs {
    mb3d_cu_mc_record *recs;          // width * height, updated
    const mb3d_cu_mc_record *snap;    // the records at the start of the pass
    int *total;                       // per pixel: the rays of its coming round (0: none)
    int w, h;
    int skip_nonzero, max_new, sqr;
    uint32_t pass_nr;
    double avrg_vari;
    float avrg_rcount;
};

}  // namespace mb3dcu
