// The flat per-render parameter block the kernels read: the fields of
// mb3d-rs's CalcParams (src/calc.rs:21-134) that the march, the post passes
// and the Monte Carlo tracer use, plus single precision copies for the
// mixed-precision march.  Passed to every kernel by value (kernel
// parameters live in the constant bank, uniform across the grid), so
// concurrent contexts with different scenes never share state.
#pragma once
#include <stdint.h>

#define MB3D_MAX_SLOTS 6
#define MB3D_MAX_LIGHTS 6
#define MB3D_MAX_AO_RAYS 40

struct DevSlot {
    int32_t formula;    // MB3D_CU_F_*
    int32_t iterations; // >= 0
    int32_t uncounted;
    int32_t ade;
    int32_t julia_add;
    int32_t ipow;       // the integer power (IntPow, FoldingIntPow)
    int32_t kind;       // FKIND_* bit of the formula (IntPow 8 apart from the other powers)
    int32_t pad;
    double o[8];        // options (Aexion C reads eight)
    float of[8];        // options, single precision
};

struct DevParams {
    DevSlot slots[MB3D_MAX_SLOTS];
    int32_t n_slots, end_to, repeat_from, is_custom_de;
    int32_t de_option, max_it, min_it, de_add_steps;
    int32_t sm_normals, color_option, color_on_it, dfog_on_it;
    int32_t normals_on_de, first_step_random, do_julia, width;
    int32_t height, all_fp64, n_lights, shadow_soft;
    int32_t fmask;        // FKIND_* bits of the formulas the scene uses
    int32_t finish_slow;  // every surface in the FP64 marcher (smoothed normals, colour on iteration, ...)
    float d_de_scale, de_stop, z_step_div, mh04zsd;
    float de_stop_factor, ln_rstop, de_offset, de_offset006;
    float mcts_m, ms_de_sub, d_col_plus, col_var;
    float fovx_off, fovx_mul, pl_optic_z, mct_color_mul;
    float fhln[6];
    float hand_margin;  // the mixed march hands over from where DE >= this x DE stop
    int32_t hand_back;  // ... at most this many steps back
    int32_t refill_min, blocks_per_sm;  // wavefront: idle lanes that trigger a refill; resident blocks
    int32_t refill_shadow, refill_ao;   // ... of the shadow and DE AO ray kernels
    int32_t blocks_march32;             // resident blocks of the single precision march
    int32_t sched;                      // SCHED_*: the slots' order when it is one the DE loop has unrolled
    float d_rstop_f, rstop3d_f, soft_radius, hs_max_len_mul;
    double d_rstop, rstop3d, zcorr, zc_mul;
    double zend, step_width, fov_y, coord_eps;
    double ju[4];
    float ju_f[4];
    double vgrads[3][3];
    double ystart[3];
    // the shadow pass: light index and HSvecs (world, -step width long)
    int32_t light_idx[MB3D_MAX_LIGHTS];
    double light_vec[MB3D_MAX_LIGHTS][3];
    // the DE AO pass (src/deao.rs:75-104): ray directions of the quality
    int32_t ao_quality, ao_rays, ao_first_step_random, pad1;
    float ao_d_step_mul, ao_d_min_a_dif, ao_corr_weight, ao_max_len;
    float ao_dirs[MB3D_MAX_AO_RAYS][3];
    double ao_rot[3][3];  // camera rows, step width long (normalise_matrix_to(sw, vgrads))
    // the call's device time budget (0: none): the march and finish kernels
    // take no new rays once this many nanoseconds have passed since the
    // first warp of the call asked (their queue counters stay resumable)
    unsigned long long budget_ns;
    // an interpolation hybrid (HybridMode::Ipol3D): the two first slots'
    // formulas blended in every iteration with the normalised weights
    int32_t ipol, pad_ipol;
    float ipol_w[2];
    // a 4D hybrid (HybridMode::Alt4D, the 4D numerical DE) and its rotation
    // (BuildSMatrix4, single precision values)
    int32_t four_d;
    // the DE runs on the sequential FP64 record (de_seq): interpolation and
    // 4D hybrids and hybrids with a Quaternion
    int32_t seq_de;
    double smatrix4[4][4];
    // a DE combination (DeComb, src/calc.rs:224-236): its kind (0: none,
    // 1..5) and its second hybrid part (HybridPart, :210-220), which runs on
    // the sequential FP64 record too
    int32_t dc_kind, dc_start2, dc_end2, dc_rep2;
    int32_t dc_max_it2, dc_de_option2, dc_custom2, dc_place;
    float dc_d_de_scale2, pad_dc;
    double dc_smooth;           // the smoothing distance in steps
    double dc_offset[3];        // Place: m * (p - offset), distances times scale
    double dc_m[3][3];
    double dc_scale;
};

// slot orders the single precision DE loop knows at compile time
#define SCHED_GENERIC 0
#define SCHED_BOX2_IP8 1  // Amazing Box x2, Integer Power 8 x1, repeating from slot 0
#define SCHED_IP8 2       // one Integer Power 8 slot
#define SCHED_MENGER_BOX 3  // Menger IFS x1, Amazing Box x1, repeating from slot 0 (the analytic DE's loop)

// the counters' slots (unsigned int) the march kernels share with the host
#define CNT_HAND 0        // hand-over list length
#define CNT_MARCH_Q 1     // the march's queue
#define CNT_SLOW 2        // slow list length
#define CNT_FINISH_Q 3    // the finish's queue
#define CNT_SLOW_Q 4      // the slow finish's queue
#define CNT_T0 32         // (two slots) %globaltimer of the call's first take
#define CNT_STATUS 34     // bits: 1 the march, 2 the finish, 4 the slow finish stopped on the budget;
                          // ST_TRIP_CAP a march or finish warp ran out of loop trips
#define ST_TRIP_CAP 8u
// the wavefront kernels' loop limit (a warp's trips; one DE per trip)
#define MB3D_TRIP_CAP 400000000u
#define CNT_OVERFLOW 35   // pixels whose single precision DE overflowed
