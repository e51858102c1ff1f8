// The distance estimate of the march loop, in double or single precision:
// only the two values the march decides on (the DE in step widths and the
// iteration count), with the four orbits of the numerical DE iterated in
// lock-step.
//
// Numerical DE (MB3D DE option 0, src/calc.rs:1515-1543): the hybrid at c,
// then at c + offset on each axis with the centre's iteration count as the
// limit and RStop3D as the bailout; DE = R ln R * s / (sqrt(sum (R - R_k)^2)
// + o006).  In lock-step the offset orbits stop where the centre stops (its
// count is their limit) or at their own bailout, exactly as the sequential
// runs do, so the double precision form gives the reference's values.
//
// The single precision form keeps the reference's formula, rewritten so that
// it stays accurate and overflow-free in single precision:
//     d_k = (v - v_k).(v + v_k) / |v|^2 (scaled by the largest component),
//     DE  = ln R * s / (sqrt(sum (d_k * h/h_k)^2) + o006 / R),
// where h_k is the offset each rounded offset point actually got, so that
// the rounding of the coordinates does not bias the gradient.
//
// Analytic DE (options 2 / 11, src/iteration.rs:539-574): one orbit with the
// running derivative in w; sqrt(R) / |w|.
#pragma once
#include "devparams.h"
#include "formulas.cuh"
#include "marcher64.cuh"

namespace mb3dcu {

struct DEr {
    double de;
    int it;
    int max_its;    // the iteration limit of the part that ruled (max_its_result; a DE combination's)
    bool need64;    // single precision cannot resolve the offset here
    bool overflow;  // ... because its DE overflowed (not finite)
};

// The iteration state a full DE leaves for the colouring (the record's
// fields after calc_de, src/calc.rs:1536-1542: rout and it_result of the
// centre; rold, otrap and the vector of the last run, the z offset's for the
// numerical DE) and the centre's smoothed iteration count.
struct DEstate {
    double rout, rold, otrap, v[3];
    float smooth_it;
};

// The iteration count at which a DE's point counts as in the set: the
// scene's maximum, or in a DE combination the ruling part's (only the
// all-formula kernels meet one)
template <int FM>
__device__ __forceinline__ int its_cap(const DevParams &p, const DEr &r) {
    if constexpr (FM == FKIND_ALL) return r.max_its;
    return p.max_it;
}

__device__ __forceinline__ float fsqrt_fast(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }

// ln |v|^2 without overflow
__device__ __forceinline__ float log_len2_f(const float v[4]) {
    float m = fmaxf(fabsf(v[0]), fmaxf(fabsf(v[1]), fabsf(v[2])));
    if (!(m > 0.0f)) return -1e30f;
    float s = __frcp_rn(m);
    float a = v[0] * s, b = v[1] * s, c = v[2] * s;
    return __logf(a * a + b * b + c * c) + 2.0f * __logf(m);
}

template <typename R>
__device__ __forceinline__ R param_f(const DevParams &p, double d, float f);
template <>
__device__ __forceinline__ double param_f<double>(const DevParams &, double d, float) { return d; }
template <>
__device__ __forceinline__ float param_f<float>(const DevParams &, double, float f) { return f; }

// One counted-or-not hybrid step on the Q orbits (run_with's body,
// src/iteration.rs:289-301).  The slot's formula is chosen once for all
// orbits, so that their independent chains share one block of code.
template <typename R, int Q, int FM>
__device__ __forceinline__ void step_orbits(const DevSlot &s, R (&v)[Q][4], R (&j)[Q][3], const R (&rout)[Q]) {
    if ((FM & FKIND_IP8) && (FM == FKIND_IP8 || s.kind == FKIND_IP8)) {
        const R zmul = Num<R>::opt(s, 1);
#pragma unroll
        for (int q = 0; q < Q; q++) f_int_pow<R>(8, zmul, v[q], j[q]);
    } else if ((FM & FKIND_BOX) && s.kind == FKIND_BOX) {
        const R scale = Num<R>::opt(s, 0), min_r = Num<R>::opt(s, 1), fold = Num<R>::opt(s, 2);
        const bool ade = s.ade != 0;
#pragma unroll
        for (int q = 0; q < Q; q++) f_amazing_box<R>(scale, min_r, fold, v[q], j[q], ade);
    } else if ((FM & FKIND_MENGER) && s.kind == FKIND_MENGER) {
        const R sc = Num<R>::opt(s, 0), cx = Num<R>::opt(s, 1), cy = Num<R>::opt(s, 2), cz = Num<R>::opt(s, 3);
        const bool ade = s.ade != 0;
#pragma unroll
        for (int q = 0; q < Q; q++) f_menger<R>(sc, cx, cy, cz, v[q], ade);
    } else if (FM == FKIND_ALL) {
#pragma unroll
        for (int q = 0; q < Q; q++) formula_iterate<R, FM>(s, v[q], j[q], rout[q]);
    }
#pragma unroll
    for (int q = 0; q < Q; q++) {
        if (s.julia_add) {
            v[q][0] += j[q][0];
            v[q][1] += j[q][1];
            v[q][2] += j[q][2];
        }
    }
}

// Counting (bench and roofline only): orbit iterations per slot and DE
// evaluations, kept per thread and added to global counters at the end.
// The march kernel adds its warps' lane use: [0] the rays' lock-step
// iterations, [1] per warp trip the most iterations of its lanes, [2] the
// warp trips that evaluated DEs, [3] the lanes busy in them.
struct DECount {
    unsigned long long its[MB3D_MAX_SLOTS];
    unsigned long long evals;
    unsigned long long lanes[4];
    __device__ void clear() {
        for (int k = 0; k < MB3D_MAX_SLOTS; k++) its[k] = 0;
        evals = 0;
        for (int k = 0; k < 4; k++) lanes[k] = 0;
    }
    __device__ void flush(unsigned long long *g) {
        for (int k = 0; k < MB3D_MAX_SLOTS; k++)
            if (its[k]) atomicAdd(&g[k], its[k]);
        if (evals) atomicAdd(&g[MB3D_MAX_SLOTS], evals);
        for (int k = 0; k < 4; k++)
            if (lanes[k]) atomicAdd(&g[MB3D_MAX_SLOTS + 1 + k], lanes[k]);
    }
};

// CalcSmoothIterations (src/iteration.rs:140-152) on the centre's lengths,
// given as ln(rout) and ln(rold) (single precision: from the scaled vector,
// so that an overflowed length still has its logarithm)
__device__ __forceinline__ float smooth_iterations_d(const DevParams &p, bool rout_le1, bool rold_lt1, double lr,
                                                     double lro, int it, int n) {
    if (rout_le1) return (float)it;
    if (rold_lt1) {
        double d = log(lr * 0.5) * (double)p.fhln[n];
        return (float)((double)it + (double)p.ln_rstop - d);
    }
    double d = log(0.5 * lr);
    double e = d - log(0.5 * lro);
    return (float)(((double)p.ln_rstop - d) / (e + 1e-100) + (double)it);
}

template <typename R>
__device__ __forceinline__ float smooth_of(const DevParams &p, R rout, R rold, const R v[4], int it, int n) {
    if (sizeof(R) == 8) {
        double ro = (double)rout, rl = (double)rold;
        if (ro <= 1.0) return (float)it;
        return smooth_iterations_d(p, false, rl < 1.0, log(ro), rl < 1.0 ? 0.0 : log(rl), it, n);
    } else {
        float ro = (float)rout, rl = (float)rold;
        if (ro <= 1.0f) return (float)it;
        float vf[4] = {(float)v[0], (float)v[1], (float)v[2], 0.f};
        double lr = (ro < 1e30f) ? (double)__logf(ro) : (double)log_len2_f(vf);
        return smooth_iterations_d(p, false, rl < 1.0f, lr, rl < 1.0f ? 0.0 : (double)__logf(rl), it, n);
    }
}

// The DE of the hybrids the lock-step loop does not carry -- interpolation
// hybrids, 4D hybrids, any hybrid with a Quaternion (its j has four
// components) -- in double precision, one orbit at a time on the
// sequential FP64 iteration record: calc_de_part (src/calc.rs:1495-1557)
// with mand_function / mand_function_de of the scene's mode, the numerical
// DE's three offset points limited by the centre's count and bailing out at
// RStop3D, as the reference runs them.  Kept out of line: it is no part of
// the ordinary hybrids' loop.
template <int FM, bool FULL, typename P>
__device__ __noinline__ DEr de_seq(const DevParams &p, const P c[3], float ms_de_stop, DEstate *st, bool calc_sit,
                                   int max_add) {
    DEr out;
    out.need64 = false;
    out.overflow = false;
    It64<FM> it;
    for (int k = 0; k < 3; k++) it.c[k] = (double)c[k];
    for (int k = 0; k < 4; k++) it.v[k] = 0.0;
    it.rout = it.rold = it.otrap = 0.0;
    it.it_result = 0;
    it.max_it = p.max_it + max_add;
    it.rstop = p.d_rstop;
    it.calc_sit = FULL && calc_sit;
    it.part2 = false;
    it.smooth_it = 0.f;
    out.max_its = it.max_it;
    if (p.dc_kind) {
        out.de = de_comb<FM>(p, it, ms_de_stop, out.max_its);
        out.it = it.it_result;
        if (FULL) {
            st->rout = it.rout;
            st->rold = it.rold;
            st->otrap = it.otrap;
            st->v[0] = it.v[0]; st->v[1] = it.v[1]; st->v[2] = it.v[2];
            st->smooth_it = it.smooth_it;
        }
        return out;
    }
    if (p.is_custom_de) {
        out.de = it.hybrid_3d_de(p) * (double)p.d_de_scale;
        out.it = it.it_result;
        if (FULL) {
            st->rout = it.rout;
            st->rold = it.rold;
            st->otrap = it.otrap;
            st->v[0] = it.v[0]; st->v[1] = it.v[1]; st->v[2] = it.v[2];
            st->smooth_it = it.smooth_it;
        }
    } else {
        it.hybrid_3d(p);
        const double R0 = it.rout;
        const int it0 = it.it_result;
        const float sit = it.smooth_it;
        if (R0 < 1e-200) {
            out.de = 0.0;
        } else {
            it.calc_sit = false;
            it.max_it = it0;
            it.rstop = p.rstop3d;
            double g = 0.0;
            for (int k = 0; k < 3; k++) {
                const double b = it.c[k];
                it.c[k] = b + (double)p.de_offset;
                it.hybrid_3d(p);
                g += (R0 - it.rout) * (R0 - it.rout);
                it.c[k] = b;
            }
            out.de = R0 * log(R0) * (double)p.d_de_scale / (sqrt(g) + (double)p.de_offset006);
        }
        out.it = it0;
        if (FULL) {
            st->rout = R0;
            st->rold = it.rold;
            st->otrap = it.otrap;
            st->v[0] = it.v[0]; st->v[1] = it.v[1]; st->v[2] = it.v[2];
            st->smooth_it = sit;
        }
    }
    const double mn = (double)ms_de_stop * 0.25;
    if (out.de < mn || isnan(out.de)) out.de = mn;
    return out;
}

// The position c is double (the FP64 march, and the single precision DE of
// a double precision position) or, for the single precision DE only, float
// (P = float: the bulk march keeps its position in single precision).
template <typename R, int FM, bool COUNT = false, bool FULL = false, typename P = double>
__device__ __forceinline__ DEr de_lock(const DevParams &p, const P c[3], float ms_de_stop, DECount *cnt = nullptr,
                                       DEstate *st = nullptr, bool calc_sit = false, int max_add = 0) {
    static_assert(sizeof(P) == 8 || sizeof(R) == 4, "a single precision position needs the single precision DE");
    if (COUNT) cnt->evals++;
    // (those hybrids run in double precision only and in the all-formula
    // kernels: their scenes are all-FP64 and carry every formula bit)
    if constexpr (sizeof(R) == 8 && FM == FKIND_ALL) {
        if (p.seq_de) return de_seq<FM, FULL, P>(p, c, ms_de_stop, st, calc_sit, max_add);
    }
    DEr out;
    out.need64 = false;
    out.overflow = false;
    const int max_it = p.max_it + max_add;  // (max_add: doBinSearchIt's one more iteration)
    out.max_its = max_it;
    const R rstop = param_f<R>(p, p.d_rstop, p.d_rstop_f);
    if (p.is_custom_de) {
        R v[1][4], j[1][3], rout[1];
        v[0][0] = (R)c[0];
        v[0][1] = (R)c[1];
        v[0][2] = (R)c[2];
        if (p.do_julia) {
            j[0][0] = param_f<R>(p, p.ju[0], p.ju_f[0]);
            j[0][1] = param_f<R>(p, p.ju[1], p.ju_f[1]);
            j[0][2] = param_f<R>(p, p.ju[2], p.ju_f[2]);
        } else {
            j[0][0] = v[0][0]; j[0][1] = v[0][1]; j[0][2] = v[0][2];
        }
        rout[0] = v[0][0] * v[0][0] + v[0][1] * v[0][1] + v[0][2] * v[0][2];
        v[0][3] = ((p.de_option & 0x38) == 16) ? rout[0] : R(1);
        R rold0 = 0, otrap0 = rout[0];
        int n = 0, btmp = p.slots[0].iterations, it = 0;
        unsigned int unc = 0;
        if constexpr ((FM & FKIND_MENGER) && (FM & FKIND_BOX)) {
            if (p.sched == SCHED_MENGER_BOX) {
                // Menger IFS, Amazing Box, repeating, every iteration counted:
                // the slots' order unrolled (the same formulas in the same
                // order as the slot loop below, without its bookkeeping)
                const DevSlot &s0 = p.slots[0], &s1 = p.slots[1];
                const R m_s = Num<R>::opt(s0, 0), m_cx = Num<R>::opt(s0, 1), m_cy = Num<R>::opt(s0, 2),
                        m_cz = Num<R>::opt(s0, 3);
                const R b_s = Num<R>::opt(s1, 0), b_min = Num<R>::opt(s1, 1), b_fold = Num<R>::opt(s1, 2);
                const bool m_ade = s0.ade != 0, b_ade = s1.ade != 0;
                for (;;) {
                    if (FULL) rold0 = rout[0];
                    f_menger<R>(m_s, m_cx, m_cy, m_cz, v[0], m_ade);
                    if (COUNT) cnt->its[0] += 1;
                    it += 1;
                    rout[0] = v[0][0] * v[0][0] + v[0][1] * v[0][1] + v[0][2] * v[0][2];
                    if (FULL && rout[0] < otrap0) otrap0 = rout[0];
                    if (it >= max_it || rout[0] > rstop) {
                        n = 0;
                        break;
                    }
                    if (FULL) rold0 = rout[0];
                    f_amazing_box<R>(b_s, b_min, b_fold, v[0], j[0], b_ade);
                    if (COUNT) cnt->its[1] += 1;
                    it += 1;
                    rout[0] = v[0][0] * v[0][0] + v[0][1] * v[0][1] + v[0][2] * v[0][2];
                    if (FULL && rout[0] < otrap0) otrap0 = rout[0];
                    if (it >= max_it || rout[0] > rstop) {
                        n = 1;
                        break;
                    }
                }
                goto done_a;
            }
        }
        for (;;) {
            if (FULL) rold0 = rout[0];
            int guard = 0;
            while (btmp <= 0) {
                n += 1;
                if (n > p.end_to) n = p.repeat_from;
                btmp = p.slots[n].iterations;
                if (++guard > 64) goto done_a;
            }
            {
                const DevSlot &s = p.slots[n];
                step_orbits<R, 1, FM>(s, v, j, rout);
                if (COUNT) cnt->its[n] += 1;
                btmp -= 1;
                if (s.uncounted) {
                    if (++unc > 100000u) goto done_a;
                    continue;
                }
            }
            it += 1;
            rout[0] = v[0][0] * v[0][0] + v[0][1] * v[0][1] + v[0][2] * v[0][2];
            if (FULL && rout[0] < otrap0) otrap0 = rout[0];
            if (it >= max_it || rout[0] > rstop) break;
        }
    done_a:
        if (FULL) {
            st->rout = (double)rout[0];
            st->rold = (double)rold0;
            st->otrap = (double)otrap0;
            st->v[0] = (double)v[0][0]; st->v[1] = (double)v[0][1]; st->v[2] = (double)v[0][2];
            st->smooth_it = calc_sit ? smooth_of<R>(p, rout[0], rold0, v[0], it, n) : 0.f;
        }
        double r;
        if (sizeof(R) == 8) {
            double w = (double)v[0][3];
            r = ((p.de_option & 7) == 4) ? fabs((double)v[0][1]) * log(fabs((double)v[0][1])) / w
                                         : sqrt((double)rout[0]) / fabs(w);
        } else {
            float vf[4] = {(float)v[0][0], (float)v[0][1], (float)v[0][2], (float)v[0][3]};
            float rf;
            if ((p.de_option & 7) == 4) {
                rf = __fdividef(fabsf(vf[1]) * __logf(fabsf(vf[1])), vf[3]);
            } else {
                float len = fsqrt_fast((float)rout[0]);
                if (!((float)rout[0] < 1e30f)) len = __expf(0.5f * log_len2_f(vf));
                rf = __fdividef(len, fabsf(vf[3]));
            }
            r = (double)rf;
        }
        out.de = r * (double)p.d_de_scale;
        out.it = it;
    } else {
        // four orbits: 0 = the centre, 1..3 = the offsets on x, y, z
        R v[4][4], j[4][3], rout[4];
        float corr[3] = {1.f, 1.f, 1.f};
        const double off = (double)p.de_offset;
        R cr[3], orr[3];  // the centre and the offset coordinates
        if (sizeof(R) == 4) {
            // (o - cf is exact in single precision where the two are within a
            // factor of 2 of each other, i.e. wherever |c| >= the offset)
#pragma unroll
            for (int k = 0; k < 3; k++) {
                float cf = (float)c[k];
                float o = sizeof(P) == 4 ? cf + p.de_offset : (float)((double)c[k] + off);
                float h = o - cf;
                if (!(h > 0.0f)) out.need64 = true;
                corr[k] = __fdividef(p.de_offset, fmaxf(h, 1e-30f));
                cr[k] = (R)cf;
                orr[k] = (R)o;
            }
        } else {
#pragma unroll
            for (int k = 0; k < 3; k++) {
                cr[k] = (R)c[k];
                orr[k] = (R)((double)c[k] + off);
            }
        }
#pragma unroll
        for (int q = 0; q < 4; q++) {
#pragma unroll
            for (int k = 0; k < 3; k++) v[q][k] = (q == k + 1) ? orr[k] : cr[k];
            v[q][3] = R(0);
            if (p.do_julia) {
                j[q][0] = param_f<R>(p, p.ju[0], p.ju_f[0]);
                j[q][1] = param_f<R>(p, p.ju[1], p.ju_f[1]);
                j[q][2] = param_f<R>(p, p.ju[2], p.ju_f[2]);
            } else {
                j[q][0] = v[q][0]; j[q][1] = v[q][1]; j[q][2] = v[q][2];
            }
            rout[q] = v[q][0] * v[q][0] + v[q][1] * v[q][1] + v[q][2] * v[q][2];
        }
        const R rstop3d = param_f<R>(p, p.rstop3d, p.rstop3d_f);
        bool live[4] = {true, true, true, true};
        float lr_frozen[4] = {0.f, 0.f, 0.f, 0.f};
        R rold0 = 0, rold3 = 0, otrap3 = rout[3];
        int n = 0, btmp = p.slots[0].iterations, it = 0;
        unsigned int unc = 0;
        // single precision with Integer Power 8 and the Amazing Box only: the
        // orbits in two packed pairs (formulas.cuh), the same loop
        constexpr bool PACKED = sizeof(R) == 4 && (FM == FKIND_IP8 || FM == (FKIND_IP8 | FKIND_BOX));
        if constexpr (PACKED) {
            float2 V[2][3], J[2][3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                V[0][k] = make_float2((float)v[0][k], (float)v[1][k]);
                V[1][k] = make_float2((float)v[2][k], (float)v[3][k]);
                J[0][k] = make_float2((float)j[0][k], (float)j[1][k]);
                J[1][k] = make_float2((float)j[2][k], (float)j[3][k]);
            }
            // after a counted iteration: the lengths, the offset orbits' own
            // bailouts, and whether the centre stops
            auto counted = [&]() -> bool {
                it += 1;
                const float2 r01 = psq3(V[0]), r23 = psq3(V[1]);
                rout[0] = r01.x;
                const float rn[4] = {0.0f, r01.y, r23.x, r23.y};
                // (an offset orbit bails out at RStop3D = 64 RStop^4, far above
                // the centre's bailout, so it rarely stops first: one test of
                // the largest length skips the per-orbit bookkeeping, but for
                // the z offset orbit's length that the colour state keeps --
                // fmaxf drops a NaN, which never stops)
                if (!(fmaxf(rn[1], fmaxf(rn[2], rn[3])) > (float)rstop3d)) {
                    if (FULL) {  // (the colour state follows the z offset orbit)
                        otrap3 = (live[3] && rn[3] < otrap3) ? rn[3] : otrap3;
                        rout[3] = live[3] ? rn[3] : rout[3];
                    }
                    return it >= max_it || rout[0] > rstop;
                }
#pragma unroll
                for (int q = 1; q < 4; q++) {
                    const bool stop = live[q] && rn[q] > (float)rstop3d;
                    if (FULL && q == 3) otrap3 = (live[3] && rn[3] < otrap3) ? rn[3] : otrap3;
                    rout[q] = live[q] ? rn[q] : rout[q];
                    if (stop) {
                        const int pq = q >> 1;
                        float vf[4];
#pragma unroll
                        for (int k = 0; k < 3; k++) vf[k] = (q & 1) ? V[pq][k].y : V[pq][k].x;
                        vf[3] = 0.f;
                        lr_frozen[q] = log_len2_f(vf);
                    }
                    live[q] = live[q] && !stop;
                }
                return it >= max_it || rout[0] > rstop;
            };
            auto before = [&]() {
                if (FULL) {
                    rold0 = rout[0];
                    rold3 = live[3] ? rout[3] : rold3;
                }
            };
            if ((FM & FKIND_BOX) && p.sched == SCHED_BOX2_IP8) {
                // Amazing Box, Amazing Box, Integer Power 8, repeating from the
                // first iteration, all counted: the slots' order as a phase
                // counter (one body of each formula, so the loop stays small)
                const float scale = p.slots[0].of[0], min_r = p.slots[0].of[1], fold = p.slots[0].of[2];
                const float zmul = p.slots[1].of[1];
                int ph = 0;
                for (int g = 0; g < (1 << 20); g++) {
                    before();
                    if (ph < 2) {
                        f_amazing_box_x2(scale, min_r, fold, V[0], J[0]);
                        f_amazing_box_x2(scale, min_r, fold, V[1], J[1]);
                        if (COUNT) cnt->its[0] += 4;
                        n = 0;
                    } else {
                        f_int_pow8_x2(zmul, V[0], J[0]);
                        f_int_pow8_x2(zmul, V[1], J[1]);
                        if (COUNT) cnt->its[1] += 4;
                        n = 1;
                    }
                    ph = ph == 2 ? 0 : ph + 1;
                    if (counted()) break;
                }
                goto done_x2;
            }
            if (p.sched == SCHED_IP8) {
                // one Integer Power 8 slot, all iterations counted
                const float zmul = p.slots[0].of[1];
                for (int g = 0; g < (1 << 20); g++) {
                    before();
                    f_int_pow8_x2(zmul, V[0], J[0]);
                    f_int_pow8_x2(zmul, V[1], J[1]);
                    if (COUNT) cnt->its[0] += 4;
                    if (counted()) break;
                }
                goto done_x2;
            }
            for (;;) {
                before();
                int guard = 0;
                while (btmp <= 0) {
                    n += 1;
                    if (n > p.end_to) n = p.repeat_from;
                    btmp = p.slots[n].iterations;
                    if (++guard > 64) goto done_x2;
                }
                {
                    const DevSlot &s = p.slots[n];
                    if (FM == FKIND_IP8 || s.kind == FKIND_IP8) {
                        const float zmul = s.of[1];
                        f_int_pow8_x2(zmul, V[0], J[0]);
                        f_int_pow8_x2(zmul, V[1], J[1]);
                    } else if (s.kind == FKIND_BOX) {
                        const float scale = s.of[0], min_r = s.of[1], fold = s.of[2];
                        f_amazing_box_x2(scale, min_r, fold, V[0], J[0]);
                        f_amazing_box_x2(scale, min_r, fold, V[1], J[1]);
                    }
                    if (s.julia_add) {
#pragma unroll
                        for (int k = 0; k < 3; k++) {
                            V[0][k] = padd(V[0][k], J[0][k]);
                            V[1][k] = padd(V[1][k], J[1][k]);
                        }
                    }
                    if (COUNT) cnt->its[n] += 4;
                    btmp -= 1;
                    if (s.uncounted) {
                        if (++unc > 100000u) goto done_x2;
                        continue;
                    }
                }
                if (counted()) break;
            }
        done_x2:
#pragma unroll
            for (int k = 0; k < 3; k++) {
                v[0][k] = V[0][k].x;
                v[1][k] = V[0][k].y;
                v[2][k] = V[1][k].x;
                v[3][k] = V[1][k].y;
            }
        } else
        for (;;) {
            if (FULL) {
                rold0 = rout[0];
                rold3 = live[3] ? rout[3] : rold3;
            }
            int guard = 0;
            while (btmp <= 0) {
                n += 1;
                if (n > p.end_to) n = p.repeat_from;
                btmp = p.slots[n].iterations;
                if (++guard > 64) goto done_n;
            }
            {
                const DevSlot &s = p.slots[n];
                step_orbits<R, 4, FM>(s, v, j, rout);
                if (COUNT) cnt->its[n] += 4;
                btmp -= 1;
                if (s.uncounted) {
                    if (++unc > 100000u) goto done_n;
                    continue;
                }
            }
            it += 1;
            rout[0] = v[0][0] * v[0][0] + v[0][1] * v[0][1] + v[0][2] * v[0][2];
            // (a stopped offset orbit keeps its last length, by selects; in
            // single precision the log of its length is taken from the vector
            // when it stops, since the squared length may overflow there)
#pragma unroll
            for (int q = 1; q < 4; q++) {
                const R rn = v[q][0] * v[q][0] + v[q][1] * v[q][1] + v[q][2] * v[q][2];
                const bool stop = live[q] && rn > rstop3d;
                if (FULL && q == 3) otrap3 = (live[3] && rn < otrap3) ? rn : otrap3;
                rout[q] = live[q] ? rn : rout[q];
                if (sizeof(R) == 4 && stop) {
                    float vf[4] = {(float)v[q][0], (float)v[q][1], (float)v[q][2], 0.f};
                    lr_frozen[q] = log_len2_f(vf);
                }
                live[q] = live[q] && !stop;
            }
            if (it >= max_it || rout[0] > rstop) break;
            // (a stopped offset orbit keeps being iterated in the lock-step;
            // its values are no longer used)
        }
    done_n:
        if (FULL) {
            st->rout = (double)rout[0];
            st->rold = (double)rold3;
            st->otrap = (double)otrap3;
            st->v[0] = (double)v[3][0]; st->v[1] = (double)v[3][1]; st->v[2] = (double)v[3][2];
            st->smooth_it = calc_sit ? smooth_of<R>(p, rout[0], rold0, v[0], it, n) : 0.f;
        }
        if (sizeof(R) == 8) {
            double R0 = (double)rout[0];
            if (R0 < 1e-200) {
                out.de = 0.0;
            } else {
                double g0 = (R0 - (double)rout[1]) * (R0 - (double)rout[1]);
                double g1 = (R0 - (double)rout[2]) * (R0 - (double)rout[2]);
                double g2 = (R0 - (double)rout[3]) * (R0 - (double)rout[3]);
                out.de = R0 * log(R0) * (double)p.d_de_scale / (sqrt(g0 + g1 + g2) + (double)p.de_offset006);
            }
        } else {
            float m0 = fmaxf(fabsf((float)v[0][0]), fmaxf(fabsf((float)v[0][1]), fabsf((float)v[0][2])));
            if (!(m0 > 0.0f)) {
                out.de = 0.0;
            } else {
                float sc = m0 > 1e15f ? __frcp_rn(m0) : 1.0f;
                float c0 = (float)v[0][0] * sc, c1 = (float)v[0][1] * sc, c2 = (float)v[0][2] * sc;
                float Rs = c0 * c0 + c1 * c1 + c2 * c2;
                float lr = __logf(Rs) - 2.0f * __logf(sc);
                float inv = __frcp_rn(Rs);
                float g = 0.0f;
#pragma unroll
                for (int q = 1; q < 4; q++) {
                    float d;
                    if (live[q]) {
                        float a0 = ((float)v[0][0] - (float)v[q][0]) * sc, b0 = ((float)v[0][0] + (float)v[q][0]) * sc;
                        float a1 = ((float)v[0][1] - (float)v[q][1]) * sc, b1 = ((float)v[0][1] + (float)v[q][1]) * sc;
                        float a2 = ((float)v[0][2] - (float)v[q][2]) * sc, b2 = ((float)v[0][2] + (float)v[q][2]) * sc;
                        d = (a0 * b0 + a1 * b1 + a2 * b2) * inv;
                    } else {
                        d = 1.0f - __expf(lr_frozen[q] - lr);
                    }
                    d *= corr[q - 1];
                    g += d * d;
                }
                out.de = (double)__fdividef(lr * p.d_de_scale, fsqrt_fast(g) + p.de_offset006 * __expf(-lr));
            }
        }
        out.it = it;
    }
    // (single precision that overflowed, e.g. a vanishing gradient sum with
    // exp(-ln R) underflowing: the double precision DE decides)
    if (sizeof(R) == 4 && !isfinite(out.de)) out.need64 = out.overflow = true;
    double mn = (double)ms_de_stop * 0.25;
    if (out.de < mn || isnan(out.de)) out.de = mn;
    return out;
}

}  // namespace mb3dcu
