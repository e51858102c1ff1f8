// The kernels of the ray march and its post passes (sm_100a), templated on
// the formula set FM (FKIND_* bits) they are built for; one compilation unit
// per set (kern_*.cu) instantiates Launch<FM>.
//
//  k_march       the march as a persistent wavefront (double precision: the
//                plain FP64 drop-in; single precision: the bulk march).
//  k_finish      the double precision finish of every ray the march handed
//                over: the rest of the reference's loop, the binary search,
//                normals, colour and depth.
//  k_surface     the post passes' bookkeeping on every pixel (shadow bits
//                cleared, DE AO zeroed) and the list of surface pixels.
//  k_post_start  per surface pixel: the surface found again from the stored
//                depth, once for the shadow pass (8 binary search steps) and
//                once for the DE AO (5 steps); a persistent wavefront.
//  k_shadow_rays one lane per (surface pixel, light) ray, persistent, refill.
//  k_ao_rays     one lane per (surface pixel, AO direction) ray, likewise.
//  k_ao_final    per surface pixel: the AO rays' correction and mean.
//  k_de_probe    the DE at given points.
//
// Every loop carries an iteration cap (the reference's guards).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include "devparams.h"
#include "marcher64.cuh"
#include "delock.cuh"
#include "kernels.h"

// resident blocks of 256 threads the wavefront kernels are compiled for
#ifndef MB3D_MIN_BLOCKS
#define MB3D_MIN_BLOCKS 3
#endif
#ifndef MB3D_MIN_BLOCKS_MARCH
#define MB3D_MIN_BLOCKS_MARCH MB3D_MIN_BLOCKS
#endif
// (the single precision march: 4 blocks of 64 registers, its spills cost
// less than the warps it gains)
#ifndef MB3D_MIN_BLOCKS_FINISH
#define MB3D_MIN_BLOCKS_FINISH MB3D_MIN_BLOCKS
#endif
#ifndef MB3D_MIN_BLOCKS_POST
#define MB3D_MIN_BLOCKS_POST MB3D_MIN_BLOCKS
#endif
#ifndef MB3D_MIN_BLOCKS_AO32
#define MB3D_MIN_BLOCKS_AO32 4
#endif
#ifndef MB3D_MIN_BLOCKS_MARCH32
#define MB3D_MIN_BLOCKS_MARCH32 4
#endif

namespace mb3dcu {

__device__ __forceinline__ int32_t pixel_seed_d(int64_t y, int64_t x) {  // src/calc.rs:1125-1140
    uint32_t row = (uint32_t)(int32_t)((int64_t)0x24563487u + (y + 1) * (int64_t)0x324594A1);
    uint32_t a = 214013u, c = 2531011u, ra = 1u, rc = 0u;
    uint64_t n = x > 0 ? (uint64_t)x : 0;
    while (n > 0) {
        if (n & 1) {
            rc = rc * a + c;
            ra = ra * a;
        }
        c = c * a + c;
        a = a * a;
        n >>= 1;
    }
    return (int32_t)(ra * row + rc);
}

// the warp's lanes that want to append write their item at consecutive
// places: one atomicAdd per warp, ranks from the ballot
template <typename T>
__device__ __forceinline__ void warp_append(bool want, unsigned int *count, const T &h, T *list) {
    unsigned int mask = __ballot_sync(0xffffffffu, want);
    if (mask == 0) return;
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    unsigned int base = 0;
    if (lane == leader) base = atomicAdd(count, (unsigned int)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (want) list[base + __popc(mask & ((1u << lane) - 1u))] = h;
}

// refill: the idle lanes of the warp take the next items of the queue
// (when at least `min_idle` are idle, or all are); returns the lane's item
// or UINT32_MAX; `open` turns false once the queue is drained
__device__ __forceinline__ uint32_t warp_take(bool idle_lane, unsigned int *queue, uint32_t n_items, int min_idle,
                                              bool &open) {
    unsigned int idle = __ballot_sync(0xffffffffu, idle_lane);
    if (!open || !(__popc(idle) >= min_idle || idle == 0xffffffffu)) return UINT32_MAX;
    int lane = threadIdx.x & 31;
    int leader = __ffs(idle) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(queue, (unsigned int)__popc(idle));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (base + (uint32_t)__popc(idle) >= n_items) open = false;
    if (!idle_lane) return UINT32_MAX;
    uint32_t item = base + (uint32_t)__popc(idle & ((1u << lane) - 1u));
    return item < n_items ? item : UINT32_MAX;
}

// The call's device time budget: true once p.budget_ns nanoseconds have
// passed since the call's first take (the first warp to ask stamps it);
// sets `bit` in the status word.  Asked by one lane before a take, so a
// warp that stops has finished every ray it took.
__device__ __forceinline__ bool budget_spent(const DevParams &p, unsigned int *counters, unsigned int bit) {
    if (p.budget_ns == 0) return false;
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    unsigned long long *t0p = reinterpret_cast<unsigned long long *>(counters + CNT_T0);
    unsigned long long t0 = atomicCAS(t0p, 0ull, now);
    if (t0 == 0ull) t0 = now;
    if (now - t0 <= p.budget_ns) return false;
    atomicOr(counters + CNT_STATUS, bit);
    return true;
}

// warp_take under the budget: no new items once it is spent (the queue's
// counter then says how far the call got; a later launch goes on from there)
__device__ __forceinline__ uint32_t warp_take_b(const DevParams &p, bool idle_lane, unsigned int *counters, int queue,
                                                uint32_t n_items, int min_idle, bool &open, unsigned int bit) {
    if (p.budget_ns != 0 && open) {
        unsigned int idle = __ballot_sync(0xffffffffu, idle_lane);
        if (__popc(idle) >= min_idle || idle == 0xffffffffu) {
            int spent = 0;
            if ((threadIdx.x & 31) == 0) spent = budget_spent(p, counters, bit) ? 1 : 0;
            if (__shfl_sync(0xffffffffu, spent, 0)) open = false;
        }
    }
    return warp_take(idle_lane, &counters[queue], n_items, min_idle, open);
}

__device__ __forceinline__ void item_pixel(uint32_t item, int tiles_x, int &x, int &ly) {
    uint32_t t = item >> 5, l = item & 31u;
    x = (int)(t % (uint32_t)tiles_x) * 8 + (int)(l & 7u);
    ly = (int)(t / (uint32_t)tiles_x) * 4 + (int)(l >> 3);
}

__device__ __forceinline__ float de_stop_at(const DevParams &p, double zz) {
    return (float)((double)p.de_stop * (1.0 + zz * (double)p.de_stop_factor));
}
// (the same in single precision, for the mixed march's predicting steps)
__device__ __forceinline__ float de_stop_at_f(const DevParams &p, double zz) {
    return p.de_stop * fmaf((float)zz, p.de_stop_factor, 1.0f);
}

// ---------------------------------------------------------------------------
// The march as a persistent wavefront: every lane of a warp holds one ray;
// each trip of the loop evaluates one DE for every lane that has a ray (the
// reference loop's two DE sites, a step and the half step back, are states
// of a small per-lane machine), and lanes whose ray ended take new pixels
// as soon as `refill_min` lanes of the warp are idle.  Queue items are
// numbered by 8 x 4 tiles, so that the rays of a refill are neighbours.
// R = double: the plain FP64 march (exactly the reference's loop); its
// surfaces are handed to the finish where they were found.  R = float: the
// single precision bulk march; a surface is handed over from the last point
// where the DE was still >= hand_margin x the DE stop (at most hand_back
// steps back) and the finish marches on from there in double precision; a
// ray whose single precision DE cannot decide (need64) is handed over from
// where it is, and only one that needs double precision at the start plane
// is marched whole by the per-thread finish.

#define PH_IDLE 0
#define PH_START 1
#define PH_STEP 2
#define PH_HALF 3

template <typename R, int FM, bool COUNT>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? MB3D_MIN_BLOCKS_MARCH32 : MB3D_MIN_BLOCKS_MARCH) k_march(const __grid_constant__ DevParams p, int row0, int rows,
                                               mb3d_cu_silight *out, Hand *list, unsigned int *counters,
                                               unsigned long long *gcount) {
    constexpr bool MIXED = sizeof(R) == 4;
    // the step logic's type: single precision in the mixed march (its
    // steps only predict; the FP64 finish decides), double in the plain
    // march (the reference's arithmetic); mzz is double in both
    typedef R T;
    DECount cnt;
    if (COUNT) cnt.clear();
    const int tiles_x = (p.width + 7) / 8;
    const uint32_t n_items = (uint32_t)tiles_x * (uint32_t)((rows + 3) / 4) * 32u;
    int phase = PH_IDLE;
    bool open = true;
    uint32_t pix = 0;
    int x = 0, ly = 0;
    double c[3] = {0, 0, 0}, vf[3] = {0, 0, 0};
    // (the single precision march keeps its start point and direction in
    // single precision and its position as start + direction x mzz)
    float cf0[3] = {0.f, 0.f, 0.f}, vff[3] = {0.f, 0.f, 0.f};
    double mzz = 0.0;
    T last_step = 0, last_de = 0;
    float ms = 0.f, rsf = 1.f, step_count = 0.f;
    int32_t seed = 0;
    bool first = false;
    // the mixed march's last two states before a step (where a surface is
    // handed over from), a ring of two slots per thread in shared memory
    // (hs: the slot of the newest); registers stay free for the DE
    __shared__ double h_mzz[2][256];
    __shared__ float h_ls[2][256], h_ld[2][256], h_cnt[2][256];
    const int tid = (int)threadIdx.x;
    int hs = 0;
    int nb = 0;
    unsigned int trip = 0;
    for (; trip < MB3D_TRIP_CAP; trip++) {
        uint32_t item = warp_take_b(p, phase == PH_IDLE, counters, CNT_MARCH_Q, n_items, p.refill_min, open, 1u);
        if (item != UINT32_MAX) {
            item_pixel(item, tiles_x, x, ly);
            if (x < p.width && ly < rows) {
                pix = (uint32_t)ly * (uint32_t)p.width + (uint32_t)x;
                pixel_ray(p, x, row0 + ly, c, vf);
                seed = pixel_seed_d(row0 + ly, x);
                if constexpr (MIXED) {
#pragma unroll
                    for (int k = 0; k < 3; k++) {
                        cf0[k] = (float)c[k];
                        vff[k] = (float)vf[k];
                    }
                }
                mzz = 0.0;
                ms = p.de_stop;
                phase = PH_START;
            }
        }
        unsigned int busy = __ballot_sync(0xffffffffu, phase != PH_IDLE);
        if (busy == 0) {
            if (!open) break;
            continue;
        }
        bool hand = false, full = false, done_bg = false, resume = false, overflowed = false;
        T cur_de = 0;
        int cur_it = 0;
        if (phase != PH_IDLE) {
            DEr r;
            if constexpr (MIXED) {
                const float t = (float)mzz;
                const float cp[3] = {fmaf(vff[0], t, cf0[0]), fmaf(vff[1], t, cf0[1]), fmaf(vff[2], t, cf0[2])};
                r = de_lock<R, FM, COUNT, false, float>(p, cp, ms, &cnt);
            } else {
                r = de_lock<R, FM, COUNT>(p, c, ms, &cnt);
            }
            cur_it = r.it;
            T dtmp = (T)r.de;
            int it = r.it;
            const int itc = its_cap<FM>(p, r);
            bool skip_half = false, decide = true;
            if (MIXED && r.need64) {
                overflowed = r.overflow;
                hand = true;
                full = phase == PH_START;
                resume = !full;
                decide = false;
            } else if (phase == PH_START) {
                if (it >= itc || dtmp < (T)ms) {
                    hand = true;  // inside the set at the start plane
                    full = true;
                    decide = false;
                } else {
                    last_step = dtmp * (T)p.z_step_div;
                    rsf = 1.0f;
                    first = p.first_step_random != 0;
                    step_count = 0.f;
                    nb = -1;
                }
            } else if (phase == PH_STEP) {
                if (dtmp > last_de + last_step) dtmp = last_de + last_step;
                if (last_de > dtmp + (T)1e-30) {
                    if constexpr (MIXED) {
                        const float t = __fdividef(last_step, last_de - dtmp);
                        rsf = t < 1.0f ? fmaxf(0.5f, t) : 1.0f;
                    } else {
                        const double t = last_step / (last_de - dtmp);
                        rsf = t < 1.0 ? (float)fmax(0.5, t) : 1.0f;
                    }
                } else {
                    rsf = 1.0f;
                }
            } else {  // PH_HALF: the DE after the half step back
                skip_half = true;
            }
            if (decide) {
                if (!skip_half && it >= itc) {
                    // src/calc.rs:2544-2551: half a step back
                    const T dt1 = (T)-0.5 * last_step;
                    mzz += (double)dt1;
                    if (!MIXED) add_w(c, vf, (double)dt1);
                    ms = MIXED ? de_stop_at_f(p, mzz) : de_stop_at(p, mzz);
                    last_step = -dt1;
                    phase = PH_HALF;
                } else if (it < p.min_it || (it < itc && dtmp >= (T)ms)) {
                    if (MIXED) {
                        if (dtmp >= (T)p.hand_margin * (T)ms && !first) nb = 0;
                        else if (nb >= 0 && nb < p.hand_back) nb++;
                        hs ^= 1;
                        h_mzz[hs][tid] = mzz;
                        h_ls[hs][tid] = (float)last_step;
                        h_ld[hs][tid] = (float)last_de;
                        h_cnt[hs][tid] = step_count;
                    }
                    last_de = dtmp;
                    T d = fmax((T)0.11, (dtmp - (T)p.ms_de_sub * (T)ms) * (T)p.z_step_div * (T)rsf);
                    const T s1 = (T)(fmaxf(ms, 0.4f) * p.mh04zsd);
                    bool count = p.dfog_on_it == 0 || it == p.dfog_on_it;
                    if (s1 < d) {
                        if (count) step_count += MIXED ? __fdividef((float)s1, (float)d) : (float)(s1 / d);
                        d = s1;
                    } else if (count) {
                        step_count += 1.0f;
                    }
                    if (first) {
                        first = false;
                        seed = (int32_t)((uint32_t)seed * 214013u + 2531011u);
                        d *= (T)((double)(seed & 0x7FFFFFFF) * (1.0 / 2147483647.0));
                    }
                    mzz += (double)d;
                    if (mzz > p.zend) {
                        done_bg = true;  // background
                    } else {
                        last_step = d;
                        if (!MIXED) add_w(c, vf, (double)d);
                        ms = MIXED ? de_stop_at_f(p, mzz) : de_stop_at(p, mzz);
                        phase = PH_STEP;
                    }
                } else {
                    hand = true;  // a surface
                }
            }
            cur_de = dtmp;
        }
        if (COUNT) {
            const int itl = cur_it;  // (0: no DE this trip)
            const int mx = __reduce_max_sync(0xffffffffu, itl);
            cnt.lanes[0] += (unsigned long long)itl;
            if ((threadIdx.x & 31) == 0) {
                cnt.lanes[1] += (unsigned long long)mx;
                cnt.lanes[2] += 1;
                cnt.lanes[3] += (unsigned long long)__popc(busy);
            }
        }
        Hand h;
        if (hand) {
            h.pix = pix;
            h.seed = seed;
            h.rsf = rsf;
            h.flags = full ? HAND_FULL : 0u;
            if (!full) {
                if (!MIXED) {
                    h.mzz = mzz;
                    h.last_step = last_step;
                    h.last_de = last_de;
                    h.dtmp = cur_de;
                    h.it = cur_it;
                    h.step_count = step_count;
                    h.c[0] = c[0]; h.c[1] = c[1]; h.c[2] = c[2];
                } else if (resume) {
                    h.flags = HAND_REMARCH | (phase == PH_HALF ? HAND_HALF : 0u);
                    h.mzz = mzz;
                    h.last_step = last_step;
                    h.last_de = last_de;
                    h.step_count = step_count;
                } else if (nb < 0) {
                    h.flags = HAND_FULL;  // no state to go back to: all in double
                } else {
                    const int slot = nb >= 1 ? hs ^ 1 : hs;
                    h.flags = HAND_REMARCH;
                    h.mzz = h_mzz[slot][tid];
                    h.last_step = h_ls[slot][tid];
                    h.last_de = h_ld[slot][tid];
                    h.step_count = h_cnt[slot][tid];
                }
            }
            phase = PH_IDLE;
        } else if (done_bg) {
            G si;
            si.clear();
            si.amb_shadow = 5000;
            si.shadow = (uint16_t)rintf(fminf(fmaxf(step_count, 0.0f), 1023.0f));
            si.store(out + pix);
            phase = PH_IDLE;
        }
        warp_append(hand, &counters[CNT_HAND], h, list);
        if (MIXED) {
            // (a ray hands over once: this counts pixels)
            const unsigned int ov = __ballot_sync(0xffffffffu, overflowed);
            if (ov && (threadIdx.x & 31) == __ffs(ov) - 1) atomicAdd(&counters[CNT_OVERFLOW], (unsigned int)__popc(ov));
        }
    }
    // (a warp that ran out of trips left rays unmarched: the host fails the call)
    if (trip >= MB3D_TRIP_CAP && (threadIdx.x & 31) == 0) atomicOr(counters + CNT_STATUS, ST_TRIP_CAP);
    if (COUNT) cnt.flush(gcount);
}

// The finish of the rare rays (slow list): the FP64 marcher per thread --
// a pixel inside the set at the start plane, a surface whose binary search
// is on the iteration count (RMdoBinSearchIt), the smoothed normals, normals
// on the smooth iterations, colour on an iteration.
// Its items are taken one per thread from a queue (CNT_SLOW_Q), so that a
// launch stopped by the budget has finished exactly the items before the
// queue's counter.
template <int FM>
__global__ void __launch_bounds__(128) k_finish_slow(const __grid_constant__ DevParams p, int row0, const Hand *list,
                                                     unsigned int *counters, mb3d_cu_silight *out) {
    const unsigned int n = counters[CNT_SLOW];
    for (int guard = 0; guard < (1 << 30); guard++) {
        if (p.budget_ns != 0 && budget_spent(p, counters, 4u)) break;
        const unsigned int i = atomicAdd(&counters[CNT_SLOW_Q], 1u);
        if (i >= n) break;
        Hand h = list[i];
        int x = (int)(h.pix % (uint32_t)p.width);
        int y = row0 + (int)(h.pix / (uint32_t)p.width);
        M64<FM> m(p);
        G si;
        if (h.flags & HAND_FULL) {
            m.seed = pixel_seed_d(y, x);
            m.march_pixel(si, x, y);
        } else {
            si.clear();
            si.amb_shadow = 5000;
            double c0[3];
            pixel_ray(p, x, y, c0, m.vfov);
            m.mzz = h.mzz;
            m.update_de_stop();
            m.it.calc_sit = false;
            m.seed = h.seed;
            if (h.flags & HAND_REMARCH) {
                for (int k = 0; k < 3; k++) m.it.c[k] = c0[k] + m.vfov[k] * h.mzz;
                double dtmp = m.calc_de();
                const bool half = (h.flags & HAND_HALF) != 0;
                float rsf = half ? h.rsf : 1.0f;
                if (h.mzz > 0.0 && !half) {
                    if (dtmp > h.last_de + h.last_step) dtmp = h.last_de + h.last_step;
                    if (h.last_de > dtmp + 1e-30) {
                        double t = h.last_step / (h.last_de - dtmp);
                        rsf = t < 1.0 ? (float)fmax(0.5, t) : 1.0f;
                    }
                }
                m.march_from(si, dtmp, h.last_step, rsf, false, h.step_count, half);
            } else {
                // a surface, exactly where it was found
                m.it.c[0] = h.c[0]; m.it.c[1] = h.c[1]; m.it.c[2] = h.c[2];
                m.calc_de();
                m.surface_found(si, h.dtmp, h.last_step);
                si.shadow = (uint16_t)rintf(fminf(fmaxf(h.step_count, 0.0f), 1023.0f));
            }
        }
        si.store(out + h.pix);
    }
}

// The finish of every handed-over ray as a wavefront, in double precision:
// the rest of the reference's loop from the hand-over state
// (src/calc.rs:2539-2640), RMdoBinSearch (:1706-1734) on a DE-limited
// surface, RMdoBinSearchIt (:1737-1791) on one the iteration count limits,
// RMCalculateNormals (:1813-1906, unsmoothed), the colour and the depth
// (:2496-2507).  One DE per trip; the rare cases (a ray marched whole, the
// smoothed normals, normals on the iteration count, colour on an iteration)
// go to the slow list.
#define F_IDLE 0
#define F_REMARCH 1
#define F_STEP 2
#define F_HALF 3
#define F_BISECT 4
#define F_NC 5
#define F_NSP 6
#define F_NSM 7
#define F_BSI1 8  // RMdoBinSearchIt: the DE at the stepped position
#define F_BSI2 9  // ... and 0.001 behind it

template <int FM>
__global__ void __launch_bounds__(256, MB3D_MIN_BLOCKS_FINISH) k_finish(const __grid_constant__ DevParams p, int row0, const Hand *list,
                                                unsigned int *counters, Hand *slow, mb3d_cu_silight *out) {
    const uint32_t n_items = counters[0];
    // RMdoBinSearchIt's target count and its limit (the search iterates once more)
    const float bsi_yp = (float)p.max_it - 0.99f, bsi_top = (float)(p.max_it + 1) - 0.1f;
    int phase = F_IDLE;
    bool open = true;
    uint32_t pix = 0;
    double c[3] = {0, 0, 0}, vf[3] = {0, 0, 0}, ct[3] = {0, 0, 0}, nrm[3] = {0, 0, 0};
    double mzz = 0, last_step = 0, last_de = 0, dt1 = 0, noffset = 0, a_plus = 0, dtmp = 0, dmul = 1.0;
    float ms = 0.f, rsf = 1.f, step_count = 0.f, nn = 0.f, b_last_si = 0.f, b_last_dif = 0.f;
    int itmp = 0, k_ax = 0;
    bool it_limited = false, b_first = false;
    unsigned int guard = 0;
    unsigned int trip = 0;
    for (; trip < MB3D_TRIP_CAP; trip++) {
        uint32_t item = warp_take_b(p, phase == F_IDLE, counters, CNT_FINISH_Q, n_items, p.refill_min, open, 2u);
        bool to_slow = false;
        Hand hs;
        int entry = 0;  // 2: a surface already evaluated (the plain march)
        int it_in = 0;
        if (item != UINT32_MAX) {
            Hand h = list[item];
            if ((h.flags & HAND_FULL) || p.finish_slow) {
                to_slow = true;
                hs = h;
            } else {
                pix = h.pix;
                int x = (int)(pix % (uint32_t)p.width), y = row0 + (int)(pix / (uint32_t)p.width);
                double c0[3];
                pixel_ray(p, x, y, c0, vf);
                mzz = h.mzz;
                ms = de_stop_at(p, mzz);
                step_count = h.step_count;
                last_step = h.last_step;
                last_de = h.last_de;
                rsf = 1.0f;
                guard = 0;
                it_limited = false;
                if (h.flags & HAND_REMARCH) {
                    for (int k = 0; k < 3; k++) c[k] = c0[k] + vf[k] * mzz;
                    if (h.flags & HAND_HALF) {
                        rsf = h.rsf;
                        phase = F_HALF;
                    } else {
                        phase = F_REMARCH;
                    }
                } else {
                    c[0] = h.c[0]; c[1] = h.c[1]; c[2] = h.c[2];
                    dtmp = h.dtmp;
                    it_in = h.it;
                    entry = 2;
                    phase = F_STEP;  // (handled below without a DE)
                }
            }
        }
        if (item != UINT32_MAX && to_slow) phase = F_IDLE;
        // ---- one DE for the lanes whose phase asks for one (the iteration
        // count search: with the smoothed count and one more iteration)
        DEr r;
        r.de = 0.0;
        r.it = 0;
        r.max_its = p.max_it;
        r.need64 = false;
        DEstate st;
        st.rout = st.rold = st.otrap = 0.0;
        st.v[0] = st.v[1] = st.v[2] = 0.0;
        st.smooth_it = 0.f;
        if (phase != F_IDLE && entry != 2) {
            const bool bsi = phase >= F_BSI1;
            r = de_lock<double, FM, false, true>(p, c, ms, nullptr, &st, phase == F_NC || bsi, bsi ? 1 : 0);
        }
        if (entry == 2) {
            r.de = dtmp;
            r.it = it_in;
        }
        // ---- the per-lane machine
        bool done_bg = false, done_surf = false;
        if (phase != F_IDLE) {
            // 1: decide the march step, 2: the surface, 3: bisection loop,
            // 5: iteration count search loop, 4: normals begin
            int go = 0;
            bool skip_half = false;
            if (++guard > 4000000u) {
                done_bg = true;  // (a cap the reference's guards never reach)
            } else if (entry == 2) {
                dtmp = r.de;
                go = 2;
            } else if (phase == F_REMARCH || phase == F_STEP) {
                dtmp = r.de;
                if (phase == F_STEP || mzz > 0.0) {
                    if (dtmp > last_de + last_step) dtmp = last_de + last_step;
                    if (last_de > dtmp + 1e-30) {
                        double t = last_step / (last_de - dtmp);
                        rsf = t < 1.0 ? (float)fmax(0.5, t) : 1.0f;
                    } else {
                        rsf = 1.0f;
                    }
                }
                go = 1;
            } else if (phase == F_HALF) {
                dtmp = r.de;
                skip_half = true;
                go = 1;
            } else if (phase == F_BISECT) {
                dtmp = r.de;
                if (r.it >= its_cap<FM>(p, r)) dt1 = -fabs(dt1);
                else dt1 = (dtmp - (double)ms) < 0.0 ? fabs(dt1) * -0.55 : fabs(dt1) * 0.55;
                go = 3;
            } else if (phase == F_BSI1) {
                float si_now = st.smooth_it;
                if (!b_first && b_last_dif < fabsf(bsi_yp - si_now)) {
                    // worse than the last position: back there, smaller steps
                    mzz -= dt1;
                    add_w(c, vf, -dt1);
                    si_now = b_last_si;
                    dmul *= dt1 > 0.0 ? 0.5 : 0.7;
                }
                b_last_dif = fabsf(bsi_yp - si_now);
                b_last_si = si_now;
                if (si_now > bsi_top) {
                    dt1 = -3.0;
                    go = 5;
                } else {
                    mzz -= 0.001;
                    add_w(c, vf, -0.001);
                    phase = F_BSI2;
                }
            } else if (phase == F_BSI2) {
                float s2 = st.smooth_it;
                float rr = b_last_si - s2;
                if (fabsf(rr) < 1e-30f) dt1 = (b_last_si < s2 ? 1.0 : 0.0) - 0.5;
                else if (rr < 0.0f) dt1 = (double)__fdiv_rn(bsi_yp - s2, rr * 500.0f);
                else dt1 = (double)__fdiv_rn(bsi_yp - s2, rr * 1000.0f);
                if (dt1 > 4.0) dt1 = sqrt(dt1) * 2.0;
                else if (dt1 < -9.0) dt1 = sqrt(-dt1) * -3.0;
                dt1 = dt1 * dmul + 0.0005;
                go = 5;
            } else if (phase == F_NC) {
                nn = st.smooth_it;
                k_ax = 0;
                for (int k = 0; k < 3; k++) c[k] = ct[k] + p.vgrads[2][k] * noffset;
                phase = F_NSP;
            } else if (phase == F_NSP) {
                a_plus = r.de;
                int ax = k_ax == 0 ? 2 : k_ax - 1;
                add_w(c, p.vgrads[ax], -2.0 * noffset);
                phase = F_NSM;
            } else if (phase == F_NSM) {
                int ax = k_ax == 0 ? 2 : k_ax - 1;
                nrm[ax] = (a_plus - r.de) * 0.5;
                k_ax++;
                if (k_ax < 3) {
                    int nx = k_ax - 1;
                    for (int k = 0; k < 3; k++) c[k] = ct[k] + p.vgrads[nx][k] * noffset;
                    phase = F_NSP;
                } else {
                    done_surf = true;
                }
            }
            if (go == 1) {
                if (!skip_half && r.it >= its_cap<FM>(p, r)) {
                    double h1 = -0.5 * last_step;
                    mzz += h1;
                    add_w(c, vf, h1);
                    ms = de_stop_at(p, mzz);
                    last_step = -h1;
                    phase = F_HALF;
                } else if (r.it < p.min_it || (r.it < its_cap<FM>(p, r) && dtmp >= (double)ms)) {
                    last_de = dtmp;
                    double d = fmax(0.11, (dtmp - (double)p.ms_de_sub * (double)ms) * (double)p.z_step_div * (double)rsf);
                    double s1 = (double)(fmaxf(ms, 0.4f) * p.mh04zsd);
                    bool count = p.dfog_on_it == 0 || r.it == p.dfog_on_it;
                    if (s1 < d) {
                        if (count) step_count += (float)(s1 / d);
                        d = s1;
                    } else if (count) {
                        step_count += 1.0f;
                    }
                    mzz += d;
                    if (mzz > p.zend) {
                        done_bg = true;
                    } else {
                        last_step = d;
                        add_w(c, vf, d);
                        ms = de_stop_at(p, mzz);
                        phase = F_STEP;
                    }
                } else {
                    go = 2;
                }
            }
            if (go == 2) {
                // surface_found: the binary search on the DE or on the
                // iteration count, then the normals
                it_limited = !(r.it < its_cap<FM>(p, r) || dtmp < (double)ms);
                if (p.de_add_steps == 0) {
                    go = 4;
                } else if (it_limited) {
                    itmp = p.de_add_steps;
                    dt1 = 0.0;
                    dmul = 1.0;
                    b_first = true;
                    add_w(c, vf, 0.0);  // (the search's first step is 0)
                    phase = F_BSI1;
                } else {
                    itmp = p.de_add_steps;
                    dt1 = last_step * -0.5;
                    go = 3;
                }
            }
            if (go == 3) {
                if (fabs(dtmp - (double)ms) <= 0.001) {
                    go = 4;
                } else {
                    mzz += dt1;
                    add_w(c, vf, dt1);
                    ms = de_stop_at(p, mzz);
                    if (--itmp <= 0) go = 4;
                    else phase = F_BISECT;
                }
            }
            if (go == 5) {
                b_first = false;
                if (--itmp < 0) {
                    go = 4;
                } else {
                    mzz += dt1;
                    add_w(c, vf, dt1);
                    phase = F_BSI1;
                }
            }
            if (go == 4) {
                noffset = (double)fminf(p.de_stop, 1.0f) * (1.0 + mzz * (double)p.de_stop_factor) * 0.15;
                ct[0] = c[0]; ct[1] = c[1]; ct[2] = c[2];
                phase = F_NC;
            }
        }
        if (done_bg || done_surf) {
            G si;
            si.clear();
            si.amb_shadow = 5000;
            if (done_surf) {
                M64<FM>::store_normal(si, nrm);
                float v;
                if (it_limited) {
                    v = 32767.0f - nn * p.mcts_m;
                } else {
                    float l = (float)log((double)fmaxf(p.de_stop, ms) * p.step_width);
                    v = 32767.0f - (nn + p.d_col_plus + p.col_var * l) * p.mcts_m;
                }
                si.si_gradient = clip15(v);
                // RMdoColor with the last DE's state, at the surface point
                const double PI = 3.14159265358979323846;
                double xv = st.v[0], yv = st.v[1], zv = st.v[2], s;
                switch (p.color_option) {
                    case 1: s = log(st.rout / (st.rold + 1.0)) * (double)p.mct_color_mul; break;
                    case 2: s = (atan2(yv - ct[1], xv - ct[0]) + PI) * 5200.0; break;
                    case 3: s = (atan2(zv - ct[2], xv - ct[0]) + PI) * 5200.0; break;
                    case 4: s = (atan2(zv - ct[2], yv - ct[1]) + PI) * 5200.0; break;
                    case 5: {
                        s = (atan2(xv, yv) + PI) * 5215.0;
                        double rr = sqrt(xv * xv + yv * yv + 1e-100 + zv * zv);
                        si.si_gradient = clip15((float)((PI + asin(clampd(zv / rr, -1.0, 1.0)) * 2.0) * 5215.0));
                        break;
                    }
                    default: s = st.otrap * 4096.0; break;
                }
                si.otrap = clip15((float)s);
                // CalcZposAndRough (no roughness without smoothed normals)
                double zz = fmax(mzz, 0.0);
                long long zv2 = sat_i64d(rint(p.zc_mul * (sqrt(zz * p.zcorr + 1.0) - 1.0)));
                long long dz = 8388352LL - zv2;
                if (dz < 0) dz = 0;
                if (dz > 8388352) dz = 8388352;
                si.zpos_fine = (unsigned int)dz << 8;
            }
            si.shadow = (uint16_t)rintf(fminf(fmaxf(step_count, 0.0f), 1023.0f));
            si.store(out + pix);
            phase = F_IDLE;
        }
        warp_append(to_slow, &counters[2], hs, slow);
        unsigned int busy = __ballot_sync(0xffffffffu, phase != F_IDLE);
        if (busy == 0 && !open) break;
    }
    if (trip >= MB3D_TRIP_CAP && (threadIdx.x & 31) == 0) atomicOr(counters + CNT_STATUS, ST_TRIP_CAP);
}

// ---------------------------------------------------------------------------
// post passes

__device__ __forceinline__ double dot_normalize_d(const double a[3], const double b[3]) {
    return dot3d(a, b) / fmax(sqrt(dot3d(a, a) * dot3d(b, b)), 1e-300);
}

#ifdef MB3D_COMMON_KERNELS
// the per-pixel part of the post passes on every pixel, and the list of the
// surface pixels (src/calc.rs:2786-2797, 2909-2915; src/deao.rs:277-281)
__global__ void k_surface(const __grid_constant__ DevParams p, int npix, int passes, mb3d_cu_silight *gbuf,
                          uint32_t *list, unsigned int *count) {
    uint16_t clear_mask = 0;
    for (int l = 0; l < p.n_lights; l++) clear_mask |= (uint16_t)(0x400 << p.light_idx[l]);
    int n_round = (npix + 31) & ~31;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_round; i += gridDim.x * blockDim.x) {
        bool surf = false;
        if (i < npix) {
            uint32_t *w = reinterpret_cast<uint32_t *>(gbuf + i);
            uint32_t zf = w[2], sh = w[3], sg = w[4] & 0xFFFFu;
            surf = (zf >> 16) < 32768u && sg < 32768u;
            uint32_t shadow = sh & 0xFFFFu, amb = sh >> 16;
            if ((passes & MB3D_CU_POST_SHADOW) && p.n_lights > 0) {
                if (p.shadow_soft) shadow |= 0xFC00u;
                else shadow &= ~(uint32_t)clear_mask;
            }
            if ((passes & MB3D_CU_POST_DEAO) && p.ao_rays > 0) amb = 0;
            w[3] = (shadow & 0xFFFFu) | (amb << 16);
        }
        warp_append(surf, count, (uint32_t)i, list);
    }
}
#endif


// The post passes' start points as a wavefront: per surface pixel, the
// surface found again from the stored depth -- hs_surface_start
// (src/calc.rs:2741-2764: RMdoBinSearch with 8 steps, or RMdoBinSearchIt
// where the iteration count limits the surface) for the shadow pass, then
// surface_point (src/calc.rs:2157-2191: a 5-step search to 0.004, or
// RMdoBinSearchIt) for the DE AO.  One DE per lane and trip; a lane whose
// item is done takes the next surface pixel.  MIXED: a search limited by the
// DE runs in single precision first; where single precision cannot decide
// (need64, or the iteration count limits the surface) the task starts over
// from the stored depth in double precision, as the plain march does it.
#define Q_IDLE 0
#define Q_D0 1    // the DE at the stored depth
#define Q_BIS 2   // RMdoBinSearch (the shadow start)
#define Q_LIM 3   // the DE AO start's short search
#define Q_BSI1 4  // RMdoBinSearchIt: the DE at the stepped position
#define Q_BSI2 5  // ... and 0.001 behind it

template <int FM, bool MIXED>
__global__ void __launch_bounds__(256, MB3D_MIN_BLOCKS_POST) k_post_start(const __grid_constant__ DevParams p, int row0, int passes,
                                                    const mb3d_cu_silight *gbuf, const uint32_t *list,
                                                    const unsigned int *count, unsigned int *queue, PostStart *ps) {
    const uint32_t n_items = count[0];
    const bool do_sh = (passes & MB3D_CU_POST_SHADOW) && p.n_lights > 0;
    const bool do_ao = (passes & MB3D_CU_POST_DEAO) && p.ao_rays > 0;
    const float bsi_yp = (float)p.max_it - 0.99f, bsi_top = (float)(p.max_it + 1) - 0.1f;
    int phase = Q_IDLE;
    bool open = true;
    uint32_t idx = 0;
    double c0[3] = {0, 0, 0}, vf[3] = {0, 0, 0}, c[3] = {0, 0, 0};
    double mzz0 = 0, digit = 0, mzz = 0, dt1 = 0, dmul = 1.0, dcur = 0;
    float ms = 0.f, b_last_si = 0.f, b_last_dif = 0.f;
    int itmp = 0;
    bool ao = false, p64 = !MIXED, b_first = false;
    // (snap: the shadow task's iteration count search is the one the DE AO
    // task would run -- both from the same DE at the same stored depth, in
    // the same precision -- and the DE AO search is its first six rounds:
    // the shadow search leaves the DE AO start at its sixth round and the
    // DE AO task is not run again)
    bool snap = !MIXED, ao_done = false;
    for (unsigned int trip = 0; trip < MB3D_TRIP_CAP; trip++) {
        uint32_t item = warp_take(phase == Q_IDLE, queue, n_items, p.refill_min, open);
        bool begin = false;
        if (item != UINT32_MAX) {
            idx = item;
            uint32_t pix = list[item];
            int x = (int)(pix % (uint32_t)p.width), y = row0 + (int)(pix / (uint32_t)p.width);
            G si;
            si.load(gbuf[pix]);
            pixel_ray(p, x, y, c0, vf);
            double zf = (double)(si.zpos_fine >> 8);
            double q1 = (8388351.5 - zf) / p.zc_mul + 1.0, q2 = (8388351.9 - zf) / p.zc_mul + 1.0;
            mzz0 = (q1 * q1 - 1.0) / p.zcorr;
            digit = (q2 * q2 - 1.0) / p.zcorr - mzz0;
            uint32_t flags = 0;
            if (do_sh) {
                double nv0[3] = {si.n0 / 32767.0, si.n1 / 32767.0, si.n2 / 32767.0}, nvec[3];
                rot_rev(nv0, p.vgrads, nvec);
                for (int l = 0; l < p.n_lights; l++)
                    if (dot3d(nvec, p.light_vec[l]) > 0.0) flags |= 1u << l;
            }
            ps[idx].pix = pix;
            ps[idx].flags = flags;
            ps[idx].pad = 0;
            ao = !do_sh;
            p64 = !MIXED;
            snap = !MIXED;
            ao_done = false;
            begin = do_sh || do_ao;
        }
        // ---- a task starts (or starts over in double precision) at the stored depth
#define POST_BEGIN()                                   \
    do {                                               \
        mzz = mzz0;                                    \
        c[0] = c0[0]; c[1] = c0[1]; c[2] = c0[2];      \
        add_w(c, vf, mzz);                             \
        ms = de_stop_at(p, mzz);                       \
        phase = Q_D0;                                  \
    } while (0)
        if (begin) POST_BEGIN();
        unsigned int busy = __ballot_sync(0xffffffffu, phase != Q_IDLE);
        if (busy == 0) {
            if (!open) break;
            continue;
        }
        // ---- one DE for the lanes whose phase asks for one
        DEr r;
        r.de = 0.0;
        r.it = 0;
        r.max_its = p.max_it;
        r.need64 = false;
        DEstate st;
        st.smooth_it = 0.f;
        if (phase != Q_IDLE) {
            if (MIXED && !p64) {
                r = de_lock<float, FM>(p, c, ms);
            } else {
                const bool bsi = phase >= Q_BSI1;
                r = de_lock<double, FM, false, true>(p, c, ms, nullptr, &st, bsi, bsi ? 1 : 0);
            }
            // ---- the per-lane machine.  go: 1 the shadow search's test, 2 the
            // DE AO search's test, 3 the iteration count search's next step,
            // 4 the task is done
            int go = 0;
            // (RMdoBinSearchIt's steps: 8 for the shadow start, 5 for the DE AO start)
            constexpr int BSI_SH = 8, BSI_AO = 5;
            const int bsi_steps = ao ? BSI_AO : BSI_SH;
            if (phase == Q_D0) {
                if (!ao) {
                    const bool limited = r.it < its_cap<FM>(p, r) || r.de < (double)ms;
                    if (!p64 && (r.need64 || !limited)) {
                        p64 = true;
                        snap = true;
                        POST_BEGIN();
                    } else if (limited) {
                        dcur = r.de;
                        itmp = 8;
                        dt1 = digit * -0.5;
                        go = 1;
                    } else {
                        phase = Q_BSI1;
                    }
                } else {
                    dcur = fmin(r.de, (double)ms * 2.0);
                    const bool limited = r.it < its_cap<FM>(p, r) || dcur < (double)ms;
                    if (!p64 && (r.need64 || !limited)) {
                        p64 = true;
                        POST_BEGIN();
                    } else if (limited) {
                        itmp = 5;
                        dt1 = digit;
                        go = 2;
                    } else {
                        phase = Q_BSI1;
                    }
                }
                if (phase == Q_BSI1) {
                    // RMdoBinSearchIt from here (its first step is 0)
                    itmp = bsi_steps;
                    dt1 = 0.0;
                    dmul = 1.0;
                    b_first = true;
                    add_w(c, vf, 0.0);
                }
            } else if (phase == Q_BIS || phase == Q_LIM) {
                if (MIXED && !p64 && r.need64) {
                    p64 = true;
                    snap = false;
                    POST_BEGIN();
                } else {
                    dcur = r.de;
                    if (phase == Q_BIS) {
                        if (r.it >= its_cap<FM>(p, r)) dt1 = -fabs(dt1);
                        else dt1 = (dcur - (double)ms) < 0.0 ? fabs(dt1) * -0.55 : fabs(dt1) * 0.55;
                        go = 1;
                    } else {
                        dt1 = dcur < (double)ms ? fabs(dt1) * -0.55 : fabs(dt1) * 0.55;
                        go = 2;
                    }
                }
            } else if (phase == Q_BSI1) {
                float si_now = st.smooth_it;
                if (!b_first && b_last_dif < fabsf(bsi_yp - si_now)) {
                    mzz -= dt1;
                    add_w(c, vf, -dt1);
                    si_now = b_last_si;
                    dmul *= dt1 > 0.0 ? 0.5 : 0.7;
                }
                b_last_dif = fabsf(bsi_yp - si_now);
                b_last_si = si_now;
                if (si_now > bsi_top) {
                    dt1 = -3.0;
                    go = 3;
                } else {
                    mzz -= 0.001;
                    add_w(c, vf, -0.001);
                    phase = Q_BSI2;
                }
            } else if (phase == Q_BSI2) {
                float s2 = st.smooth_it;
                float rr = b_last_si - s2;
                if (fabsf(rr) < 1e-30f) dt1 = (b_last_si < s2 ? 1.0 : 0.0) - 0.5;
                else if (rr < 0.0f) dt1 = (double)__fdiv_rn(bsi_yp - s2, rr * 500.0f);
                else dt1 = (double)__fdiv_rn(bsi_yp - s2, rr * 1000.0f);
                if (dt1 > 4.0) dt1 = sqrt(dt1) * 2.0;
                else if (dt1 < -9.0) dt1 = sqrt(-dt1) * -3.0;
                dt1 = dt1 * dmul + 0.0005;
                go = 3;
            }
            if (go == 1) {  // RMdoBinSearch's loop test and step
                if (fabs(dcur - (double)ms) <= 0.001) {
                    go = 4;
                } else {
                    mzz += dt1;
                    add_w(c, vf, dt1);
                    ms = de_stop_at(p, mzz);
                    if (--itmp <= 0) go = 4;
                    else phase = Q_BIS;
                }
            } else if (go == 2) {  // surface_point's loop test and step
                if (!(itmp > 0 && fabs(dcur - (double)ms) > 0.004)) {
                    go = 4;
                } else {
                    mzz += dt1;
                    add_w(c, vf, dt1);
                    ms = de_stop_at(p, mzz);
                    itmp -= 1;
                    if (itmp > 0) phase = Q_LIM;
                    else go = 4;
                }
            } else if (go == 3) {
                b_first = false;
                if (!ao && snap && do_ao && itmp == BSI_SH - BSI_AO) {
                    // (the sixth round of the shadow search, before its step:
                    // where the DE AO search, 5 steps, ends)
                    ps[idx].ao_c[0] = c[0]; ps[idx].ao_c[1] = c[1]; ps[idx].ao_c[2] = c[2];
                    ps[idx].ao_ms = (float)((double)p.de_stop * (1.0 + fabs(mzz) * (double)p.de_stop_factor));
                    ao_done = true;
                }
                if (--itmp < 0) {
                    // surface_point's DE stop after the iteration count search
                    if (ao) ms = (float)((double)p.de_stop * (1.0 + fabs(mzz) * (double)p.de_stop_factor));
                    go = 4;
                } else {
                    mzz += dt1;
                    add_w(c, vf, dt1);
                    phase = Q_BSI1;
                }
            }
            if (go == 4) {
                if (!ao) {
                    // 0.1 step in front of the surface (src/calc.rs:2799-2802)
                    mzz = p.shadow_soft ? mzz - 0.1 : fmax(mzz - 0.1, 0.0);
                    add_w(c, vf, -0.1);
                    ps[idx].sh_c[0] = c[0]; ps[idx].sh_c[1] = c[1]; ps[idx].sh_c[2] = c[2];
                    ps[idx].sh_mzz = mzz;
                    if (do_ao && !ao_done) {
                        ao = true;
                        p64 = !MIXED;
                        POST_BEGIN();
                    } else {
                        phase = Q_IDLE;
                    }
                } else {
                    ps[idx].ao_c[0] = c[0]; ps[idx].ao_c[1] = c[1]; ps[idx].ao_c[2] = c[2];
                    ps[idx].ao_ms = ms;
                    phase = Q_IDLE;
                }
            }
        }
#undef POST_BEGIN
    }
}

// the DE of a secondary ray: single precision in the mixed mode (double
// where single cannot resolve the offset), else double
template <typename R, int FM>
__device__ __forceinline__ DEr ray_de(const DevParams &p, const double c[3], float ms) {
    DEr r = de_lock<R, FM>(p, c, ms);
    if (sizeof(R) == 4 && r.need64) r = de_lock<double, FM>(p, c, ms);
    return r;
}
// (a single precision position: the mixed mode's secondary rays)
template <typename R, int FM>
__device__ __forceinline__ DEr ray_de(const DevParams &p, const float c[3], float ms) {
    DEr r = de_lock<float, FM, false, false, float>(p, c, ms);
    if (r.need64) {
        const double cd[3] = {(double)c[0], (double)c[1], (double)c[2]};
        r = de_lock<double, FM>(p, cd, ms);
    }
    return r;
}

// One lane per shadow ray (surface pixel, light): the march toward the
// light of hard_shadow_row / soft_shadow_row (src/calc.rs:2836-2893,
// 2931-2977), one DE per trip of the loop, lanes refilled from the queue.
template <typename R, int FM>
__global__ void __launch_bounds__(256, MB3D_MIN_BLOCKS) k_shadow_rays(const __grid_constant__ DevParams p, int row0,
                                                     const PostStart *ps, const unsigned int *count,
                                                     mb3d_cu_silight *gbuf, unsigned int *queue) {
    const uint32_t npx = count[0];
    const uint32_t n_items = npx * (uint32_t)p.n_lights;
    bool open = true, active = false;
    uint32_t pix = 0;
    int li = 0, guard = 0;
    double c[3] = {0, 0, 0}, dt1 = 0, dmax = 0, zz2 = 0, zz2mul = 0, d = 0, last_de = 0, st = 0, max_lhs = 1;
    // (the mixed mode's DE position in single precision: the start point
    // and the light's direction, and the length marched so far)
    float cs[3] = {0.f, 0.f, 0.f}, lv[3] = {0.f, 0.f, 0.f};
    float ms = 0.f, rsf = 2.f, zr = 1.f, zrs_mul = 0.f;
    bool stepped = false;
    for (unsigned int trip = 0; trip < MB3D_TRIP_CAP; trip++) {
        uint32_t item = warp_take(!active, queue, n_items, p.refill_shadow, open);
        if (item != UINT32_MAX) {
            uint32_t i = item % npx;
            li = (int)(item / npx);
            const PostStart &s = ps[i];
            pix = s.pix;
            int y = row0 + (int)(pix / (uint32_t)p.width), x = (int)(pix % (uint32_t)p.width);
            uint32_t *w = reinterpret_cast<uint32_t *>(gbuf + pix);
            // MaxLHS (src/calc.rs:2767-2773) at the shadow start's depth
            float a = (float)(p.width + y) * 0.6f;
            float b = 1.0f + __fdiv_rn(0.5f * (float)fmin(s.sh_mzz, p.zend * 0.4) * (float)fmax(p.fov_y, 0.0), (float)p.height);
            max_lhs = (double)(a * b * p.hs_max_len_mul);
            if (s.flags & (1u << li)) {
                // the surface faces away from the light: in shadow
                if (p.shadow_soft) atomicAnd(&w[3], 0xFFFF03FFu);
                else atomicOr(&w[3], 0x400u << p.light_idx[li]);
            } else if (max_lhs > 0.0) {
                double c0[3], vf[3];
                pixel_ray(p, x, y, c0, vf);
                c[0] = s.sh_c[0]; c[1] = s.sh_c[1]; c[2] = s.sh_c[2];
                if (sizeof(R) == 4) {
                    for (int k = 0; k < 3; k++) {
                        cs[k] = (float)s.sh_c[k];
                        lv[k] = (float)p.light_vec[li][k];
                    }
                }
                zz2 = s.sh_mzz;
                zz2mul = -dot_normalize_d(p.light_vec[li], vf);
                dt1 = max_lhs;
                dmax = max_lhs;
                ms = de_stop_at(p, fabs(zz2));
                rsf = 2.0f;
                zr = 1.0f;
                zrs_mul = __fdiv_rn(80.0f, fmaxf(p.soft_radius, 0.001f));
                stepped = false;
                guard = 0;
                active = true;
            } else if (p.shadow_soft) {
                // no ray to march: the soft value stays 63 (lit)
            }
        }
        unsigned int busy = __ballot_sync(0xffffffffu, active);
        if (busy == 0) {
            if (!open) break;
            continue;
        }
        if (active) {
            DEr r;
            if constexpr (sizeof(R) == 4) {
                const float t = -(float)(dmax - dt1);
                const float cp[3] = {fmaf(lv[0], t, cs[0]), fmaf(lv[1], t, cs[1]), fmaf(lv[2], t, cs[2])};
                r = ray_de<R, FM>(p, cp, ms);
            } else {
                r = ray_de<R, FM>(p, c, ms);
            }
            bool end = false, shadowed = false;
            if (!stepped) {
                d = r.de;  // the DE at the ray's start
            } else {
                double dn = r.de;
                if (p.shadow_soft) {
                    double rr = (dmax - dt1) / max_lhs;
                    double r8 = (rr * rr) * (rr * rr);
                    zr = fminf(zr, (float)((dn - (double)ms) * (double)zrs_mul / (dmax - dt1 + 0.11) + r8 * r8));
                }
                if (r.it >= its_cap<FM>(p, r) || dn <= (double)ms) {
                    end = true;  // a surface in the way
                    shadowed = dt1 > 0.0;
                } else {
                    if (dn > last_de + st) dn = last_de + st;
                    if (last_de > dn + 1e-30) {
                        float t = sizeof(R) == 4 ? __fdividef((float)st, (float)(last_de - dn)) : (float)(st / (last_de - dn));
                        rsf = t < 1.0f ? fmaxf(t, 0.5f) : 1.0f;
                    } else {
                        rsf = 1.0f;
                    }
                    d = dn;
                    if (dt1 < 0.0) end = true;  // the whole way open
                }
            }
            if (!end && ++guard > 1000000) {
                end = true;
                shadowed = dt1 > 0.0;
            }
            if (!end) {
                last_de = d;
                st = (double)fminf(
                    fmaxf(0.11f, (float)((d - (double)p.ms_de_sub * (double)ms) * (double)p.z_step_div * (double)rsf)),
                    fmaxf(ms, 0.4f) * p.mh04zsd);
                dt1 -= st;
                if (sizeof(R) == 8) add_w(c, p.light_vec[li], -st);
                zz2 += st * zz2mul;
                ms = de_stop_at(p, fabs(zz2));
                stepped = true;
            } else {
                uint32_t *w = reinterpret_cast<uint32_t *>(gbuf + pix);
                if (p.shadow_soft) {
                    float zc = fminf(fmaxf(zr, 0.0f), 1.0f);
                    uint32_t v = (uint32_t)rintf(zc * 63.4f);
                    atomicAnd(&w[3], 0xFFFF03FFu | (v << 10));
                } else if (shadowed) {
                    atomicOr(&w[3], 0x400u << p.light_idx[li]);
                }
                active = false;
            }
        }
    }
}

// MakeRotQuatFromSNormals + CreateSMatrixFromQuat (src/deao.rs:45-62)
__device__ __forceinline__ void normal_matrix_d(const float n[3], float m[3][3]) {
    double a = acos(clampd((double)-n[2], -1.0, 1.0)) * 0.5;
    double sa, ca;
    sincos(a, &sa, &ca);
    double nn = sqrt((double)(n[1] * n[1] + n[0] * n[0]));
    double q0, q1, q2 = 0.0, q3 = ca;
    if (nn < 1e-25) {
        q0 = 0.0;
        q1 = 0.0;
    } else {
        sa /= nn;
        q0 = -(double)n[1] * sa;
        q1 = (double)n[0] * sa;
    }
    m[0][0] = (float)(1.0 - 2.0 * (q1 * q1 + q2 * q2));
    m[0][1] = (float)(2.0 * (q0 * q1 + q2 * q3));
    m[0][2] = (float)(2.0 * (q0 * q2 - q1 * q3));
    m[1][0] = (float)(2.0 * (q0 * q1 - q2 * q3));
    m[1][1] = (float)(1.0 - 2.0 * (q0 * q0 + q2 * q2));
    m[1][2] = (float)(2.0 * (q2 * q1 + q0 * q3));
    m[2][0] = (float)(2.0 * (q0 * q2 + q1 * q3));
    m[2][1] = (float)(2.0 * (q1 * q2 - q0 * q3));
    m[2][2] = (float)(1.0 - 2.0 * (q0 * q0 + q1 * q1));
}

__device__ __forceinline__ float sdot3(const float a[3], const float b[3]) {
    return __fadd_rn(__fadd_rn(__fmul_rn(a[0], b[0]), __fmul_rn(a[1], b[1])), __fmul_rn(a[2], b[2]));
}

// the per-pixel constants of the DE AO rays (src/deao.rs:285-300)
struct AOc {
    double msd, step_ao, max_dist, md_d10, de_mul;
};
__device__ __forceinline__ AOc ao_consts(const DevParams &p, float ms_surface) {
    AOc a;
    double de_stop = (double)p.de_stop;
    double s_max_d = (double)p.ao_max_len * 0.5 * sqrt((double)p.height * (double)p.height + (double)p.width * (double)p.width);
    double msd = fmin((double)ms_surface, 1e6);
    a.step_ao = msd / de_stop;
    a.max_dist = s_max_d * sqrt(a.step_ao);
    double dsm = (double)p.ao_d_step_mul;
    a.msd = (p.de_stop_factor == 0.0f) ? de_stop / (dsm * dsm) : msd / (dsm * dsm);
    a.de_mul = sqrt((double)p.ao_rays * 0.5);
    a.md_d10 = 0.1 / (a.max_dist * a.de_mul);
    return a;
}

// One lane per DE AO ray (surface pixel, direction): the ray loop of
// deao_row (src/deao.rs:317-359) outside rendering, one DE per trip;
// min_ra[k * npx + i] receives the ray's openness.
template <typename R, int FM>
__global__ void __launch_bounds__(256, sizeof(R) == 4 ? MB3D_MIN_BLOCKS_AO32 : MB3D_MIN_BLOCKS) k_ao_rays(const __grid_constant__ DevParams p, const PostStart *ps,
                                                 const mb3d_cu_silight *gbuf, const unsigned int *count,
                                                 float *min_ra, unsigned int *queue) {
    // the ray's type: single precision in the mixed mode (the DE AO's
    // openness is a smooth minimum), double in the plain mode
    typedef R T;
    const uint32_t npx = count[0];
    const uint32_t n_items = npx * (uint32_t)p.ao_rays;
    bool open = true, active = false, b_end = false;
    uint32_t slot = 0;
    T ic[3] = {0, 0, 0}, sv[3] = {0, 0, 0}, dt1 = 0, s_tmp = 1, msd = 0, max_dist = 0, md_d10 = 0;
    float ms_s = 0.f;
    int guard = 0;
    const T dsm = (T)p.ao_d_step_mul;
    const double de_mul = sqrt((double)p.ao_rays * 0.5);
    for (unsigned int trip = 0; trip < MB3D_TRIP_CAP; trip++) {
        uint32_t item = warp_take(!active, queue, n_items, p.refill_ao, open);
        if (item != UINT32_MAX) {
            uint32_t i = item % npx;
            int k = (int)(item / npx);
            const PostStart &s = ps[i];
            slot = item;
            ic[0] = (T)s.ao_c[0]; ic[1] = (T)s.ao_c[1]; ic[2] = (T)s.ao_c[2];
            ms_s = s.ao_ms;
            msd = (T)s.ao_msd;
            max_dist = (T)s.ao_max_dist;
            md_d10 = (T)s.ao_md_d10;
            // the ray's direction: the table direction turned to the normal,
            // then to world space, one step width long
            const float *dk = p.ao_dirs[k];
            float vv[3] = {sdot3(s.ao_rot[0], dk), sdot3(s.ao_rot[1], dk), sdot3(s.ao_rot[2], dk)};
            double vd[3] = {(double)vv[0], (double)vv[1], (double)vv[2]}, svd[3];
            rot_rev(vd, p.ao_rot, svd);
            sv[0] = (T)svd[0]; sv[1] = (T)svd[1]; sv[2] = (T)svd[2];
            dt1 = (T)s.ao_step0;
            s_tmp = (T)1;
            b_end = false;
            guard = 0;
            active = true;
        }
        unsigned int busy = __ballot_sync(0xffffffffu, active);
        if (busy == 0) {
            if (!open) break;
            continue;
        }
        if (active) {
            if (dt1 > max_dist) {
                dt1 = max_dist;
                b_end = true;
            }
            T c[3] = {ic[0] + sv[0] * dt1, ic[1] + sv[1] * dt1, ic[2] + sv[2] * dt1};
            DEr r;
            if constexpr (sizeof(R) == 4) {
                // a DE single precision cannot decide: the ray goes on in
                // double precision in k_ao_slow (kept out of this kernel:
                // the double DE's registers would cost this loop occupancy)
                r = de_lock<float, FM, false, false, float>(p, c, ms_s);
                if (r.need64) {
                    AoSlow *list = ao_slow_list(min_ra, n_items);
                    const unsigned int at = atomicAdd(queue + 2, 1u);
                    list[at] = AoSlow{slot, (float)dt1, (float)s_tmp, (unsigned int)guard | (b_end ? 0x80000000u : 0u)};
                    active = false;
                    continue;
                }
            } else {
                r = ray_de<R, FM>(p, c, ms_s);
            }
            const T dt2 = (T)r.de;
            if constexpr (sizeof(R) == 4) s_tmp = fminf(s_tmp, __fdividef(dt2 - msd + dt1 * md_d10, dt1));
            else s_tmp = fmin(s_tmp, (dt2 - msd + dt1 * md_d10) / dt1);
            bool end = s_tmp < (T)0.02 || b_end || ++guard > 100000;
            if (!end) dt1 += fmax(dt2, dt1 * dsm);
            if (end) {
                min_ra[slot] = (float)(fmax((double)s_tmp, 0.0) * de_mul);
                active = false;
            }
        }
    }
}

// the DE AO rays the single precision kernel handed over (AoSlow records),
// one thread per ray, in double precision from where they stopped: the DE
// there, then the rest of the ray as k_ao_rays<double> marches it
template <int FM>
__global__ void __launch_bounds__(128) k_ao_slow(const __grid_constant__ DevParams p, const PostStart *ps,
                                                 const unsigned int *count, float *min_ra, unsigned int *queue) {
    const uint32_t npx = count[0];
    const uint32_t n_items = npx * (uint32_t)p.ao_rays;
    const AoSlow *list = ao_slow_list(min_ra, n_items);
    const unsigned int n = queue[2];
    const double dsm = (double)p.ao_d_step_mul;
    const double de_mul = sqrt((double)p.ao_rays * 0.5);
    for (;;) {
        const unsigned int at = atomicAdd(queue + 3, 1u);
        if (at >= n) break;
        const AoSlow rec = list[at];
        const uint32_t i = rec.item % npx;
        const int k = (int)(rec.item / npx);
        const PostStart &s = ps[i];
        const double ic[3] = {s.ao_c[0], s.ao_c[1], s.ao_c[2]};
        const float *dk = p.ao_dirs[k];
        const float vv[3] = {sdot3(s.ao_rot[0], dk), sdot3(s.ao_rot[1], dk), sdot3(s.ao_rot[2], dk)};
        const double vd[3] = {(double)vv[0], (double)vv[1], (double)vv[2]};
        double sv[3];
        rot_rev(vd, p.ao_rot, sv);
        const double msd = s.ao_msd, max_dist = s.ao_max_dist, md_d10 = s.ao_md_d10;
        double dt1 = (double)rec.dt1, s_tmp = (double)rec.s;
        int guard = (int)(rec.guard & 0x7FFFFFFFu);
        bool b_end = (rec.guard & 0x80000000u) != 0;
        for (;;) {
            if (dt1 > max_dist) {
                dt1 = max_dist;
                b_end = true;
            }
            const double c[3] = {ic[0] + sv[0] * dt1, ic[1] + sv[1] * dt1, ic[2] + sv[2] * dt1};
            const DEr r = de_lock<double, FM>(p, c, s.ao_ms);
            s_tmp = fmin(s_tmp, (r.de - msd + dt1 * md_d10) / dt1);
            if (s_tmp < 0.02 || b_end || ++guard > 100000) break;
            dt1 += fmax(r.de, dt1 * dsm);
        }
        min_ra[rec.item] = (float)(fmax(s_tmp, 0.0) * de_mul);
    }
}

#ifdef MB3D_COMMON_KERNELS
// per surface pixel, before the DE AO rays: the turn of the ray table to
// the surface normal (src/deao.rs:301-316) and the per-pixel constants
// (src/deao.rs:285-300), once for all of the pixel's rays
__global__ void k_ao_prep(const __grid_constant__ DevParams p, PostStart *ps, const mb3d_cu_silight *gbuf,
                          const unsigned int *count) {
    const uint32_t npx = count[0];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npx; i += gridDim.x * blockDim.x) {
        PostStart &s = ps[i];
        G si;
        si.load(gbuf[s.pix]);
        float nrm[3];
        {
            float v[3] = {(float)si.n0, (float)si.n1, (float)si.n2};
            float l = fmaxf(__fsqrt_rn(sdot3(v, v)), 1e-30f);
            nrm[0] = __fdiv_rn(v[0], l);
            nrm[1] = __fdiv_rn(v[1], l);
            nrm[2] = __fdiv_rn(v[2], l);
        }
        normal_matrix_d(nrm, s.ao_rot);
        AOc a = ao_consts(p, s.ao_ms);
        s.ao_step0 = a.step_ao * (double)p.ao_d_step_mul;
        s.ao_max_dist = a.max_dist;
        s.ao_msd = a.msd;
        s.ao_md_d10 = a.md_d10;
    }
}

// per surface pixel: the correction of the closed rays by their open
// neighbours and the mean (src/deao.rs:361-413)
__global__ void k_ao_final(const __grid_constant__ DevParams p, const PostStart *ps, const unsigned int *count,
                           const float *min_ra, mb3d_cu_silight *gbuf) {
    const uint32_t npx = count[0];
    const int nr = p.ao_rays;
    const double de_mul = sqrt((double)nr * 0.5);
    const double abr = 1.2 / asin(clampd(1.0 / de_mul, -1.0, 1.0));
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npx; i += gridDim.x * blockDim.x) {
        float mr[MB3D_MAX_AO_RAYS];
        for (int k = 0; k < nr; k++) mr[k] = min_ra[(size_t)k * npx + i];
        double amount = 0.0;
        for (int k = 0; k < nr; k++) {
            float s_add = 0.f;
            if (mr[k] < 1.0f) {
                float max_add = 1.0f - mr[k];
                for (int k2 = 0; k2 < nr; k2++) {
                    if (k2 == k) continue;
                    float dt = sdot3(p.ao_dirs[k], p.ao_dirs[k2]);
                    if (dt > p.ao_d_min_a_dif) {
                        float ov = mr[k2] - (float)((double)acosf(fminf(fmaxf(dt, -1.0f), 1.0f)) * abr) + 1.0f;
                        if (ov > 0.0f) s_add += fminf(max_add, ov) * p.ao_corr_weight;
                    }
                }
            }
            amount += (double)fminf(s_add + mr[k], 1.0f);
        }
        uint16_t v = sat_u16d(fmax(rint(16383.0 * (1.0 - amount / (double)nr)), 0.0));
        uint32_t *w = reinterpret_cast<uint32_t *>(gbuf + ps[i].pix);
        w[3] = (w[3] & 0xFFFFu) | ((uint32_t)v << 16);
    }
}
#endif

template <int FM>
__global__ void k_de_probe(const __grid_constant__ DevParams p, const double *pos, int n, double *de, int *its,
                           int mixed) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    double c[3] = {pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]};
    DEr r = mixed ? ray_de<float, FM>(p, c, p.de_stop) : de_lock<double, FM>(p, c, p.de_stop);
    de[i] = r.de * p.step_width;
    its[i] = r.it;
}

}  // namespace mb3dcu
#include "reflect.cuh"
namespace mb3dcu {

// ---------------------------------------------------------------------------
// the launches of one formula set (instantiated per set in kern_*.cu)
template <int FM>
struct Launch {
    static void march(const DevParams &p, bool mixed, int row0, int rows, mb3d_cu_silight *out, Hand *list,
                      unsigned int *counters, unsigned long long *gcount, int blocks, cudaStream_t s) {
        if (gcount) {
            if (mixed) k_march<float, FM, true><<<blocks, 256, 0, s>>>(p, row0, rows, out, list, counters, gcount);
            else k_march<double, FM, true><<<blocks, 256, 0, s>>>(p, row0, rows, out, list, counters, gcount);
        } else {
            if (mixed) k_march<float, FM, false><<<blocks, 256, 0, s>>>(p, row0, rows, out, list, counters, nullptr);
            else k_march<double, FM, false><<<blocks, 256, 0, s>>>(p, row0, rows, out, list, counters, nullptr);
        }
    }
    static void finish(const DevParams &p, bool mixed, int row0, const Hand *list, unsigned int *counters,
                       Hand *slow, mb3d_cu_silight *out, int blocks, cudaStream_t s) {
        k_finish<FM><<<blocks, 256, 0, s>>>(p, row0, list, counters, slow, out);
        k_finish_slow<FM><<<blocks, 128, 0, s>>>(p, row0, slow, counters, out);
    }
    static void finish_fast(const DevParams &p, bool, int row0, const Hand *list, unsigned int *counters,
                            Hand *slow, mb3d_cu_silight *out, int blocks, cudaStream_t s) {
        k_finish<FM><<<blocks, 256, 0, s>>>(p, row0, list, counters, slow, out);
    }
    static void finish_slow(const DevParams &p, bool, int row0, const Hand *, unsigned int *counters,
                            Hand *slow, mb3d_cu_silight *out, int blocks, cudaStream_t s) {
        k_finish_slow<FM><<<blocks, 128, 0, s>>>(p, row0, slow, counters, out);
    }
    static void post_start(const DevParams &p, bool mixed, int row0, int passes, const mb3d_cu_silight *gbuf,
                           const uint32_t *list, const unsigned int *count, unsigned int *queue, PostStart *ps,
                           int blocks, cudaStream_t s) {
        if (mixed) k_post_start<FM, true><<<blocks, 256, 0, s>>>(p, row0, passes, gbuf, list, count, queue, ps);
        else k_post_start<FM, false><<<blocks, 256, 0, s>>>(p, row0, passes, gbuf, list, count, queue, ps);
    }
    static void shadow_rays(const DevParams &p, bool mixed, int row0, const PostStart *ps, const unsigned int *count,
                            mb3d_cu_silight *gbuf, unsigned int *queue, int blocks, cudaStream_t s) {
        if (mixed) k_shadow_rays<float, FM><<<blocks, 256, 0, s>>>(p, row0, ps, count, gbuf, queue);
        else k_shadow_rays<double, FM><<<blocks, 256, 0, s>>>(p, row0, ps, count, gbuf, queue);
    }
    static void ao_rays(const DevParams &p, bool mixed, const PostStart *ps, const mb3d_cu_silight *gbuf,
                        const unsigned int *count, float *min_ra, unsigned int *queue, int blocks, cudaStream_t s) {
        if (mixed) {
            k_ao_rays<float, FM><<<blocks, 256, 0, s>>>(p, ps, gbuf, count, min_ra, queue);
            k_ao_slow<FM><<<blocks, 128, 0, s>>>(p, ps, count, min_ra, queue);
        } else {
            k_ao_rays<double, FM><<<blocks, 256, 0, s>>>(p, ps, gbuf, count, min_ra, queue);
        }
    }
    static void reflect(const DevParams &p, const mb3d_cu_reflect_ray *rays, uint32_t n, int far_fog, const ReflAO *tab,
                        mb3d_cu_reflect_hit *hits, int blocks, cudaStream_t s) {
        k_reflect<FM><<<blocks, 128, 0, s>>>(p, rays, n, far_fog, tab, hits);
    }
    static void reflect_first(const DevParams &p, const mb3d_cu_silight *gbuf, mb3d_cu_reflect_ray *tmp,
                              unsigned char *valid, int blocks, cudaStream_t s) {
        k_reflect_first<FM><<<blocks, 128, 0, s>>>(p, gbuf, tmp, valid);
    }
    static void de_probe(const DevParams &p, const double *pos, int n, double *de, int *its, bool mixed, cudaStream_t s) {
        k_de_probe<FM><<<(n + 127) / 128, 128, 0, s>>>(p, pos, n, de, its, mixed ? 1 : 0);
    }
};

}  // namespace mb3dcu
