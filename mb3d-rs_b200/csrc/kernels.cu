// The kernels of the ray march and its post passes (sm_100a).
//
//  k_march64   the plain double precision march, one thread per pixel: the
//              drop-in for mb3d-rs's FP64 CPU march (Marcher::march_pixel).
//  k_march32   the single precision bulk march (double precision origin and
//              ray parameter): a persistent kernel whose warps take pixel
//              tiles from a queue; a ray that reaches a surface (or starts
//              inside the set, or needs double precision) is handed to the
//              finish kernel through a list filled with warp-aggregated
//              atomics; a ray into the background is written at once.
//  k_finish64  the double precision finish of every handed-over ray: the
//              surface re-check (the march goes on in double precision when
//              the single precision hit was not one), the binary search,
//              normals, colour and depth (the reference's own mixed mode,
//              Marcher::finish_pixel, src/calc.rs:2439-2465, on the card).
//  k_shadow    hard (or soft) shadows per pixel (src/calc.rs:2777-2979 without
//              the row-sequential open-air shortcut, as the reference's card
//              pass, src/gpu_march.wgsl:3343-3500).
//  k_deao      DE ambient occlusion per pixel (src/deao.rs:268-414).
//  k_de_probe  the DE at given points (gpu::de_probe, calc::de_at).
//
// Every loop has an iteration cap (the reference's guards), so no kernel can
// spin without end.
#include <cuda_runtime.h>
#include <stdint.h>
#include "devparams.h"
#include "marcher64.cuh"
#include "de32.cuh"
#include "kernels.h"

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

// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(128) k_march64(const __grid_constant__ DevParams p, int row0, int rows, mb3d_cu_silight *out) {
    int x = blockIdx.x * 16 + (threadIdx.x & 15);
    int ly = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= p.width || ly >= rows) return;
    int y = row0 + ly;
    M64 m(p);
    m.seed = pixel_seed_d(y, x);
    G si;
    m.march_pixel(si, x, y);
    si.store(out + (size_t)ly * p.width + x);
}

// ---------------------------------------------------------------------------
// tiles of 8 x 4 pixels per warp (neighbouring rays march alike)
#define TILE_W 8
#define TILE_H 4

__device__ __forceinline__ void warp_append(bool want, unsigned int *count, const Hand &h, Hand *list) {
    unsigned int mask = __ballot_sync(0xffffffffu, want);
    if (mask == 0) return;
    int lane = threadIdx.x & 31;
    int leader = __ffs(mask) - 1;
    unsigned int base = 0;
    if (lane == leader) base = atomicAdd(count, (unsigned int)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (want) list[base + __popc(mask & ((1u << lane) - 1u))] = h;
}

__global__ void __launch_bounds__(256) k_march32(const __grid_constant__ DevParams p, int row0, int rows, mb3d_cu_silight *out,
                                                 Hand *list, unsigned int *counters) {
    const int lane = threadIdx.x & 31;
    const int tiles_x = (p.width + TILE_W - 1) / TILE_W;
    const int tiles = tiles_x * ((rows + TILE_H - 1) / TILE_H);
    for (;;) {
        int t = 0;
        if (lane == 0) t = (int)atomicAdd(&counters[1], 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= tiles) break;
        int x = (t % tiles_x) * TILE_W + (lane & (TILE_W - 1));
        int ly = (t / tiles_x) * TILE_H + lane / TILE_W;
        bool valid = x < p.width && ly < rows;
        int y = row0 + ly;
        Hand h;
        bool hand = false;
        if (valid) {
            double c0[3], vf[3], c[3];
            pixel_ray(p, x, y, c0, vf);
            h.pix = (uint32_t)(ly * p.width + x);
            h.flags = 0;
            double mzz = 0.0;
            float ms = p.de_stop;
            DE32 r = de32(p, c0, ms);
            float step_count = 0.f;
            if (r.need64 || r.it >= p.max_it || (double)r.de < (double)ms) {
                h.flags = HAND_FULL;  // start inside (or no single precision): all in double
                hand = true;
            } else {
                double dtmp = r.de;
                int it = r.it;
                double last_step = dtmp * (double)p.z_step_div, last_de = 0.0;
                float rsf = 1.0f;
                bool first = p.first_step_random != 0;
                int32_t seed = pixel_seed_d(y, x);
                bool stepped = false;
                for (unsigned int guard = 0; guard < 2000000u; guard++) {
                    if (it >= p.max_it) {
                        double dt1 = -0.5 * last_step;
                        mzz += dt1;
                        ms = (float)((double)p.de_stop * (1.0 + mzz * (double)p.de_stop_factor));
                        c[0] = c0[0] + vf[0] * mzz; c[1] = c0[1] + vf[1] * mzz; c[2] = c0[2] + vf[2] * mzz;
                        r = de32(p, c, ms);
                        dtmp = r.de;
                        it = r.it;
                        last_step = -dt1;
                        stepped = false;
                    }
                    if (r.need64) {
                        hand = true;
                        break;
                    }
                    if (it < p.min_it || (it < p.max_it && dtmp >= (double)ms)) {
                        last_de = dtmp;
                        double d = fmax(0.11, (dtmp - (double)p.ms_de_sub * (double)ms) * (double)p.z_step_div * (double)rsf);
                        double s1 = (double)(fmaxf(ms, 0.4f) * p.mh04zsd);
                        bool count = p.dfog_on_it == 0 || it == p.dfog_on_it;
                        if (s1 < d) {
                            if (count) step_count += (float)(s1 / d);
                            d = s1;
                        } else if (count) {
                            step_count += 1.0f;
                        }
                        if (first) {
                            first = false;
                            seed = (int32_t)((uint32_t)seed * 214013u + 2531011u);
                            d *= (double)(seed & 0x7FFFFFFF) * (1.0 / 2147483647.0);
                        }
                        mzz += d;
                        if (mzz > p.zend) break;  // background
                        last_step = d;
                        ms = (float)((double)p.de_stop * (1.0 + mzz * (double)p.de_stop_factor));
                        c[0] = c0[0] + vf[0] * mzz; c[1] = c0[1] + vf[1] * mzz; c[2] = c0[2] + vf[2] * mzz;
                        r = de32(p, c, ms);
                        dtmp = r.de;
                        it = r.it;
                        if (dtmp > last_de + last_step) dtmp = last_de + last_step;
                        if (last_de > dtmp + 1e-30) {
                            double tt = last_step / (last_de - dtmp);
                            rsf = tt < 1.0 ? (float)fmax(0.5, tt) : 1.0f;
                        } else {
                            rsf = 1.0f;
                        }
                        stepped = true;
                    } else {
                        hand = true;  // a surface: the finish decides in double precision
                        break;
                    }
                }
                if (hand) {
                    h.flags = (stepped ? HAND_STEPPED : 0u) | (first ? HAND_FIRST : 0u) | (r.need64 ? HAND_FULL : 0u);
                    h.mzz = mzz;
                    h.last_step = last_step;
                    h.last_de = last_de;
                    h.rsf = rsf;
                    h.step_count = step_count;
                    h.seed = seed;
                } else {
                    G si;
                    si.clear();
                    si.amb_shadow = 5000;
                    float sc = fminf(fmaxf(step_count, 0.0f), 1023.0f);
                    si.shadow = (uint16_t)rintf(sc);
                    si.store(out + h.pix);
                }
            }
        }
        warp_append(hand, &counters[0], h, list);
    }
}

__global__ void __launch_bounds__(128) k_finish64(const __grid_constant__ DevParams p, int row0, const Hand *list,
                                                  const unsigned int *counters, mb3d_cu_silight *out) {
    unsigned int n = counters[0];
    for (unsigned int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        Hand h = list[i];
        int x = (int)(h.pix % (uint32_t)p.width);
        int ly = (int)(h.pix / (uint32_t)p.width);
        int y = row0 + ly;
        M64 m(p);
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
            for (int k = 0; k < 3; k++) m.it.c[k] = c0[k] + m.vfov[k] * h.mzz;
            m.update_de_stop();
            m.it.calc_sit = false;
            m.seed = h.seed;
            double dtmp = m.calc_de();
            if ((h.flags & HAND_STEPPED) && dtmp > h.last_de + h.last_step) dtmp = h.last_de + h.last_step;
            m.march_from(si, dtmp, h.last_step, h.rsf, (h.flags & HAND_FIRST) != 0, h.step_count);
        }
        si.store(out + h.pix);
    }
}

// ---------------------------------------------------------------------------
// post passes

__device__ __forceinline__ double dot_normalize_d(const double a[3], const double b[3]) {
    return dot3d(a, b) / fmax(sqrt(dot3d(a, a) * dot3d(b, b)), 1e-300);
}

// the DE along a secondary ray: double precision, or single precision with
// the double precision position
template <bool MIXED>
__device__ __forceinline__ double ray_de(M64 &m, int &it) {
    if (MIXED) {
        DE32 r = de32(m.p, m.it.c, m.ms_de_stop);
        if (!r.need64) {
            it = r.it;
            m.max_its_result = m.p.max_it;
            return (double)r.de;
        }
    }
    double d = m.calc_de();
    it = m.it.it_result;
    return d;
}

template <bool MIXED>
__global__ void __launch_bounds__(128) k_shadow(const __grid_constant__ DevParams p, int row0, int rows, mb3d_cu_silight *gbuf) {
    int x = blockIdx.x * 16 + (threadIdx.x & 15);
    int ly = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= p.width || ly >= rows) return;
    int y = row0 + ly;
    mb3d_cu_silight *rec = gbuf + (size_t)ly * p.width + x;
    G si;
    si.load(*rec);
    M64 m(p);
    m.seed = (int32_t)((int64_t)0x24563487u + ((int64_t)y + 1) * (int64_t)0x324594A1);
    double nv0[3] = {si.n0 / 32767.0, si.n1 / 32767.0, si.n2 / 32767.0}, nvec[3];
    rot_rev(nv0, p.vgrads, nvec);
    if (p.shadow_soft) {
        // calcHSsoft (src/calc.rs:2901-2979)
        si.shadow |= 0xFC00;
        if (m.hs_surface_start(x, y, si)) {
            m.mzz -= 0.1;
            add_w(m.it.c, m.vfov, -0.1);
            double max_lhs = m.hs_max_len(y);
            double zz2 = m.mzz;
            m.update_de_stop();
            const double *lvec = p.light_vec[0];
            double zz2mul = -dot_normalize_d(lvec, m.vfov);
            if (dot3d(nvec, lvec) > 0.0) {
                si.shadow &= 0x3FF;
            } else {
                float zrs_mul = __fdiv_rn(80.0f, fmaxf(p.soft_radius, 0.001f));
                float zr = 1.0f;
                double dmax = max_lhs, dt1 = max_lhs;
                if (dt1 > 0.0) {
                    m.ms_de_stop = (float)((double)p.de_stop * (1.0 + fabs(zz2) * (double)p.de_stop_factor));
                    float rsf = 2.0f;
                    int it;
                    double d = ray_de<MIXED>(m, it);
                    for (int guard = 0; guard < 1000000; guard++) {
                        double last_de = d;
                        double st = (double)fminf(
                            fmaxf(0.11f, (float)((d - (double)p.ms_de_sub * (double)m.ms_de_stop) * (double)p.z_step_div * (double)rsf)),
                            fmaxf(m.ms_de_stop, 0.4f) * p.mh04zsd);
                        dt1 -= st;
                        add_w(m.it.c, lvec, -st);
                        zz2 += st * zz2mul;
                        m.ms_de_stop = (float)((double)p.de_stop * (1.0 + fabs(zz2) * (double)p.de_stop_factor));
                        d = ray_de<MIXED>(m, it);
                        double rr = (dmax - dt1) / max_lhs;
                        double r8 = (rr * rr) * (rr * rr);
                        zr = fminf(zr, (float)((d - (double)m.ms_de_stop) * (double)zrs_mul / (dmax - dt1 + 0.11) + r8 * r8));
                        if (it >= m.max_its_result || d <= (double)m.ms_de_stop) break;
                        if (d > last_de + st) d = last_de + st;
                        if (last_de > d + 1e-30) {
                            float t = (float)(st / (last_de - d));
                            rsf = t < 1.0f ? fmaxf(t, 0.5f) : 1.0f;
                        } else {
                            rsf = 1.0f;
                        }
                        if (dt1 < 0.0) break;
                    }
                }
                float zc = fminf(fmaxf(zr, 0.0f), 1.0f);
                si.shadow = (uint16_t)((si.shadow & 0x3FF) | ((uint16_t)rintf(zc * 63.4f) << 10));
            }
        }
    } else {
        // THardShadowCalcThread.Execute per pixel (src/calc.rs:2777-2898)
        uint16_t clear_mask = 0;
        for (int l = 0; l < p.n_lights; l++) clear_mask |= (uint16_t)(0x400 << p.light_idx[l]);
        si.shadow &= (uint16_t)~clear_mask;
        if (m.hs_surface_start(x, y, si)) {
            m.mzz = fmax(m.mzz - 0.1, 0.0);
            add_w(m.it.c, m.vfov, -0.1);
            m.update_de_stop();
            double ic[3] = {m.it.c[0], m.it.c[1], m.it.c[2]};
            double max_lhs = m.hs_max_len(y);
            for (int l = 0; l < p.n_lights; l++) {
                int li = p.light_idx[l];
                m.it.c[0] = ic[0]; m.it.c[1] = ic[1]; m.it.c[2] = ic[2];
                double zz2 = m.mzz;
                const double *lvec = p.light_vec[l];
                double zz2mul = -dot_normalize_d(lvec, m.vfov);
                if (dot3d(nvec, lvec) > 0.0) {
                    si.shadow |= (uint16_t)(0x400 << li);
                    continue;
                }
                double dt1 = max_lhs;
                if (dt1 > 0.0) {
                    m.ms_de_stop = (float)((double)p.de_stop * (1.0 + fabs(zz2) * (double)p.de_stop_factor));
                    float rsf = 2.0f;
                    int it;
                    double d = ray_de<MIXED>(m, it);
                    for (int guard = 0; guard < 1000000; guard++) {
                        double last_de = d;
                        double st = (double)fminf(
                            fmaxf(0.11f, (float)((d - (double)p.ms_de_sub * (double)m.ms_de_stop) * (double)p.z_step_div * (double)rsf)),
                            fmaxf(m.ms_de_stop, 0.4f) * p.mh04zsd);
                        dt1 -= st;
                        add_w(m.it.c, lvec, -st);
                        zz2 += st * zz2mul;
                        m.ms_de_stop = (float)((double)p.de_stop * (1.0 + fabs(zz2) * (double)p.de_stop_factor));
                        d = ray_de<MIXED>(m, it);
                        if (it >= m.max_its_result || d <= (double)m.ms_de_stop) break;
                        if (d > last_de + st) d = last_de + st;
                        if (last_de > d + 1e-30) {
                            float t = (float)(st / (last_de - d));
                            rsf = t < 1.0f ? fmaxf(t, 0.5f) : 1.0f;
                        } else {
                            rsf = 1.0f;
                        }
                        if (dt1 < 0.0) break;
                    }
                }
                if (dt1 > 0.0) si.shadow |= (uint16_t)(0x400 << li);
            }
        }
    }
    si.store(rec);
}

// MakeRotQuatFromSNormals + CreateSMatrixFromQuat (src/deao.rs:45-62)
__device__ void normal_matrix_d(const float n[3], float m[3][3]) {
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

template <bool MIXED>
__global__ void __launch_bounds__(128) k_deao(const __grid_constant__ DevParams p, int row0, int rows, mb3d_cu_silight *gbuf) {
    int x = blockIdx.x * 16 + (threadIdx.x & 15);
    int ly = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= p.width || ly >= rows) return;
    int y = row0 + ly;
    mb3d_cu_silight *rec = gbuf + (size_t)ly * p.width + x;
    G si;
    si.load(*rec);
    si.amb_shadow = 0;
    M64 m(p);
    if (!(si.zpos() >= 32768 || si.si_gradient >= 32768)) {
        int32_t rnd = (int32_t)((int64_t)0x24563487u + ((int64_t)y + 1) * (int64_t)0x324594A1);
        // DEAO uses 5 binary search steps
        m.surface_point(x, y, si, 5, 0.004);
        double sw = p.step_width;
        double s_max_d = (double)p.ao_max_len * 0.5 * sqrt((double)p.height * (double)p.height + (double)p.width * (double)p.width);
        double de_stop = (double)p.de_stop;
        double msd = fmin((double)m.ms_de_stop, 1e6);
        double ic[3] = {m.it.c[0], m.it.c[1], m.it.c[2]};
        double step_ao = msd / de_stop;
        double max_dist = s_max_d * sqrt(step_ao);
        double dsm = (double)p.ao_d_step_mul;
        msd = (p.de_stop_factor == 0.0f) ? de_stop / (dsm * dsm) : msd / (dsm * dsm);
        int nr = p.ao_rays;
        double de_mul = sqrt((double)nr * 0.5);
        double abr = 1.2 / asin(clampd(1.0 / de_mul, -1.0, 1.0));
        double md_d10 = 0.1 / (max_dist * de_mul);
        float nrm[3];
        {
            float v[3] = {(float)si.n0, (float)si.n1, (float)si.n2};
            float l = fmaxf(__fsqrt_rn(sdot3(v, v)), 1e-30f);
            nrm[0] = __fdiv_rn(v[0], l);
            nrm[1] = __fdiv_rn(v[1], l);
            nrm[2] = __fdiv_rn(v[2], l);
        }
        float rot_w[3][3];
        normal_matrix_d(nrm, rot_w);
        // the rotation to world space, step width long (normalise_matrix_to(sw, vgrads))
        double rv[3][3];
        for (int i = 0; i < 3; i++) {
            double d = sw / sqrt(dot3d(p.vgrads[i], p.vgrads[i]));
            for (int k = 0; k < 3; k++) rv[i][k] = p.vgrads[i][k] * d;
        }
        float min_ra[MB3D_MAX_AO_RAYS];
        for (int k = 0; k < nr; k++) {
            const float *dk = p.ao_dirs[k];
            float vv[3] = {sdot3(rot_w[0], dk), sdot3(rot_w[1], dk), sdot3(rot_w[2], dk)};
            double vd[3] = {(double)vv[0], (double)vv[1], (double)vv[2]}, sv[3];
            rot_rev(vd, rv, sv);
            double dt1 = step_ao * dsm;
            double s_tmp = 1.0;
            bool b_end = false, b_first = p.ao_first_step_random != 0;
            for (int guard = 0; guard < 100000; guard++) {
                if (b_first) {
                    b_first = false;
                    rnd = (int32_t)((uint32_t)rnd * 0x343FDu + 0x269EC3u);
                    dt1 *= (double)(((uint32_t)rnd >> 8) & 0x7FFFFF) / (double)0x7FFFFF * 1.5 + 0.5;
                } else if (dt1 > max_dist) {
                    dt1 = max_dist;
                    b_end = true;
                }
                m.it.c[0] = ic[0]; m.it.c[1] = ic[1]; m.it.c[2] = ic[2];
                add_w(m.it.c, sv, dt1);
                int it;
                double dt2 = ray_de<MIXED>(m, it);
                s_tmp = fmin(s_tmp, (dt2 - msd + dt1 * md_d10) / dt1);
                if (s_tmp < 0.02) break;
                dt1 += fmax(dt2, dt1 * dsm);
                if (b_end) break;
            }
            min_ra[k] = (float)(fmax(s_tmp, 0.0) * de_mul);
        }
        double amount = 0.0;
        for (int k = 0; k < nr; k++) {
            float s_add = 0.f;
            if (min_ra[k] < 1.0f) {
                float max_add = 1.0f - min_ra[k];
                for (int k2 = 0; k2 < nr; k2++) {
                    if (k2 == k) continue;
                    float dt = sdot3(p.ao_dirs[k], p.ao_dirs[k2]);
                    if (dt > p.ao_d_min_a_dif) {
                        float ov = min_ra[k2] - (float)((double)acosf(fminf(fmaxf(dt, -1.0f), 1.0f)) * abr) + 1.0f;
                        if (ov > 0.0f) s_add += fminf(max_add, ov) * p.ao_corr_weight;
                    }
                }
            }
            amount += (double)fminf(s_add + min_ra[k], 1.0f);
        }
        si.amb_shadow = sat_u16d(fmax(rint(16383.0 * (1.0 - amount / (double)nr)), 0.0));
    }
    si.store(rec);
}

__global__ void k_de_probe(const __grid_constant__ DevParams p, const double *pos, int n, double *de, int *its, int mixed) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    M64 m(p);
    m.it.c[0] = pos[3 * i];
    m.it.c[1] = pos[3 * i + 1];
    m.it.c[2] = pos[3 * i + 2];
    double d;
    int it;
    if (mixed) d = ray_de<true>(m, it);
    else d = ray_de<false>(m, it);
    de[i] = d * p.step_width;
    its[i] = it;
}

// ---------------------------------------------------------------------------
// launchers

int launch_march64(const DevParams &p, int row0, int rows, mb3d_cu_silight *out, cudaStream_t s) {
    dim3 grid((p.width + 15) / 16, (rows + 7) / 8);
    k_march64<<<grid, 128, 0, s>>>(p, row0, rows, out);
    return 1;
}

int launch_march32(const DevParams &p, int row0, int rows, mb3d_cu_silight *out, Hand *list, unsigned int *counters,
                   int sms, cudaStream_t s) {
    int tiles = ((p.width + TILE_W - 1) / TILE_W) * ((rows + TILE_H - 1) / TILE_H);
    int blocks = sms * 8;  // 8 blocks of 8 warps resident per SM
    int need = (tiles + 7) / 8;
    if (blocks > need) blocks = need > 0 ? need : 1;
    k_march32<<<blocks, 256, 0, s>>>(p, row0, rows, out, list, counters);
    return 1;
}

int launch_finish64(const DevParams &p, int row0, const Hand *list, const unsigned int *counters, mb3d_cu_silight *out,
                    int sms, cudaStream_t s) {
    k_finish64<<<sms * 8, 128, 0, s>>>(p, row0, list, counters, out);
    return 1;
}

int launch_shadow(const DevParams &p, int row0, int rows, mb3d_cu_silight *gbuf, bool mixed, cudaStream_t s) {
    dim3 grid((p.width + 15) / 16, (rows + 7) / 8);
    if (mixed) k_shadow<true><<<grid, 128, 0, s>>>(p, row0, rows, gbuf);
    else k_shadow<false><<<grid, 128, 0, s>>>(p, row0, rows, gbuf);
    return 1;
}

int launch_deao(const DevParams &p, int row0, int rows, mb3d_cu_silight *gbuf, bool mixed, cudaStream_t s) {
    dim3 grid((p.width + 15) / 16, (rows + 7) / 8);
    if (mixed) k_deao<true><<<grid, 128, 0, s>>>(p, row0, rows, gbuf);
    else k_deao<false><<<grid, 128, 0, s>>>(p, row0, rows, gbuf);
    return 1;
}

int launch_de_probe(const DevParams &p, const double *pos, int n, double *de, int *its, bool mixed, cudaStream_t s) {
    k_de_probe<<<(n + 127) / 128, 128, 0, s>>>(p, pos, n, de, its, mixed ? 1 : 0);
    return 1;
}

}  // namespace mb3dcu
