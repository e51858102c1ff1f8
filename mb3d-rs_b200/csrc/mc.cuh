// The Monte Carlo tracer of mb3d-rs (src/mc.rs) on the card, as one
// persistent wavefront kernel.
//
// Every lane of a warp carries one work item through a state machine: a
// whole ray of Tracer::ray (render mode) or one march request of
// McMarch::run (batch mode, the drop-in for gpu::mc_batch).  Each trip of
// the loop runs every lane's logic up to its next distance estimate and
// then evaluates one DE for all lanes together, whatever part of the ray
// they are in (primary march, secant / binary search, normal samples,
// shadow march, bounce march), so the lanes stay converged in the DE, where
// the time goes.  Lanes whose item is done take new ones with a ballot and
// one warp-aggregated atomicAdd on the queue once enough of them are idle.
//
// Restated functions (src/mc.rs): seed_of 1107-1116, rand_of 472-475,
// halton_2d_shifts 131-142, Tracer::ray 2467-2627 (common camera, no
// salt, no depth of field, no cutting planes, no water), CalcRay 1904-2348
// (no reflections, transparency, material, clouds; the ambient bounce),
// McMarch::ray 665-865 with the 10-step binary search or the 4-step secant
// search and doBinSearchIt 588-643, McMarch::normals 533-585,
// surface_colour 647-662, McMarch::shadow without transparency 869-914,
// CalcHSMC 1513-1625 and CalcPhongLight 1699-1768 for global lights,
// CalcVisLights 1301-1401 without visible lights, CalcBGLight 1406-1510
// without a background picture, CalcColor 1250-1285 with the palette of
// LightVals (src/lighting.rs:1563-1614).
#pragma once
#include "devparams.h"
#include "marcher64.cuh"
#include "delock.cuh"
#include "mc.h"

namespace mb3dcu {

__device__ __forceinline__ int32_t mc_seed_of(int32_t x, int32_t y, uint32_t b) {
    auto mix = [](uint32_t h) {
        h ^= h >> 16;
        h *= 0x7FEB352Du;
        h ^= h >> 15;
        h *= 0x846CA68Bu;
        return h ^ (h >> 16);
    };
    return (int32_t)mix(((uint32_t)x * 0x9E3779B1u) ^ mix(((uint32_t)y * 0x85EBCA77u) ^ mix(b + 0x165667B1u)));
}
__device__ __forceinline__ int32_t mc_lcg(int32_t s) { return (int32_t)((uint32_t)s * 0x343FDu + 0x269EC3u); }
__device__ __forceinline__ double mc_rand(int32_t &seed) {
    seed = mc_lcg(seed);
    return (double)(seed & 0x7FFFFFFF) * (1.0 / 2147483647.0);
}
__device__ __forceinline__ float frac_s(float s) { return s - truncf(s); }
__device__ __forceinline__ void mc_normalize(const double a[3], double o[3]) {
    double l = sqrt(dot3d(a, a));
    if (l > 0.0) {
        double s = 1.0 / l;
        for (int k = 0; k < 3; k++) o[k] = a[k] * s;
    } else {
        for (int k = 0; k < 3; k++) o[k] = a[k];
    }
}
__device__ __forceinline__ void mc_norm_to(double n, const double v[3], double o[3]) {
    double d = n / sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + 1e-100);
    for (int k = 0; k < 3; k++) o[k] = v[k] * d;
}
__device__ __forceinline__ void mc_make_ortho(const double v[3], double o0[3], double o1[3]) {
    double n[3];
    mc_normalize(v, n);
    double a[3];
    if (fabs(n[0]) > 0.1) {
        double d = 1.0 / sqrt(n[0] * n[0] + n[2] * n[2]);
        a[0] = n[2] * d; a[1] = 0.0; a[2] = -n[0] * d;
    } else {
        double d = 1.0 / sqrt(n[1] * n[1] + n[2] * n[2]);
        a[0] = 0.0; a[1] = -n[2] * d; a[2] = n[1] * d;
    }
    for (int k = 0; k < 3; k++) o0[k] = (double)(float)a[k];
    double b[3] = {o0[1] * n[2] - o0[2] * n[1], o0[2] * n[0] - o0[0] * n[2], o0[0] * n[1] - o0[1] * n[0]};
    for (int k = 0; k < 3; k++) o1[k] = (double)(float)b[k];
}
__device__ __forceinline__ uint32_t mc_zpos_of(const DevParams &p, double zz) {
    double v = rint(p.zc_mul * (sqrt(fmax(zz, 0.0) * p.zcorr + 1.0) - 1.0));
    double d = clampd(8388352.0 - v, 0.0, 8388352.0);
    return (uint32_t)d << 8;
}

// RMdoColor (src/calc.rs:2068-2088) on the state of the last DE at c
__device__ __forceinline__ void mc_do_color(const DevParams &p, const DEstate &st, const double c[3], uint16_t &si_gradient,
                                            uint16_t &otrap) {
    const double PI = 3.14159265358979323846;
    double x = st.v[0], y = st.v[1], z = st.v[2], s;
    switch (p.color_option) {
        case 1: s = log(st.rout / (st.rold + 1.0)) * (double)p.mct_color_mul; break;
        case 2: s = (atan2(y - c[1], x - c[0]) + PI) * 5200.0; break;
        case 3: s = (atan2(z - c[2], x - c[0]) + PI) * 5200.0; break;
        case 4: s = (atan2(z - c[2], y - c[1]) + PI) * 5200.0; break;
        case 5: {
            s = (atan2(x, y) + PI) * 5215.0;
            double r = sqrt(x * x + y * y + 1e-100 + z * z);
            double s2 = (PI + asin(clampd(z / r, -1.0, 1.0)) * 2.0) * 5215.0;
            si_gradient = clip15((float)s2);
            break;
        }
        default: s = st.otrap * 4096.0; break;
    }
    otrap = clip15((float)s);
}

// The lane's phases: L_* run logic, W_* wait for the DE the lane asked for.
enum McPhase : int {
    L_IDLE = 0, L_RAY, L_CALC_RAY, L_MSTEP, L_SEC, L_BIS, L_BIT, L_BIT_END, L_NORM, L_NTRY, L_NSAMP, L_MHIT, L_MOPEN,
    L_LIGHT, L_SSTEP, L_SDONE, L_PHONG_END, L_RAY_END, L_ITEM_END,
    W_M0, W_MSTEP, W_SEC, W_BIS, W_BIT1, W_BIT2, W_N0, W_NK, W_S0, W_SSTEP,
    A_RAY, A_SHADOW  // (split render: the path waits for the march kernel's result)
};

// Everything one lane carries.
struct McLane {
    int phase;
    uint32_t item;
    // the DE the lane asks for
    double c[3];
    float ms;
    bool sit;
    int max_add;
    // the ray (Tracer)
    int x1, y, b;
    uint32_t pix;
    int32_t seed;
    double vfov[3], normals[3], dir[3];
    double mzz;
    bool hit, calc_amb_shadow, rit1, probe, aov;
    int rit, guard;
    float halton_x, halton_y, disc_x, disc_y;
    float tl[3], ta[3];
    uint32_t main_zpos;
    float t_dyn_fog, zpos_dyn_fog;
    // the march (kind 0, and the shadow march)
    double zz, zz2, zzplus, max_l, dtmp, rlast_de, rlast_sw, ds;
    float rsf, m_dyn_fog;
    bool first, de_limited;
    uint32_t mguard;
    int itmp, it_last;
    // doBinSearchIt
    double bdt1, bdmul, bzz0;
    float last_si, last_dif, yp;
    bool bfirst;
    // the normals
    double no, n[3], tsave;
    float nn, sca;
    int ntry, nq;
    uint16_t si_grad, otrap;
    // the surface of CalcRay
    double cc[3], hzz;
    float obj_spe[3], obj_dif[3];
    float bg_dec, d1;
    // the lights
    int li;
    float max_lhs, lsd[2][3];
    double dmaxl, sdir[3];
};

template <bool BATCH>
struct McRun {
    const DevParams &p;
    const McDev &m;
    __device__ McRun(const DevParams &pp, const McDev &mm) : p(pp), m(mm) {}

    __device__ __forceinline__ float de_stop(double zz) const {
        return (float)((double)p.de_stop * (1.0 + fabs(zz) * (double)p.de_stop_factor));
    }
    __device__ __forceinline__ void ask(McLane &L, int wait, bool sit = false, int max_add = 0) const {
        L.phase = wait;
        L.sit = sit;
        L.max_add = max_add;
    }

    // Tracer::ray's set-up of ray b of pixel (x1, y)
    __device__ void ray_begin(McLane &L) const {
        L.guard = 0;
        uint32_t act = L.b < 65535 ? (uint32_t)L.b : 65535u;
        L.seed = mc_seed_of(L.x1, L.y, (uint32_t)L.b);
        int32_t i = mc_lcg(L.x1), i2 = mc_lcg(L.y);
        int32_t t = (int32_t)(((uint32_t)L.x1 << 15) ^ (uint32_t)L.y ^ ((uint32_t)i << 9) ^ ((uint32_t)i2 << 5));
        t = mc_lcg(mc_lcg(t));
        float sx = (float)((double)(t & 0x7FFFFFFF) * (1.0 / 2147483647.0));
        t = mc_lcg(t);
        float sy = (float)((double)(t & 0x7FFFFFFF) * (1.0 / 2147483647.0));
        uint2 h = m.halton[act];
        const float D1D65535 = 1.0f / 65535.0f;
        L.halton_x = frac_s((float)(h.x & 0xFFFFu) * D1D65535 + sx);
        L.halton_y = frac_s((float)(h.x >> 16) * D1D65535 + sy);
        L.disc_x = frac_s((float)(h.y & 0xFFFFu) * D1D65535 + sx);
        L.disc_y = frac_s((float)(h.y >> 16) * D1D65535 + sy);
        L.main_zpos = 32768u << 16;
        float xx, yy;
        if (L.b < 4) {
            xx = (float)L.x1 - (float)(L.b & 1) * 0.5f - 0.75f;
            yy = (float)L.y + (float)(L.b & 2) * 0.25f - 0.25f;
        } else {
            float gx = (float)(mc_rand(L.seed) - 0.5), gy = (float)(mc_rand(L.seed) - 0.5);
            xx = gx + (float)L.x1 - 1.0f;
            yy = gy + (float)L.y;
        }
        double cafx = (double)((p.fovx_off - xx - 1.0f) * p.fovx_mul);
        double cafy = ((double)yy / (double)p.height - 0.5) * p.fov_y;
        double sx1, cx1, sy1, cy1;
        sincos(cafy, &sx1, &cx1);
        sincos(cafx, &sy1, &cy1);
        double v[3] = {-sy1, sx1, cx1 * cy1};
        double nv = 1.0 / sqrt(dot3d(v, v));
        for (int k = 0; k < 3; k++) v[k] *= nv;
        rot_rev(v, p.vgrads, L.vfov);
        for (int k = 0; k < 3; k++) L.c[k] = p.ystart[k] + p.vgrads[1][k] * (double)yy + p.vgrads[0][k] * (double)xx;
        for (int k = 0; k < 3; k++) {
            L.tl[k] = 0.0f;
            L.ta[k] = 1.0f;
            L.dir[k] = L.vfov[k];
        }
        L.calc_amb_shadow = false;
        L.rit1 = true;
        L.t_dyn_fog = 0.0f;
        L.hit = false;
        L.rit = 0;
        L.probe = true;
        L.zz = 0.0;
    }

    __device__ void surface_colour(McLane &L, const DEstate &st) const {
        float v = L.de_limited ? 32767.0f - (L.nn + p.d_col_plus + p.col_var * (float)log((double)L.ms * p.step_width)) * p.mcts_m
                               : 32767.0f - L.nn * p.mcts_m;
        L.si_grad = clip15(v);
        mc_do_color(p, st, L.c, L.si_grad, L.otrap);
    }

    // CalcBGLight without a background picture
    __device__ void bg_light(const McLane &L, const double vec[3], bool use_amb, float res[3]) const {
        const mb3d_cu_mc_light &lv = m.lv;
        double t0[3] = {dot3d(p.vgrads[0], vec), dot3d(p.vgrads[1], vec), dot3d(p.vgrads[2], vec)}, t[3];
        mc_normalize(t0, t);
        if (use_amb) {
            float d = (float)(t[1] * 0.5 + 0.5);
            for (int k = 0; k < 3; k++) res[k] = (lv.amb_col[k] + d * (lv.amb_col2[k] - lv.amb_col[k])) * (1.0f / 256.0f);
        } else {
            float d = L.rit1 ? (float)L.y / (float)p.height
                             : (float)clampd(asin(clampd(t[1], -1.0, 1.0)) * (double)m.fovy1d + 0.5, 0.0, 1.0);
            if (lv.depth_func == 1) d *= d;
            else if (lv.depth_func == 2) d = sqrtf(fmaxf(d, 0.0f));
            for (int k = 0; k < 3; k++)
                res[k] = (lv.depth_col[k] + d * (lv.depth_col2[k] - lv.depth_col[k])) * (1.0f / 256.0f);
        }
    }

    // CalcVisLights without visible lights
    __device__ void vis_lights(const McLane &L, const double view[3], uint32_t zpos_fine, float &bg_dec, float &depth_dec,
                               float res[3]) const {
        const mb3d_cu_mc_light &lv = m.lv;
        int32_t zp = (int32_t)(zpos_fine >> 16);
        float bgz = zp < 32768 ? fmaxf(1.0f + (float)(zp - 28000) * lv.s_depth, 0.0f)
                               : fmaxf(1.0f - (float)(60768 - zp) * lv.s_depth, 0.0f);
        if (bgz < 1.0f) {
            bgz = lv.sqr ? (1.0f - bgz) * (1.0f - bgz) : 1.0f - bgz;
            if (lv.far_fog) bgz *= bgz;
            bgz = 1.0f - bgz;
        }
        depth_dec = bgz;
        bg_dec = 1.0f;
        float svbg[3];
        bg_light(L, view, false, svbg);
        float dfog = (L.t_dyn_fog - lv.s_shad - lv.s_shad_zmul * L.zpos_dyn_fog) * lv.s_shad_gr;
        if (lv.dfog_options & 2) dfog = fmaxf(dfog, 0.0f);
        float stmp = fminf(L.t_dyn_fog * lv.s_dyn_fog_mul, 1.0f) * dfog;
        float w = fmaxf(1.0f - bgz, 0.0f);
        for (int k = 0; k < 3; k++) res[k] = 0.0f + svbg[k] * w;
        if (lv.dfog_options & 1) {
            dfog = fminf(fmaxf(dfog, 0.0f), 1.0f);
            stmp = fminf(fmaxf(stmp, 0.0f), 1.0f);
            for (int k = 0; k < 3; k++) res[k] = res[k] * (1.0f - dfog);
            depth_dec *= 1.0f - dfog;
        }
        float w1 = (dfog - stmp) / 255.0f, w2 = stmp / 255.0f;
        for (int k = 0; k < 3; k++) res[k] += lv.dyn_fog_col[k] * w1;
        for (int k = 0; k < 3; k++) res[k] += lv.dyn_fog_col2[k] * w2;
    }

    // CalcColor: the palette's specular and diffuse colours of the surface
    __device__ void calc_color(McLane &L, float z_pos) const {
        const mb3d_cu_mc_light &lv = m.lv;
        float idif0 = lv.s_col_zmul * z_pos;
        float irf = lv.col_on_otrap ? (float)(L.otrap & 0x7FFF) : (float)L.si_grad;
        float x = ((irf - lv.s_c_start) * lv.s_c_mul + idif0) * 16384.0f;
        x = fminf(fmaxf(x, -1e9f), 1e9f);
        int32_t ir = isnan(x) ? 0 : (int32_t)roundf(x);
        int a = -1, b = -1;
        float t = 0.0f;
        if (lv.col_cycling) ir &= 32767;
        else if (ir < 0) a = 0;
        else if (ir >= lv.col_pos[9]) a = 9;
        if (a < 0) {
            int il2 = 5;
            if (lv.col_pos[il2] < ir) {
                for (;;) {
                    il2 += 1;
                    if (il2 == 10 || lv.col_pos[il2] >= ir) break;
                }
            } else {
                while (il2 > 1 && lv.col_pos[il2 - 1] >= ir) il2 -= 1;
            }
            a = il2 - 1;
            if (!lv.no_col_ipol) {
                b = il2 > 9 ? 0 : il2;
                t = (float)(ir - lv.col_pos[a]) * lv.s_c_div[a];
            }
        }
        for (int k = 0; k < 3; k++) {
            if (b < 0) {
                L.obj_dif[k] = lv.col_dif[a][k];
                L.obj_spe[k] = lv.col_spe[a][k];
            } else {
                L.obj_dif[k] = lv.col_dif[a][k] + t * (lv.col_dif[b][k] - lv.col_dif[a][k]);
                L.obj_spe[k] = lv.col_spe[a][k] + t * (lv.col_spe[b][k] - lv.col_spe[a][k]);
            }
        }
    }

    // light i's terms of CalcPhongLight's second loop, shadow factor f
    __device__ void phong_add(McLane &L, int i, float f) const {
        const mb3d_cu_mc_light &lv = m.lv;
        const double sw = p.step_width;
        if (f == 0.0f) return;
        float l0[3];
        const double *t = m.hs_vecs[i];
        for (int k = 0; k < 3; k++) l0[k] = lv.col[i][k] * f;
        double nd = 2.0 * dot3d(L.normals, L.dir);
        double reflect[3] = {L.dir[0] - L.normals[0] * nd, L.dir[1] - L.normals[1] * nd, L.dir[2] - L.normals[2] * nd};
        float base = (float)(dot3d(reflect, t) * 1.0 / -(sw * sw));
        float sp = 0.0f;
        if (!(base < 0.0f)) {  // FastIntPow (src/math.rs:273-285)
            sp = base;
            for (int e = lv.pow_func[i] >> 1; e > 0; e >>= 1) sp *= sp;
        }
        sp = sp * lv.s_spec / 255.0f;
        for (int k = 0; k < 3; k++) L.lsd[0][k] += l0[k] * sp;
        float cs = (float)(dot3d(L.normals, t) / -sw);
        float mm = fmaxf(cs, 0.0f);
        float df = mm * mm * lv.s_diff / 255.0f;
        for (int k = 0; k < 3; k++) L.lsd[1][k] += l0[k] * df;
    }

    __device__ void put_res(const McLane &L, mb3d_cu_mc_res *res, int kind, const double pos[3], const double nrm[3],
                            double zz, double zz2, double len, float dyn_fog, float ms, uint16_t sg, uint16_t ot,
                            bool de_limited) const {
        mb3d_cu_mc_res &o = res[L.item];
        for (int k = 0; k < 3; k++) {
            o.pos[k] = pos[k];
            o.normals[k] = nrm[k];
        }
        o.zz = zz;
        o.zz2 = zz2;
        o.len = len;
        o.dyn_fog = dyn_fog;
        o.ms_de_stop = ms;
        o.seed = L.seed;
        o.si_grad = sg;
        o.otrap = ot;
        o.kind = (uint8_t)kind;
        o.de_limited = de_limited ? 1 : 0;
        o.inside = 0;
        o.pad = 0;
        o.pad2 = 0;
    }

    // Runs the lane's logic on the result r (st) of the DE it asked for,
    // up to the next DE it asks for (or the end of its item).
    __device__ __forceinline__ void advance(McLane &L, const DEr &r, const DEstate &st, McAcc &acc, mb3d_cu_mc_res *res) const {
        const double sw = p.step_width;
        const double zero3[3] = {0.0, 0.0, 0.0};
        for (int turn = 0; turn < 64; turn++) {
            switch (L.phase) {
            case L_RAY:
                if (BATCH) {  // (render logic: not in the march kernels)
                    L.phase = L_IDLE;
                    return;
                }
                ray_begin(L);
                L.phase = L_CALC_RAY;
                break;
            case L_CALC_RAY: {
                if (BATCH) {  // (render logic: not in the march kernels)
                    L.phase = L_IDLE;
                    return;
                }
                // CalcRay's entry
                if (fabsf(L.ta[0]) * 0.3f + fabsf(L.ta[1]) * 0.59f + fabsf(L.ta[2]) * 0.11f < 1e-4f) {
                    L.phase = L_RAY_END;
                    break;
                }
                L.guard += 1;
                if (L.guard > 4096) {
                    L.phase = L_RAY_END;
                    break;
                }
                if (L.calc_amb_shadow) {
                    double q = mc_rand(L.seed);
                    L.max_l = m.amb_max_l * (q * q + 0.75);
                } else {
                    L.max_l = p.zend;
                }
                L.rit += 1;
                L.rit1 = L.rit == 1;
                L.zz2 = L.rit1 ? L.zz : 0.0;
                L.bg_dec = 1.0f;
                L.zzplus = dot3d(L.dir, L.vfov) / (sw * sw);  // (the march starts at c)
                L.ms = de_stop(L.zz);
                ask(L, W_M0);
                return;
            }
            case W_M0:
                L.dtmp = r.de;
                if (L.probe && (r.it >= r.max_its || r.de < (double)L.ms)) {
                    // the start is inside the set
                    if (BATCH) {
                        uint16_t sg = 0, ot = 0;
                        mc_do_color(p, st, L.c, sg, ot);
                        if (p.color_option > 4) sg |= 32768;
                        else sg = (uint16_t)(32768 + (uint16_t)rint(32767.0 * clampd(st.rout / p.d_rstop, 0.0, 1.0)));
                        put_res(L, res, 2, L.c, zero3, 0.0, 0.0, 0.0, 0.0f, 0.0f, sg, ot, false);
                        L.phase = L_ITEM_END;
                    } else {
                        if (acc.counters) atomicAdd(&acc.counters[2], 1ull);
                        L.hit = true;  // (Tracer::ray takes the start inside for a hit)
                        for (int k = 0; k < 3; k++) L.tl[k] = 0.0f;
                        L.phase = L_RAY_END;
                    }
                    break;
                }
                L.m_dyn_fog = 0.0f;
                L.first = true;
                L.de_limited = true;
                L.rsf = 1.0f;
                L.rlast_sw = L.dtmp * (double)p.z_step_div;
                L.mguard = 0;
                L.it_last = r.it;
                L.phase = L_MSTEP;
                break;
            case L_MSTEP: {
                L.rlast_de = L.dtmp;
                double dstep = fmax((L.dtmp - (double)p.ms_de_sub * (double)L.ms) * (double)p.z_step_div * (double)L.rsf, 0.11);
                double d1 = (double)(fmaxf(L.ms, 0.4f) * p.mh04zsd);
                bool count = p.dfog_on_it == 0 || L.it_last == p.dfog_on_it;
                if (d1 < dstep) {
                    if (count) L.m_dyn_fog += (float)(d1 / dstep);
                    dstep = d1;
                } else if (count) {
                    L.m_dyn_fog += 1.0f;
                }
                if (L.first) {
                    L.first = false;
                    dstep *= mc_rand(L.seed);
                }
                L.rlast_sw = dstep;
                L.zz2 += dstep;
                if (L.zz2 > L.max_l) {
                    L.phase = L_MOPEN;
                    break;
                }
                add_w(L.c, L.dir, dstep);
                L.zz += dstep * L.zzplus;
                L.ms = de_stop(L.zz);
                ask(L, W_MSTEP);
                return;
            }
            case W_MSTEP:
                L.dtmp = r.de;
                L.it_last = r.it;
                if (r.it >= r.max_its) {
                    // doBinSearchIt on the iteration-limited surface
                    L.de_limited = false;
                    L.bzz0 = L.zz;
                    L.ds = L.zz;
                    L.bdt1 = 0.0;
                    L.bdmul = 1.0;
                    L.bfirst = true;
                    L.last_si = 0.0f;
                    L.last_dif = 0.0f;
                    L.yp = (float)p.max_it - 0.99f;
                    L.itmp = 10;
                    L.phase = L_BIT;
                    break;
                }
                if (!(L.dtmp >= (double)L.ms) && r.it >= p.min_it) {
                    if (m.secant) {
                        L.itmp = 4;
                        L.phase = L_SEC;
                    } else {
                        L.itmp = 10;
                        L.ds = L.rlast_sw * -0.5;
                        L.phase = L_BIS;
                    }
                    break;
                }
                if (L.dtmp > L.rlast_de + L.rlast_sw) L.dtmp = L.rlast_de + L.rlast_sw;
                if (L.rlast_de > L.dtmp + 1e-30) {
                    double d = L.rlast_sw / (L.rlast_de - L.dtmp);
                    L.rsf = d < 1.0 ? (float)fmax(d, 0.5) : 1.0f;
                } else {
                    L.rsf = 1.0f;
                }
                if (++L.mguard > 1000000u) {
                    L.phase = L_MOPEN;
                    break;
                }
                L.phase = L_MSTEP;
                break;
            case L_SEC: {
                if (!(L.itmp > 0 && fabs(L.dtmp - (double)L.ms) > 0.001)) {
                    L.phase = L_NORM;
                    break;
                }
                double nz = L.rlast_de - L.dtmp;
                if (fabs(nz) < 1e-40) nz = nz < 0.0 ? -1e-40 : 1e-40;
                L.rlast_de = nz;
                double f = L.rlast_sw * (L.dtmp - (double)L.ms) / L.rlast_de;
                if (L.dtmp < (double)L.ms)
                    L.rlast_sw = (f >= 0.0 || f < fabs(L.rlast_sw) * -0.94) ? fabs(L.rlast_sw) * -0.5 : f;
                else
                    L.rlast_sw = (f <= 0.0 || f > fabs(L.rlast_sw) * 0.94) ? fabs(L.rlast_sw) * 0.5 : f;
                L.rlast_de = L.dtmp;
                L.zz += L.rlast_sw * L.zzplus;
                add_w(L.c, L.dir, L.rlast_sw);
                L.ms = de_stop(L.zz);
                L.itmp -= 1;
                if (L.itmp <= 0) {
                    L.phase = L_NORM;
                    break;
                }
                ask(L, W_SEC);
                return;
            }
            case W_SEC:
                L.dtmp = r.de;
                L.phase = L_SEC;
                break;
            case L_BIS:
                if (!(fabs(L.dtmp - (double)L.ms) > 0.001)) {
                    L.phase = L_NORM;
                    break;
                }
                L.zz += L.ds * L.zzplus;
                add_w(L.c, L.dir, L.ds);
                L.ms = de_stop(L.zz);
                L.itmp -= 1;
                if (L.itmp <= 0) {
                    L.phase = L_NORM;
                    break;
                }
                ask(L, W_BIS);
                return;
            case W_BIS:
                L.dtmp = r.de;
                L.ds = L.dtmp < (double)L.ms ? fabs(L.ds) * -0.55 : fabs(L.ds) * 0.55;
                L.phase = L_BIS;
                break;
            case L_BIT:
                // doBinSearchIt's loop head: on by dt1, the DE with the smoothed count
                L.ds += L.bdt1;
                add_w(L.c, L.dir, L.bdt1);
                ask(L, W_BIT1, true, 1);
                return;
            case W_BIT1: {
                float s = st.smooth_it;
                if (!L.bfirst && L.last_dif < fabsf(L.yp - s)) {
                    L.ds -= L.bdt1;
                    add_w(L.c, L.dir, -L.bdt1);
                    s = L.last_si;
                    if (L.bdt1 > 0.0) L.bdmul *= 0.5;
                    else L.bdmul *= 0.7;
                }
                L.last_dif = fabsf(L.yp - s);
                L.last_si = s;
                if (s > (float)(p.max_it + 1) - 0.1f) {
                    L.bdt1 = -3.0;
                    L.bfirst = false;
                    L.itmp -= 1;
                    L.phase = L.itmp < 0 ? L_BIT_END : L_BIT;
                    break;
                }
                L.ds -= 0.001;
                add_w(L.c, L.dir, -0.001);
                ask(L, W_BIT2, true, 1);
                return;
            }
            case W_BIT2: {
                float s = st.smooth_it;
                float rr = L.last_si - s;
                double dt1;
                if (fabsf(rr) < 1e-30f) dt1 = (L.last_si < s ? 1.0 : 0.0) - 0.5;
                else if (rr < 0.0f) dt1 = (double)((L.yp - s) / (rr * 500.0f));
                else dt1 = (double)((L.yp - s) / (rr * 1000.0f));
                if (dt1 > 4.0) dt1 = sqrt(dt1) * 2.0;
                else if (dt1 < -9.0) dt1 = sqrt(-dt1) * -3.0;
                L.bdt1 = dt1 * L.bdmul + 0.0005;
                L.bfirst = false;
                L.itmp -= 1;
                L.phase = L.itmp < 0 ? L_BIT_END : L_BIT;
                break;
            }
            case L_BIT_END:
                // zz moves by the search's way times zzplus
                L.zz += (L.ds - L.bzz0) * L.zzplus;
                L.phase = L_NORM;
                break;
            case L_NORM:
                // McMarch::normals: the centre with the smoothed count
                L.mzz = fabs(L.zz);
                L.sca = (L.seed & 128) == 0 ? 0.15f : -0.15f;
                L.ntry = 4;
                ask(L, W_N0, true);
                return;
            case W_N0:
                L.no = r.de;
                L.nn = st.smooth_it;
                L.phase = L_NTRY;
                break;
            case L_NTRY:
                if (L.ntry < 4) L.sca = (float)((mc_rand(L.seed) - 0.5) * 0.5);
                L.nq = 0;
                L.phase = L_NSAMP;
                break;
            case L_NSAMP: {
                // the one-sided sample on axis k = 2, 0, 1 (q = 0, 1, 2)
                double off = (double)fminf(p.de_stop, 1.0f) * (1.0 + L.mzz * (double)p.de_stop_factor) * (double)L.sca * p.step_width;
                if (L.nq == 0) {
                    L.tsave = L.c[2];
                    L.c[2] = L.tsave + off;
                } else if (L.nq == 1) {
                    L.tsave = L.c[0];
                    L.c[0] = L.tsave + off;
                } else {
                    L.tsave = L.c[1];
                    L.c[1] = L.tsave + off;
                }
                ask(L, W_NK);
                return;
            }
            case W_NK: {
                double g = (r.de - L.no) * (double)L.sca;
                if (L.nq == 0) {
                    L.n[2] = g;
                    L.c[2] = L.tsave;
                } else if (L.nq == 1) {
                    L.n[0] = g;
                    L.c[0] = L.tsave;
                } else {
                    L.n[1] = g;
                    L.c[1] = L.tsave;
                }
                L.nq += 1;
                if (L.nq < 3) {
                    L.phase = L_NSAMP;
                    break;
                }
                double l = L.n[0] * L.n[0] + L.n[1] * L.n[1] + L.n[2] * L.n[2];
                if (l > 1e-100 && dot3d(L.n, L.dir) < 0.0) {
                    double s = 1.0 / sqrt(l);
                    for (int q = 0; q < 3; q++) L.normals[q] = L.n[q] * s;
                } else {
                    L.ntry -= 1;
                    if (L.ntry != 0) {
                        L.phase = L_NTRY;
                        break;
                    }
                    mc_norm_to(-1.0, L.dir, L.normals);
                }
                surface_colour(L, st);
                L.phase = L_MHIT;
                break;
            }
            case L_MOPEN:
                if (BATCH) {
                    put_res(L, res, 0, L.c, zero3, L.zz, L.zz2, 0.0, L.m_dyn_fog, 0.0f, 0, 0, false);
                    L.phase = L_ITEM_END;
                } else {
                    // CalcRay in open air: the background
                    L.t_dyn_fog = L.m_dyn_fog;
                    const mb3d_cu_mc_light &lv = m.lv;
                    L.zpos_dyn_fog = (float)(p.zend * sw + m.zz_stmit_dif);
                    uint32_t cr_zpos;
                    if ((lv.far_fog || lv.sqr) && fabsf(lv.s_depth) > 1e-10f) {
                        int32_t main_z = (int32_t)(L.main_zpos >> 16);
                        bool both = lv.far_fog && lv.sqr;
                        float e1 = 1.0f - fmaxf(1.0f + (float)(main_z - 28000) * lv.s_depth, 0.0f);
                        if (e1 > 0.0f) {
                            e1 *= e1;
                            if (both) e1 *= e1;
                        }
                        float e2 = 1.0f - fmaxf(1.0f - 28000.0f * lv.s_depth, 0.0f);
                        if (e2 > 0.0f) {
                            e2 *= e2;
                            if (both) e2 *= e2;
                        }
                        float e = e2 - e1;
                        if (e > 0.0f) {
                            e = sqrtf(e);
                            if (both) e = sqrtf(e);
                        }
                        cr_zpos = (uint32_t)rintf(fminf(fmaxf(60768.0f - e / lv.s_depth, 32768.0f), 65535.0f)) << 16;
                    } else {
                        cr_zpos = 32768u << 16;
                    }
                    if (L.rit1) L.main_zpos = cr_zpos;
                    float rsf = 0.0f, sv[3], bgl[3];
                    vis_lights(L, L.dir, cr_zpos, L.bg_dec, rsf, sv);
                    bg_light(L, L.dir, L.calc_amb_shadow, bgl);
                    L.bg_dec *= rsf;
                    for (int k = 0; k < 3; k++) sv[k] += bgl[k] * L.bg_dec;
                    for (int k = 0; k < 3; k++) L.tl[k] = L.tl[k] + sv[k] * L.ta[k];
                    L.phase = L_RAY_END;
                }
                break;
            case L_MHIT:
                if (BATCH) {
                    put_res(L, res, 1, L.c, L.normals, L.zz, L.zz2, 0.0, L.m_dyn_fog, L.ms, L.si_grad, L.otrap, L.de_limited);
                    L.phase = L_ITEM_END;
                } else {
                    // CalcRay on a surface, up to the lights
                    L.t_dyn_fog = L.m_dyn_fog;
                    L.hit = true;
                    L.mzz = fabs(L.zz);
                    for (int k = 0; k < 3; k++) L.cc[k] = L.c[k];
                    uint32_t cr_zpos = mc_zpos_of(p, L.zz2);
                    if (L.rit1) L.main_zpos = cr_zpos;
                    calc_color(L, (float)(L.mzz * sw + m.zz_stmit_dif));
                    if (L.rit1 && L.aov) {
                        L.aov = false;
                        if (acc.albedo)
                            for (int k = 0; k < 3; k++) acc.albedo[3 * L.pix + k] = L.obj_dif[k];
                        if (acc.normal)
                            for (int k = 0; k < 3; k++) acc.normal[3 * L.pix + k] = (float)L.normals[k];
                        if (acc.depth) acc.depth[L.pix] = (float)(L.zz * sw);
                    }
                    L.zpos_dyn_fog = (float)(L.zz2 * sw + m.zz_stmit_dif);
                    float sv[3];
                    vis_lights(L, L.dir, cr_zpos, L.bg_dec, L.d1, sv);
                    for (int k = 0; k < 3; k++) L.tl[k] = L.tl[k] + sv[k] * L.ta[k];
                    float bd = L.bg_dec * L.d1;
                    for (int k = 0; k < 3; k++) L.ta[k] = L.ta[k] * bd;
                    L.hzz = L.zz;
                    L.mzz = L.zz;
                    for (int a = 0; a < 2; a++)
                        for (int k = 0; k < 3; k++) L.lsd[a][k] = 0.0f;
                    float zzf = (float)fabs(L.mzz);
                    L.max_lhs = m.hs_max_lmul * (1.0f + 0.5f * fminf(zzf, (float)p.zend * 0.4f) * fmaxf((float)p.fov_y, 0.0f) / (float)p.height);
                    L.li = 0;
                    L.phase = L_LIGHT;
                }
                break;
            case L_LIGHT: {
                if (BATCH) {  // (render logic: not in the march kernels)
                    L.phase = L_IDLE;
                    return;
                }
                if (L.li >= m.lv.n_lights) {
                    L.phase = L_PHONG_END;
                    break;
                }
                const int i = L.li;
                // the light vector jittered on the light's disc (CalcPhongLight)
                double stmp = (double)L.disc_x, s1 = (double)L.disc_y;
                double sn, cs;
                sincos(2.0 * 3.14159265358979323846 * s1, &sn, &cs);
                double d = sqrt(stmp) * sqrt((double)m.lv.lmax_l[i]) * 2.5e-5 * (double)m.soft_shadow_radius * sw;
                double o0[3], o1[3];
                mc_make_ortho(m.hs_vecs[i], o0, o1);
                double v[3], hj[3];
                for (int q = 0; q < 3; q++) v[q] = m.hs_vecs[i][q] + (double)((float)(o0[q] * sn * d) + (float)(o1[q] * cs * d));
                mc_norm_to(sw, v, hj);
                // CalcHSMC for this light
                double dt1 = (double)L.max_lhs;
                for (int q = 0; q < 3; q++) L.sdir[q] = -hj[q];
                if (dt1 <= 0.001) {
                    phong_add(L, i, 1.0f);
                    L.li += 1;
                    break;
                }
                if (dot3d(L.normals, L.sdir) < 0.0) {
                    L.li += 1;
                    break;
                }
                L.zzplus = dot3d(L.sdir, L.vfov) / sqrt(dot3d(L.sdir, L.sdir) * dot3d(L.vfov, L.vfov));
                L.dmaxl = dt1;
                L.max_l = dt1;  // the shadow ray's length left
                L.zz2 = L.hzz;
                L.zz = (double)(float)fabs(L.hzz);
                for (int q = 0; q < 3; q++) L.c[q] = L.cc[q];
                L.ms = de_stop(L.zz);
                ask(L, W_S0);
                return;
            }
            case W_S0:
                L.dtmp = r.de;
                L.rsf = 2.0f;
                L.mguard = 0;
                L.phase = L_SSTEP;
                break;
            case L_SSTEP: {
                L.rlast_de = L.dtmp;
                double st1 = fmin(L.dtmp * (double)p.z_step_div * (double)L.rsf, (double)(fmaxf(L.ms, 0.4f) * p.mh04zsd));
                L.rlast_sw = st1;
                L.max_l -= st1;
                add_w(L.c, L.sdir, st1);
                L.zz2 += st1 * L.zzplus;
                L.ms = de_stop(L.zz2);
                ask(L, W_SSTEP);
                return;
            }
            case W_SSTEP:
                L.dtmp = r.de;
                if (r.it >= r.max_its || !(L.dtmp >= (double)L.ms) || !(L.dtmp < 1e30)) {
                    L.phase = L_SDONE;
                    break;
                }
                if (L.dtmp > L.rlast_de + L.rlast_sw) L.dtmp = L.rlast_de + L.rlast_sw;
                if (L.rlast_de > L.dtmp + 1e-30) {
                    double s = L.rlast_sw / (L.rlast_de - L.dtmp);
                    L.rsf = s < 1.0 ? (float)fmax(s, 0.5) : 1.0f;
                } else {
                    L.rsf = 1.0f;
                }
                if (!(L.max_l >= 0.0) || ++L.mguard > 1000000u) {
                    L.phase = L_SDONE;
                    break;
                }
                L.phase = L_SSTEP;
                break;
            case L_SDONE:
                if (BATCH) {
                    put_res(L, res, 0, zero3, zero3, 0.0, 0.0, L.max_l, 0.0f, 0.0f, 0, 0, false);
                    L.phase = L_ITEM_END;
                } else {
                    double dt1 = L.max_l;
                    float f = 1.0f;
                    if (dt1 > 0.01) {
                        float x = (float)((L.dmaxl - dt1) / (double)L.max_lhs);
                        float a = x * x, a2 = a * a;
                        f = fminf(a2 * a2, 1.0f);
                    }
                    phong_add(L, L.li, f);
                    L.li += 1;
                    L.phase = L_LIGHT;
                }
                break;
            case L_PHONG_END: {
                if (BATCH) {  // (render logic: not in the march kernels)
                    L.phase = L_IDLE;
                    return;
                }
                const float ws = (0.25f + 1.0f) * 0.8f;
                for (int k = 0; k < 3; k++) {
                    float spec = (L.obj_spe[k] * ws) * L.lsd[0][k];
                    float diff = (L.obj_dif[k] * 1.0f) * L.lsd[1][k];
                    L.tl[k] = L.tl[k] + (spec + diff) * L.ta[k];
                }
                if (L.d1 > 1.0f)
                    for (int k = 0; k < 3; k++) L.ta[k] = L.ta[k] * (1.0f / L.d1);
                if (!(L.rit < m.max_amb_depth || !L.calc_amb_shadow)) {
                    L.phase = L_RAY_END;
                    break;
                }
                // the ambient bounce: Halton on the first surface, random after
                double a, ml;
                if (!L.calc_amb_shadow) {
                    a = 2.0 * 3.14159265358979323846 * (double)L.halton_x;
                    ml = (double)L.halton_y;
                } else {
                    a = 2.0 * 3.14159265358979323846 * mc_rand(L.seed);
                    ml = mc_rand(L.seed);
                }
                double sa, ca;
                sincos(a, &sa, &ca);
                double d4s = (double)(float)sa, d3c = (double)(float)ca;
                double dd = sqrt(ml);
                double o0[3], o1[3];
                mc_make_ortho(L.normals, o0, o1);
                double w = sqrt(1.0 - ml);
                double nv[3];
                for (int k = 0; k < 3; k++)
                    nv[k] = (double)((float)(o0[k] * d3c * dd) + (float)(o1[k] * d4s * dd)) + L.normals[k] * w;
                mc_norm_to(sw, nv, L.dir);
                for (int k = 0; k < 3; k++) L.c[k] = L.cc[k];
                L.calc_amb_shadow = true;
                for (int k = 0; k < 3; k++) L.ta[k] = L.ta[k] * (L.obj_dif[k] * 1.0f);
                L.probe = false;
                L.zz = L.hzz;
                L.phase = L_CALC_RAY;
                break;
            }
            case L_RAY_END:
                if (!BATCH) {  // (render logic: not in the march kernels)
                    // the ray's light into its pixel's sum
                    float svs[3];
                    for (int k = 0; k < 3; k++) {
                        float sv = fminf(fmaxf(L.tl[k], 0.0f), 400.0f);
                        svs[k] = sv;
                        unsigned long long q = (unsigned long long)rint((double)sv * 4294967296.0);
                        if (q) atomicAdd(&acc.sum[3 * L.pix + k], q);
                    }
                    if (acc.ysum) {
                        // YofSVec (src/svec.rs:38-40), unfused single precision
                        const float yl = fmaxf(__fadd_rn(__fadd_rn(__fmul_rn(svs[0], 0.3f), __fmul_rn(svs[1], 0.59f)),
                                                         __fmul_rn(svs[2], 0.11f)),
                                               0.0f);
                        const double yv = (double)yl;
                        const unsigned long long q1 = (unsigned long long)rint(yv * 4294967296.0);
                        const unsigned long long q2 = (unsigned long long)rint(yv * yv * 16777216.0);
                        if (q1) atomicAdd(&acc.ysum[2 * L.pix], q1);
                        if (q2) atomicAdd(&acc.ysum[2 * L.pix + 1], q2);
                    }
                    if (L.hit) atomicOr(&acc.hit[L.pix], 1u);
                }
                L.phase = L_IDLE;
                return;
            case L_ITEM_END:
            default:
                L.phase = L_IDLE;
                return;
            }
        }
        // (no logic chain takes this many turns; end the item)
        L.phase = L_IDLE;
    }
};

// The persistent kernel.  BATCH: the items are the march requests `reqs`
// (results into `res`); else item i is ray ray0 + i / npad of pixel i % npad
// (8x4 tiles), so that neighbouring lanes trace neighbouring pixels.
// the double precision DE where single precision cannot resolve it: out of
// line in the single precision kernel (rare; keeps the loop's code small)
template <int FM>
__device__ __noinline__ DEr mc_de64(const DevParams &p, double c0, double c1, double c2, float ms, DEstate *st, bool sit,
                                    int max_add) {
    const double c[3] = {c0, c1, c2};
    return de_lock<double, FM, false, true>(p, c, ms, nullptr, st, sit, max_add);
}

#ifndef MB3D_MC_MIN_BLOCKS
#define MB3D_MC_MIN_BLOCKS 6  // (the whole C5 frame at 4 rays: 5 blocks 201.2 ms, 6 196.4, 7 205.4, 8 214.0)
#endif
template <typename R, int FM, bool BATCH>
__global__ void __launch_bounds__(128, MB3D_MC_MIN_BLOCKS) k_mc(const __grid_constant__ DevParams p, const __grid_constant__ McDev m,
                                            McAcc acc, const mb3d_cu_mc_req *reqs, mb3d_cu_mc_res *res,
                                            unsigned int *queue, uint32_t n_items, const uint32_t *list) {
    McRun<BATCH> run(p, m);
    McLane L;
    L.phase = L_IDLE;
    bool open = true;
    unsigned long long evals = 0, its = 0, fb = 0;
    DEr r;
    r.de = 0.0;
    r.it = 0;
    r.max_its = p.max_it;
    r.need64 = false;
    DEstate st;
    st.rout = 0.0; st.rold = 0.0; st.otrap = 0.0;
    st.v[0] = 0.0; st.v[1] = 0.0; st.v[2] = 0.0;
    st.smooth_it = 0.0f;
    const bool single = sizeof(R) == 4 && !p.all_fp64;
    for (;;) {
        uint32_t item = warp_take(L.phase == L_IDLE, queue, n_items, p.refill_min, open);
        if (item != UINT32_MAX) {
            L.item = item;
            if (BATCH) {
                if (list) L.item = list[item];  // (the split render: a path's slot)
                const mb3d_cu_mc_req &q = reqs[L.item];
                for (int k = 0; k < 3; k++) L.c[k] = q.pos[k];
                L.seed = q.seed;
                L.zz = q.zz;
                L.zz2 = q.zz2;
                L.zzplus = q.zzplus;
                L.max_l = q.len;
                L.ms = run.de_stop(L.zz);
                L.sit = false;
                L.max_add = 0;
                if (q.kind == 0) {
                    for (int k = 0; k < 3; k++) L.dir[k] = q.dir[k];
                    L.probe = q.probe != 0;
                    L.phase = W_M0;
                } else {
                    for (int k = 0; k < 3; k++) L.sdir[k] = q.dir[k];
                    L.phase = W_S0;
                }
            } else {
                if (m.items) {
                    const uint2 it = m.items[item];
                    L.pix = it.x;
                    L.x1 = m.x0 + (int)(it.x % (uint32_t)m.w) + 1;
                    L.y = m.y0 + (int)(it.x / (uint32_t)m.w);
                    L.b = (int)it.y;
                    L.aov = false;
                    L.phase = L_RAY;
                } else {
                    uint32_t within = item % m.npad;
                    int x, ly;
                    item_pixel(within, (int)m.tiles_x, x, ly);
                    if (x < m.w && ly < m.h) {
                        L.pix = (uint32_t)ly * (uint32_t)m.w + (uint32_t)x;
                        L.x1 = m.x0 + x + 1;
                        L.y = m.y0 + ly;
                        L.b = m.ray0 + (int)(item / m.npad);
                        L.aov = L.b == m.ray0;
                        L.phase = L_RAY;  // (its logic runs below, its first DE on the next trip)
                    }
                }
            }
        }
        unsigned int busy = __ballot_sync(0xffffffffu, L.phase != L_IDLE);
        if (busy == 0) {
            if (!open) break;
            continue;
        }
        const bool wants = L.phase >= W_M0 && L.phase <= W_SSTEP;
        if (wants) {
            if (single) {
                r = de_lock<float, FM, false, true>(p, L.c, L.ms, nullptr, &st, L.sit, L.max_add);
                if (r.need64) {
                    r = mc_de64<FM>(p, L.c[0], L.c[1], L.c[2], L.ms, &st, L.sit, L.max_add);
                    fb++;
                }
            } else {
                r = de_lock<double, FM, false, true>(p, L.c, L.ms, nullptr, &st, L.sit, L.max_add);
            }
            evals++;
            its += (unsigned long long)r.it;
        }
        if (L.phase != L_IDLE) run.advance(L, r, st, acc, res);
    }
    if (acc.counters) {
        atomicAdd(&acc.counters[0], evals);
        atomicAdd(&acc.counters[1], its);
        if (fb) atomicAdd(&acc.counters[3], fb);
    }
}

#ifdef MB3D_MC_COMMON
// The split render's logic: every path (one per slot, its state in `lanes`)
// takes in the result of its last march, runs Tracer::ray's logic up to
// its next march, writes that march's request into its slot and puts the
// slot on the march list; a path whose ray ended takes the next ray item
// (warp-aggregated atomicAdd on `next`), so the slots stay full.
__global__ void __launch_bounds__(128) k_mc_logic(const __grid_constant__ DevParams p, const __grid_constant__ McDev m,
                                                  McAcc acc, McLane *lanes, mb3d_cu_mc_req *reqs,
                                                  const mb3d_cu_mc_res *res, uint32_t n_slots, unsigned int *next,
                                                  uint32_t n_items, uint32_t *list, unsigned int *n_list) {
    McRun<false> run(p, m);
    DEr r;
    r.de = 0.0;
    r.it = 0;
    r.max_its = p.max_it;
    r.need64 = false;
    DEstate st;
    st.rout = 0.0; st.rold = 0.0; st.otrap = 0.0;
    st.v[0] = 0.0; st.v[1] = 0.0; st.v[2] = 0.0;
    st.smooth_it = 0.0f;
    const int lane = threadIdx.x & 31;
    for (uint32_t base = blockIdx.x * blockDim.x; base < n_slots; base += gridDim.x * blockDim.x) {
        const uint32_t slot = base + threadIdx.x;
        const bool mine = slot < n_slots;
        McLane L;
        L.phase = L_IDLE;
        bool queued = false;
        if (mine) {
            L = lanes[slot];
            if (L.phase == A_RAY) {
                const mb3d_cu_mc_res &o = res[slot];
                L.seed = o.seed;
                if (o.kind == 2) {
                    if (acc.counters) atomicAdd(&acc.counters[2], 1ull);
                    L.hit = true;  // (Tracer::ray takes the start inside for a hit)
                    for (int k = 0; k < 3; k++) L.tl[k] = 0.0f;
                    L.phase = L_RAY_END;
                } else {
                    for (int k = 0; k < 3; k++) L.c[k] = o.pos[k];
                    L.zz = o.zz;
                    L.zz2 = o.zz2;
                    L.m_dyn_fog = o.dyn_fog;
                    if (o.kind == 1) {
                        for (int k = 0; k < 3; k++) L.normals[k] = o.normals[k];
                        L.ms = o.ms_de_stop;
                        L.si_grad = o.si_grad;
                        L.otrap = o.otrap;
                        L.de_limited = o.de_limited != 0;
                        L.phase = L_MHIT;
                    } else {
                        L.phase = L_MOPEN;
                    }
                }
            } else if (L.phase == A_SHADOW) {
                L.max_l = res[slot].len;
                L.phase = L_SDONE;
            }
        }
        // the logic up to the next march; a finished ray takes the next item
        for (int turn = 0; turn < 8; turn++) {
            bool want_item = mine && L.phase == L_IDLE;
            unsigned int ask = __ballot_sync(0xffffffffu, want_item);
            if (ask) {
                int leader = __ffs(ask) - 1;
                uint32_t b0 = 0;
                if (lane == leader) b0 = atomicAdd(next, (unsigned int)__popc(ask));
                b0 = __shfl_sync(0xffffffffu, b0, leader);
                if (want_item) {
                    uint32_t item = b0 + (uint32_t)__popc(ask & ((1u << lane) - 1u));
                    if (item < n_items) {
                        if (m.items) {
                            const uint2 it = m.items[item];
                            L.pix = it.x;
                            L.x1 = m.x0 + (int)(it.x % (uint32_t)m.w) + 1;
                            L.y = m.y0 + (int)(it.x / (uint32_t)m.w);
                            L.b = (int)it.y;
                            L.aov = false;
                            L.item = item;
                            L.phase = L_RAY;
                        } else {
                            uint32_t within = item % m.npad;
                            int x, ly;
                            item_pixel(within, (int)m.tiles_x, x, ly);
                            if (x < m.w && ly < m.h) {
                                L.pix = (uint32_t)ly * (uint32_t)m.w + (uint32_t)x;
                                L.x1 = m.x0 + x + 1;
                                L.y = m.y0 + ly;
                                L.b = m.ray0 + (int)(item / m.npad);
                                L.aov = L.b == m.ray0;
                                L.item = item;
                                L.phase = L_RAY;
                            }
                        }
                        // (a padding item outside the rectangle: the slot asks again)
                    } else {
                        want_item = false;
                        L.phase = L_IDLE;  // (no rays left: the slot stays empty)
                        L.item = UINT32_MAX;
                    }
                }
            }
            if (mine && L.phase != L_IDLE && L.phase != W_M0 && L.phase != W_S0) run.advance(L, r, st, acc, nullptr);
            bool more = mine && L.phase == L_IDLE && L.item != UINT32_MAX;
            if (!__any_sync(0xffffffffu, more)) break;
        }
        if (mine) {
            mb3d_cu_mc_req &q = reqs[slot];
            if (L.phase == W_M0) {
                for (int k = 0; k < 3; k++) {
                    q.pos[k] = L.c[k];
                    q.dir[k] = L.dir[k];
                }
                q.zz = L.zz; q.zz2 = L.zz2; q.zzplus = L.zzplus; q.len = L.max_l;
                q.seed = L.seed; q.kind = 0; q.probe = L.probe ? 1 : 0; q.inside = 0; q.pad = 0;
                L.phase = A_RAY;
                queued = true;
            } else if (L.phase == W_S0) {
                for (int k = 0; k < 3; k++) {
                    q.pos[k] = L.c[k];
                    q.dir[k] = L.sdir[k];
                }
                q.zz = L.zz; q.zz2 = L.zz2; q.zzplus = L.zzplus; q.len = L.max_l;
                q.seed = L.seed; q.kind = 1; q.probe = 0; q.inside = 0; q.pad = 0;
                L.phase = A_SHADOW;
                queued = true;
            }
            lanes[slot] = L;
        }
        unsigned int qm = __ballot_sync(0xffffffffu, queued);
        if (qm) {
            int leader = __ffs(qm) - 1;
            uint32_t b0 = 0;
            if (lane == leader) b0 = atomicAdd(n_list, (unsigned int)__popc(qm));
            b0 = __shfl_sync(0xffffffffu, b0, leader);
            if (queued) list[b0 + (uint32_t)__popc(qm & ((1u << lane) - 1u))] = slot;
        }
    }
}

// the records: the mean light of each pixel's rays, and the hit flags
__global__ void k_mc_final(McAcc acc, uint32_t npix, int rays, float *radiance, uint8_t *hit) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        for (int k = 0; k < 3; k++)
            radiance[3 * i + k] = (float)((double)acc.sum[3 * i + k] / 4294967296.0 / (double)rays);
        if (hit) hit[i] = acc.hit[i] ? 1 : 0;
    }
}
#endif

}  // namespace mb3dcu
