// The double precision marcher on the device: the per-pixel state machine
// of mb3d-rs's CPU march (Marcher, src/calc.rs:1142-2980; the hybrid loops
// of src/iteration.rs:137-574), one thread per ray.  It is the plain FP64
// drop-in, and the finish stage of the mixed-precision march (the surface
// re-check, the binary search, normals, colour and depth of every hit).
// Single precision parts of the reference (the DE stop, colour values) keep
// their single precision; their divisions are written as __fdiv_rn so that
// they stay IEEE in any build.
#pragma once
#include "devparams.h"
#include "formulas.cuh"

namespace mb3dcu {

struct G {  // one G-buffer record in registers (SiLight)
    short n0, n1, n2;
    unsigned int zpos_fine;
    unsigned short shadow, amb_shadow, si_gradient, otrap;
    __device__ void clear() {
        n0 = n1 = n2 = 0;
        zpos_fine = 32768u << 16;
        shadow = amb_shadow = si_gradient = otrap = 0;
    }
    __device__ void load(const mb3d_cu_silight &s) {
        n0 = s.normal[0];
        n1 = s.normal[1];
        n2 = s.normal[2];
        zpos_fine = s.zpos_fine;
        shadow = s.shadow;
        amb_shadow = s.amb_shadow;
        si_gradient = s.si_gradient;
        otrap = s.otrap;
    }
    __device__ void store(mb3d_cu_silight *d) const {
        uint32_t *w = reinterpret_cast<uint32_t *>(d);
        w[0] = (uint32_t)(uint16_t)n0 | ((uint32_t)(uint16_t)n1 << 16);
        w[1] = (uint32_t)(uint16_t)n2;
        w[2] = zpos_fine;
        w[3] = (uint32_t)shadow | ((uint32_t)amb_shadow << 16);
        w[4] = (uint32_t)si_gradient | ((uint32_t)otrap << 16);
    }
    __device__ unsigned int zpos() const { return zpos_fine >> 16; }
};

__device__ __forceinline__ uint16_t clip15(float s) {  // MinMaxClip15bit
    if (isnan(s) || s < 0.0f) return 0;
    if (s > 32767.0f) return 32767;
    return (uint16_t)rintf(s);
}
__device__ __forceinline__ uint16_t sat_u16d(double x) {
    if (isnan(x) || x <= 0.0) return 0;
    if (x >= 65535.0) return 65535;
    return (uint16_t)x;
}
__device__ __forceinline__ long long sat_i64d(double x) {
    if (isnan(x)) return 0;
    if (x >= 9.2e18) return 9200000000000000000LL;
    if (x <= -9.2e18) return -9200000000000000000LL;
    return (long long)x;
}
__device__ __forceinline__ double clampd(double x, double lo, double hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
__device__ __forceinline__ void add_w(double a[3], const double b[3], double w) {
    a[0] += b[0] * w;
    a[1] += b[1] * w;
    a[2] += b[2] * w;
}
__device__ __forceinline__ double dot3d(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ void rot_rev(const double v[3], const double m[3][3], double o[3]) {
    double r0 = v[0] * m[0][0] + v[1] * m[1][0] + v[2] * m[2][0];
    double r1 = v[0] * m[0][1] + v[1] * m[1][1] + v[2] * m[2][1];
    double r2 = v[0] * m[0][2] + v[1] * m[1][2] + v[2] * m[2][2];
    o[0] = r0;
    o[1] = r1;
    o[2] = r2;
}

// RMCalculateVgradsFOV + RMCalculateStartPos (src/calc.rs:1561-1573,
// 1673-1689) for the common camera: the start of the ray of pixel (x, y) and
// its direction, one step width long.
__device__ __forceinline__ void pixel_ray(const DevParams &p, int x, int y, double c[3], double vf[3]) {
    double cafy = ((double)y / (double)p.height - 0.5) * p.fov_y;
    double cafx = (double)((p.fovx_off - (float)(x + 1)) * p.fovx_mul);
    double sx, cx, sy, cy;
    sincos(cafy, &sx, &cx);
    sincos(cafx, &sy, &cy);
    double v[3] = {-sy, sx, cx * cy};
    double n = 1.0 / sqrt(dot3d(v, v));
    v[0] *= n;
    v[1] *= n;
    v[2] *= n;
    rot_rev(v, p.vgrads, vf);
    double xd = x, yd = y;
    for (int k = 0; k < 3; k++) c[k] = p.ystart[k] + p.vgrads[0][k] * xd + p.vgrads[1][k] * yd;
}

// the iteration record (TIteration3Dext, src/iteration.rs:57-105); FM is
// the formula set the kernel is built for
template <int FM>
struct It64 {
    // (j's fourth component: the Quaternion's, only in the all-formula kernels)
    double v[4], c[3], j[FM == FKIND_ALL ? 4 : 3];
    double rout, rold, otrap, rstop;
    int it_result, max_it;
    bool calc_sit;
    // the second part of a DE combination is set (set_part, src/calc.rs:1476-1489):
    // its slot range and DE option (only the all-formula kernels meet one)
    bool part2;
    float smooth_it;

    __device__ void smooth_iterations(const DevParams &p, int n) {  // CalcSmoothIterations
        if (rout <= 1.0) {
            smooth_it = (float)it_result;
        } else if (rold < 1.0) {
            double d = log(log(rout) * 0.5) * (double)p.fhln[n];
            smooth_it = (float)((double)it_result + (double)p.ln_rstop - d);
        } else {
            double d = log(0.5 * log(rout));
            double e = d - log(0.5 * log(rold));
            smooth_it = (float)(((double)p.ln_rstop - d) / (e + 1e-100) + (double)it_result);
        }
    }
    // run_with (src/iteration.rs:268-313)
    __device__ int run(const DevParams &p) {
        int n = 0, end = p.end_to, rep = p.repeat_from;
        if constexpr (FM == FKIND_ALL) {
            if (part2) {
                n = p.dc_start2;
                end = p.dc_end2;
                rep = p.dc_rep2;
            }
        }
        int btmp = p.slots[n].iterations;
        it_result = 0;
        unsigned int unc_guard = 0;
        for (;;) {
            rold = rout;
            int guard = 0;
            while (btmp <= 0) {
                n += 1;
                if (n > end) n = rep;
                btmp = p.slots[n].iterations;
                if (++guard > 64) return n;
            }
            const DevSlot &s = p.slots[n];
            formula_iterate<double, FM, FM == FKIND_ALL>(s, v, j, rout);
            if (s.julia_add) {
                v[0] += j[0];
                v[1] += j[1];
                v[2] += j[2];
            }
            btmp -= 1;
            if (s.uncounted) {
                if (++unc_guard > 100000) return n;
                continue;
            }
            it_result += 1;
            // (4D hybrids hold a Quaternion: only the all-formula kernels meet them)
            if (FM == FKIND_ALL && p.four_d) rout = v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + v[3] * v[3];
            else rout = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
            if (rout < otrap) otrap = rout;
            if (it_result >= max_it || rout > rstop) return n;
        }
    }
    __device__ void start(const DevParams &p) {
        if (p.do_julia) {
            j[0] = p.ju[0];
            j[1] = p.ju[1];
            j[2] = p.ju[2];
        } else {
            j[0] = c[0];
            j[1] = c[1];
            j[2] = c[2];
        }
        if constexpr (FM == FKIND_ALL) j[3] = p.ju[3];
        v[0] = c[0];
        v[1] = c[1];
        v[2] = c[2];
        rout = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
        otrap = rout;
    }
    // doHybrid4DPas (src/iteration.rs:757-772): the point turned into 4D
    // (Rotate4Dex, src/math.rs:209-215), the hybrid on four components
    __device__ void hybrid_4d(const DevParams &p) {
        if constexpr (FM != FKIND_ALL) return;
        double v4[4];
        for (int i = 0; i < 4; i++) v4[i] = c[0] * p.smatrix4[i][0] + c[1] * p.smatrix4[i][1] + c[2] * p.smatrix4[i][2];
        for (int k = 0; k < 4; k++) {
            v[k] = v4[k];
            if constexpr (FM == FKIND_ALL) j[k] = p.do_julia ? p.ju[k] : v4[k];
        }
        rout = v4[0] * v4[0] + v4[1] * v4[1] + v4[2] * v4[2] + v4[3] * v4[3];
        otrap = rout;
        if (p.ipol) {  // doInterpolHybridPas4D (src/iteration.rs:457-464)
            it_result = ipol_run<double, FM>(p, v, j, rout, rold, otrap, max_it, rstop, false);
            if (calc_sit) smooth_iterations(p, 0);
            return;
        }
        int n = run(p);
        if (calc_sit) smooth_iterations(p, n);
    }
    __device__ void hybrid_3d(const DevParams &p) {  // doHybridPas; doInterpolHybridPas; a 4D hybrid
        if (FM == FKIND_ALL && p.four_d) {
            hybrid_4d(p);
            return;
        }
        start(p);
        v[3] = 0.0;
        if constexpr (FM == FKIND_ALL) {
            if (p.ipol) {
                it_result = ipol_run<double, FM>(p, v, j, rout, rold, otrap, max_it, rstop, false);
                if (calc_sit) smooth_iterations(p, 0);
                return;
            }
        }
        int n = run(p);
        if (calc_sit) smooth_iterations(p, n);
    }
    __device__ double hybrid_3d_de(const DevParams &p) {  // doHybridPasDE
        start(p);
        if constexpr (FM == FKIND_ALL) {
            if (p.ipol) {  // doInterpolHybridPasDE (src/iteration.rs:441-455)
                v[3] = ((p.de_option & 0x18) == 16) ? rout : 1.0;
                it_result = ipol_run<double, FM>(p, v, j, rout, rold, otrap, max_it, rstop, true);
                const double w = v[3];
                const double r = ((p.de_option & 7) == 4) ? fabs(v[2]) * log(fabs(v[2])) / w : sqrt(rout) / fabs(w);
                if (calc_sit) smooth_iterations(p, 0);
                return r;
            }
        }
        int deo = p.de_option;
        if constexpr (FM == FKIND_ALL) deo = part2 ? p.dc_de_option2 : deo;
        v[3] = ((deo & 0x38) == 16) ? rout : 1.0;
        int n = run(p);
        double w = v[3];
        double r = ((deo & 7) == 4) ? fabs(v[1]) * log(fabs(v[1])) / w : sqrt(rout) / fabs(w);
        if (calc_sit) smooth_iterations(p, n);
        return r;
    }
};

// calc_de_part (src/calc.rs:1495-1557) of the part the record is set to,
// outside rendering: the analytic DE or the numerical one (the offsets'
// runs to the centre's iteration count), at least a quarter of the DE stop;
// `max_its` takes the iteration limit of the part (max_its_result)
template <int FM>
__device__ __forceinline__ double de_part(const DevParams &p, It64<FM> &it, float ms_de_stop, bool custom,
                                          float d_de_scale, int &max_its) {
    double result;
    if (custom) {
        result = it.hybrid_3d_de(p) * (double)d_de_scale;
    } else {
        it.hybrid_3d(p);
        if (it.rout < 1e-200) {
            result = 0.0;
        } else {
            const bool bsit = it.calc_sit;
            const int bmax = it.max_it;
            const double brout = it.rout;
            it.calc_sit = false;
            it.max_it = it.it_result;
            it.rstop = p.rstop3d;
            double g = 0.0;
            for (int k = 0; k < 3; k++) {
                const double b = it.c[k];
                it.c[k] = b + (double)p.de_offset;
                it.hybrid_3d(p);
                g += (brout - it.rout) * (brout - it.rout);
                it.c[k] = b;
            }
            result = brout * log(brout) * (double)d_de_scale / (sqrt(g) + (double)p.de_offset006);
            it.rout = brout;
            it.it_result = it.max_it;
            it.max_it = bmax;
            it.calc_sit = bsit;
            it.rstop = p.d_rstop;
        }
    }
    max_its = it.max_it;
    const double mn = (double)ms_de_stop * 0.25;
    if (result < mn || isnan(result)) result = mn;
    return result;
}

// A DE combination (CalcDEfull with FormulaType > 0, src/calc.rs:1369-1455):
// part 1's distance, then part 2's in its own place (PrepareF1DEcomb and
// set_part), combined by min, max, max of the inverted part 2 or one of
// the smooth minima; the colour values and the iteration limit are the
// ruling part's (the smooth minima blend the colour values by distance).
// Part 1's iteration limit holds afterwards (RestoreF1DEcomb: it.max_it is
// the scene's again, which the iteration count search reads back).
template <int FM>
__device__ __noinline__ double de_comb(const DevParams &p, It64<FM> &it, float ms_de_stop, int &max_its) {
    it.part2 = false;
    double result = de_part<FM>(p, it, ms_de_stop, p.is_custom_de != 0, p.d_de_scale, max_its);
    const int b_it = it.it_result, b_max = max_its;
    const double b_otrap = it.otrap;
    const float b_sit = it.smooth_it;
    it.part2 = true;
    it.max_it = p.dc_max_it2;
    const double c0[3] = {it.c[0], it.c[1], it.c[2]};
    if (p.dc_place) {
        const double d[3] = {c0[0] - p.dc_offset[0], c0[1] - p.dc_offset[1], c0[2] - p.dc_offset[2]};
        for (int i = 0; i < 3; i++) it.c[i] = p.dc_m[i][0] * d[0] + p.dc_m[i][1] * d[1] + p.dc_m[i][2] * d[2];
    }
    const int kind = p.dc_kind;
    const double ms = (double)ms_de_stop;
    double rst = de_part<FM>(p, it, ms_de_stop, p.dc_custom2 != 0, p.dc_d_de_scale2, max_its);
    if (kind == 3) {  // the part "inside" (bCalcInside)
        rst = ms * 4.0 - rst * 3.0;
        if (rst >= ms) it.it_result -= 1;
    }
    if (p.dc_place) {
        rst *= p.dc_scale;
        for (int i = 0; i < 3; i++) it.c[i] = c0[i];
    }
    bool restore = false;
    if (kind == 1) {
        if (rst >= result) restore = true;
        else result = rst;
    } else if (kind == 2 || kind == 3) {
        if (rst > result) result = rst;
        else restore = true;
    } else {  // 4, 5: smooth minima
        if (!(rst < result)) {
            it.it_result = b_it;
            max_its = b_max;
        }
        const double sm = p.dc_smooth;
        if (kind == 4) {
            result = fmin(rst - fmax(sm - result, 0.0), result - fmax(sm - rst, 0.0));
        } else {
            const double rd1 = fmax(sm - result - ms, 0.0);
            const double d2 = fmax(sm - rst - ms, 0.0);
            result = fmin(rst - rd1 * (sm - d2) / sm, result - d2 * (sm - rd1) / sm);
        }
        const double r2 = fabs(rst), w = fabs(result);
        const double f = 1.0 / (w + r2 + 1e-10);
        it.smooth_it = (float)(((double)it.smooth_it * w + (double)b_sit * r2) * f);
        it.otrap = (it.otrap * w + b_otrap * r2) * f;
    }
    if (restore) {
        it.it_result = b_it;
        it.smooth_it = b_sit;
        it.otrap = b_otrap;
        max_its = b_max;
    }
    it.part2 = false;
    it.max_it = p.max_it;
    return result;
}

template <int FM>
struct M64 {
    const DevParams &p;
    It64<FM> it;
    float ms_de_stop;
    double mzz;
    double vfov[3];
    int max_its_result;
    float s_roughness;
    int seed;
    int add_steps;  // binary search steps (the march's; 8 for shadows, 5 for DE AO)

    __device__ M64(const DevParams &pp) : p(pp) {
        add_steps = p.de_add_steps;
        it.max_it = p.max_it;
        it.rstop = p.d_rstop;
        it.calc_sit = false;
        it.part2 = false;
        it.rout = it.rold = it.otrap = 0.0;
        it.smooth_it = 0.f;
        it.it_result = 0;
        for (int k = 0; k < 4; k++) it.v[k] = 0.0;
        ms_de_stop = p.de_stop;
        mzz = 0.0;
        max_its_result = p.max_it;
        s_roughness = 0.f;
        seed = 0;
    }

    // calc_de -> calc_de_part (src/calc.rs:1333-1557), one hybrid part
    __device__ double calc_de() {
        if constexpr (FM == FKIND_ALL) {
            if (p.dc_kind) return de_comb<FM>(p, it, ms_de_stop, max_its_result);
        }
        double result;
        if (p.is_custom_de) {
            result = it.hybrid_3d_de(p) * (double)p.d_de_scale;
        } else {
            it.hybrid_3d(p);
            if (it.rout < 1e-200) {
                result = 0.0;
            } else {
                bool bsit = it.calc_sit;
                int bmax = it.max_it;
                double brout = it.rout;
                it.calc_sit = false;
                it.max_it = it.it_result;
                it.rstop = p.rstop3d;
                double off = (double)p.de_offset;
                double g = 0.0, gk[3];
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    double b = it.c[k];
                    it.c[k] = b + off;
                    it.hybrid_3d(p);
                    gk[k] = (brout - it.rout) * (brout - it.rout);
                    it.c[k] = b;
                }
                g = gk[0] + gk[1] + gk[2];
                result = brout * log(brout) * (double)p.d_de_scale / (sqrt(g) + (double)p.de_offset006);
                it.rout = brout;
                it.it_result = it.max_it;
                it.max_it = bmax;
                it.calc_sit = bsit;
                it.rstop = p.d_rstop;
            }
        }
        max_its_result = it.max_it;
        double mn = (double)ms_de_stop * 0.25;
        if (result < mn || isnan(result)) result = mn;
        return result;
    }

    __device__ void step(double d) { add_w(it.c, vfov, d); }
    __device__ void update_de_stop() { ms_de_stop = (float)((double)p.de_stop * (1.0 + mzz * (double)p.de_stop_factor)); }

    // RMdoBinSearch (src/calc.rs:1706-1734)
    __device__ void bin_search(double &de, double last_step_width) {
        int itmp = add_steps;
        double dt1 = last_step_width * -0.5;
        while (fabs(de - (double)ms_de_stop) > 0.001) {
            mzz += dt1;
            step(dt1);
            update_de_stop();
            if (--itmp <= 0) break;
            de = calc_de();
            if (it.it_result >= max_its_result) {
                dt1 = -fabs(dt1);
                continue;
            }
            dt1 = (de - (double)ms_de_stop) < 0.0 ? fabs(dt1) * -0.55 : fabs(dt1) * 0.55;
        }
    }

    // RMdoBinSearchIt (src/calc.rs:1737-1791)
    __device__ void bin_search_it() {
        float yp = (float)it.max_it - 0.99f;
        int saved = it.max_it;
        it.max_it += 1;
        int itmp = add_steps;
        it.calc_sit = true;
        double dt1 = 0.0, dmul = 1.0;
        bool first = true;
        float last_si = 0.f, last_dif = 0.f;
        for (;;) {
            mzz += dt1;
            step(dt1);
            calc_de();
            if (!first && last_dif < fabsf(yp - it.smooth_it)) {
                mzz -= dt1;
                step(-dt1);
                it.smooth_it = last_si;
                dmul *= dt1 > 0.0 ? 0.5 : 0.7;
            }
            last_dif = fabsf(yp - it.smooth_it);
            last_si = it.smooth_it;
            if (it.smooth_it > (float)it.max_it - 0.1f) {
                dt1 = -3.0;
            } else {
                mzz -= 0.001;
                step(-0.001);
                calc_de();
                float r = last_si - it.smooth_it;
                if (fabsf(r) < 1e-30f) dt1 = (last_si < it.smooth_it ? 1.0 : 0.0) - 0.5;
                else if (r < 0.0f) dt1 = (double)__fdiv_rn(yp - it.smooth_it, r * 500.0f);
                else dt1 = (double)__fdiv_rn(yp - it.smooth_it, r * 1000.0f);
                if (dt1 > 4.0) dt1 = sqrt(dt1) * 2.0;
                else if (dt1 < -9.0) dt1 = sqrt(-dt1) * -3.0;
                dt1 = dt1 * dmul + 0.0005;
            }
            first = false;
            if (--itmp < 0) break;
        }
        it.max_it = saved;
    }

    __device__ static __forceinline__ void store_normal(G &si, const double n[3]) {  // MakeWNormalsFromDVec
        double d = 32767.0 / sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2] + 1e-100);
        short o[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double v = rint(n[k] * d);
            o[k] = isnan(v) ? 0 : (short)clampd(v, -32767.0, 32767.0);
        }
        if (o[0] == 0 && o[1] == 0) o[2] = o[2] > 0 ? 32767 : -32767;
        si.n0 = o[0];
        si.n1 = o[1];
        si.n2 = o[2];
    }

    // RMCalculateNormals (src/calc.rs:1813-1906)
    __device__ float calculate_normals(G &si) {
        const double(&vg)[3][3] = p.vgrads;
        it.calc_sit = true;
        double noffset = (double)fminf(p.de_stop, 1.0f) * (1.0 + mzz * (double)p.de_stop_factor) * 0.15;
        double ct[3] = {it.c[0], it.c[1], it.c[2]};
        double dnn = calc_de();
        float nn = it.smooth_it;
        it.calc_sit = false;
        double n[3] = {0.0, 0.0, 0.0};
        if (p.sm_normals == 8) {
            double ssn = noffset * 1.3333;
            for (int a = -2; a <= 2; a++)
                for (int b = -2; b <= 2; b++)
                    for (int c = -2; c <= 2; c++) {
                        if ((a | b | c) == 0) continue;
                        it.c[0] = ct[0]; it.c[1] = ct[1]; it.c[2] = ct[2];
                        add_w(it.c, vg[2], a * ssn);
                        add_w(it.c, vg[1], b * ssn);
                        add_w(it.c, vg[0], c * ssn);
                        double d = calc_de();
                        if (a != 0) n[2] += d / a;
                        if (b != 0) n[1] += d / b;
                        if (c != 0) n[0] += d / c;
                    }
            n[0] *= 0.0075; n[1] *= 0.0075; n[2] *= 0.0075;
        } else {
#pragma unroll
            for (int q = 0; q < 3; q++) {
                const int k = q == 0 ? 2 : q - 1;  // z, x, y
                it.c[0] = ct[0]; it.c[1] = ct[1]; it.c[2] = ct[2];
                add_w(it.c, vg[k], noffset);
                double a = calc_de();
                add_w(it.c, vg[k], -2.0 * noffset);
                n[k] = (a - calc_de()) * 0.5;
            }
        }
        if (p.sm_normals > 0) {
            noffset *= 2.0;
            if (p.sm_normals < 8) {
                it.c[0] = ct[0]; it.c[1] = ct[1]; it.c[2] = ct[2];
                add_w(it.c, vg[0], -noffset);
                dnn += calc_de();
                add_w(it.c, vg[0], 2.0 * noffset);
                dnn += calc_de();
                it.c[0] = ct[0]; it.c[1] = ct[1]; it.c[2] = ct[2];
                add_w(it.c, vg[1], -noffset);
                dnn += calc_de();
                add_w(it.c, vg[1], 2.0 * noffset);
                dnn = (dnn + calc_de()) * 0.2;
            }
            int sm = p.sm_normals;
            double ssn = noffset * 3.0 / ((double)sm + 0.5);
            double dm = (double)sm * 2.0;
            // CreateXYVecsFromNormals (src/math.rs:218-233)
            double vx0[3], vy0[3];
            double dd0 = n[1] * n[1] + n[0] * n[0];
            if (dd0 < 1e-50) {
                vx0[0] = 1; vx0[1] = 0; vx0[2] = 0;
                vy0[0] = 0; vy0[1] = 1; vy0[2] = 0;
            } else {
                double a = acos(clampd(-n[2] / sqrt(dd0 + n[2] * n[2] + 1e-100), -1.0, 1.0)) * 0.5;
                double sa, ca;
                sincos(a, &sa, &ca);
                sa /= sqrt(dd0);
                double e = -n[1] * sa, d1 = n[0] * sa;
                vx0[0] = 1.0 - 2.0 * d1 * d1; vx0[1] = 2.0 * e * d1; vx0[2] = 2.0 * d1 * ca;
                vy0[0] = vx0[1]; vy0[1] = 1.0 - 2.0 * e * e; vy0[2] = -2.0 * e * ca;
            }
            double vx[3], vy[3];
            rot_rev(vx0, vg, vx);
            rot_rev(vy0, vg, vy);
            double sums[2][2];
            for (int w = 0; w < 2; w++) {
                const double *dir = w == 0 ? vx : vy;
                it.c[0] = ct[0]; it.c[1] = ct[1]; it.c[2] = ct[2];
                add_w(it.c, dir, -(double)sm * ssn);
                double s1 = 0.0, ds = 0.0;
                for (int k = -sm; k <= sm; k++) {
                    if (k != 0) {
                        double d = (calc_de() - dnn) / (double)k;
                        s1 += d;
                        ds += d * d;
                    }
                    add_w(it.c, dir, ssn);
                }
                sums[w][0] = s1;
                sums[w][1] = ds;
            }
            double dsg = sums[0][1] * dm - sums[0][0] * sums[0][0] + sums[1][1] * dm - sums[1][0] * sums[1][0];
            double dt2 = noffset * 0.5 / (dm * ssn);
            double ra = (dsg * 7.0 * dt2 * dt2 + 1e-40) / (n[0] * n[0] + n[1] * n[1] + n[2] * n[2] + 1e-40);
            s_roughness = (float)clampd(sqrt(fmax(ra, 0.0)) - 0.05, 0.0, 1.0);
            if (p.sm_normals < 8) {
                n[0] += sums[0][0] * dt2;
                n[1] += sums[1][0] * dt2;
            }
        }
        it.c[0] = ct[0]; it.c[1] = ct[1]; it.c[2] = ct[2];
        store_normal(si, n);
        return nn;
    }

    // RMCalculateNormalsOnSmoothIt (src/calc.rs:1910-2006), unsmoothed
    __device__ float calculate_normals_on_smooth_it(G &si) {
        const double(&vg)[3][3] = p.vgrads;
        double noffset = (double)fminf(p.de_stop, 1.0f) * (1.0 + mzz * (double)p.de_stop_factor) * 0.15;
        it.calc_sit = true;
        double ct[3] = {it.c[0], it.c[1], it.c[2]};
        it.hybrid_3d(p);
        float nn = it.smooth_it;
        double n[3] = {0.0, 0.0, 0.0};
        for (int q = 0; q < 3; q++) {
            const int k = q == 0 ? 2 : q - 1;
            it.c[0] = ct[0]; it.c[1] = ct[1]; it.c[2] = ct[2];
            add_w(it.c, vg[k], noffset);
            it.hybrid_3d(p);
            double a = (double)it.smooth_it;
            add_w(it.c, vg[k], -2.0 * noffset);
            it.hybrid_3d(p);
            n[k] = ((double)it.smooth_it - a) * 0.5;
        }
        it.c[0] = ct[0]; it.c[1] = ct[1]; it.c[2] = ct[2];
        store_normal(si, n);
        return nn;
    }

    __device__ void do_color_on_it() {  // doColorOnIt
        if (p.color_on_it == 1) {
            it.v[0] = it.c[0]; it.v[1] = it.c[1]; it.v[2] = it.c[2];
        } else {
            int i = it.max_it;
            it.max_it = p.color_on_it - 1;
            it.rstop = p.rstop3d;
            calc_de();
            it.max_it = i;
            it.rstop = p.d_rstop;
        }
    }

    __device__ void do_color(G &si) {  // RMdoColor (src/calc.rs:2068-2088)
        const double PI = 3.14159265358979323846;
        double x = it.v[0], y = it.v[1], z = it.v[2];
        double s;
        switch (p.color_option) {
            case 1: s = log(it.rout / (it.rold + 1.0)) * (double)p.mct_color_mul; break;
            case 2: s = (atan2(y - it.c[1], x - it.c[0]) + PI) * 5200.0; break;
            case 3: s = (atan2(z - it.c[2], x - it.c[0]) + PI) * 5200.0; break;
            case 4: s = (atan2(z - it.c[2], y - it.c[1]) + PI) * 5200.0; break;
            case 5: {
                s = (atan2(x, y) + PI) * 5215.0;
                double r = sqrt(x * x + y * y + 1e-100 + z * z);
                double s2 = (PI + asin(clampd(z / r, -1.0, 1.0)) * 2.0) * 5215.0;
                si.si_gradient = clip15((float)s2);
                break;
            }
            default: s = it.otrap * 4096.0; break;
        }
        si.otrap = clip15((float)s);
    }

    __device__ void calc_zpos_and_rough(G &si) {  // CalcZposAndRough
        double zz = fmax(mzz, 0.0);
        long long v = sat_i64d(rint(p.zc_mul * (sqrt(zz * p.zcorr + 1.0) - 1.0)));
        long long d = 8388352LL - v;
        if (d < 0) d = 0;
        if (d > 8388352) d = 8388352;
        unsigned int r = (unsigned int)d << 8;
        if (p.sm_normals > 0) r |= (unsigned int)sat_u16d(rint((double)(s_roughness * 255.0f))) & 0xFF;
        si.zpos_fine = r;
    }

    // surface_found (src/calc.rs:2471-2511)
    __device__ void surface_found(G &si, double dtmp, double last_step) {
        bool de_limited = it.it_result < max_its_result || dtmp < (double)ms_de_stop;
        if (add_steps != 0) {
            if (de_limited) bin_search(dtmp, last_step);
            else bin_search_it();
        }
        float nn = p.normals_on_de ? calculate_normals(si) : calculate_normals_on_smooth_it(si);
        float v;
        if (de_limited) {
            float l = (float)log((double)fmaxf(p.de_stop, ms_de_stop) * p.step_width);
            v = 32767.0f - (nn + p.d_col_plus + p.col_var * l) * p.mcts_m;
        } else {
            v = 32767.0f - nn * p.mcts_m;
        }
        si.si_gradient = clip15(v);
        if (p.color_on_it != 0) do_color_on_it();
        do_color(si);
        calc_zpos_and_rough(si);
    }

    // the start-inside branch of march_pixel_from (src/calc.rs:2279-2298)
    __device__ void start_inside(G &si) {
        if (p.color_on_it != 0) do_color_on_it();
        si.zpos_fine = 0x7FFF0000u;
        si.n0 = 0; si.n1 = 0; si.n2 = -32767;
        do_color(si);
        if (p.color_option > 4) {
            si.si_gradient |= 32768;
        } else {
            double t = clampd(it.rout / p.d_rstop, 0.0, 1.0);
            si.si_gradient = (uint16_t)(32768 + sat_u16d(rint(32767.0 * t)));
        }
    }

    // march_from (src/calc.rs:2533-2655), from the state (dtmp, last_step,
    // rsf_mul, first_step, step_count) so that the mixed march can hand a
    // ray over to it in the middle (after_half: the state is right after the
    // half step back, whose DE decides without another one)
    __device__ void march_from(G &si, double dtmp, double last_step, float rsf_mul, bool first_step, float step_count,
                               bool after_half = false) {
        double last_de;
        unsigned int guard = 0;
        for (;;) {
            if (++guard > 2000000u) break;
            bool half = !after_half && it.it_result >= max_its_result;
            after_half = false;
            if (half) {
                double dt1 = -0.5 * last_step;
                mzz += dt1;
                step(dt1);
                update_de_stop();
                dtmp = calc_de();
                last_step = -dt1;
            }
            if (it.it_result < p.min_it || (it.it_result < max_its_result && dtmp >= (double)ms_de_stop)) {
                last_de = dtmp;
                double d = fmax(0.11, (dtmp - (double)p.ms_de_sub * (double)ms_de_stop) * (double)p.z_step_div * (double)rsf_mul);
                double s1 = (double)(fmaxf(ms_de_stop, 0.4f) * p.mh04zsd);
                bool count = p.dfog_on_it == 0 || it.it_result == p.dfog_on_it;
                if (s1 < d) {
                    if (count) step_count += (float)(s1 / d);
                    d = s1;
                } else if (count) {
                    step_count += 1.0f;
                }
                if (first_step) {
                    first_step = false;
                    seed = (int)((unsigned int)seed * 214013u + 2531011u);
                    d *= (double)(seed & 0x7FFFFFFF) * (1.0 / 2147483647.0);
                }
                mzz += d;
                if (mzz > p.zend) break;
                last_step = d;
                step(d);
                update_de_stop();
                dtmp = calc_de();
                if (dtmp > last_de + last_step) dtmp = last_de + last_step;
                if (last_de > dtmp + 1e-30) {
                    double t = last_step / (last_de - dtmp);
                    rsf_mul = t < 1.0 ? (float)fmax(0.5, t) : 1.0f;
                } else {
                    rsf_mul = 1.0f;
                }
            } else {
                surface_found(si, dtmp, last_step);
                break;
            }
        }
        float sc = step_count;
        if (sc < 0.0f) sc = 0.0f;
        if (sc > 1023.0f) sc = 1023.0f;
        si.shadow = (uint16_t)rintf(sc);
    }

    // march_pixel (src/calc.rs:2207-2318), outside rendering
    __device__ void march_pixel(G &si, int x, int y) {
        si.clear();
        si.amb_shadow = 5000;
        pixel_ray(p, x, y, it.c, vfov);
        it.calc_sit = false;
        mzz = 0.0;
        ms_de_stop = p.de_stop;
        double dtmp = calc_de();
        if (it.it_result >= max_its_result || dtmp < (double)ms_de_stop) {
            start_inside(si);
            return;
        }
        march_from(si, dtmp, dtmp * (double)p.z_step_div, 1.0f, p.first_step_random != 0, 0.0f);
    }

    // where the post passes start: the stored depth's position
    // (src/calc.rs:2750-2753, 2166-2170)
    __device__ void at_stored_depth(int x, int y, const G &si, double &zf) {
        pixel_ray(p, x, y, it.c, vfov);
        zf = (double)(si.zpos_fine >> 8);
        double q = (8388351.5 - zf) / p.zc_mul + 1.0;
        mzz = (q * q - 1.0) / p.zcorr;
        add_w(it.c, vfov, mzz);
        update_de_stop();
    }

    // hs_surface_start (src/calc.rs:2741-2764)
    __device__ bool hs_surface_start(int x, int y, const G &si) {
        if (si.zpos() >= 32768 || si.si_gradient >= 32768) return false;
        it.calc_sit = false;
        double zf;
        at_stored_depth(x, y, si, zf);
        double d = calc_de();
        bool de_limited = it.it_result < max_its_result || d < (double)ms_de_stop;
        if (de_limited) {
            double q2 = (8388351.9 - zf) / p.zc_mul + 1.0;
            bin_search(d, (q2 * q2 - 1.0) / p.zcorr - mzz);
        } else {
            bin_search_it();
        }
        return true;
    }

    // surface_point (src/calc.rs:2157-2191)
    __device__ bool surface_point(int x, int y, const G &si, int steps, double thr) {
        if (si.zpos() >= 32768 || si.si_gradient >= 32768) return false;
        it.calc_sit = false;
        double zf;
        at_stored_depth(x, y, si, zf);
        double d = fmin(calc_de(), (double)ms_de_stop * 2.0);
        if (it.it_result < max_its_result || d < (double)ms_de_stop) {
            double q2 = (8388351.9 - zf) / p.zc_mul + 1.0;
            double dt1 = (q2 * q2 - 1.0) / p.zcorr - mzz;
            int itmp = steps;
            while (itmp > 0 && fabs(d - (double)ms_de_stop) > thr) {
                mzz += dt1;
                add_w(it.c, vfov, dt1);
                update_de_stop();
                itmp -= 1;
                if (itmp > 0) {
                    d = calc_de();
                    dt1 = d < (double)ms_de_stop ? fabs(dt1) * -0.55 : fabs(dt1) * 0.55;
                }
            }
        } else {
            bin_search_it();
            ms_de_stop = (float)((double)p.de_stop * (1.0 + fabs(mzz) * (double)p.de_stop_factor));
        }
        return true;
    }

    // MaxLHS (src/calc.rs:2767-2773)
    __device__ double hs_max_len(int y) {
        float a = (float)(p.width + y) * 0.6f;
        float b = 1.0f + __fdiv_rn(0.5f * (float)fmin(mzz, p.zend * 0.4) * (float)fmax(p.fov_y, 0.0), (float)p.height);
        return (double)(a * b * p.hs_max_len_mul);
    }
};

}  // namespace mb3dcu
