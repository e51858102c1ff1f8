// TEST INFRASTRUCTURE — the Monte Carlo oracle: a C++ restatement of
// mb3d-rs's Monte Carlo renderer (src/mc.rs) for the scenes the card's
// tracer takes: global lights that are not visible, no reflections,
// transparency, cutting planes, depth of field, volumetric light, water,
// clouds, background picture, surface material or detail; rays that start
// inside the set are left dark.  Single precision (`f32`) values of the
// reference stay `float` here, with -ffp-contract=off as the reference's
// unfused arithmetic.  Each function cites the reference it restates.
//
// The records: the mean of the rays' light (clamped to 0..400,
// src/mc.rs:2799), summed per pixel in 32.32 fixed point so that the card,
// which takes the rays of a pixel in any order, sums exactly the same; the
// reference's running average (src/mc.rs:2805-2826) agrees with it to the
// last bits of single precision for a fixed number of rays.
//
// Parity pinning: the reference keeps no known-answer test of the Monte
// Carlo renderer that runs without its own binary, so this restatement is
// pinned through the march it shares with the Calculate 3D oracle (the DE,
// oracle.cpp) and through the tests' own checks of its pieces (the seed
// hash, the Halton numbers, the light values); image-level parity against
// mb3d-rs itself is unpinned.
#include "oracle.hpp"
#include <cstring>
#include <thread>
#include <vector>

namespace oracle {

static const double PIc = 3.14159265358979323846;
static const double SEED_MUL = 1.0 / 2147483647.0;  // src/mc.rs:34
static const float D1D65535 = 1.0f / 65535.0f;      // src/mc.rs:35

// seed_of (src/mc.rs:1107-1116)
int32_t mc_seed_of(int32_t x, int32_t y, uint32_t b) {
    auto mix = [](uint32_t h) {
        h ^= h >> 16;
        h *= 0x7FEB352Du;
        h ^= h >> 15;
        h *= 0x846CA68Bu;
        return h ^ (h >> 16);
    };
    return (int32_t)mix(((uint32_t)x * 0x9E3779B1u) ^ mix(((uint32_t)y * 0x85EBCA77u) ^ mix(b + 0x165667B1u)));
}

// rand_of / Tracer::rand (src/mc.rs:472-475, 1177-1180)
static inline double rand_of(int32_t &seed) {
    seed = wrap_lcg(seed, 0x343FDu, 0x269EC3u);
    return (double)(seed & 0x7FFFFFFF) * SEED_MUL;
}

// halton / halton_seq (src/mc.rs:103-128)
static double halton(int32_t index, int32_t base) {
    double r = 0.0, f = 1.0 / (double)base, d = f;
    int32_t i = index;
    while (i > 0) {
        r += f * (double)(i % base);
        i = sat_i32(std::trunc((double)i * d));
        f *= d;
    }
    return r;
}
struct HaltonRec {
    uint16_t hrx, hry, hdx, hdy;
};
static const std::vector<HaltonRec> &halton_seq() {
    static std::vector<HaltonRec> h = [] {
        std::vector<HaltonRec> t(65536);
        for (int i = 0; i < 65536; i++) {
            auto q = [&](int b) { return (uint16_t)rte(halton(i + 1, b) * 65535.0); };
            t[i] = HaltonRec{q(2), q(3), q(5), q(7)};
        }
        return t;
    }();
    return h;
}

// halton_2d_shifts (src/mc.rs:131-142)
static void halton_2d_shifts(int32_t x, int32_t y, float &s1, float &s2) {
    int32_t i = wrap_lcg(x, 0x343FDu, 0x269EC3u);
    int32_t i2 = wrap_lcg(y, 0x343FDu, 0x269EC3u);
    int32_t t = (int32_t)(((uint32_t)x << 15) ^ (uint32_t)y ^ ((uint32_t)i << 9) ^ ((uint32_t)i2 << 5));
    t = wrap_lcg(t, 0x343FDu, 0x269EC3u);
    t = wrap_lcg(t, 0x343FDu, 0x269EC3u);
    s1 = (float)((double)(t & 0x7FFFFFFF) * SEED_MUL);
    t = wrap_lcg(t, 0x343FDu, 0x269EC3u);
    s2 = (float)((double)(t & 0x7FFFFFFF) * SEED_MUL);
}

static inline float frac_s(float s) { return s - std::trunc(s); }

// normalize (src/math.rs:50-57)
static inline void normalize3(const double a[3], double o[3]) {
    double l = std::sqrt(dot3(a, a));
    if (l > 0.0) {
        double s = 1.0 / l;
        for (int k = 0; k < 3; k++) o[k] = a[k] * s;
    } else {
        for (int k = 0; k < 3; k++) o[k] = a[k];
    }
}

// norm_to (src/svec.rs:53-56)
static inline void norm_to(double n, const double v[3], double o[3]) {
    double d = n / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + 1e-100);
    for (int k = 0; k < 3; k++) o[k] = v[k] * d;
}

// MakeOrthoVecs (src/mc.rs:70-82)
static void make_ortho(const double v[3], double o0[3], double o1[3]) {
    double n[3];
    normalize3(v, n);
    double a[3];
    if (std::fabs(n[0]) > 0.1) {
        double d = 1.0 / std::sqrt(n[0] * n[0] + n[2] * n[2]);
        a[0] = n[2] * d; a[1] = 0.0; a[2] = -n[0] * d;
    } else {
        double d = 1.0 / std::sqrt(n[1] * n[1] + n[2] * n[2]);
        a[0] = 0.0; a[1] = -n[2] * d; a[2] = n[1] * d;
    }
    for (int k = 0; k < 3; k++) o0[k] = (double)(float)a[k];
    double b[3] = {o0[1] * n[2] - o0[2] * n[1], o0[2] * n[0] - o0[0] * n[2], o0[0] * n[1] - o0[1] * n[0]};
    for (int k = 0; k < 3; k++) o1[k] = (double)(float)b[k];
}

static inline float fpow8(float x) {  // f32::powi(8)
    float a = x * x, b = a * a;
    return b * b;
}

// FastIntPow (src/math.rs:273-285)
static inline float fast_int_pow(float base, int expo) {
    if (base < 0.0f) return 0.0f;
    float r = base;
    for (int i = expo >> 1; i > 0; i >>= 1) r *= r;
    return r;
}

// zpos_of (src/mc.rs:1120-1123)
static inline uint32_t zpos_of(const Params &p, double zz) {
    double v = rte(p.zc_mul * (std::sqrt(rmax(zz, 0.0) * p.zcorr + 1.0) - 1.0));
    return sat_u32(rclamp(8388352.0 - v, 0.0, 8388352.0)) << 8;
}

// ---- the render constants (CalcMCT, src/mc.rs:3120-3237) ----
struct McCtx {
    Params p;
    mb3d_cu_mc_light lv;
    double hs_vecs[6][3];
    int max_amb_depth;
    bool secant;
    double amb_max_l;
    float fovy1d, soft_shadow_radius, hs_max_lmul;
    int width, height;
    double zz_stmit_dif;  // CalcParams.zz_stmit_dif (src/calc.rs:858)
};

// mc_scene (src/mc.rs:2842-2850): the far plane at least a tenth of the
// picture's diagonal away
static mb3d_cu_scene mc_scene(const mb3d_cu_scene &sc) {
    mb3d_cu_scene s = sc;
    double sw = 2.1345 / (s.zoom * (double)s.width);
    double los = std::sqrt((double)s.width * (double)s.width + (double)s.height * (double)s.height);
    s.z_end = rmax(s.z_end - s.z_start, los * 0.1 * sw) + s.z_start;
    return s;
}

static bool make_ctx(const mb3d_cu_scene &sc0, const mb3d_cu_mc_light &lv, int depth, int secant, float ssr,
                     McCtx &c, std::string &err) {
    mb3d_cu_scene sc = mc_scene(sc0);
    if (!make_params(sc, c.p, err)) return false;
    c.p.sm_normals = 0;
    c.lv = lv;
    Mat3 m1;
    normalise_matrix_to(1.0, c.p.vgrads, m1);
    for (int i = 0; i < lv.n_lights && i < 6; i++) {
        double l[3] = {(double)lv.ln[i][0], (double)lv.ln[i][1], (double)lv.ln[i][2]}, v[3];
        norm_to(-c.p.step_width, l, v);
        rotate_vector_reverse(v, m1, c.hs_vecs[i]);
    }
    c.max_amb_depth = depth;
    c.secant = secant != 0;
    double los = std::sqrt((double)sc.width * (double)sc.width + (double)sc.height * (double)sc.height);
    double deao_max = (double)sc.deao_max_len;
    c.amb_max_l = rmin(deao_max * los * 3.0, c.p.zend * 255.0 / 1.75);
    c.fovy1d = (float)(1.0 / (c.p.fov_y == 0.0 ? 1e-30 : c.p.fov_y));
    c.soft_shadow_radius = ssr;
    c.hs_max_lmul = (float)(sc.width + sc.height) * 0.6f * sc.hs_max_len_mul;
    c.width = sc.width;
    c.height = sc.height;
    c.zz_stmit_dif = sc.z_start - sc.mid[2];
    return true;
}

struct McReqO {
    int kind;
    double pos[3], dir[3], zz, zz2, zzplus, len;
    int32_t seed;
    bool probe;
};
struct McResO {
    int kind = 0;
    double pos[3] = {0, 0, 0}, normals[3] = {0, 0, 0};
    double zz = 0, zz2 = 0, len = 0;
    float dyn_fog = 0, ms_de_stop = 0;
    int32_t seed = 0;
    uint16_t si_grad = 0, otrap = 0;
    bool de_limited = false;
};

// ---- McMarch (src/mc.rs:477-956) ----
struct McMarch {
    const McCtx *c;
    Marcher m;
    explicit McMarch(const McCtx *cc) : c(cc), m(&cc->p, 0) {}

    void update_de_stop(double zz) {
        const Params &p = c->p;
        m.ms_de_stop = (float)((double)p.de_stop * (1.0 + std::fabs(zz) * (double)p.de_stop_factor));
    }
    void advance(const double d[3], double s) { add_weight(m.it.c, d, s); }

    // McMarch::normals (src/mc.rs:533-585), on the DE
    void normals(const double raydir[3], int32_t &seed, float &nn, double out[3]) {
        const Params &p = c->p;
        float sca = (seed & 128) == 0 ? 0.15f : -0.15f;
        m.it.calc_sit = true;
        double no = m.calc_de();
        nn = m.it.smooth_it;
        m.it.calc_sit = false;
        int i = 4;
        double n[3] = {0, 0, 0};
        out[0] = out[1] = out[2] = 0.0;
        for (;;) {
            if (i < 4) sca = (float)((rand_of(seed) - 0.5) * 0.5);
            double off = (double)rminf(p.de_stop, 1.0f) * (1.0 + m.mzz * (double)p.de_stop_factor) * (double)sca * p.step_width;
            const int ks[3] = {2, 0, 1};
            for (int q = 0; q < 3; q++) {
                int k = ks[q];
                double t = m.it.c[k];
                m.it.c[k] = t + off;
                n[k] = (m.calc_de() - no) * (double)sca;
                m.it.c[k] = t;
            }
            double l = n[0] * n[0] + n[1] * n[1] + n[2] * n[2];
            if (l > 1e-100 && dot3(n, raydir) < 0.0) {
                double s = 1.0 / std::sqrt(l);
                for (int k = 0; k < 3; k++) out[k] = n[k] * s;
                break;
            }
            i -= 1;
            if (i == 0) break;
        }
        if (i == 0) norm_to(-1.0, raydir, out);
    }

    // doBinSearchIt (src/mc.rs:588-643)
    void bin_search_it(double &zz, const double dir[3]) {
        int saved = m.it.max_it;
        float yp = (float)saved - 0.99f;
        m.it.max_it += 1;
        int itmp = 10;
        m.it.calc_sit = true;
        double dt1 = 0.0, dmul = 1.0;
        bool first = true;
        float last_si = 0.0f, last_dif = 0.0f;
        for (;;) {
            zz += dt1;
            add_weight(m.it.c, dir, dt1);
            m.calc_de();
            if (!first && last_dif < std::fabs(yp - m.it.smooth_it)) {
                zz -= dt1;
                add_weight(m.it.c, dir, -dt1);
                m.it.smooth_it = last_si;
                if (dt1 > 0.0) dmul *= 0.5;
                else dmul *= 0.7;
            }
            last_dif = std::fabs(yp - m.it.smooth_it);
            last_si = m.it.smooth_it;
            if (m.it.smooth_it > (float)m.it.max_it - 0.1f) {
                dt1 = -3.0;
            } else {
                zz -= 0.001;
                add_weight(m.it.c, dir, -0.001);
                m.calc_de();
                float r = last_si - m.it.smooth_it;
                if (std::fabs(r) < 1e-30f) dt1 = (last_si < m.it.smooth_it ? 1.0 : 0.0) - 0.5;
                else if (r < 0.0f) dt1 = (double)((yp - m.it.smooth_it) / (r * 500.0f));
                else dt1 = (double)((yp - m.it.smooth_it) / (r * 1000.0f));
                if (dt1 > 4.0) dt1 = std::sqrt(dt1) * 2.0;
                else if (dt1 < -9.0) dt1 = std::sqrt(-dt1) * -3.0;
                dt1 = dt1 * dmul + 0.0005;
            }
            first = false;
            itmp -= 1;
            if (itmp < 0) break;
        }
        m.it.max_it = saved;
    }

    // surface_colour (src/mc.rs:647-662) without colour on iteration
    void surface_colour(float nn, bool de_limited, uint16_t &si_grad, uint16_t &otrap) {
        const Params &p = c->p;
        float v = de_limited ? 32767.0f - (nn + p.d_col_plus + p.col_var_de_stop_mul * (float)std::log((double)m.ms_de_stop * p.step_width)) * p.mcts_m
                             : 32767.0f - nn * p.mcts_m;
        SiLight si;
        si.si_gradient = min_max_clip_15bit_o(v);
        m.do_color(si);
        si_grad = si.si_gradient;
        otrap = si.otrap;
    }
    static uint16_t min_max_clip_15bit_o(float s) {
        if (std::isnan(s) || s < 0.0f) return 0;
        if (s > 32767.0f) return 32767;
        return (uint16_t)rtef(s);
    }

    // McMarch::ray (src/mc.rs:665-865)
    McResO ray(const McReqO &r) {
        const Params &p = c->p;
        int32_t seed = r.seed;
        McResO o;
        const double *dir = r.dir;
        double zz = r.zz, zz2 = r.zz2;
        double max_l = r.len, zzplus = r.zzplus;
        update_de_stop(zz);
        double dtmp = m.calc_de();
        if (r.probe && (m.it.it_result >= m.max_its_result || dtmp < (double)m.ms_de_stop)) {
            // the start is inside the set (outside rendering)
            SiLight si;
            m.do_color(si);
            m.mzz = zz;
            if (p.color_option > 4) si.si_gradient |= 32768;
            else si.si_gradient = (uint16_t)(32768 + (uint16_t)rte(32767.0 * rclamp(m.it.rout / p.d_rstop, 0.0, 1.0)));
            o.kind = 2;
            std::memcpy(o.pos, m.it.c, sizeof(o.pos));
            o.si_grad = si.si_gradient;
            o.otrap = si.otrap;
            o.seed = seed;
            return o;
        }
        float dyn_fog = 0.0f;
        bool open_air = false, de_limited = true, first_step = true;
        float rsfmul = 1.0f;
        double rlast_sw = dtmp * (double)p.z_step_div, rlast_de;
        uint32_t guard = 0;
        for (;;) {
            rlast_de = dtmp;
            double dstep = rmax((dtmp - (double)p.ms_de_sub * (double)m.ms_de_stop) * (double)p.z_step_div * (double)rsfmul, 0.11);
            double d1 = (double)(rmaxf(m.ms_de_stop, 0.4f) * p.mh04zsd);
            bool count = p.dfog_on_it == 0 || m.it.it_result == p.dfog_on_it;
            if (d1 < dstep) {
                if (count) dyn_fog += (float)(d1 / dstep);
                dstep = d1;
            } else if (count) {
                dyn_fog += 1.0f;
            }
            if (first_step) {
                first_step = false;
                dstep *= rand_of(seed);
            }
            rlast_sw = dstep;
            zz2 += dstep;
            if (zz2 > max_l) {
                open_air = true;
                break;
            }
            advance(dir, dstep);
            zz += dstep * zzplus;
            update_de_stop(zz);
            dtmp = m.calc_de();
            if (m.it.it_result >= m.max_its_result) {
                de_limited = false;
                break;
            }
            if (!(dtmp >= (double)m.ms_de_stop) && m.it.it_result >= p.min_it) break;
            if (dtmp > rlast_de + rlast_sw) dtmp = rlast_de + rlast_sw;
            if (rlast_de > dtmp + 1e-30) {
                double d = rlast_sw / (rlast_de - dtmp);
                rsfmul = d < 1.0 ? (float)rmax(d, 0.5) : 1.0f;
            } else {
                rsfmul = 1.0f;
            }
            guard += 1;
            if (guard > 1000000) {
                open_air = true;
                break;
            }
        }
        o.dyn_fog = dyn_fog;
        o.zz2 = zz2;
        if (open_air) {
            std::memcpy(o.pos, m.it.c, sizeof(o.pos));
            o.zz = zz;
            o.seed = seed;
            return o;
        }
        if (de_limited) {
            if (c->secant) {
                int itmp = 4;
                while (itmp > 0 && std::fabs(dtmp - (double)m.ms_de_stop) > 0.001) {
                    double nz = rlast_de - dtmp;
                    if (std::fabs(nz) < 1e-40) nz = nz < 0.0 ? -1e-40 : 1e-40;  // not_zero
                    rlast_de = nz;
                    double f = rlast_sw * (dtmp - (double)m.ms_de_stop) / rlast_de;
                    if (dtmp < (double)m.ms_de_stop)
                        rlast_sw = (f >= 0.0 || f < std::fabs(rlast_sw) * -0.94) ? std::fabs(rlast_sw) * -0.5 : f;
                    else
                        rlast_sw = (f <= 0.0 || f > std::fabs(rlast_sw) * 0.94) ? std::fabs(rlast_sw) * 0.5 : f;
                    rlast_de = dtmp;
                    zz += rlast_sw * zzplus;
                    advance(dir, rlast_sw);
                    update_de_stop(zz);
                    itmp -= 1;
                    if (itmp <= 0) break;
                    dtmp = m.calc_de();
                }
            } else {
                int itmp = 10;
                double ds = rlast_sw * -0.5;
                while (std::fabs(dtmp - (double)m.ms_de_stop) > 0.001) {
                    zz += ds * zzplus;
                    advance(dir, ds);
                    update_de_stop(zz);
                    itmp -= 1;
                    if (itmp <= 0) break;
                    dtmp = m.calc_de();
                    ds = dtmp < (double)m.ms_de_stop ? std::fabs(ds) * -0.55 : std::fabs(ds) * 0.55;
                }
            }
        } else {
            double ds = zz;
            bin_search_it(ds, dir);
            zz += (ds - zz) * zzplus;
        }
        m.mzz = std::fabs(zz);
        float nn;
        normals(dir, seed, nn, o.normals);
        std::memcpy(o.pos, m.it.c, sizeof(o.pos));
        surface_colour(nn, de_limited, o.si_grad, o.otrap);
        o.kind = 1;
        o.zz = zz;
        o.de_limited = de_limited;
        o.seed = seed;
        o.ms_de_stop = m.ms_de_stop;
        return o;
    }

    // McMarch::shadow without transparency (src/mc.rs:869-914)
    McResO shadow(const McReqO &r) {
        const Params &p = c->p;
        McResO o;
        const double *v = r.dir;
        double dt1 = r.len, zz2mul = r.zzplus, zz2 = r.zz2;
        update_de_stop(r.zz);
        float rsfd = 2.0f;
        double dtmp = m.calc_de();
        double rlast_de, rlast_sw;
        uint32_t guard = 0;
        for (;;) {
            rlast_de = dtmp;
            dtmp = rmin(dtmp * (double)p.z_step_div * (double)rsfd, (double)(rmaxf(m.ms_de_stop, 0.4f) * p.mh04zsd));
            rlast_sw = dtmp;
            dt1 -= dtmp;
            advance(v, dtmp);
            zz2 += dtmp * zz2mul;
            update_de_stop(zz2);
            dtmp = m.calc_de();
            if (m.it.it_result >= m.max_its_result || !(dtmp >= (double)m.ms_de_stop) || !(dtmp < 1e30)) break;
            if (dtmp > rlast_de + rlast_sw) dtmp = rlast_de + rlast_sw;
            if (rlast_de > dtmp + 1e-30) {
                double s = rlast_sw / (rlast_de - dtmp);
                rsfd = s < 1.0 ? (float)rmax(s, 0.5) : 1.0f;
            } else {
                rsfd = 1.0f;
            }
            if (!(dt1 >= 0.0)) break;
            if (++guard > 1000000) break;  // (the card's bound; the reference has none)
        }
        o.len = dt1;
        o.seed = r.seed;
        return o;
    }

    McResO run(const McReqO &r) {
        std::memcpy(m.it.c, r.pos, sizeof(double) * 3);
        m.it.calc_sit = false;
        return r.kind == 0 ? ray(r) : shadow(r);
    }
};

// ---- the tracer (src/mc.rs:1063-2627) ----
struct Tracer {
    const McCtx *c;
    McMarch mm;
    int32_t seed = 0;
    double pos[3] = {0, 0, 0}, vfov[3] = {0, 0, 0}, normals[3] = {0, 0, 0};
    double mzz = 0.0;
    bool hit = false, calc_amb_shadow = false, rit1 = true, inside_start = false;
    float halton_x = 0, halton_y = 0, disc_x = 0, disc_y = 0;
    float total_light[3] = {0, 0, 0};
    uint32_t main_zpos_fine = 0;
    float dyn_fog = 0, zpos_dyn_fog = 0;
    int row_y = 0;
    int guard = 0;
    float hs6[6][4];
    double hs_vecs[6][3];
    // the first surface of the ray (the denoiser's guides)
    bool aov = false;
    float aov_albedo[3] = {0, 0, 0};
    double aov_normal[3] = {0, 0, 0};
    double aov_depth = 0.0;

    explicit Tracer(const McCtx *cc) : c(cc), mm(cc) { std::memcpy(hs_vecs, cc->hs_vecs, sizeof(hs_vecs)); }

    double rand() { return rand_of(seed); }

    // CalcBGLight without a background picture (src/mc.rs:1406-1510)
    void calc_bg_light(const double vec[3], bool use_amb, float res[3]) {
        const mb3d_cu_mc_light &lv = c->lv;
        const Params &p = c->p;
        double t0[3] = {dot3(p.vgrads[0], vec), dot3(p.vgrads[1], vec), dot3(p.vgrads[2], vec)}, t[3];
        normalize3(t0, t);
        if (use_amb) {
            float d = (float)(t[1] * 0.5 + 0.5);
            for (int k = 0; k < 3; k++) res[k] = (lv.amb_col[k] + d * (lv.amb_col2[k] - lv.amb_col[k])) * (1.0f / 256.0f);
        } else {
            float d = rit1 ? (float)row_y / (float)c->height
                           : (float)rclamp(std::asin(rclamp(t[1], -1.0, 1.0)) * (double)c->fovy1d + 0.5, 0.0, 1.0);
            if (lv.depth_func == 1) d *= d;
            else if (lv.depth_func == 2) d = std::sqrt(rmaxf(d, 0.0f));
            for (int k = 0; k < 3; k++) res[k] = (lv.depth_col[k] + d * (lv.depth_col2[k] - lv.depth_col[k])) * (1.0f / 256.0f);
        }
    }

    // CalcVisLights without visible lights (src/mc.rs:1301-1401)
    void calc_vis_lights(const double view[3], uint32_t zpos_fine, float &bg_dec, float &depth_dec, float res[3]) {
        const mb3d_cu_mc_light &lv = c->lv;
        int32_t zp = (int32_t)(zpos_fine >> 16);
        float bgz = zp < 32768 ? rmaxf(1.0f + (float)(zp - 28000) * lv.s_depth, 0.0f)
                               : rmaxf(1.0f - (float)(60768 - zp) * lv.s_depth, 0.0f);
        if (bgz < 1.0f) {
            bgz = lv.sqr ? (1.0f - bgz) * (1.0f - bgz) : 1.0f - bgz;
            if (lv.far_fog) bgz *= bgz;
            bgz = 1.0f - bgz;
        }
        depth_dec = bgz;
        bg_dec = 1.0f;
        float svbg[3];
        calc_bg_light(view, false, svbg);
        for (int k = 0; k < 3; k++) res[k] = 0.0f;
        float dfog = (dyn_fog - lv.s_shad - lv.s_shad_zmul * zpos_dyn_fog) * lv.s_shad_gr;
        if (lv.dfog_options & 2) dfog = rmaxf(dfog, 0.0f);
        float stmp = rminf(dyn_fog * lv.s_dyn_fog_mul, 1.0f) * dfog;
        float w = rmaxf(1.0f - bgz, 0.0f);
        for (int k = 0; k < 3; k++) res[k] += svbg[k] * w;
        if (lv.dfog_options & 1) {
            dfog = rclampf(dfog, 0.0f, 1.0f);
            stmp = rclampf(stmp, 0.0f, 1.0f);
            for (int k = 0; k < 3; k++) res[k] = res[k] * (1.0f - dfog);
            depth_dec *= 1.0f - dfog;
        }
        float w1 = (dfog - stmp) / 255.0f, w2 = stmp / 255.0f;
        for (int k = 0; k < 3; k++) res[k] += lv.dyn_fog_col[k] * w1;
        for (int k = 0; k < 3; k++) res[k] += lv.dyn_fog_col2[k] * w2;
    }

    // CalcColor (src/mc.rs:1250-1285) -> calc_colors_alpha / palette_place
    // (src/lighting.rs:1563-1614) for a surface outside the set
    void calc_color(uint16_t si_gradient, uint16_t otrap, float z_pos, float spe[4], float dif[4]) {
        const mb3d_cu_mc_light &lv = c->lv;
        float idif0 = lv.s_col_zmul * z_pos;
        float irf = lv.col_on_otrap ? (float)(otrap & 0x7FFF) : (float)si_gradient;
        float x = ((irf - lv.s_c_start) * lv.s_c_mul + idif0) * 16384.0f;
        x = rclampf(x, -1e9f, 1e9f);
        int32_t ir = std::isnan(x) ? 0 : (int32_t)std::round(x);
        int a = -1, b = -1;
        float t = 0.0f;
        if (lv.col_cycling) {
            ir &= 32767;
        } else if (ir < 0) {
            a = 0;
        } else if (ir >= lv.col_pos[9]) {
            a = 9;
        }
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
            if (lv.no_col_ipol) {
                a = il2 - 1;
            } else {
                a = il2 - 1;
                b = il2 > 9 ? 0 : il2;
                t = (float)(ir - lv.col_pos[a]) * lv.s_c_div[a];
            }
        }
        if (b < 0) {
            for (int k = 0; k < 3; k++) {
                dif[k] = lv.col_dif[a][k];
                spe[k] = lv.col_spe[a][k];
            }
            spe[3] = lv.col_spe_a[a];
        } else {
            for (int k = 0; k < 3; k++) {
                dif[k] = lv.col_dif[a][k] + t * (lv.col_dif[b][k] - lv.col_dif[a][k]);
                spe[k] = lv.col_spe[a][k] + t * (lv.col_spe[b][k] - lv.col_spe[a][k]);
            }
            spe[3] = lv.col_spe_a[a] + t * (lv.col_spe_a[b] - lv.col_spe_a[a]);
        }
        dif[3] = 0.0f;
    }

    McResO march(const McReqO &r) { return mm.run(r); }

    // CalcHSMC for global lights without transparency (src/mc.rs:1513-1625)
    void calc_hs_mc() {
        const Params &p = c->p;
        float zz = (float)std::fabs(mzz);
        double ic[3] = {pos[0], pos[1], pos[2]};
        float max_lhs = c->hs_max_lmul * (1.0f + 0.5f * rminf(zz, (float)p.zend * 0.4f) * rmaxf((float)p.fov_y, 0.0f) / (float)c->height);
        for (int i = 0; i < c->lv.n_lights; i++) {
            for (int k = 0; k < 4; k++) hs6[i][k] = 1.0f;
            std::memcpy(pos, ic, sizeof(ic));
            double zz2 = mzz;
            double dt1 = (double)max_lhs;
            double v[3] = {-hs_vecs[i][0], -hs_vecs[i][1], -hs_vecs[i][2]};
            if (dt1 <= 0.001) continue;
            if (dot3(normals, v) < 0.0) {
                for (int k = 0; k < 4; k++) hs6[i][k] = 0.0f;
                continue;
            }
            double zz2mul = dot3(v, vfov) / std::sqrt(dot3(v, v) * dot3(vfov, vfov));
            double dmaxl = dt1;
            McReqO q;
            q.kind = 1;
            std::memcpy(q.pos, ic, sizeof(ic));
            std::memcpy(q.dir, v, sizeof(v));
            q.zz = (double)zz;
            q.zz2 = zz2;
            q.zzplus = zz2mul;
            q.len = dt1;
            q.seed = seed;
            q.probe = false;
            McResO h = march(q);
            seed = h.seed;
            dt1 = h.len;
            if (dt1 <= 0.01) continue;
            float fade = rminf(fpow8((float)((dmaxl - dt1) / (double)max_lhs)), 1.0f);
            for (int k = 0; k < 3; k++) hs6[i][k] *= fade;
        }
        std::memcpy(pos, ic, sizeof(ic));
    }

    // CalcPhongLight for global lights (src/mc.rs:1699-1768): [specular, diffuse]
    void calc_phong_light(const double reflect[3], float res[2][3]) {
        const mb3d_cu_mc_light &lv = c->lv;
        const double sw = c->p.step_width;
        for (int a = 0; a < 2; a++)
            for (int k = 0; k < 3; k++) res[a][k] = 0.0f;
        for (int i = 0; i < lv.n_lights; i++) {
            double stmp = (double)disc_x, s1 = (double)disc_y;
            double sn = std::sin(2.0 * PIc * s1), cs = std::cos(2.0 * PIc * s1);
            double k = 2.5e-5;
            double d = std::sqrt(stmp) * std::sqrt((double)lv.lmax_l[i]) * k * (double)c->soft_shadow_radius * sw;
            double o0[3], o1[3];
            make_ortho(c->hs_vecs[i], o0, o1);
            double v[3];
            for (int q = 0; q < 3; q++) v[q] = c->hs_vecs[i][q] + (double)((float)(o0[q] * sn * d) + (float)(o1[q] * cs * d));
            norm_to(sw, v, hs_vecs[i]);
        }
        calc_hs_mc();
        for (int i = 0; i < lv.n_lights; i++) {
            const float *hs = hs6[i];
            if (hs[0] != 0.0f || hs[1] != 0.0f || hs[2] != 0.0f) {
                float l0[3];
                const double *t = c->hs_vecs[i];
                for (int k = 0; k < 3; k++) l0[k] = lv.col[i][k] * hs[k];
                float sp = fast_int_pow((float)(dot3(reflect, t) * (double)hs[3] / -(sw * sw)), lv.pow_func[i]) * lv.s_spec / 255.0f;
                for (int k = 0; k < 3; k++) res[0][k] += l0[k] * sp;
                float cs = (float)(dot3(normals, t) / -sw);
                float m = rmaxf(cs, 0.0f);
                float df = m * m * lv.s_diff / 255.0f;
                for (int k = 0; k < 3; k++) res[1][k] += l0[k] * df;
            }
            std::memcpy(hs_vecs[i], c->hs_vecs[i], sizeof(double) * 3);
        }
    }

    // CalcRay (src/mc.rs:1904-2348), the recursion of the ambient bounce as a loop
    void calc_ray(double zz, double dir0[3], float t_absorb0[3], int rit, bool probe) {
        const Params &p = c->p;
        const mb3d_cu_mc_light &lv = c->lv;
        const double sw = p.step_width;
        double dir[3] = {dir0[0], dir0[1], dir0[2]};
        float ta[3] = {t_absorb0[0], t_absorb0[1], t_absorb0[2]};
        for (;;) {
            if (std::fabs(ta[0]) * 0.3f + std::fabs(ta[1]) * 0.59f + std::fabs(ta[2]) * 0.11f < 1e-4f) return;
            guard += 1;
            if (guard > 4096) return;
            double max_l;
            if (calc_amb_shadow) {
                double r = rand();
                max_l = c->amb_max_l * (r * r + 0.75);
            } else {
                max_l = p.zend;
            }
            rit += 1;
            rit1 = rit == 1;
            uint32_t cr_zpos = rit1 ? main_zpos_fine : 0u;
            double zz2 = rit1 ? zz : 0.0;
            float bg_dec = 1.0f;
            double zzplus = dot3(dir, vfov) / (sw * sw);
            McReqO q;
            q.kind = 0;
            std::memcpy(q.pos, pos, sizeof(pos));
            std::memcpy(q.dir, dir, sizeof(dir));
            q.zz = zz;
            q.zz2 = zz2;
            q.zzplus = zzplus;
            q.len = max_l;
            q.seed = seed;
            q.probe = probe;
            McResO h = march(q);
            seed = h.seed;
            std::memcpy(pos, h.pos, sizeof(pos));
            if (h.kind == 2) {
                inside_start = true;  // (Tracer::ray takes the start inside for a hit; left dark)
                hit = true;
                total_light[0] = total_light[1] = total_light[2] = 0.0f;
                return;
            }
            zz = h.zz;
            zz2 = h.zz2;
            dyn_fog = h.dyn_fog;
            bool open_air = h.kind == 0;
            float d1 = 1.0f;
            float obj[2][4];
            double cc[3];
            if (!open_air) {
                hit = true;
                mzz = std::fabs(zz);
                std::memcpy(normals, h.normals, sizeof(normals));
                std::memcpy(cc, pos, sizeof(cc));
                cr_zpos = zpos_of(p, zz2);
                if (rit1) main_zpos_fine = cr_zpos;
                calc_color(h.si_grad, h.otrap, (float)(mzz * sw + c->zz_stmit_dif), obj[0], obj[1]);
                if (rit1 && aov) {
                    for (int k = 0; k < 3; k++) {
                        aov_albedo[k] = obj[1][k];
                        aov_normal[k] = normals[k];
                    }
                    aov_depth = zz * sw;
                    aov = false;
                }
                zpos_dyn_fog = (float)(zz2 * sw + c->zz_stmit_dif);
                float sv[3];
                calc_vis_lights(dir, cr_zpos, bg_dec, d1, sv);
                for (int k = 0; k < 3; k++) total_light[k] = total_light[k] + sv[k] * ta[k];
            } else {
                zpos_dyn_fog = (float)(p.zend * sw + c->zz_stmit_dif);
                int32_t main_z = (int32_t)(main_zpos_fine >> 16);  // (cr is main_si on the first ray)
                if ((lv.far_fog || lv.sqr) && std::fabs(lv.s_depth) > 1e-10f) {
                    bool both = lv.far_fog && lv.sqr;
                    float e1 = 1.0f - rmaxf(1.0f + (float)(main_z - 28000) * lv.s_depth, 0.0f);
                    if (e1 > 0.0f) {
                        e1 *= e1;
                        if (both) e1 *= e1;
                    }
                    float e2 = 1.0f - rmaxf(1.0f - 28000.0f * lv.s_depth, 0.0f);
                    if (e2 > 0.0f) {
                        e2 *= e2;
                        if (both) e2 *= e2;
                    }
                    float e = e2 - e1;
                    if (e > 0.0f) {
                        e = std::sqrt(e);
                        if (both) e = std::sqrt(e);
                    }
                    uint32_t z = (uint32_t)rtef(rclampf(60768.0f - e / lv.s_depth, 32768.0f, 65535.0f));
                    cr_zpos = z << 16;
                } else {
                    cr_zpos = 32768u << 16;  // set_zpos_word(cr, 32768)
                }
                if (rit1) main_zpos_fine = cr_zpos;
                float rsf = 0.0f, sv[3], bgl[3];
                calc_vis_lights(dir, cr_zpos, bg_dec, rsf, sv);
                calc_bg_light(dir, calc_amb_shadow, bgl);
                bg_dec *= rsf;
                for (int k = 0; k < 3; k++) sv[k] += bgl[k] * bg_dec;
                for (int k = 0; k < 3; k++) total_light[k] = total_light[k] + sv[k] * ta[k];
                return;
            }
            float bd = bg_dec * d1;
            for (int k = 0; k < 3; k++) ta[k] = ta[k] * bd;
            double nd = 2.0 * dot3(normals, dir);
            double reflect[3] = {dir[0] - normals[0] * nd, dir[1] - normals[1] * nd, dir[2] - normals[2] * nd};
            mzz = zz;
            float light_sd[2][3];
            calc_phong_light(reflect, light_sd);
            const float d2 = 1.0f, d3v = 1.0f;
            float ws = (0.25f + d3v) * 0.8f;
            for (int k = 0; k < 3; k++) {
                float spec = (obj[0][k] * ws) * light_sd[0][k];
                float diff = (obj[1][k] * d2) * light_sd[1][k];
                total_light[k] = total_light[k] + (spec + diff) * ta[k];
            }
            if (d1 > 1.0f)
                for (int k = 0; k < 3; k++) ta[k] = ta[k] * (1.0f / d1);
            double nvec[3] = {normals[0], normals[1], normals[2]};
            if (!(rit < c->max_amb_depth || !calc_amb_shadow)) return;
            double a, ml;
            if (!calc_amb_shadow) {
                a = 2.0 * PIc * (double)halton_x;
                ml = (double)halton_y;
            } else {
                a = 2.0 * PIc * rand();
                ml = rand();
            }
            double d4s = (double)(float)std::sin(a), d3c = (double)(float)std::cos(a);
            double dd = std::sqrt(ml);
            double o0[3], o1[3];
            make_ortho(nvec, o0, o1);
            double w = std::sqrt(1.0 - ml);
            double nv[3];
            for (int k = 0; k < 3; k++) nv[k] = (double)((float)(o0[k] * d3c * dd) + (float)(o1[k] * d4s * dd)) + nvec[k] * w;
            norm_to(sw, nv, dir);
            std::memcpy(pos, cc, sizeof(cc));
            calc_amb_shadow = true;
            for (int k = 0; k < 3; k++) ta[k] = ta[k] * (obj[1][k] * d2);
            probe = false;
        }
    }

    // Tracer::ray (src/mc.rs:2467-2627) for the common camera, no salt,
    // no depth of field, no cutting planes, no water: x1 the 1-based column
    void ray(int x1, int y, uint32_t b, float out[3]) {
        const Params &p = c->p;
        guard = 0;
        row_y = y;
        uint32_t act = b < 65535u ? b : 65535u;
        seed = mc_seed_of(x1, y, b);
        float sx, sy;
        halton_2d_shifts(x1, y, sx, sy);
        const HaltonRec &h = halton_seq()[act];
        halton_x = frac_s((float)h.hrx * D1D65535 + sx);
        halton_y = frac_s((float)h.hry * D1D65535 + sy);
        main_zpos_fine = 32768u << 16;
        float xx, yy;
        if (b < 4) {
            xx = (float)x1 - (float)(b & 1) * 0.5f - 0.75f;
            yy = (float)y + (float)(b & 2) * 0.25f - 0.25f;
        } else {
            float gx = (float)(rand() - 0.5), gy = (float)(rand() - 0.5);  // sub_pixel_shift (box)
            xx = gx + (float)x1 - 1.0f;
            yy = gy + (float)y;
        }
        // calc_vgrads_fov (src/mc.rs:2418-2431)
        double cafx = (double)((p.fovx_off - xx - 1.0f) * p.fovx_mul);
        double cafy = ((double)yy / (double)p.height - 0.5) * p.fov_y;
        double v[3];
        build_view_vector_dfov(cafy, cafx, v);
        rotate_vector_reverse(v, p.vgrads, vfov);
        for (int k = 0; k < 3; k++) pos[k] = p.ystart[k] + p.vgrads[1][k] * (double)yy + p.vgrads[0][k] * (double)xx;
        disc_x = frac_s((float)h.hdx * D1D65535 + sx);
        disc_y = frac_s((float)h.hdy * D1D65535 + sy);
        total_light[0] = total_light[1] = total_light[2] = 0.0f;
        calc_amb_shadow = false;
        rit1 = true;
        dyn_fog = 0.0f;
        hit = false;
        inside_start = false;
        double vf[3] = {vfov[0], vfov[1], vfov[2]};
        float one[3] = {1.0f, 1.0f, 1.0f};
        calc_ray(0.0, vf, one, 0, true);
        for (int k = 0; k < 3; k++) out[k] = total_light[k];
    }
};

// SVecRGB2Lab (src/mc.rs:3906-3919), single precision
static void rgb_to_lab(const float v[3], float o[3]) {
    const float sftc = 216.0f / (29.0f * 29.0f * 29.0f), s4d29 = 4.0f / 29.0f, smul = 29.0f * 29.0f / 108.0f;
    float x[3] = {(0.412453f * v[0] + 0.35758f * v[1] + 0.180423f * v[2]) * 1.052111f,
                  0.212671f * v[0] + 0.71516f * v[1] + 0.072169f * v[2],
                  (0.019334f * v[0] + 0.119193f * v[1] + 0.950227f * v[2]) * 0.918417f};
    for (float &c : x) c = c > sftc ? std::cbrt(c) : smul * c + s4d29;
    o[0] = 1.16f * x[1] - 0.16f;
    o[1] = x[0] - x[1];
    o[2] = x[1] - x[2];
}

// SVecLab2RGB (src/mc.rs:3922-3938)
static void lab_to_rgb(const float v[3], float o[3]) {
    const float sftc = 6.0f / 29.0f, s4d29 = 4.0f / 29.0f, smul = 108.0f / 841.0f;
    float y = (v[0] + 0.16f) / 1.16f;
    float x[3] = {y + v[1], y, y - v[2]};
    for (float &c : x) c = c > sftc ? c * c * c : (c - s4d29) * smul;
    x[0] *= 0.95047f;
    x[2] *= 1.08883f;
    o[0] = 3.240479f * x[0] - 1.537150f * x[1] - 0.498535f * x[2];
    o[1] = -0.969256f * x[0] + 1.875992f * x[1] + 0.041556f * x[2];
    o[2] = 0.055648f * x[0] - 0.204043f * x[1] + 1.057311f * x[2];
}

// paint_recs (src/mc.rs:3957-4005): records' colours to 8-bit RGB
static void paint_recs(const float *col, const uint8_t *rays, size_t n, const mb3d_cu_mc_paint_opts &mc, uint8_t *out) {
    float contrast = (float)mc.contrast / 256.0f + 0.5f;
    contrast = contrast * contrast;
    const bool soft_clip = (mc.options & 1) != 0;
    const float saturation = (float)(mc.saturation & 0x7F) / 32.0f;
    // (gamma.round() as i32).clamp(0, 63): the cast saturates, NaN gives 0
    float gr = std::round(mc.gamma);
    int ig = std::isnan(gr) ? 0 : gr < 0.0f ? 0 : gr > 63.0f ? 63 : (int)gr;
    int igamma = (ig << 2) & 0xFC;
    if (soft_clip) {
        igamma = std::max(igamma - 20, 0);
        contrast *= 1.1f;
    }
    int gmode;
    float sgamma;
    if (igamma > 128) {
        gmode = 1;
        sgamma = (float)(igamma - 128) / 127.0f;
    } else if (igamma < 128) {
        gmode = -1;
        sgamma = 1.0f - (float)igamma / 128.0f;
    } else {
        gmode = 0;
        sgamma = 1.0f;
    }
    for (size_t i = 0; i < n; i++) {
        uint8_t *o = out + 3 * i;
        o[0] = o[1] = o[2] = 0;
        if (rays && !rays[i]) continue;
        float v[3];
        for (int k = 0; k < 3; k++) {
            float c = std::max(col[3 * i + k] * contrast, 0.0f);
            v[k] = c * c;
        }
        float lab[3];
        rgb_to_lab(v, lab);
        float scol = saturation;
        if (lab[0] > 0.0f) {
            if (gmode != 0) {
                float s2 = lab[0];
                float s = gmode > 0 ? std::sqrt(lab[0]) : lab[0] * lab[0];
                lab[0] += (s - lab[0]) * sgamma;
                if (gmode > 0 && s2 > 1.0f) scol *= lab[0] / s2;
            }
            if (soft_clip) {
                float s = lab[0];
                float x2 = s * s;
                float q = x2 * 0.9f;
                lab[0] = std::sqrt(x2 / std::sqrt(q * q + 1.0f));
                scol *= lab[0] / s;
            }
        }
        lab[1] *= scol;
        lab[2] *= scol;
        float rgb[3];
        lab_to_rgb(lab, rgb);
        for (int k = 0; k < 3; k++) {
            float c = std::sqrt(std::max(rgb[k], 0.0f));
            c = std::min(std::max(c, 0.0f), 1.0f) * 255.0f;
            o[k] = (uint8_t)std::round(c);
        }
    }
}

// ---------------------------------------------------------------------------
// the adaptive pass (src/mc.rs:2657-2834 calc_n and pixel, :3110-3300
// pass_inner's set-up, :329-358 stats and avg_sqr_noise)

static const double MC_MAX = 1096.6331584284585 - 2.718281828459045 + 2.0;  // src/mc.rs:37
static inline double clamp_mc(double d) { return rclamp(d, -1.0, MC_MAX); }
// YofSVec (src/svec.rs:38-40)
static inline float luma_s(const float v[3]) { return rmaxf(v[0] * 0.3f + v[1] * 0.59f + v[2] * 0.11f, 0.0f); }
static inline double rec_y(const mb3d_cu_mc_record &r) { return (double)r.ysum; }
static inline double rec_noise(const mb3d_cu_mc_record &r) { return (double)r.ysqr - rec_y(r) * rec_y(r); }

struct PassArgs {
    const mb3d_cu_mc_record *snap;
    int w, h;
    bool skip_nonzero;
    double avrg_vari;
    float avrg_rcount;
    int max_new;
    uint32_t pass_nr;
};

// CalcN: how many more rays the pixel gets in this pass (x1, y1 1-based)
static int calc_n(Tracer &t, const PassArgs &a, int x1, int y1, const mb3d_cu_mc_record &rec) {
    const int w = a.w, h = a.h;
    auto at = [&](int x, int y) -> const mb3d_cu_mc_record & { return a.snap[(size_t)(y - 1) * w + (x - 1)]; };
    double maxyd = 0, maxyd2 = 0, maxnoise = 0;
    int n = 0, n2 = 0, avg_rc = 0;
    const double dt2 = rec_y(rec);
    if (y1 > 1) {
        const auto &r = at(x1, y1 - 1);
        double dt = rec_y(r);
        maxyd = (dt - dt2) * (dt - dt2);
        maxnoise = rec_noise(r);
        avg_rc = r.ray_count;
        n += 1;
        if (x1 > 1) {
            const auto &r3 = at(x1 - 1, y1 - 1);
            double dt3 = rec_y(r3);
            maxyd += (dt2 - dt3) * (dt2 - dt3);
            maxyd2 = (dt - dt3) * (dt - dt3);
            maxnoise = rmax(maxnoise, rec_noise(r3));
            avg_rc += r3.ray_count;
            n += 1;
            n2 += 1;
        }
        if (x1 < w) {
            const auto &r3 = at(x1 + 1, y1 - 1);
            double dt3 = rec_y(r3);
            maxyd += (dt2 - dt3) * (dt2 - dt3);
            maxyd2 += (dt - dt3) * (dt - dt3);
            maxnoise = rmax(maxnoise, rec_noise(r3));
            avg_rc += r3.ray_count;
            n += 1;
            n2 += 1;
        }
    }
    double dt = 0;
    if (x1 > 1) {
        const auto &r = at(x1 - 1, y1);
        dt = rec_y(r);
        maxyd += (dt - dt2) * (dt - dt2);
        maxnoise = rmax(maxnoise, rec_noise(r));
        avg_rc += r.ray_count;
        n += 1;
    }
    if (x1 < w) {
        const auto &r = at(x1 + 1, y1);
        double dt3 = rec_y(r);
        maxyd += (dt3 - dt2) * (dt3 - dt2);
        if (x1 > 1) {
            maxyd2 += (dt - dt3) * (dt - dt3);
            n2 += 1;
        }
        maxnoise = rmax(maxnoise, rec_noise(r));
        avg_rc += r.ray_count;
        n += 1;
    }
    if (y1 < h) {
        const auto &r = at(x1, y1 + 1);
        double dty = rec_y(r);
        maxyd += (dty - dt2) * (dty - dt2);
        maxnoise = rmax(maxnoise, rec_noise(r));
        avg_rc += r.ray_count;
        n += 1;
        if (x1 > 1) {
            const auto &r3 = at(x1 - 1, y1 + 1);
            double dt3 = rec_y(r3);
            maxyd += (dt2 - dt3) * (dt2 - dt3);
            maxyd2 += (dty - dt3) * (dty - dt3);
            maxnoise = rmax(maxnoise, rec_noise(r3));
            avg_rc += r3.ray_count;
            n += 1;
            n2 += 1;
        }
        if (x1 < w) {
            const auto &r3 = at(x1 + 1, y1 + 1);
            double dt3 = rec_y(r3);
            maxyd += (dt2 - dt3) * (dt2 - dt3);
            maxyd2 += (dty - dt3) * (dty - dt3);
            maxnoise = rmax(maxnoise, rec_noise(r3));
            avg_rc += r3.ray_count;
            n += 1;
            n2 += 1;
        }
    }
    const double nf = (double)(n > 1 ? n : 1), n2f = (double)(n2 > 1 ? n2 : 1);
    maxyd /= nf;
    maxyd2 /= n2f;
    const double dt3 = ((double)rec.ysqr - dt2 * dt2) / (rmax(dt2, 0.0) + 0.01);
    const double dm = !rec.hit ? 0.0
                               : rmax(rmax(maxyd, maxyd2) - 20.0 * a.avrg_vari, 0.0) *
                                     rclamp((double)rec.ray_count - (double)avg_rc / nf, -4.0, 4.0);
    const double q = dt2 / std::sqrt(1.0 + (dt2 * 0.9) * (dt2 * 0.9));
    const double d = rmax(rmax(dt3, maxnoise) / rmax(q * (double)rec.ray_count, 0.3) - dm, 0.0);
    const double d2 = d * 4.0 / a.avrg_vari;
    if (d2 >= 1.0) return (int)rte(rmin((double)a.avrg_rcount * 0.5 + 8.0, d2));
    if (t.rand() * 1.1 - 0.1 > rmax(d2, 0.0)) return 0;
    return 1;
}

// one pixel of TMCCalcThread.Execute: rays in rounds until its noise is low
static void mc_pixel(Tracer &t, const PassArgs &a, bool sqr, int x1, int y, mb3d_cu_mc_record &rec) {
    t.seed = mc_seed_of(x1, y, 0x80000000u | a.pass_nr);
    int total;
    if (rec.ray_count == 0) total = 4;
    else if (a.skip_nonzero) return;
    else total = calc_n(t, a, x1, y + 1, rec);
    bool hit = rec.hit != 0;
    for (int round = 0; round < 100000; round++) {
        if (total + (int)rec.ray_count > 65535) total = 65535 - (int)rec.ray_count;
        float at[3] = {0.f, 0.f, 0.f};
        double sum = 0.0, sqr_sum = 0.0;
        int itcount = 0;
        const uint32_t rc = rec.ray_count;
        for (int i = 0; i < total; i++) {
            float L[3];
            t.aov = false;
            t.ray(x1, y, rc + (uint32_t)i, L);
            hit = hit || t.hit;
            float sv[3];
            for (int k = 0; k < 3; k++) sv[k] = rclampf(L[k], 0.0f, 400.0f);
            double yv = (double)luma_s(sv);
            sqr_sum += yv * yv;
            sum += yv;
            for (int k = 0; k < 3; k++) at[k] = at[k] + sv[k];
            itcount += 1;
        }
        rec.hit = hit ? 1 : 0;
        if (itcount == 0) return;
        const double dtmp = (double)rec.ysum, zz = (double)rec.ysqr;
        const int itmp = rec.ray_count;
        const double yy = itmp != 0 ? rmax((zz - dtmp * dtmp) * 10.0, 0.03) : 0.0;
        float light[3];
        if (sqr) {
            const float inv = 1.0f / (float)itcount;
            for (int k = 0; k < 3; k++) {
                float v = at[k] * inv;
                light[k] = (v > 0.0f ? std::sqrt(v) : v) * (float)itcount;
            }
        } else {
            for (int k = 0; k < 3; k++) light[k] = at[k];
        }
        const double xx = 1.0 / (double)(itmp + itcount);
        for (int k = 0; k < 3; k++) rec.col[k] = (float)clamp_mc(((double)rec.col[k] * itmp + (double)light[k]) * xx);
        rec.ysum = (float)clamp_mc((dtmp * itmp + sum) * xx);
        rec.ysqr = (float)clamp_mc((zz * itmp + sqr_sum) * xx);
        rec.ray_count = (uint16_t)(itmp + itcount);
        const double mean = sum / (double)itcount;
        if (itmp != 0 && (int)rec.ray_count < a.max_new && (mean - dtmp) * (mean - dtmp) > yy) {
            const int m = std::max(std::min(itmp, itcount), 4);
            total = (int)rte(std::sqrt((mean - dtmp) * (mean - dtmp) / yy) * (double)m);
            continue;
        }
        return;
    }
}

}  // namespace oracle

using namespace oracle;

extern "C" {

/* paint_recs of n records' colours (3 floats each); rays (n bytes) may be
 * NULL. */
void oracle_mc_paint(const float *col, const uint8_t *rays, size_t n, const mb3d_cu_mc_paint_opts *opts, uint8_t *rgb) {
    paint_recs(col, rays, n, *opts, rgb);
}

/* The Monte Carlo tracer's rays (ray0 .. ray0+rays-1) on the pixels of the
 * options' rectangle.  Outputs (w*h*3 doubles: radiance, albedo, normal; w*h:
 * depth; w*h bytes: hit) may be NULL except radiance; inside (may be NULL):
 * the rays that started inside the set. */
int oracle_mc_render(const mb3d_cu_scene *sc, const mb3d_cu_mc_light *lv, const mb3d_cu_mc_opts *o, double *radiance,
                     double *albedo, double *normal, double *depth_out, uint8_t *hit, uint64_t *inside, int threads) {
    McCtx c;
    std::string err;
    if (!make_ctx(*sc, *lv, o->depth, o->secant, o->soft_shadow_radius, c, err)) return -22;
    int x0 = o->x0, y0 = o->y0, w = o->w, h = o->h;
    if (w <= 0) {
        x0 = 0;
        y0 = 0;
        w = sc->width;
        h = sc->height;
    }
    if (threads < 1) threads = (int)std::thread::hardware_concurrency();
    if (threads < 1) threads = 1;
    halton_seq();
    std::atomic<uint64_t> n_inside{0};
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; t++)
        ts.emplace_back([&, t]() {
            Tracer tr(&c);
            for (int r = t; r < h; r += threads)
                for (int col = 0; col < w; col++) {
                    uint64_t acc[3] = {0, 0, 0};
                    bool any = false;
                    size_t i = (size_t)r * w + col;
                    for (int b = 0; b < o->rays; b++) {
                        float L[3];
                        tr.aov = b == 0;
                        tr.aov_depth = 0.0;
                        for (int k = 0; k < 3; k++) {
                            tr.aov_albedo[k] = 0.0f;
                            tr.aov_normal[k] = 0.0;
                        }
                        tr.ray(x0 + col + 1, y0 + r, (uint32_t)(o->ray0 + b), L);
                        if (tr.inside_start) n_inside++;
                        any = any || tr.hit;
                        for (int k = 0; k < 3; k++) {
                            float sv = rclampf(L[k], 0.0f, 400.0f);
                            acc[k] += (uint64_t)std::nearbyint((double)sv * 4294967296.0);
                        }
                        if (b == 0) {
                            if (albedo)
                                for (int k = 0; k < 3; k++) albedo[3 * i + k] = (double)tr.aov_albedo[k];
                            if (normal)
                                for (int k = 0; k < 3; k++) normal[3 * i + k] = tr.aov_normal[k];
                            if (depth_out) depth_out[i] = tr.aov_depth;
                        }
                    }
                    for (int k = 0; k < 3; k++) radiance[3 * i + k] = (double)acc[k] / 4294967296.0 / (double)o->rays;
                    if (hit) hit[i] = any ? 1 : 0;
                }
        });
    for (auto &t : ts) t.join();
    if (inside) *inside = n_inside.load();
    return 0;
}

/* One pass of the adaptive Monte Carlo renderer over the whole picture
 * (mc::pass, src/mc.rs:3110-3300 with the CPU's per-pixel loop): recs holds
 * width*height records, updated in place.  The options' rays, ray0 and
 * rectangle are not used. */
int oracle_mc_pass(const mb3d_cu_scene *sc, const mb3d_cu_mc_light *lv, const mb3d_cu_mc_opts *o, uint32_t pass_nr,
                   mb3d_cu_mc_record *recs, int threads) {
    McCtx c;
    std::string err;
    if (!make_ctx(*sc, *lv, o->depth, o->secant, o->soft_shadow_radius, c, err)) return -22;
    const int w = sc->width, h = sc->height;
    const size_t n = (size_t)w * h;
    // StartCalc / CalcAvrgNoise (src/mc.rs:3226-3235, stats :329-358)
    bool fresh = true, zero_counts = false;
    double rsum = 0.0, noise_sum = 0.0;
    for (size_t i = 0; i < n; i++) {
        if (recs[i].ray_count != 0) fresh = false;
        if (recs[i].ray_count == 0) {
            zero_counts = true;
            continue;
        }
        rsum += (double)recs[i].ray_count;
        noise_sum += rmax(rec_noise(recs[i]) / (double)recs[i].ray_count, 0.0);
    }
    const double l = (double)(n > 0 ? n : 1);
    const double avrg_sqr_noise = fresh ? 1.0 : rmax(noise_sum / l + 0.002, 0.002);
    const float avrg_rcount = fresh ? 0.0f : (float)(rsum / l);
    PassArgs a;
    std::vector<mb3d_cu_mc_record> snap(recs, recs + n);
    a.snap = snap.data();
    a.w = w;
    a.h = h;
    a.skip_nonzero = fresh ? true : zero_counts;
    a.avrg_vari = rmax(avrg_sqr_noise, 0.001);
    a.avrg_rcount = avrg_rcount;
    a.max_new = (int)std::round((avrg_rcount + avrg_rcount * avrg_rcount * 0.2f) * 10.0f);  // (f32, as the reference)
    a.pass_nr = pass_nr;
    if (threads < 1) threads = (int)std::thread::hardware_concurrency();
    if (threads < 1) threads = 1;
    halton_seq();
    const bool sqr = lv->sqr != 0;
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; t++)
        ts.emplace_back([&, t]() {
            Tracer tr(&c);
            for (int y = t; y < h; y += threads)
                for (int x = 0; x < w; x++) mc_pixel(tr, a, sqr, x + 1, y, recs[(size_t)y * w + x]);
        });
    for (auto &t : ts) t.join();
    return 0;
}

/* McMarch::run on n requests (kinds 0, 1). */
int oracle_mc_batch(const mb3d_cu_scene *sc, int secant, const mb3d_cu_mc_req *reqs, uint32_t n, mb3d_cu_mc_res *res,
                    int threads) {
    McCtx c;
    std::string err;
    mb3d_cu_mc_light lv;
    std::memset(&lv, 0, sizeof(lv));
    if (!make_ctx(*sc, lv, 0, secant, 1.0f, c, err)) return -22;
    if (threads < 1) threads = (int)std::thread::hardware_concurrency();
    if (threads < 1) threads = 1;
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; t++)
        ts.emplace_back([&, t]() {
            McMarch mm(&c);
            for (uint32_t i = (uint32_t)t; i < n; i += (uint32_t)threads) {
                const mb3d_cu_mc_req &r = reqs[i];
                McReqO q;
                q.kind = r.kind;
                std::memcpy(q.pos, r.pos, sizeof(q.pos));
                std::memcpy(q.dir, r.dir, sizeof(q.dir));
                q.zz = r.zz;
                q.zz2 = r.zz2;
                q.zzplus = r.zzplus;
                q.len = r.len;
                q.seed = r.seed;
                q.probe = r.probe != 0;
                McResO o = mm.run(q);
                mb3d_cu_mc_res &d = res[i];
                std::memset(&d, 0, sizeof(d));
                std::memcpy(d.pos, o.pos, sizeof(d.pos));
                std::memcpy(d.normals, o.normals, sizeof(d.normals));
                d.zz = o.zz;
                d.zz2 = o.zz2;
                d.len = o.len;
                d.dyn_fog = o.dyn_fog;
                d.ms_de_stop = o.ms_de_stop;
                d.seed = o.seed;
                d.si_grad = o.si_grad;
                d.otrap = o.otrap;
                d.kind = (uint8_t)o.kind;
                d.de_limited = o.de_limited ? 1 : 0;
            }
        });
    for (auto &t : ts) t.join();
    return 0;
}

/* The Halton record of ray number i and the shifts of pixel (x1, y). */
void oracle_mc_halton(int i, int x1, int y, uint16_t rec[4], float shifts[2]) {
    const HaltonRec &h = halton_seq()[i & 0xFFFF];
    rec[0] = h.hrx;
    rec[1] = h.hry;
    rec[2] = h.hdx;
    rec[3] = h.hdy;
    halton_2d_shifts(x1, y, shifts[0], shifts[1]);
}

int32_t oracle_mc_seed_of(int32_t x, int32_t y, uint32_t b) { return mc_seed_of(x, y, b); }

}  // extern "C"
