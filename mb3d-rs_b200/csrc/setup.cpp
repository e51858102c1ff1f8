// Host set-up of the per-render parameters: the scene (mb3d_cu_scene) turned
// into the flat DevParams block, as mb3d-rs's CalcParams::new does it
// (`GetMCTparasFromHeader`, src/calc.rs:375-891), for the alternating 3D
// hybrid with the built-in formulas; plus the shadow light vectors
// (render::shadow_job, src/render.rs:2383-2415) and the DE AO ray table
// (deao::build_rays, src/deao.rs:75-104).
#include "setup.h"
#include "kernels.h"
#include <cmath>
#include <cstring>
#include <algorithm>
#include <string>

namespace mb3dcu {

static const double kPi = 3.14159265358979323846;
static inline double deg2rad(double d) { return d * (kPi / 180.0); }

// Formula meta data (src/formulas.rs:492-569); the Menger IFS has its .m3f
// header's values (.DEoption 2, .DEscale 0.2, .RStop 1024).
static int f_de_option(int f) {
    return f == MB3D_CU_F_AMAZINGBOX ? 11 : f == MB3D_CU_F_MENGERIFS ? 2 : f == MB3D_CU_F_QUATERNION ? 4 : 0;
}
static double f_de_scale(int f) {
    if (f == MB3D_CU_F_AMAZINGBOX || f == MB3D_CU_F_BULBOX || f == MB3D_CU_F_MENGERIFS) return 0.2;
    if (f == MB3D_CU_F_FOLDINGINTPOW) return 0.5;
    return 1.0;
}
static double f_rstop(int f) {
    return (f == MB3D_CU_F_AMAZINGBOX || f == MB3D_CU_F_BULBOX || f == MB3D_CU_F_FOLDINGINTPOW || f == MB3D_CU_F_MENGERIFS)
               ? 1024.0
               : 16.0;
}
static int f_ipow(const mb3d_cu_slot &s) {
    double r = std::round(s.options[0]);
    int p = std::isnan(r) ? 0 : (r > 1e9 ? 1000000000 : (r < -1e9 ? -1000000000 : (int)r));
    return std::min(8, std::max(2, p));
}
static double f_si_pow(const mb3d_cu_slot &s) {
    switch (s.formula) {
        case MB3D_CU_F_INTPOW: return (double)f_ipow(s);
        case MB3D_CU_F_REALPOWER: case MB3D_CU_F_AEXIONC: return s.options[0] == 0.0 ? 1e-40 : s.options[0];
        case MB3D_CU_F_MENGERIFS: return 0.0;
        default: return 2.0;
    }
}
static bool f_first_is_zmul(int f) { return f == MB3D_CU_F_INTPOW || f == MB3D_CU_F_FOLDINGINTPOW; }
static double f_first_option(const mb3d_cu_slot &s) { return f_first_is_zmul(s.formula) ? s.options[1] : s.options[0]; }
static bool f_known(int f) {
    return f == MB3D_CU_F_INTPOW || f == MB3D_CU_F_REALPOWER || f == MB3D_CU_F_TRICORN || f == MB3D_CU_F_AMAZINGBOX ||
           f == MB3D_CU_F_BULBOX || f == MB3D_CU_F_FOLDINGINTPOW || f == MB3D_CU_F_MENGERIFS ||
           f == MB3D_CU_F_QUATERNION || f == MB3D_CU_F_AEXIONC;
}

// CheckFormulaOptions (combine_de_options_range, src/calc.rs:315-372): the
// DE option of slots start..end
static int de_option_of(const int *des, const int *its, int start, int end) {
    int opt = -1;
    for (int x = start; x <= end; x++) {
        if (its[x] == 0) continue;
        int de = des[x];
        if (de < 0 || de == opt) continue;
        if (opt == -1 || opt == 21 || opt == 22) opt = de;
        else if (opt == 2) opt = (de == 2 || de == 5 || de == 6 || de == 11) ? 2 : 0;
        else if (opt == 4) opt = (de == 5 || de == 6) ? 4 : 0;
        else if (opt == 5) opt = de == 4 ? 4 : (de == 2 || de == 11) ? 2 : (de != 6 ? 0 : 5);
        else if (opt == 6) opt = (de == 2 || de == 4 || de == 5 || de == 11) ? de : 0;
        else if (opt == 11) opt = (de == 2 || de == 5) ? 2 : (de != 6 ? 0 : 11);
    }
    return opt;
}

// BuildSMatrix4 (src/math.rs:176-206): the 4D rotation from the XW, YW and
// ZW plane angles, each element rounded to single precision
static void build_smatrix4(double xw, double yw, double zw, double out[4][4]) {
    auto ini = [](double m[4][4]) {
        for (int i = 0; i < 4; i++)
            for (int k = 0; k < 4; k++) m[i][k] = i == k ? 1.0 : 0.0;
    };
    auto mul = [](const double a[4][4], const double b[4][4], double r[4][4]) {
        for (int i = 0; i < 4; i++)
            for (int k = 0; k < 4; k++) {
                double acc = 0.0;
                for (int q = 0; q < 4; q++) acc += a[i][q] * b[q][k];
                r[i][k] = acc;
            }
    };
    double m1[4][4], m2[4][4], m3[4][4], t[4][4];
    ini(m1);
    m1[0][0] = std::cos(xw); m1[3][3] = std::cos(xw); m1[0][3] = -std::sin(xw); m1[3][0] = std::sin(xw);
    ini(m2);
    m2[1][1] = std::cos(yw); m2[3][3] = std::cos(yw); m2[1][3] = -std::sin(yw); m2[3][1] = std::sin(yw);
    mul(m2, m1, t);
    ini(m3);
    m3[2][2] = std::cos(zw); m3[3][3] = std::cos(zw); m3[2][3] = -std::sin(zw); m3[3][2] = std::sin(zw);
    mul(m3, t, out);
    for (int i = 0; i < 4; i++)
        for (int k = 0; k < 4; k++) out[i][k] = (double)(float)out[i][k];
}

// ipol_de_option (src/calc.rs:255-308): CheckDEoption of the two weighted
// formulas (a weight counts when its bits as a signed integer are > 0)
static int ipol_de_option(const int *des, const float *raw) {
    int opt = -1;
    for (int x = 0; x < 2; x++) {
        int32_t bits;
        std::memcpy(&bits, &raw[x], 4);
        if (bits <= 0) continue;
        const int de = des[x];
        if (de < 0 || de > 20 || de == opt) continue;
        if ((opt >= 0 && opt < 20 && de > 19) || (opt > 19 && de >= 0 && de < 20)) return -1;
        if (opt == -1) opt = de;
        else if (opt == 2) opt = (de == 2 || de == 5 || de == 6 || de == 11) ? 2 : 0;
        else if (opt == 4) opt = (de == 5 || de == 6) ? 4 : 0;
        else if (opt == 5) opt = de == 4 ? 4 : (de == 2 || de == 11) ? 2 : (de != 6 ? 0 : 5);
        else if (opt == 6) opt = (de == 2 || de == 4 || de == 5 || de == 11) ? de : 0;
        else if (opt == 11) opt = (de == 2 || de == 5) ? 2 : (de != 6 ? 0 : 11);
    }
    return opt > 19 ? 20 : opt;
}

int unsupported_reason(const mb3d_cu_scene &sc, std::string &why) {
    if (sc.width <= 0 || sc.height <= 0 || sc.width > 65536 || sc.height > 65536) {
        why = "the picture size must be 1..65536 pixels each way";
        return MB3D_CU_EINVAL;
    }
    if (sc.n_slots < 1 || sc.n_slots > MB3D_CU_SLOTS) {
        why = "n_slots must be 1..6";
        return MB3D_CU_EINVAL;
    }
    if (!(sc.zoom > 0.0) || !(sc.fov_y > 0.0) || sc.iterations < 1) {
        why = "zoom and fov must be positive and iterations at least 1";
        return MB3D_CU_EINVAL;
    }
    const bool ipol = sc.interpolation != 0;
    if (ipol && sc.n_slots < 2) {
        why = "an interpolation hybrid needs two formulas";
        return MB3D_CU_EINVAL;
    }
    bool any = false;
    for (int i = 0; i < (ipol ? 2 : sc.n_slots); i++) {
        if (sc.slots[i].iterations == 0 && !ipol) continue;
        any = true;
        if (!f_known(sc.slots[i].formula)) {
            why = "formula #" + std::to_string(sc.slots[i].formula) + " is not built into this backend";
            return 1;
        }
    }
    if (!any) {
        why = "no formula with iterations > 0";
        return MB3D_CU_EINVAL;
    }
    if (sc.deao_quality >= 0 && (sc.deao_dither != 0 || sc.deao_first_step_random != 0)) {
        why = "DE ambient occlusion with dithering or a random first step is not on the card";
        return 1;
    }
    return 0;
}

int setup_params(const mb3d_cu_scene &sc, DevParams &p, std::string &err) {
    int u = unsupported_reason(sc, err);
    if (u < 0) return u;
    if (u > 0) return MB3D_CU_ENOTSUP;
    std::memset(&p, 0, sizeof(p));
    // an interpolation hybrid (src/calc.rs:378-409): the two first formulas,
    // one iteration each, counted, with their weights normalised to a sum
    // of 1 in single precision
    const bool ipol = sc.interpolation != 0;
    float ipw[2] = {1.0f, 0.0f};
    if (ipol) {
        float x1 = sc.ipol_weights[0], x2 = sc.ipol_weights[1];
        float y1 = x1 + x2;
        if (y1 < 1e-10f) {
            y1 = 1.0f;
            x1 = 1.0f;
            x2 = 0.0f;
        } else {
            y1 = 1.0f / y1;
        }
        ipw[0] = x1 * y1;
        ipw[1] = x2 * y1;
    }
    int n = ipol ? 2 : sc.n_slots;
    int its[6] = {0}, des[6] = {0}, fs[6] = {0};
    bool unc[6] = {false};
    for (int i = 0; i < n; i++) {
        its[i] = ipol ? 1 : std::abs(sc.slots[i].iterations);
        unc[i] = !ipol && sc.slots[i].iterations < 0;
        fs[i] = (sc.slots[i].iterations != 0 || ipol) ? sc.slots[i].formula : MB3D_CU_F_INTPOW;
        des[i] = f_de_option(fs[i]);
    }
    // CheckHybridOptions: the last slot with iterations ends the hybrid
    int last = n - 1;
    while (last > 0 && its[last] == 0) last--;
    int nsl = last + 1;
    int end_to = last;
    // a DE combination (src/calc.rs:421-431): part 1 ends at decomb_end1
    // when both parts have slots; none in an interpolation hybrid
    if (sc.decomb < 0 || sc.decomb > 6) {
        err = "decomb must be 0..6";
        return MB3D_CU_EINVAL;
    }
    auto slot_of = [](int v) { return std::min(std::max(v, 0), 5); };
    const bool dc = !ipol && sc.decomb != 0 && slot_of(sc.decomb_end1) < last && slot_of(sc.decomb_start2) <= last;
    if (dc) end_to = slot_of(sc.decomb_end1);
    int rep = std::min(std::max(sc.repeat_from, 0), end_to);
    while (rep > 0 && its[rep] <= 0) rep--;
    int de_option = de_option_of(des, its, 0, end_to);
    if (sc.disable_analytic_de) {
        if (de_option == 2 || de_option == 11) de_option = 0;
        else if (de_option == 5 || de_option == 6) de_option = 4;
    }
    if (ipol) {
        de_option = ipol_de_option(des, sc.ipol_weights);
        if (de_option >= 20) {
            err = "dIFS formulas do not work in an interpolation hybrid";
            return MB3D_CU_EINVAL;
        }
    }
    if (de_option < 0) {
        err = "formula option is not valid";
        return MB3D_CU_EINVAL;
    }
    // a 4D hybrid (HybridMode::Alt4D) with the 4D numerical DE (option 4);
    // the analytic 4D DE (options 5, 6) and 4D interpolation are not built
    const bool four_d = de_option >= 4 && de_option <= 6;
    if (four_d && de_option != 4) {
        err = "4D hybrids with the analytic DE are not built into this backend";
        return MB3D_CU_ENOTSUP;
    }
    bool custom = de_option == 2 || de_option == 5 || de_option == 6 || de_option == 11 || de_option == 20;
    // the second part of a DE combination (src/calc.rs:491-520; the card
    // has no dIFS formulas, options 20 and up)
    int s2 = 0, e2 = 0, rep2 = 0, de2 = -1;
    if (dc) {
        s2 = std::min(slot_of(sc.decomb_start2), last);
        e2 = std::min(std::max(slot_of(sc.decomb_end2), s2), last);
        de2 = de_option_of(des, its, s2, e2);
        if (sc.disable_analytic_de) {
            if (de2 == 2 || de2 == 11) de2 = 0;
            else if (de2 == 5 || de2 == 6) de2 = 4;
        }
        if (de2 < 0) {
            err = "DE combination: the second formula part has no valid DE option";
            return MB3D_CU_EINVAL;
        }
        if (sc.decomb == 6 && de2 != 20) {
            err = "DE combination 'mix': the second hybrid part must be dIFS";
            return MB3D_CU_EINVAL;
        }
        if (four_d || (de2 >= 4 && de2 <= 6)) {
            err = "4D hybrids in a DE combination are not built into this backend";
            return MB3D_CU_ENOTSUP;
        }
        rep2 = std::min(std::max(slot_of(sc.decomb_repeat2), s2), e2);
        while (rep2 > s2 && its[rep2] <= 0) rep2--;
    }
    const bool custom2 = dc && (de2 == 2 || de2 == 5 || de2 == 6 || de2 == 11 || de2 == 20);
    for (int i = 0; i < nsl; i++) unc[i] = unc[i] || des[i] < 0 || des[i] > 20;

    // DE scale, colour helpers and the smooth iteration logs
    const bool custom_p1 = custom;
    float fhln[6];
    for (int k = 0; k < 6; k++) fhln[k] = (float)(1.0 / std::log(2.0));
    double cnt_n = 0, sum_x = 0, sum_y = 0, cnt_i = 0;
    // (a DE combination: part 1's scale is taken at part 2's first slot and
    // the sums start again)
    bool have_p1 = false;
    double dde_p1 = 1.0;
    for (int x = 0; x < nsl; x++) {
        if (its[x] == 0) continue;
        const bool second = dc && x > end_to;
        if (second && !have_p1) {
            dde_p1 = (cnt_n > 0.0 && de_option != 20) ? sum_x / cnt_n : 1.0;
            have_p1 = true;
            cnt_n = sum_x = sum_y = cnt_i = 0.0;
        }
        const bool custom = second ? custom2 : custom_p1;
        const mb3d_cu_slot &s = sc.slots[x];
        if (ipol || !unc[x]) {
            double sip = f_si_pow(s);
            double z1 = sip > 1.0 ? sip : f_first_option(s);
            fhln[x] = (float)(1.0 / std::log(std::fmax(2.0, std::fabs(z1))));
        }
        // (an interpolation hybrid: weighted by the weights, counted once)
        double w = ipol ? (double)ipw[x] : (double)its[x];
        const double cnt = ipol ? 1.0 : w;
        int j = des[x];
        if (custom && (ipol || !unc[x]) && (j == 5 || j == 11)) {
            cnt_n += cnt;
            cnt_i += cnt;
            double x2 = f_first_option(s);
            if (x2 == 0.0) x2 = 1e-40;
            sum_x += x2 < 0.0 ? 0.65 * w : (x2 * 1.2 + 1.0) / x2 * w;
            sum_y += std::fabs(x2) * w;
        } else if (j >= 0 || ipol) {
            cnt_n += cnt;
            sum_x += (custom ? 1.0 : f_de_scale(fs[x])) * w;
        }
    }
    double dde = 1.0, dde2 = 1.0;
    float col_plus = 0.f;
    if (have_p1) {
        dde = dde_p1;
        if (cnt_n > 0.0 && de2 != 20) dde2 = sum_x / cnt_n;
    } else if (cnt_n > 0.0 && de_option != 20) {
        dde = ipol ? sum_x : sum_x / cnt_n;
    }
    if (cnt_n > 0.0 && cnt_i > 0.0) col_plus = (float)(std::pow(std::fabs(sum_y / cnt_i), 0.25) * 40.0 - 49.0);
    // mctColVarDEstopMul (src/calc.rs:591-652): of the first part, or of a
    // DE combination's part with more iterations
    float col_var = 0.6f;
    {
        double a = 0, b = 0, b1 = 0;
        int ia = 0, itmp = 0;
        bool second = false;
        for (int x = 0; x < nsl; x++) {
            if (!(ipol || (its[x] > 0 && !unc[x]))) {
                if (its[x] > 0) (x > end_to ? ia : itmp)++;
                continue;
            }
            if (x > end_to && !second) {
                second = true;
                col_var = b > 0.0 ? (float)(a / b) : 0.6f;
                b1 = b;
                a = b = 0.0;
                if (!dc || de2 == 20) break;
            }
            double w = ipol ? (double)ipw[x] : (double)its[x];
            int de = des[x];
            if (de == 0 || de == 4) {
                a += w * 0.6;
                b += w;
            } else if (((de >= 1 && de <= 3) || (de >= 5 && de <= 40)) && !f_first_is_zmul(fs[x])) {
                double v = f_first_option(sc.slots[x]);
                if (v > 1.0) {
                    if (v < 1.2) v = 1.1 + (v - 1.0) * (v - 1.0) * 2.5;
                    a += w * 0.5 / (std::log(v) + 0.03);
                    b += w;
                } else if (v < -1.0) {
                    if (v > -1.2) v = -1.1 - (v + 1.0) * (v + 1.0) * 2.5;
                    a += w * 0.5 / (std::log(-v) + 0.03);
                    b += w;
                }
            }
        }
        if ((b >= b1 && b > 1e-3) || (ia > itmp && std::fabs(b - b1) < 1e-3 && b > 1e-3)) col_var = (float)(a / b);
        else if (b1 < 1e-3) col_var = 0.6f;
    }
    double rstop = sc.rstop;
    if (!(rstop > 0.0)) {
        rstop = 0.0;
        for (int i = 0; i < n; i++)
            if (sc.slots[i].iterations > 0) rstop = std::fmax(rstop, f_rstop(sc.slots[i].formula));
        rstop = std::fmax(rstop, 1.0001);
    }
    const double W = sc.width, H = sc.height;
    double sw = 2.1345 / (sc.zoom * W);
    double fov = deg2rad(sc.fov_y);
    float zsd0 = (float)std::fmax(sc.z_step_div, 0.0001);
    float de_stop = (float)std::fmax(sc.de_stop, 0.001);
    double half = fov * 0.5;
    if (half < 0.01) half = 0.01;
    if (half > 1.5) half = 1.5;
    p.pl_optic_z = (float)(std::cos(half) * half / std::sin(half));
    p.fovx_off = 0.5f * (float)sc.width;
    p.fovx_mul = (float)(fov / H);
    // CalcPPZvals
    p.zcorr = std::sin(std::fmax(deg2rad(sc.fov_y), 1.0) / H);
    p.zc_mul = 32767.0 * 256.0 / (std::sqrt((sc.z_end - sc.z_start) * p.zcorr / sw + 1.0) - 0.999999999);
    p.zend = std::fmax(1e-10, (sc.z_end - sc.z_start) / sw);
    p.mh04zsd = (float)((double)std::max(sc.width, sc.height) * 0.5 * std::sqrt((double)zsd0 + 0.001) *
                        std::fmax(0.01, sc.raystep_limiter));
    // GetDEstopFactor
    if (sc.vary_de_stop_on_fov) {
        double ze = std::fmax(1e-16, (sc.z_end - sc.z_start) / sw);
        double a = 0.01 * H / (std::sin(0.01) * std::fmax(1.0 / 65535.0, deg2rad(sc.fov_y)));
        double b = sw * (a + ze) / a;
        p.de_stop_factor = (float)((b - sw) / (sw * std::fmax(1e-6, ze)));
    }
    // the camera's start plane: its corner and the per-pixel/per-step rows
    double z1 = (sc.z_start - sc.mid[2]) / sw;
    for (int i = 0; i < 3; i++) {
        const double *r = sc.vgrads[i];
        double d = sw / std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        for (int k = 0; k < 3; k++) p.vgrads[i][k] = r[k] * d;
    }
    for (int k = 0; k < 3; k++)
        p.ystart[k] = sc.mid[k] + z1 * p.vgrads[2][k] - (H * 0.5) * p.vgrads[1][k] - (W * 0.5) * p.vgrads[0][k];
    float de_off = std::fmin(de_stop * 0.1f, 0.004f);
    p.d_de_scale = custom ? (float)((double)(float)dde / sw) : (float)dde * de_off;
    p.dc_d_de_scale2 = custom2 ? (float)((double)(float)dde2 / sw) : (float)dde2 * de_off;
    p.de_offset006 = de_off * 0.06f;
    p.de_offset = (float)((double)de_off * sw);
    p.z_step_div = zsd0;
    p.ms_de_sub = 0.f;
    if (sc.step_sub_de_stop) {
        float s = zsd0 * zsd0 + (1.2f * zsd0) * (1.0f - zsd0);
        p.z_step_div = s;
        p.ms_de_sub = std::fmin(std::sqrt(s), 0.9f);
    }
    p.ln_rstop = (float)std::log(std::log(rstop));
    p.d_rstop = (double)(float)(rstop * rstop);
    p.rstop3d = (double)(float)((p.d_rstop * p.d_rstop) * 64.0);
    p.d_rstop_f = (float)p.d_rstop;
    p.rstop3d_f = (float)p.rstop3d;
    // the iterations of both parts of a DE combination (iMaxitF2)
    const int it2 = sc.decomb_iterations2 > 0 ? sc.decomb_iterations2 : sc.iterations;
    const int its_all = !dc ? sc.iterations : sc.decomb > 5 ? sc.iterations + it2 : std::max(sc.iterations, it2);
    p.mcts_m = 32767.0f / (float)std::max(its_all + 1, 1);
    p.d_col_plus = col_plus + (float)its_all * 0.1f;
    p.col_var = col_var;
    p.mct_color_mul = (float)(sc.color_mul * 512.0);
    p.de_stop = de_stop;
    p.step_width = sw;
    p.fov_y = fov;
    p.n_slots = nsl;
    p.end_to = end_to;
    p.repeat_from = rep;
    p.is_custom_de = custom;
    p.de_option = de_option;
    p.max_it = sc.iterations;
    p.min_it = std::min(sc.min_iterations, sc.iterations);
    p.de_add_steps = sc.bin_search_steps;
    p.sm_normals = std::min(8, std::max(0, sc.smooth_normals));
    p.color_option = std::min(sc.color_option, 5);
    p.color_on_it = sc.color_on_it;
    p.dfog_on_it = sc.dfog_on_it;
    p.normals_on_de = (sc.normals_on_de || custom || dc) ? 1 : 0;
    p.first_step_random = sc.first_step_random ? 1 : 0;
    p.do_julia = sc.julia ? 1 : 0;
    p.width = sc.width;
    p.height = sc.height;
    for (int k = 0; k < 6; k++) p.fhln[k] = fhln[k];
    for (int k = 0; k < 4; k++) {
        p.ju[k] = sc.julia_c[k];
        p.ju_f[k] = (float)sc.julia_c[k];
    }
    for (int i = 0; i < nsl; i++) {
        DevSlot &d = p.slots[i];
        d.formula = fs[i];
        d.iterations = its[i];
        d.uncounted = unc[i];
        d.ade = (dc && i > end_to) ? custom2 : custom;
        d.julia_add = sc.julia && fs[i] == MB3D_CU_F_MENGERIFS;
        d.ipow = f_ipow(sc.slots[i]);
        switch (fs[i]) {
            case MB3D_CU_F_INTPOW: d.kind = d.ipow == 8 ? 1 : 2; break;
            case MB3D_CU_F_AMAZINGBOX: d.kind = 4; break;
            case MB3D_CU_F_MENGERIFS: d.kind = 8; break;
            case MB3D_CU_F_REALPOWER: d.kind = 16; break;
            case MB3D_CU_F_TRICORN: d.kind = 32; break;
            case MB3D_CU_F_BULBOX: d.kind = 64; break;
            case MB3D_CU_F_QUATERNION: d.kind = 256; break;
            case MB3D_CU_F_AEXIONC: d.kind = 512; break;
            default: d.kind = 128; break;
        }
        if (its[i] > 0) p.fmask |= d.kind;
        for (int k = 0; k < 8; k++) {
            d.o[k] = sc.slots[i].options[k];
            d.of[k] = (float)sc.slots[i].options[k];
        }
    }
    // slot orders the single precision DE loop has unrolled
    p.sched = SCHED_GENERIC;
    if (nsl == 2 && end_to == 1 && rep == 0 && its[0] == 2 && its[1] == 1 && !unc[0] && !unc[1] &&
        fs[0] == MB3D_CU_F_AMAZINGBOX && p.slots[1].kind == 1 && !p.slots[0].julia_add && !p.slots[1].julia_add)
        p.sched = SCHED_BOX2_IP8;
    else if (nsl == 1 && its[0] >= 1 && !unc[0] && p.slots[0].kind == 1 && !p.slots[0].julia_add)
        p.sched = SCHED_IP8;
    else if (nsl == 2 && end_to == 1 && rep == 0 && its[0] == 1 && its[1] == 1 && !unc[0] && !unc[1] &&
             fs[0] == MB3D_CU_F_MENGERIFS && fs[1] == MB3D_CU_F_AMAZINGBOX && !p.slots[0].julia_add &&
             !p.slots[1].julia_add)
        p.sched = SCHED_MENGER_BOX;
    // single precision coordinates are good enough when the numerical DE
    // offset spans >= 3 single steps at the size of the coordinates, or a
    // pixel step >= 64 of them with an analytic DE (gpu::precision,
    // gpu::step_precision, src/gpu.rs:1019-1040)
    double coord = std::fmax(std::fabs(p.ystart[0]), std::fmax(std::fabs(p.ystart[1]), std::fabs(p.ystart[2]))) +
                   sw * (W + H) + 2.0;
    double eps32 = 1.1920928955078125e-07;
    double prec = custom ? sw / (coord * eps32) : (double)p.de_offset / (coord * eps32);
    p.all_fp64 = custom ? (prec < 64.0) : (prec < 3.0);
    // an interpolation hybrid: the double precision DE only (the single
    // precision march and rays do not carry its blend)
    p.ipol = ipol ? 1 : 0;
    p.ipol_w[0] = ipw[0];
    p.ipol_w[1] = ipw[1];
    p.four_d = four_d ? 1 : 0;
    build_smatrix4(sc.rot_4d[0], sc.rot_4d[1], sc.rot_4d[2], p.smatrix4);
    bool quat = false;
    // (the Quaternion reads a fourth component of j, Aexion C writes j: both
    // only on the sequential record)
    for (int i = 0; i < nsl; i++)
        quat = quat || ((fs[i] == MB3D_CU_F_QUATERNION || fs[i] == MB3D_CU_F_AEXIONC) && its[i] > 0);
    // the DE combination's second part (DeComb, src/calc.rs:730-760): its
    // place turns the point into the part's own space, m * (p - offset)
    // with m the rotation divided by the size, and scales its distances
    if (dc) {
        p.dc_kind = sc.decomb;
        p.dc_start2 = s2;
        p.dc_end2 = e2;
        p.dc_rep2 = rep2;
        p.dc_max_it2 = std::max(it2, 1);
        p.dc_de_option2 = de2;
        p.dc_custom2 = custom2 ? 1 : 0;
        p.dc_smooth = (double)std::max(sc.decomb_smooth, 1e-30f) / sw;
        const double scale = sc.part2_scale > 0.0 ? sc.part2_scale : 1.0;
        const double *o = sc.part2_offset, *r = sc.part2_rotation;
        const bool placed = o[0] != 0.0 || o[1] != 0.0 || o[2] != 0.0 || r[0] != 0.0 || r[1] != 0.0 || r[2] != 0.0 ||
                            scale != 1.0;
        p.dc_place = (placed && sc.decomb != 6) ? 1 : 0;
        if (p.dc_place) {
            // build_rot_matrix (src/math.rs:466-475), rows to length 1 / scale
            const double sx = std::sin(deg2rad(r[0])), cx = std::cos(deg2rad(r[0]));
            const double sy = std::sin(deg2rad(r[1])), cy = std::cos(deg2rad(r[1]));
            const double sz = std::sin(deg2rad(r[2])), cz = std::cos(deg2rad(r[2]));
            const double m[3][3] = {{cy * cz, -cy * sz, sy},
                                    {sx * sy * cz + cx * sz, cx * cz - sx * sy * sz, -sx * cy},
                                    {sx * sz - cx * sy * cz, cx * sy * sz + sx * cz, cx * cy}};
            const double len = 1.0 / std::fmax(scale, 1e-300);
            for (int i = 0; i < 3; i++) {
                const double d = len / std::sqrt(m[i][0] * m[i][0] + m[i][1] * m[i][1] + m[i][2] * m[i][2]);
                for (int k = 0; k < 3; k++) p.dc_m[i][k] = m[i][k] * d;
                p.dc_offset[i] = o[i];
            }
            p.dc_scale = scale;
        }
    }
    p.seq_de = (ipol || four_d || quat || dc) ? 1 : 0;
    if (p.seq_de) {
        p.all_fp64 = 1;
        p.sched = SCHED_GENERIC;
        p.fmask |= KSET_ALL;  // (only the all-formula kernels carry the sequential DE)
    }
    p.coord_eps = coord * eps32;
    p.hand_margin = 4.0f;
    p.hand_back = 2;
    // (a DE combination's surfaces too: the FP64 marcher keeps the ruling
    // part's iteration limit between its DEs, as the reference's marcher)
    p.finish_slow = (p.sm_normals > 0 || !p.normals_on_de || p.color_on_it != 0 || dc) ? 1 : 0;
    // (measured on the 1920x1080 hybrid frame: the march and its finish are
    // fastest when a warp takes new rays only once all of its lanes are idle
    // -- rays that start together iterate alike -- the shadow and DE AO rays
    // when a quarter of the lanes are idle)
    p.refill_min = 32;
    p.refill_shadow = 8;
    p.refill_ao = 8;
    p.blocks_march32 = 4;
    p.blocks_per_sm = 3;

    // shadow lights (render::shadow_job): HSvecs = RotateVectorReverse(-sw * LN, M)
    p.n_lights = 0;
    double m[3][3];
    for (int i = 0; i < 3; i++) {
        const double *r = p.vgrads[i];
        double d = 1.0 / std::sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]);
        for (int k = 0; k < 3; k++) m[i][k] = r[k] * d;
    }
    for (int idx = 0; idx < 6; idx++) {
        const mb3d_cu_light &li = sc.lights[idx];
        if (!li.on || !((sc.shadow_lights >> idx) & 1)) continue;
        double a = -li.x_angle, b = li.y_angle;
        double v[3] = {-std::sin(a), std::sin(b), std::cos(b) * std::cos(a)};
        double nv = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        double ln[3] = {(double)(float)(-v[0] / nv), (double)(float)(-v[1] / nv), (double)(float)(-v[2] / nv)};
        double l = std::sqrt(ln[0] * ln[0] + ln[1] * ln[1] + ln[2] * ln[2]);
        if (l > 0.0)
            for (int k = 0; k < 3; k++) ln[k] = ln[k] * (1.0 / l);
        double w[3] = {-ln[0] * sw, -ln[1] * sw, -ln[2] * sw};
        int q = p.n_lights++;
        p.light_idx[q] = idx;
        for (int k = 0; k < 3; k++) p.light_vec[q][k] = w[0] * m[0][k] + w[1] * m[1][k] + w[2] * m[2][k];
    }
    if (sc.shadow_soft && p.n_lights > 1) {
        p.light_idx[0] = p.light_idx[p.n_lights - 1];
        for (int k = 0; k < 3; k++) p.light_vec[0][k] = p.light_vec[p.n_lights - 1][k];
        p.n_lights = 1;
    }
    p.shadow_soft = sc.shadow_soft ? 1 : 0;
    p.soft_radius = sc.soft_radius;
    p.hs_max_len_mul = sc.hs_max_len_mul;

    for (int i = 0; i < 3; i++) {
        double d = sw / std::sqrt(p.vgrads[i][0] * p.vgrads[i][0] + p.vgrads[i][1] * p.vgrads[i][1] + p.vgrads[i][2] * p.vgrads[i][2]);
        for (int k = 0; k < 3; k++) p.ao_rot[i][k] = p.vgrads[i][k] * d;
    }
    // DE AO rays (deao::build_rays)
    p.ao_quality = sc.deao_quality;
    p.ao_max_len = sc.deao_max_len;
    p.ao_first_step_random = sc.deao_first_step_random;
    if (sc.deao_quality >= 0) {
        int q = std::min(sc.deao_quality, 3);
        int nr = 0;
        auto put = [&](double ya, double za) {
            double sy = std::sin(ya), cy = std::cos(ya), sz = std::sin(za), cz = std::cos(za);
            p.ao_dirs[nr][0] = (float)(sy * cz);
            p.ao_dirs[nr][1] = (float)(-sy * sz);
            p.ao_dirs[nr][2] = (float)(-cy);
            nr++;
        };
        const double tau = 2.0 * kPi;
        if (q == 0) {
            double abr = deg2rad(60.0);
            for (int x = 0; x < 3; x++) put(0.5 * abr, (double)x * tau / 3.0);
            p.ao_d_step_mul = 1.8f;
            p.ao_d_min_a_dif = -1.0f;
            p.ao_corr_weight = 0.3f;
        } else {
            put(0.0, 0.0);
            double abr = (kPi / 2.0) / ((double)q + 0.9);
            for (int y = 1; y <= q; y++) {
                double t = (double)y * abr;
                int cnt = (int)std::nearbyint(std::sin(t) * tau / abr);
                for (int x = 0; x < cnt && nr < MB3D_MAX_AO_RAYS; x++) put(t, (double)x * tau / (double)cnt);
            }
            p.ao_d_step_mul = (float)(1.0 + std::sin(abr));
            p.ao_d_min_a_dif = (float)std::cos(abr * 1.2);
            p.ao_corr_weight = q == 1 ? 0.2f : 0.1666f;
        }
        p.ao_rays = nr;
    }
    return 0;
}

// deao_1pos's directions (ray_dir, src/reflect.rs:968-972) and constants
// (:975-998) per quality, with the pairs' angle terms of its correction
// (:1058-1084), in the reference's precisions
void reflect_ao_table(ReflAO &t) {
    std::memset(&t, 0, sizeof(t));
    const double PI_ = 3.14159265358979323846, TAU_ = 2.0 * PI_;
    auto ray_dir = [](double ya, double za, float *o) {
        const double sy = std::sin(ya), cy = std::cos(ya), sz = std::sin(za), cz = std::cos(za);
        o[0] = (float)(sy * cz);
        o[1] = (float)(-sy * sz);
        o[2] = (float)(-cy);
    };
    int at = 0;
    for (int q = 0; q < 4; q++) {
        t.first[q] = at;
        float d_min_a_dif;
        if (q == 0) {
            const double abr = 60.0 * (PI_ / 180.0);
            for (int i = 0; i < 3; i++) ray_dir(0.5 * abr, (double)i * TAU_ / 3.0, t.dirs[at++]);
            t.d_step_mul[q] = 1.8;
            d_min_a_dif = -1.0f;
            t.corr_w[q] = 0.3f;
        } else {
            const double abr = (PI_ / 2.0) / ((double)q + 0.9);
            ray_dir(0.0, 0.0, t.dirs[at++]);
            for (int iy = 1; iy <= q; iy++) {
                const int n = (int)std::nearbyint(std::sin(0.25) * TAU_ / abr);
                for (int ix = 0; ix < n; ix++) ray_dir(abr * (double)iy, (double)ix * TAU_ / (double)n, t.dirs[at++]);
            }
            t.d_step_mul[q] = 1.0 + std::sin(abr);
            d_min_a_dif = (float)std::cos(abr * 1.2);
            t.corr_w[q] = q == 1 ? 0.2f : 0.1666f;
        }
        t.count[q] = at - t.first[q];
        const double de_mul = std::sqrt((double)t.count[q] * 0.5);
        const double abr_c = 1.2 / std::asin(std::fmin(std::fmax(1.0 / de_mul, -1.0), 1.0));
        for (int k = 0; k < t.count[q]; k++)
            for (int k2 = 0; k2 < t.count[q]; k2++) {
                const float *a = t.dirs[t.first[q] + k], *b = t.dirs[t.first[q] + k2];
                const float dt = a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
                t.ang[q][k][k2] = k != k2 && dt > d_min_a_dif
                                      ? (float)((double)std::acos(std::fmin(std::fmax(dt, -1.0f), 1.0f)) * abr_c)
                                      : REFL_AO_NO;
            }
    }
}

}  // namespace mb3dcu
