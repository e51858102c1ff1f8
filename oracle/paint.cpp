// TEST INFRASTRUCTURE: the Calculate 3D painter of the reference on the CPU,
// for the parity metric "PSNR of one painter applied to both G-buffers" (the
// card's march and the oracle's).  A single precision restatement of
// render::paint (src/render.rs:2499-2501, paint_core :2676-2720) for the
// scenes of this project: Lighting::default (src/lighting.rs:290-391) with
// the scene's lights switched on and turned, LightVals::build
// (:978-1190), effective_lighting (src/render.rs:2275-2283), the paint
// camera (:2340-2370, common optic, no stereo), plv_for_pixel
// (src/lighting.rs:1764-1796), shade (:1802-2162) and pixel_color_s
// (:1739-1760) in 8 bits, along the default path: directional lights not
// visible in the picture, no internal gamma 2, no light or colour maps, no
// background picture, no surface detail or material, no ground, no clouds,
// reflections or depth of field.
#include <cmath>
#include <cstdint>
#include <array>
#include <cstring>
#include <string>
#include <vector>

#include "../include/mb3d_cu.h"
#include "oracle.hpp"

namespace oracle {
namespace {

using SV = std::array<float, 3>;

SV sv(float a, float b, float c) { return SV{a, b, c}; }
SV add(SV a, SV b) { return sv(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
SV scale(SV a, float s) { return sv(a[0] * s, a[1] * s, a[2] * s); }
SV mul(SV a, SV b) { return sv(a[0] * b[0], a[1] * b[1], a[2] * b[2]); }
void add_w(SV &a, SV b, float w) {
    a[0] += b[0] * w;
    a[1] += b[1] * w;
    a[2] += b[2] * w;
}
// lerp(sv1, sv2, w1) = sv2 + w1 (sv1 - sv2) (src/lighting.rs:563-569)
SV lerp(SV a, SV b, float w) { return sv(b[0] + w * (a[0] - b[0]), b[1] + w * (a[1] - b[1]), b[2] + w * (a[2] - b[2])); }
float dot(SV a, SV b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

// Delphi TColor ($BBGGRR) -> r, g, b (src/lighting.rs:285-288)
SV col255(uint32_t c) { return sv((float)(c & 0xFF), (float)((c >> 8) & 0xFF), (float)((c >> 16) & 0xFF)); }
SV col1(uint32_t c) { return scale(col255(c), 1.0f / 255.0f); }

// SetCosTabFunction (src/lighting.rs:464-499)
struct CosTabs {
    float diff[8][128];
    CosTabs() {
        for (int i = 0; i < 128; i++) {
            double d = 1.0 - ((double)i - 2.0) / 60.0;
            diff[0][i] = d > 0.15 ? (float)((d - 0.08) * 1.0869565) : d <= 0.0 ? 0.0f : (float)std::pow(d, std::fmax(1.0, (0.505 - d) * 3.8));
            double dc = std::fmax(d, 0.0);
            diff[1][i] = (float)(dc * dc);
            diff[2][i] = (float)(d * 0.5 + 0.5);
            diff[3][i] = (float)((d * 0.5 + 0.5) * (d * 0.5 + 0.5));
        }
        for (int k = 0; k < 4; k++) {
            float tmp[128];
            for (int j = 0; j < 128; j++) tmp[j] = std::sqrt(std::fmax(diff[k][j], 0.0f));
            for (int j = 0; j < 128; j++) {
                double e = 0.0;
                for (int i = 0; i <= 60; i++) {
                    int l = std::abs(j + i - 30);
                    if (l < 128) e += (double)tmp[l];
                }
                double a = e * 0.011 + (e * 0.007) * (e * 0.007);
                diff[k + 4][j] = (float)(a * a);
            }
        }
    }
};
const CosTabs &cos_tabs() {
    static const CosTabs t;
    return t;
}

// make_spline_coeff (src/math.rs:263-269)
void spline_coeff(double xs, float w[4]) {
    double r3 = xs * xs * xs / 6.0;
    double r0 = 1.0 / 6.0 + 0.5 * xs * (xs - 1.0) - r3;
    double r2 = xs + r0 - 2.0 * r3;
    double r1 = 1.0 - r0 - r2 - r3;
    w[0] = (float)r0;
    w[1] = (float)r1;
    w[2] = (float)r2;
    w[3] = (float)r3;
}

// GetCosTabVal (src/lighting.rs:501-532), no internal gamma 2
float cos_tab_val(int tnr, float dotp, float rough) {
    const CosTabs &tabs = cos_tabs();
    float t = 62.0f - 60.0f * dotp;
    int ip = (int)std::trunc(t) - 1;
    if (ip < 0) {
        ip = 0;
        t = 0.0f;
    } else if (ip > 124) {
        ip = 124;
        t = 1.0f;
    } else {
        t = t - std::trunc(t);
    }
    float w[4];
    spline_coeff((double)t, w);
    float a = 0.0f, b = 0.0f;
    for (int k = 0; k < 4; k++) a += tabs.diff[tnr][ip + k] * w[k];
    for (int k = 0; k < 4; k++) b += tabs.diff[tnr + 4][ip + k] * w[k];
    return a + rough * (b - a);
}

// FastIntPow (src/math.rs:273-285)
float fast_int_pow(float base, int expo) {
    if (base < 0.0f) return 0.0f;
    float r = base;
    for (int i = expo >> 1; i > 0; i >>= 1) r *= r;
    return r;
}

struct Light {
    SV ln, col;
    int pow_func, diff_func, idx;
    bool sub_amb_sh, hs_calced;
    uint16_t hs_mask;
};

struct Lv {
    std::vector<Light> lights;
    SV amb_col, amb_col2, depth_col, depth_col2, dyn_fog_col, dyn_fog_col2;
    float s_depth, s_shad, s_shad_gr, s_shad_zmul, s_dyn_fog_mul, s_amb_shad, s_diff, s_spec, s_ind_light_reflect;
    float s_col_zmul, s_c_start, s_c_mul, s_ci_start, s_ci_mul, s_roughness_factor, s_diffuse_shadowing;
    SV col_dif[10], col_spe[10], col_int[4];
    float col_spe_a[10], s_c_div[10], col_int_spec[4], s_ic_div[4];
    int col_pos[10], icol_pos[4];
};

// LightVals::build for Lighting::default with the scene's lights, as
// light_vals (src/render.rs:2285-2331) calls it for a still picture
Lv light_vals(const mb3d_cu_scene &sc, double step_width) {
    Lv o;
    const uint32_t cols[9] = {5873889, 8837614, 0x8B491D, 2988346, 12248958, 0xFFC49F, 11287584, 14579248, 7481121};
    for (int idx = 0; idx < 6; idx++) {
        const mb3d_cu_light &li = sc.lights[idx];
        if (!li.on) continue;
        // the preset's light 0 and 1, and defaultLight8 (src/lighting.rs:125-145, 309-330)
        uint32_t color = idx == 0 ? 0xA0E8FFu : idx == 1 ? 2307911u : 0xFFFFFFu;
        int spec_func = idx == 0 ? (53 & 7) : idx == 1 ? (16 & 7) : 4;
        int diff_func = idx == 0 ? ((53 >> 4) & 3) : idx == 1 ? ((16 >> 4) & 3) : 0;
        // effective_lighting: hs_calced, hs_soft from the scene's shadow pass
        const bool hs_calced = ((sc.shadow_lights & 0x3F) >> idx) & 1;
        const bool hs_soft = sc.shadow_soft != 0, hs_set_cos = false, hs_enabled = true;
        double dtmp = -li.x_angle, dtmp2 = li.y_angle;
        double v[3] = {-std::sin(dtmp), std::sin(dtmp2), std::cos(dtmp2) * std::cos(dtmp)};
        double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        Light L;
        L.ln = sv((float)(-v[0] / n), (float)(-v[1] / n), (float)(-v[2] / n));
        L.col = scale(scale(col255(color), 1.0f), 1.0f);  // x light_scale, x amplitude
        L.pow_func = 2 << (spec_func & 7);
        L.diff_func = hs_calced && hs_set_cos ? 0 : (diff_func & 3);
        L.idx = idx;
        L.sub_amb_sh = hs_calced != hs_enabled;
        L.hs_calced = hs_calced;
        L.hs_mask = hs_soft && hs_calced ? 0xFFFF : (uint16_t)(0x400 << idx);
        o.lights.push_back(L);
    }
    const float zsd = (float)sc.z_step_div;
    o.s_depth = 27.0f * 0.8e-6f;
    float gr = (53.0f - 53.0f) * 1.0f * zsd * 0.00065f, dt = 2.2f / zsd, mul = zsd * 0.015f, stmp = 128.0f;
    if (sc.dfog_on_it > 0) {
        dt *= 0.25f;
        gr *= 4.0f;
        mul *= 4.0f;
    } else {
        stmp = 137.0f;
    }
    o.s_shad_gr = gr;
    o.s_dyn_fog_mul = mul;
    o.s_shad = (stmp - std::sqrt(std::fmax(128.0f, 0.0f)) * 11.313708f) * dt * 0.28f;
    const double z_range = sc.z_end - sc.z_start;
    o.s_shad_zmul = dt * 0.7f / (float)z_range * (128.0f - std::sqrt(std::fmax(128.0f, 0.0f)) * 11.313708f);
    o.s_amb_shad = 53.0f / 53.0f;
    float a = (68.0f + 30.0f) / 90.0f, b = (72.0f + 30.0f) / 90.0f;
    float s_c_start = a * a * 32767.0f - 10900.0f;
    float s_c_mul = b * b * 32767.0f - 10900.0f - s_c_start;
    o.s_c_mul = std::fabs(s_c_mul) > 0.001f ? 2.0f / s_c_mul : (s_c_mul < 0.0f ? -2000.0f : 2000.0f);
    o.s_c_start = s_c_start;
    const float ti = 60.0f;
    float dti = ti * ti * ti * ti;
    o.s_ci_start = dti * 0.000158025f + 32768.0f;
    float cim = (ti * ti * ti * ti - dti) * 0.5f * 0.00031605f;
    o.s_ci_mul = std::fabs(cim) > 1e-10f ? 1.0f / cim : cim;
    const float amb_mul = 90.0f / 90.0f;
    o.amb_col = scale(col255(0x8B491D), amb_mul);
    o.amb_col2 = scale(col255(0xFFC49F), amb_mul);
    o.depth_col = col255(0x8B491D);
    o.depth_col2 = col255(0xFFC49F);
    o.dyn_fog_col = sv(255.0f, 255.0f, 255.0f);
    o.dyn_fog_col2 = sv(255.0f, 255.0f, 255.0f);
    // the palette: three colours at 0, 10922, 21844, then colour 0 from 32200 on
    uint32_t dif[10], spe[10];
    for (int i = 0; i < 10; i++) {
        int j = i < 3 ? i : 0;
        dif[i] = cols[j * 3];
        spe[i] = cols[j * 3 + 1];
        o.col_pos[i] = i < 3 ? i * 10922 : 32200 + (i - 3) * 84;
        o.col_dif[i] = col1(dif[i]);
        o.col_spe[i] = col1(spe[i]);
        SV s = col255(spe[i]);
        float al = std::fmax(s[0], std::fmax(s[1], s[2]));  // palette_alpha
        o.col_spe_a[i] = al / 255.0f;
    }
    for (int i = 0; i < 10; i++) {
        int j = i < 9 ? o.col_pos[i + 1] - o.col_pos[i] : 32767 - o.col_pos[9];
        o.s_c_div[i] = j > 1 ? 1.0f / (float)j : 1.0f;
    }
    // the interior colours (0, 10922, 21844: the palette's, 32700: colour 0)
    for (int i = 0; i < 4; i++) {
        o.icol_pos[i] = i < 3 ? i * 10922 : 32700;
        o.col_int[i] = col1(cols[(i < 3 ? i : 0) * 3]);
        o.col_int_spec[i] = 160.0f / 255.0f;
    }
    for (int i = 0; i < 4; i++) {
        int j = i < 3 ? o.icol_pos[i + 1] - o.icol_pos[i] : 32767 - o.icol_pos[3];
        o.s_ic_div[i] = j > 1 ? 1.0f / (float)j : 1.0f;
    }
    float ind = std::round(std::fmin(std::fmax(53.0f - 53.0f, -128.0f), 127.0f));
    float r = (ind + 53.0f) * 0.022f;
    o.s_ind_light_reflect = r * r;
    o.s_diff = 120.0f * 0.02f;
    o.s_spec = std::fmax(50.0f * 0.02f, 0.004f);
    o.s_col_zmul = (float)(0.0 * -0.005 / (step_width * (double)sc.width));
    o.s_roughness_factor = 0.0f / (255.0f * 255.0f);
    o.s_diffuse_shadowing = 0.0f;
    return o;
}

// CalcColors (src/lighting.rs:1563-1615): diffuse, specular colour, alpha
void colors_alpha(const Lv &lv, uint16_t si_gradient, float idif0, SV &d, SV &s, float &a) {
    float irf = ((float)si_gradient - lv.s_c_start) * lv.s_c_mul + idif0;
    irf = std::fmin(std::fmax(irf * 16384.0f, -1e9f), 1e9f);
    int ir = (int)std::round(irf);
    int il1, il2 = 5;
    float t;
    if (ir < 0) {
        d = lv.col_dif[0], s = lv.col_spe[0], a = lv.col_spe_a[0];
        return;
    }
    if (ir >= lv.col_pos[9]) {
        d = lv.col_dif[9], s = lv.col_spe[9], a = lv.col_spe_a[9];
        return;
    }
    if (lv.col_pos[il2] < ir) {
        do {
            il2 += 1;
        } while (!(il2 == 10 || lv.col_pos[il2] >= ir));
    } else {
        while (il2 > 1 && lv.col_pos[il2 - 1] >= ir) il2 -= 1;
    }
    il1 = il2 - 1;
    if (il2 > 9) il2 = 0;
    t = (float)(ir - lv.col_pos[il1]) * lv.s_c_div[il1];
    d = lerp(lv.col_dif[il2], lv.col_dif[il1], t);
    s = lerp(lv.col_spe[il2], lv.col_spe[il1], t);
    a = lv.col_spe_a[il1] + t * (lv.col_spe_a[il2] - lv.col_spe_a[il1]);
}

// CalcColorsInside (src/lighting.rs:1656-1685)
void colors_inside(const Lv &lv, uint16_t si_gradient, float idif0, SV &d, SV &s) {
    int ir = (int)std::round((((float)si_gradient - lv.s_ci_start) * lv.s_ci_mul + idif0) * 16384.0f);
    float spe;
    if (ir < 0) {
        d = lv.col_int[0];
        spe = lv.col_int_spec[0];
    } else if (ir > lv.icol_pos[3]) {
        d = lv.col_int[3];
        spe = lv.col_int_spec[3];
    } else {
        int il2 = 1;
        while (il2 < 4 && lv.icol_pos[il2] < ir) il2 += 1;
        int il1 = il2 - 1;
        il2 &= 3;
        float t = (float)(ir - lv.icol_pos[il1]) * lv.s_ic_div[il1];
        d = lerp(lv.col_int[il2], lv.col_int[il1], t);
        spe = lv.col_int_spec[il2] + t * (lv.col_int_spec[il1] - lv.col_int_spec[il2]);
    }
    s = sv(spe, spe, spe);
}

struct Cam {
    int width, height;
    float fov, aspect, x_off;
    double zcorr, zc_mul, step_width, zz_stmit_dif;
};

// CalcViewVec, common optic (src/lighting.rs:749-771)
SV view_vec(const Cam &c, float x_pos, float y_pos) {
    float cx = (c.x_off - x_pos) * c.fov * c.aspect;
    float cy = (y_pos - 0.5f) * c.fov;
    SV v = sv(-std::sin(cx), std::sin(cy), std::cos(cy) * std::cos(cx));
    float n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    return scale(v, 1.0f / n);
}

// shade + pixel_color_s of one record
void pixel_color(const Lv &lv, const Cam &cam, const mb3d_cu_silight &si, int x, int y, uint8_t out[3]) {
    // plv_for_pixel
    const float x_pos = (float)(x + 1) / (float)cam.width, y_pos = (float)y / (float)cam.height;
    const SV view = view_vec(cam, x_pos, y_pos);
    const uint32_t zpos_word = si.zpos_fine >> 16;
    double z1;
    if (zpos_word > 32767) {
        double q = 8388352.0 / cam.zc_mul + 1.0;
        z1 = (q * q - 1.0) * cam.step_width / cam.zcorr;
    } else {
        double q = (double)(8388352 - (int64_t)(si.zpos_fine >> 8)) / cam.zc_mul + 1.0;
        z1 = (q * q - 1.0) * cam.step_width / cam.zcorr;
    }
    const float z_pos = (float)(z1 + cam.zz_stmit_dif);
    const SV dep_c = lerp(lv.depth_col2, lv.depth_col, y_pos);  // depth_func 0
    SV o;
    float dtmp;
    if (zpos_word < 32768) {
        const float d_rough = (float)(si.zpos_fine & 0xFF) * lv.s_roughness_factor;
        const float shadow = si.amb_shadow >= 16383 ? 1.0f : (float)si.amb_shadow / 16383.0f;
        float d_amb_sh;
        if (lv.s_amb_shad < 1.0f) {
            d_amb_sh = 1.0f - lv.s_amb_shad * shadow;
        } else {
            float a = 1.0f - shadow;
            d_amb_sh = a + (lv.s_amb_shad - 1.0f) * (a * a - a);
        }
        const SV lns = sv((float)si.normal[0] * 3.0518509476e-5f, (float)si.normal[1] * 3.0518509476e-5f,
                          (float)si.normal[2] * 3.0518509476e-5f);
        SV li_dif = sv(0, 0, 0), li_spe = sv(0, 0, 0), li_amb = sv(0, 0, 0);
        const float d_fog = lv.s_diffuse_shadowing * (d_amb_sh - 1.0f) + 1.0f;
        for (const Light &L : lv.lights) {
            const bool soft = L.hs_mask == 0xFFFF;
            const bool no_hs = soft || (si.shadow & L.hs_mask) == 0 || !L.hs_calced;
            const float soft_mul = soft ? (float)(si.shadow >> 10) * (1.0f / 63.0f) : 1.0f;
            const float att = 1.0f;
            float dt = lns[0] * L.ln[0] + lns[1] * L.ln[1] + lns[2] * L.ln[2];
            float d = cos_tab_val(L.diff_func, dt, d_rough) * att;
            add_w(li_amb, L.col, d);
            if (no_hs) {
                d *= L.sub_amb_sh ? d_amb_sh : d_fog;
                d *= soft_mul;
                add_w(li_dif, L.col, d);
            }
            float d2 = 2.0f * (lns[0] * view[0] + lns[1] * view[1] + lns[2] * view[2]);
            float ds = L.ln[0] * (view[0] - lns[0] * d2) + L.ln[1] * (view[1] - lns[1] * d2) + L.ln[2] * (view[2] - lns[2] * d2);
            if (ds > 0.0f) {
                float pf = (float)L.pow_func;
                float t2 = (att + std::fmin(d_rough * 2.0f, 1.0f) * (1.0f / pf - att)) * lv.s_spec;
                if (t2 > 0.0f) {
                    add_w(li_amb, L.col, t2 / pf);
                    if (no_hs) {
                        t2 *= fast_int_pow(ds, L.pow_func);
                        t2 *= L.sub_amb_sh ? d_amb_sh : d_fog;
                        t2 *= soft_mul;
                        add_w(li_spe, L.col, t2);
                    }
                }
            }
        }
        const float idif0 = lv.s_col_zmul * z_pos;
        SV idif, ispe;
        float ia;
        if (si.si_gradient > 32767) {
            colors_inside(lv, si.si_gradient, idif0, idif, ispe);
            ia = ispe[0];
        } else {
            colors_alpha(lv, si.si_gradient, idif0, idif, ispe, ia);
        }
        (void)ia;
        // ambient light top / bottom
        const float t2 = (lns[1] * 0.5f + 0.5f) * d_amb_sh, t1 = d_amb_sh - t2;
        SV iamb = add(scale(lv.amb_col, t1), scale(lv.amb_col2, t2));
        iamb = mul(iamb, idif);
        const SV dif_s = scale(idif, lv.s_diff);
        const SV total = add(add(iamb, mul(dif_s, li_dif)), mul(ispe, li_spe));
        // CalcTotalLight1
        const SV l3 = add(iamb, scale(mul(dif_s, li_amb), d_amb_sh * 0.3f));
        const float st = std::fmax(1.0f - d_amb_sh, 0.0f);
        const float st2 = st * st * st * st;
        const SV refl = sv(idif[0] * st2 * lv.s_ind_light_reflect + (st - st2), idif[1] * st2 * lv.s_ind_light_reflect + (st - st2),
                           idif[2] * st2 * lv.s_ind_light_reflect + (st - st2));
        o = add(total, mul(l3, mul(idif, refl)));
        dtmp = std::fmax(((float)zpos_word - 28000.0f) * lv.s_depth + 1.0f, 0.0f);
    } else {
        o = dep_c;
        dtmp = std::fmax(1.0f - (float)(60768 - (int32_t)zpos_word) * lv.s_depth, 0.0f);
    }
    // the depth fog and the dynamic fog (no far fog, no background picture)
    o = scale(o, dtmp);
    const float ir = (float)(si.shadow & 0x3FF);
    float dfog = (ir - lv.s_shad - lv.s_shad_zmul * z_pos) * lv.s_shad_gr;
    const float dtmp3 = std::fmin(ir * lv.s_dyn_fog_mul, 1.0f) * dfog;
    o = add(o, scale(dep_c, std::fmax(1.0f - dtmp, 0.0f)));
    o = add(o, add(scale(lv.dyn_fog_col, dfog - dtmp3), scale(lv.dyn_fog_col2, dtmp3)));
    // pixel_color_s in 8 bits: clipped to 0..255, no gamma curve, rounded
    for (int k = 0; k < 3; k++) {
        float c = std::fmin(std::fmax(o[k], 0.0f), 255.0f);
        out[k] = (uint8_t)std::round(c);
    }
}

}  // namespace
}  // namespace oracle

using namespace oracle;

extern "C" {

/* render::paint of rows row0 .. row0+rows-1 of the scene's picture from their
 * G-buffer records (rows * width), 8-bit RGB out. */
int oracle_paint(const mb3d_cu_scene *sc, const mb3d_cu_silight *gbuf, int row0, int rows, uint8_t *rgb) {
    Params p;
    std::string err;
    if (!make_params(*sc, p, err)) return -1;
    Cam cam;
    cam.width = sc->width;
    cam.height = sc->height;
    cam.fov = (float)(sc->fov_y * (3.14159265358979323846 / 180.0));  // f64::to_radians
    cam.aspect = (float)sc->width / (float)sc->height;
    cam.x_off = 0.5f;
    cam.zcorr = p.zcorr;
    cam.zc_mul = p.zc_mul;
    cam.step_width = p.step_width;
    cam.zz_stmit_dif = sc->z_start - sc->mid[2];
    const Lv lv = light_vals(*sc, p.step_width);
    for (int y = 0; y < rows; y++)
        for (int x = 0; x < sc->width; x++) {
            size_t i = (size_t)y * sc->width + x;
            pixel_color(lv, cam, gbuf[i], x, row0 + y, rgb + 3 * i);
        }
    return 0;
}
}
