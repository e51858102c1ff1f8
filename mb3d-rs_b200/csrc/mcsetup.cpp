// Host set-up of the Monte Carlo tracer: the light values of MB3D's start-up
// lighting, the render constants of CalcMCT and the Halton table.
#include <cmath>
#include <cstring>
#include <vector>
#include "mcsetup.h"
#include "setup.h"

namespace mb3dcu {

// Delphi TColor ($BBGGRR) -> r, g, b (src/lighting.rs:285-288)
static void rgb_of(uint32_t c, int o[3]) {
    o[0] = (int)(c & 0xFF);
    o[1] = (int)((c >> 8) & 0xFF);
    o[2] = (int)((c >> 16) & 0xFF);
}

// LightVals::build (src/lighting.rs:978-1190) for Lighting::default
// (src/lighting.rs:290-391) with the scene's lights switched on and turned
// as the scene says; no internal gamma 2, no fine colour adjustment.
int mc_light_default(const mb3d_cu_scene &sc, mb3d_cu_mc_light &o) {
    std::memset(&o, 0, sizeof(o));
    const uint32_t cols[9] = {5873889, 8837614, 0x8B491D, 2988346, 12248958, 0xFFC49F, 11287584, 14579248, 7481121};
    // the lights' colours and specular functions of the preset (light 0,
    // light 1, and defaultLight8 for the others)
    for (int idx = 0; idx < 6; idx++) {
        const mb3d_cu_light &li = sc.lights[idx];
        if (!li.on) continue;
        int c[3];
        rgb_of(idx == 0 ? 0xA0E8FFu : (idx == 1 ? 2307911u : 0xFFFFFFu), c);
        int spec_func = idx == 0 ? (53 & 7) : (idx == 1 ? (16 & 7) : 4);
        double dtmp = -li.x_angle, dtmp2 = li.y_angle;
        double v[3] = {-std::sin(dtmp), std::sin(dtmp2), std::cos(dtmp2) * std::cos(dtmp)};
        double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        int i = o.n_lights++;
        for (int k = 0; k < 3; k++) o.ln[i][k] = (float)(-v[k] / n);
        float raw[3];
        for (int k = 0; k < 3; k++) raw[k] = (float)c[k] * 1.0f;  // col255 x light_scale
        const float amplitude = 1.0f;
        for (int k = 0; k < 3; k++) o.col[i][k] = raw[k] * amplitude;
        o.lmax_l[i] = 800.0f * (raw[0] + raw[1] + raw[2] + 128.0f) * amplitude;
        o.pow_func[i] = 2 << (spec_func & 7);
    }
    int at[3], ab[3], fog[3] = {255, 255, 255};
    rgb_of(0x8B491D, at);
    rgb_of(0xFFC49F, ab);
    const float amb_mul = 90.0f / 90.0f;
    for (int k = 0; k < 3; k++) {
        o.amb_col[k] = (float)at[k] * amb_mul;
        o.amb_col2[k] = (float)ab[k] * amb_mul;
        o.depth_col[k] = (float)at[k];
        o.depth_col2[k] = (float)ab[k];
        o.dyn_fog_col[k] = (float)fog[k];
        o.dyn_fog_col2[k] = (float)fog[k];
    }
    const float depth_fog = 27.0f, dyn_fog = 53.0f, fog_offset = 128.0f, fog_far_offset = 128.0f;
    const float zsd = (float)sc.z_step_div;
    o.s_depth = depth_fog * 0.8e-6f;
    float gr = (dyn_fog - 53.0f) * 1.0f * zsd * 0.00065f;
    float dt = 2.2f / zsd;
    float mul = zsd * 0.015f;
    float stmp = 128.0f;
    if (sc.dfog_on_it > 0) {
        dt *= 0.25f;
        gr *= 4.0f;
        mul *= 4.0f;
    } else {
        stmp = 137.0f;
    }
    o.s_shad_gr = gr;
    o.s_dyn_fog_mul = mul;
    o.s_shad = (stmp - std::sqrt(std::fmax(fog_offset, 0.0f)) * 11.313708f) * dt * 0.28f;
    // z range of the Monte Carlo scene (mc_scene, src/mc.rs:2842-2850)
    double sw = 2.1345 / (sc.zoom * (double)sc.width);
    double los = std::sqrt((double)sc.width * (double)sc.width + (double)sc.height * (double)sc.height);
    double z_range = std::fmax(sc.z_end - sc.z_start, los * 0.1 * sw);
    o.s_shad_zmul = dt * 0.7f / (float)z_range * (128.0f - std::sqrt(std::fmax(fog_far_offset, 0.0f)) * 11.313708f);
    const float color_start = 68.0f, color_end = 72.0f;
    float a = (color_start + 30.0f) / 90.0f, b = (color_end + 30.0f) / 90.0f;
    float s_c_start = a * a * 32767.0f - 10900.0f;
    float s_c_mul = b * b * 32767.0f - 10900.0f - s_c_start;
    s_c_mul = std::fabs(s_c_mul) > 0.001f ? 2.0f / s_c_mul : (s_c_mul < 0.0f ? -2000.0f : 2000.0f);
    o.s_c_start = s_c_start;
    o.s_c_mul = s_c_mul;
    const float diffuse = 120.0f, specular = 50.0f, var_col_z = 0.0f;
    o.s_diff = diffuse * 0.02f;
    o.s_spec = std::fmax(specular * 0.02f, 0.004f);
    o.s_col_zmul = (float)((double)var_col_z * -0.005 / (sw * (double)sc.width));
    // the palette: three colours at 0, 10922, 21844, then colour 0 from 32200 on
    int dif[10][3], spe[10][3], pos[10];
    for (int i = 0; i < 3; i++) {
        pos[i] = i * 10922;
        rgb_of(cols[i * 3], dif[i]);
        rgb_of(cols[i * 3 + 1], spe[i]);
    }
    for (int i = 3; i < 10; i++) {
        std::memcpy(dif[i], dif[0], sizeof(dif[0]));
        std::memcpy(spe[i], spe[0], sizeof(spe[0]));
        pos[i] = 32200 + (i - 3) * 84;
    }
    const float d255 = 1.0f / 255.0f;
    for (int i = 0; i < 10; i++) {
        for (int k = 0; k < 3; k++) {
            o.col_dif[i][k] = (float)dif[i][k] * d255;
            o.col_spe[i][k] = (float)spe[i][k] * d255;
        }
        int al = std::max(spe[i][0], std::max(spe[i][1], spe[i][2]));  // palette_alpha
        o.col_spe_a[i] = (float)al / 255.0f;
        o.col_pos[i] = pos[i];
    }
    for (int i = 0; i < 10; i++) {
        int j = i < 9 ? o.col_pos[i + 1] - o.col_pos[i] : 32767 - o.col_pos[9];
        o.s_c_div[i] = j > 1 ? 1.0f / (float)j : 1.0f;
    }
    return 0;
}

// halton / halton_seq (src/mc.rs:103-128)
static double halton(int32_t index, int32_t base) {
    double r = 0.0, f = 1.0 / (double)base, d = f;
    int32_t i = index;
    while (i > 0) {
        r += f * (double)(i % base);
        i = (int32_t)std::trunc((double)i * d);
        f *= d;
    }
    return r;
}

const std::vector<uint32_t> &mc_halton_table() {
    static std::vector<uint32_t> t = [] {
        std::vector<uint32_t> v(2 * 65536);
        for (int i = 0; i < 65536; i++) {
            auto q = [&](int b) { return (uint32_t)std::nearbyint(halton(i + 1, b) * 65535.0); };
            v[2 * i] = q(2) | q(3) << 16;
            v[2 * i + 1] = q(5) | q(7) << 16;
        }
        return v;
    }();
    return t;
}

int mc_setup(const mb3d_cu_scene &sc0, const mb3d_cu_mc_light &lv, int depth, int secant, float ssr, DevParams &p,
             McDev &m, std::string &err) {
    if (lv.n_lights < 0 || lv.n_lights > 6) {
        err = "n_lights must be 0..6";
        return MB3D_CU_EINVAL;
    }
    for (int i = 0; i < lv.n_lights; i++) {
        int pf = lv.pow_func[i];
        if (pf < 1 || (pf & (pf - 1)) != 0) {
            err = "pow_func must be a power of two";
            return MB3D_CU_EINVAL;
        }
    }
    if (sc0.color_on_it != 0) {
        err = "the Monte Carlo tracer on the card has no colour on iteration";
        return MB3D_CU_ENOTSUP;
    }
    // mc_scene (src/mc.rs:2842-2850)
    mb3d_cu_scene sc = sc0;
    double sw = 2.1345 / (sc.zoom * (double)sc.width);
    double los = std::sqrt((double)sc.width * (double)sc.width + (double)sc.height * (double)sc.height);
    sc.z_end = std::fmax(sc.z_end - sc.z_start, los * 0.1 * sw) + sc.z_start;
    sc.smooth_normals = 0;
    int r = setup_params(sc, p, err);
    if (r < 0) return r;
    p.sm_normals = 0;
    p.refill_min = 8;  // (measured best of 8, 16, 24 for the march kernel of the Monte Carlo tracer)
    std::memset(&m, 0, sizeof(m));
    m.lv = lv;
    double n1[3][3];
    for (int i = 0; i < 3; i++) {
        double d = 1.0 / std::sqrt(p.vgrads[i][0] * p.vgrads[i][0] + p.vgrads[i][1] * p.vgrads[i][1] + p.vgrads[i][2] * p.vgrads[i][2]);
        for (int j = 0; j < 3; j++) n1[i][j] = p.vgrads[i][j] * d;
    }
    for (int i = 0; i < lv.n_lights; i++) {
        double l[3] = {(double)lv.ln[i][0], (double)lv.ln[i][1], (double)lv.ln[i][2]};
        double d = -p.step_width / std::sqrt(l[0] * l[0] + l[1] * l[1] + l[2] * l[2] + 1e-100);
        double v[3] = {l[0] * d, l[1] * d, l[2] * d};
        for (int j = 0; j < 3; j++) m.hs_vecs[i][j] = v[0] * n1[0][j] + v[1] * n1[1][j] + v[2] * n1[2][j];
    }
    double deao_max = (double)sc.deao_max_len;
    m.amb_max_l = std::fmin(deao_max * los * 3.0, p.zend * 255.0 / 1.75);
    m.zz_stmit_dif = sc.z_start - sc.mid[2];
    m.fovy1d = (float)(1.0 / (p.fov_y == 0.0 ? 1e-30 : p.fov_y));
    m.soft_shadow_radius = ssr;
    m.hs_max_lmul = (float)(sc.width + sc.height) * 0.6f * sc.hs_max_len_mul;
    m.max_amb_depth = depth;
    m.secant = secant ? 1 : 0;
    return 0;
}

}  // namespace mb3dcu
