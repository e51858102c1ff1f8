// The Calculate 3D painter on the card: render::paint (src/render.rs:
// 2499-2501, paint_core :2676-2720) of a G-buffer to 8-bit RGB, one thread
// per pixel, for the lighting this library renders with: Lighting::default
// (src/lighting.rs:290-391) with the scene's lights switched on and turned,
// directional and not visible in the picture; no internal gamma 2, light or
// colour maps, background picture, surface detail or material, ground,
// clouds, reflections or depth of field.  The light values (LightVals::build,
// src/lighting.rs:978-1190, as light_vals src/render.rs:2285-2331 makes them
// for a still picture) and the diffuse light tables (SetCosTabFunction,
// src/lighting.rs:464-499) are made on the host; the kernel is shade
// (src/lighting.rs:1802-2162) and pixel_color_s (:1739-1760) along that path.
// Built with -fmad=false: the reference's single precision is unfused.
#include <cuda_runtime.h>
#include <stdint.h>
#include <cmath>
#include <cstring>
#include "kernels.h"

namespace mb3dcu {

namespace {

struct PaintLight {
    float ln[3], col[3];
    int32_t pow_func, diff_func, sub_amb_sh, hs_calced;
    uint32_t hs_mask;
};

struct PaintK {
    PaintLight lights[6];
    int32_t n_lights, width, height, row0;
    float amb_col[3], amb_col2[3], depth_col[3], depth_col2[3], dyn_fog_col[3], dyn_fog_col2[3];
    float s_depth, s_shad, s_shad_gr, s_shad_zmul, s_dyn_fog_mul, s_amb_shad, s_diff, s_spec, s_ind_light_reflect;
    float s_col_zmul, s_c_start, s_c_mul, s_ci_start, s_ci_mul, s_roughness_factor, s_diffuse_shadowing;
    float col_dif[10][3], col_spe[10][3], col_int[4][3];
    float s_c_div[10], col_int_spec[4], s_ic_div[4];
    int32_t col_pos[10], icol_pos[4];
    float fov, aspect, x_off;
    double zcorr, zc_mul, step_width, zz_stmit_dif;
    float cos_tab[8][128];
};

// Delphi TColor ($BBGGRR) -> r, g, b (src/lighting.rs:285-288)
void col255(uint32_t c, float o[3]) {
    o[0] = (float)(c & 0xFF);
    o[1] = (float)((c >> 8) & 0xFF);
    o[2] = (float)((c >> 16) & 0xFF);
}

void make_paint_k(const mb3d_cu_scene &sc, const DevParams &p, uint32_t row0, PaintK &k) {
    std::memset(&k, 0, sizeof(k));
    const uint32_t cols[9] = {5873889, 8837614, 0x8B491D, 2988346, 12248958, 0xFFC49F, 11287584, 14579248, 7481121};
    for (int idx = 0; idx < 6; idx++) {
        const mb3d_cu_light &li = sc.lights[idx];
        if (!li.on) continue;
        // the preset's light 0 and 1, and defaultLight8 (src/lighting.rs:125-145, 309-330)
        uint32_t color = idx == 0 ? 0xA0E8FFu : idx == 1 ? 2307911u : 0xFFFFFFu;
        int spec_func = idx == 0 ? (53 & 7) : idx == 1 ? (16 & 7) : 4;
        int diff_func = idx == 0 ? ((53 >> 4) & 3) : idx == 1 ? ((16 >> 4) & 3) : 0;
        // effective_lighting (src/render.rs:2275-2283): the scene's shadow pass
        const bool hs_calced = ((sc.shadow_lights & 0x3F) >> idx) & 1;
        const bool hs_soft = sc.shadow_soft != 0, hs_set_cos = false, hs_enabled = true;
        double dtmp = -li.x_angle, dtmp2 = li.y_angle;
        double v[3] = {-std::sin(dtmp), std::sin(dtmp2), std::cos(dtmp2) * std::cos(dtmp)};
        double n = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        PaintLight &L = k.lights[k.n_lights++];
        for (int c = 0; c < 3; c++) L.ln[c] = (float)(-v[c] / n);
        col255(color, L.col);  // (x light_scale 1, x amplitude 1)
        L.pow_func = 2 << (spec_func & 7);
        L.diff_func = hs_calced && hs_set_cos ? 0 : (diff_func & 3);
        L.sub_amb_sh = hs_calced != hs_enabled;
        L.hs_calced = hs_calced;
        L.hs_mask = hs_soft && hs_calced ? 0xFFFFu : (0x400u << idx);
    }
    const float zsd = (float)sc.z_step_div;
    k.s_depth = 27.0f * 0.8e-6f;
    float gr = (53.0f - 53.0f) * 1.0f * zsd * 0.00065f, dt = 2.2f / zsd, mul = zsd * 0.015f, stmp = 128.0f;
    if (sc.dfog_on_it > 0) {
        dt *= 0.25f;
        gr *= 4.0f;
        mul *= 4.0f;
    } else {
        stmp = 137.0f;
    }
    k.s_shad_gr = gr;
    k.s_dyn_fog_mul = mul;
    k.s_shad = (stmp - std::sqrt(std::fmax(128.0f, 0.0f)) * 11.313708f) * dt * 0.28f;
    const double z_range = sc.z_end - sc.z_start;
    k.s_shad_zmul = dt * 0.7f / (float)z_range * (128.0f - std::sqrt(std::fmax(128.0f, 0.0f)) * 11.313708f);
    k.s_amb_shad = 53.0f / 53.0f;
    float a = (68.0f + 30.0f) / 90.0f, b = (72.0f + 30.0f) / 90.0f;
    float s_c_start = a * a * 32767.0f - 10900.0f;
    float s_c_mul = b * b * 32767.0f - 10900.0f - s_c_start;
    k.s_c_mul = std::fabs(s_c_mul) > 0.001f ? 2.0f / s_c_mul : (s_c_mul < 0.0f ? -2000.0f : 2000.0f);
    k.s_c_start = s_c_start;
    const float ti = 60.0f;
    float dti = ti * ti * ti * ti;
    k.s_ci_start = dti * 0.000158025f + 32768.0f;
    float cim = (ti * ti * ti * ti - dti) * 0.5f * 0.00031605f;
    k.s_ci_mul = std::fabs(cim) > 1e-10f ? 1.0f / cim : cim;
    col255(0x8B491D, k.amb_col);  // x amb_mul 90 / 90 = 1
    col255(0xFFC49F, k.amb_col2);
    col255(0x8B491D, k.depth_col);
    col255(0xFFC49F, k.depth_col2);
    for (int c = 0; c < 3; c++) k.dyn_fog_col[c] = k.dyn_fog_col2[c] = 255.0f;
    // the palette: three colours at 0, 10922, 21844, then colour 0 from 32200 on
    const float d255 = 1.0f / 255.0f;
    for (int i = 0; i < 10; i++) {
        int j = i < 3 ? i : 0;
        float d[3], s[3];
        col255(cols[j * 3], d);
        col255(cols[j * 3 + 1], s);
        for (int c = 0; c < 3; c++) {
            k.col_dif[i][c] = d[c] * d255;
            k.col_spe[i][c] = s[c] * d255;
        }
        k.col_pos[i] = i < 3 ? i * 10922 : 32200 + (i - 3) * 84;
    }
    for (int i = 0; i < 10; i++) {
        int j = i < 9 ? k.col_pos[i + 1] - k.col_pos[i] : 32767 - k.col_pos[9];
        k.s_c_div[i] = j > 1 ? 1.0f / (float)j : 1.0f;
    }
    // the interior colours (0, 10922, 21844: the palette's, 32700: colour 0)
    for (int i = 0; i < 4; i++) {
        k.icol_pos[i] = i < 3 ? i * 10922 : 32700;
        float d[3];
        col255(cols[(i < 3 ? i : 0) * 3], d);
        for (int c = 0; c < 3; c++) k.col_int[i][c] = d[c] * d255;
        k.col_int_spec[i] = 160.0f / 255.0f;
    }
    for (int i = 0; i < 4; i++) {
        int j = i < 3 ? k.icol_pos[i + 1] - k.icol_pos[i] : 32767 - k.icol_pos[3];
        k.s_ic_div[i] = j > 1 ? 1.0f / (float)j : 1.0f;
    }
    float ind = std::round(std::fmin(std::fmax(53.0f - 53.0f, -128.0f), 127.0f));
    float r = (ind + 53.0f) * 0.022f;
    k.s_ind_light_reflect = r * r;
    k.s_diff = 120.0f * 0.02f;
    k.s_spec = std::fmax(50.0f * 0.02f, 0.004f);
    k.s_col_zmul = (float)(0.0 * -0.005 / (p.step_width * (double)sc.width));
    k.s_roughness_factor = 0.0f / (255.0f * 255.0f);
    k.s_diffuse_shadowing = 0.0f;
    // the camera (paint_camera, src/render.rs:2340-2370, common optic)
    k.width = sc.width;
    k.height = sc.height;
    k.row0 = (int32_t)row0;
    k.fov = (float)(sc.fov_y * (3.14159265358979323846 / 180.0));
    k.aspect = (float)sc.width / (float)sc.height;
    k.x_off = 0.5f;
    k.zcorr = p.zcorr;
    k.zc_mul = p.zc_mul;
    k.step_width = p.step_width;
    k.zz_stmit_dif = sc.z_start - sc.mid[2];
    // SetCosTabFunction
    for (int i = 0; i < 128; i++) {
        double d = 1.0 - ((double)i - 2.0) / 60.0;
        k.cos_tab[0][i] = d > 0.15 ? (float)((d - 0.08) * 1.0869565) : d <= 0.0 ? 0.0f : (float)std::pow(d, std::fmax(1.0, (0.505 - d) * 3.8));
        double dc = std::fmax(d, 0.0);
        k.cos_tab[1][i] = (float)(dc * dc);
        k.cos_tab[2][i] = (float)(d * 0.5 + 0.5);
        k.cos_tab[3][i] = (float)((d * 0.5 + 0.5) * (d * 0.5 + 0.5));
    }
    for (int t = 0; t < 4; t++) {
        float tmp[128];
        for (int j = 0; j < 128; j++) tmp[j] = std::sqrt(std::fmax(k.cos_tab[t][j], 0.0f));
        for (int j = 0; j < 128; j++) {
            double e = 0.0;
            for (int i = 0; i <= 60; i++) {
                int l = std::abs(j + i - 30);
                if (l < 128) e += (double)tmp[l];
            }
            double aa = e * 0.011 + (e * 0.007) * (e * 0.007);
            k.cos_tab[t + 4][j] = (float)(aa * aa);
        }
    }
}

// lerp(sv1, sv2, w1) = sv2 + w1 (sv1 - sv2) (src/lighting.rs:563-569)
__device__ __forceinline__ void lerp3(const float a[3], const float b[3], float w, float o[3]) {
#pragma unroll
    for (int c = 0; c < 3; c++) o[c] = b[c] + w * (a[c] - b[c]);
}

// GetCosTabVal (src/lighting.rs:501-532), no internal gamma 2
__device__ float cos_tab_val(const PaintK &k, int tnr, float dotp, float rough) {
    float t = 62.0f - 60.0f * dotp;
    int ip = (int)truncf(t) - 1;
    if (ip < 0) {
        ip = 0;
        t = 0.0f;
    } else if (ip > 124) {
        ip = 124;
        t = 1.0f;
    } else {
        t = t - truncf(t);
    }
    // make_spline_coeff (src/math.rs:263-269)
    double xs = (double)t;
    double r3 = xs * xs * xs / 6.0;
    double r0 = 1.0 / 6.0 + 0.5 * xs * (xs - 1.0) - r3;
    double r2 = xs + r0 - 2.0 * r3;
    double r1 = 1.0 - r0 - r2 - r3;
    const float w[4] = {(float)r0, (float)r1, (float)r2, (float)r3};
    float a = 0.0f, b = 0.0f;
#pragma unroll
    for (int q = 0; q < 4; q++) a += k.cos_tab[tnr][ip + q] * w[q];
#pragma unroll
    for (int q = 0; q < 4; q++) b += k.cos_tab[tnr + 4][ip + q] * w[q];
    return a + rough * (b - a);
}

// FastIntPow (src/math.rs:273-285)
__device__ __forceinline__ float fast_int_pow(float base, int expo) {
    if (base < 0.0f) return 0.0f;
    float r = base;
    for (int i = expo >> 1; i > 0; i >>= 1) r *= r;
    return r;
}

__global__ void k_paint(const __grid_constant__ PaintK k, const mb3d_cu_silight *gbuf, uint32_t n, uint8_t *rgb) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const mb3d_cu_silight si = gbuf[i];
        const int x = (int)(i % (uint32_t)k.width), y = k.row0 + (int)(i / (uint32_t)k.width);
        // plv_for_pixel (src/lighting.rs:1764-1796)
        const float x_pos = (float)(x + 1) / (float)k.width, y_pos = (float)y / (float)k.height;
        float view[3];
        {
            float cx = (k.x_off - x_pos) * k.fov * k.aspect, cy = (y_pos - 0.5f) * k.fov;
            float v0 = -sinf(cx), v1 = sinf(cy), v2 = cosf(cy) * cosf(cx);
            float nn = sqrtf(v0 * v0 + v1 * v1 + v2 * v2);
            float inv = 1.0f / nn;
            view[0] = v0 * inv;
            view[1] = v1 * inv;
            view[2] = v2 * inv;
        }
        const uint32_t zpos_word = si.zpos_fine >> 16;
        double q = zpos_word > 32767 ? 8388352.0 / k.zc_mul + 1.0
                                     : (double)(8388352 - (int64_t)(si.zpos_fine >> 8)) / k.zc_mul + 1.0;
        const double z1 = (q * q - 1.0) * k.step_width / k.zcorr;
        const float z_pos = (float)(z1 + k.zz_stmit_dif);
        float dep_c[3];
        lerp3(k.depth_col2, k.depth_col, y_pos, dep_c);  // depth_func 0
        float o[3], dtmp;
        if (zpos_word < 32768) {
            const float d_rough = (float)(si.zpos_fine & 0xFF) * k.s_roughness_factor;
            const float shadow = si.amb_shadow >= 16383 ? 1.0f : (float)si.amb_shadow / 16383.0f;
            float d_amb_sh;
            if (k.s_amb_shad < 1.0f) {
                d_amb_sh = 1.0f - k.s_amb_shad * shadow;
            } else {
                float a = 1.0f - shadow;
                d_amb_sh = a + (k.s_amb_shad - 1.0f) * (a * a - a);
            }
            const float lns[3] = {(float)si.normal[0] * 3.0518509476e-5f, (float)si.normal[1] * 3.0518509476e-5f,
                                  (float)si.normal[2] * 3.0518509476e-5f};
            float li_dif[3] = {0, 0, 0}, li_spe[3] = {0, 0, 0}, li_amb[3] = {0, 0, 0};
            const float d_fog = k.s_diffuse_shadowing * (d_amb_sh - 1.0f) + 1.0f;
            for (int l = 0; l < k.n_lights; l++) {
                const PaintLight &L = k.lights[l];
                const bool soft = L.hs_mask == 0xFFFFu;
                const bool no_hs = soft || (si.shadow & L.hs_mask) == 0 || !L.hs_calced;
                const float soft_mul = soft ? (float)(si.shadow >> 10) * (1.0f / 63.0f) : 1.0f;
                const float att = 1.0f;
                float dt = lns[0] * L.ln[0] + lns[1] * L.ln[1] + lns[2] * L.ln[2];
                float d = cos_tab_val(k, L.diff_func, dt, d_rough) * att;
#pragma unroll
                for (int c = 0; c < 3; c++) li_amb[c] += L.col[c] * d;
                if (no_hs) {
                    d *= L.sub_amb_sh ? d_amb_sh : d_fog;
                    d *= soft_mul;
#pragma unroll
                    for (int c = 0; c < 3; c++) li_dif[c] += L.col[c] * d;
                }
                float d2 = 2.0f * (lns[0] * view[0] + lns[1] * view[1] + lns[2] * view[2]);
                float ds = L.ln[0] * (view[0] - lns[0] * d2) + L.ln[1] * (view[1] - lns[1] * d2) +
                           L.ln[2] * (view[2] - lns[2] * d2);
                if (ds > 0.0f) {
                    float pf = (float)L.pow_func;
                    float t2 = (att + fminf(d_rough * 2.0f, 1.0f) * (1.0f / pf - att)) * k.s_spec;
                    if (t2 > 0.0f) {
#pragma unroll
                        for (int c = 0; c < 3; c++) li_amb[c] += L.col[c] * (t2 / pf);
                        if (no_hs) {
                            t2 *= fast_int_pow(ds, L.pow_func);
                            t2 *= L.sub_amb_sh ? d_amb_sh : d_fog;
                            t2 *= soft_mul;
#pragma unroll
                            for (int c = 0; c < 3; c++) li_spe[c] += L.col[c] * t2;
                        }
                    }
                }
            }
            const float idif0 = k.s_col_zmul * z_pos;
            float idif[3], ispe[3];
            if (si.si_gradient > 32767) {
                // CalcColorsInside (src/lighting.rs:1656-1685)
                int ir = (int)roundf((((float)si.si_gradient - k.s_ci_start) * k.s_ci_mul + idif0) * 16384.0f);
                float spe;
                if (ir < 0) {
                    for (int c = 0; c < 3; c++) idif[c] = k.col_int[0][c];
                    spe = k.col_int_spec[0];
                } else if (ir > k.icol_pos[3]) {
                    for (int c = 0; c < 3; c++) idif[c] = k.col_int[3][c];
                    spe = k.col_int_spec[3];
                } else {
                    int il2 = 1;
                    while (il2 < 4 && k.icol_pos[il2] < ir) il2 += 1;
                    int il1 = il2 - 1;
                    il2 &= 3;
                    float t = (float)(ir - k.icol_pos[il1]) * k.s_ic_div[il1];
                    lerp3(k.col_int[il2], k.col_int[il1], t, idif);
                    spe = k.col_int_spec[il2] + t * (k.col_int_spec[il1] - k.col_int_spec[il2]);
                }
                ispe[0] = ispe[1] = ispe[2] = spe;
            } else {
                // CalcColors (src/lighting.rs:1563-1615)
                float irf = ((float)si.si_gradient - k.s_c_start) * k.s_c_mul + idif0;
                irf = fminf(fmaxf(irf * 16384.0f, -1e9f), 1e9f);
                int ir = (int)roundf(irf);
                if (ir < 0 || ir >= k.col_pos[9]) {
                    const int a = ir < 0 ? 0 : 9;
                    for (int c = 0; c < 3; c++) {
                        idif[c] = k.col_dif[a][c];
                        ispe[c] = k.col_spe[a][c];
                    }
                } else {
                    int il2 = 5;
                    if (k.col_pos[il2] < ir) {
                        do {
                            il2 += 1;
                        } while (!(il2 == 10 || k.col_pos[il2] >= ir));
                    } else {
                        while (il2 > 1 && k.col_pos[il2 - 1] >= ir) il2 -= 1;
                    }
                    const int il1 = il2 - 1;
                    if (il2 > 9) il2 = 0;
                    const float t = (float)(ir - k.col_pos[il1]) * k.s_c_div[il1];
                    lerp3(k.col_dif[il2], k.col_dif[il1], t, idif);
                    lerp3(k.col_spe[il2], k.col_spe[il1], t, ispe);
                }
            }
            // ambient light top / bottom
            const float t2 = (lns[1] * 0.5f + 0.5f) * d_amb_sh, t1 = d_amb_sh - t2;
            const float st = fmaxf(1.0f - d_amb_sh, 0.0f), st2 = st * st * st * st;
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float iamb = (k.amb_col[c] * t1 + k.amb_col2[c] * t2) * idif[c];
                const float dif_s = idif[c] * k.s_diff;
                const float total = (iamb + dif_s * li_dif[c]) + ispe[c] * li_spe[c];
                // CalcTotalLight1
                const float l3 = iamb + (dif_s * li_amb[c]) * (d_amb_sh * 0.3f);
                const float refl = idif[c] * st2 * k.s_ind_light_reflect + (st - st2);
                o[c] = total + l3 * (idif[c] * refl);
            }
            dtmp = fmaxf(((float)zpos_word - 28000.0f) * k.s_depth + 1.0f, 0.0f);
        } else {
            o[0] = dep_c[0];
            o[1] = dep_c[1];
            o[2] = dep_c[2];
            dtmp = fmaxf(1.0f - (float)(60768 - (int32_t)zpos_word) * k.s_depth, 0.0f);
        }
        // the depth fog and the dynamic fog (no far fog, no background picture)
        const float ir = (float)(si.shadow & 0x3FF);
        const float dfog = (ir - k.s_shad - k.s_shad_zmul * z_pos) * k.s_shad_gr;
        const float dtmp3 = fminf(ir * k.s_dyn_fog_mul, 1.0f) * dfog;
        uint8_t out[3];
#pragma unroll
        for (int c = 0; c < 3; c++) {
            float v = o[c] * dtmp;
            v = v + dep_c[c] * fmaxf(1.0f - dtmp, 0.0f);
            v = v + (k.dyn_fog_col[c] * (dfog - dtmp3) + k.dyn_fog_col2[c] * dtmp3);
            // pixel_color_s in 8 bits: clipped to 0..255, no gamma curve, rounded
            out[c] = (uint8_t)roundf(fminf(fmaxf(v, 0.0f), 255.0f));
        }
        rgb[3 * i] = out[0];
        rgb[3 * i + 1] = out[1];
        rgb[3 * i + 2] = out[2];
    }
}

}  // namespace

void paint_launch(const mb3d_cu_scene &sc, const DevParams &p, uint32_t row0, const mb3d_cu_silight *gbuf, uint32_t n,
                  uint8_t *rgb, int blocks, cudaStream_t s) {
    PaintK k;
    make_paint_k(sc, p, row0, k);
    k_paint<<<blocks, 256, 0, s>>>(k, gbuf, n, rgb);
}

}  // namespace mb3dcu
