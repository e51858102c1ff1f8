// The reflection pass's rays on the card (gpu::reflect_batch,
// src/gpu.rs:2521): the march of a reflected or refracted ray from a surface
// point to its hit, and the hit's normal, colour, depth, hard or soft shadow
// and DE ambient occlusion -- SrTracer::march_ray (src/reflect.rs:1464-1675)
// with calc_hs (:805-952) and deao_1pos (:954-1090), one thread per ray, in
// double precision on the device marcher M64 (the primary march's FP64
// state machine), so that a bounce is the same march the picture's own rays
// take.  Every ray sets its marcher up at its pixel (pixel_marcher,
// :1840-1845: the pixel's view vector decides the depth along the ray).
// Outside rendering, no cutting planes, no ground plane, no volumetric
// light, the scene's global lights, no random first step of the AO.
#pragma once
#include "marcher64.cuh"

namespace mb3dcu {

// update_de_stop (src/reflect.rs:414-418)
__device__ __forceinline__ float refl_de_stop(const DevParams &p, double zz) {
    return (float)((double)p.de_stop * (1.0 + fabs(zz) * (double)p.de_stop_factor));
}

// the march toward a light (the closure of calc_hs, src/reflect.rs:815-848);
// the soft shadow's zrsoft when zrs_mul > 0
template <int FM>
__device__ float refl_hs_march(M64<FM> &m, const double hv[3], double &dt1, double &zz2, double zz2mul,
                               float zrs_mul, double max_lhs) {
    const DevParams &p = m.p;
    float rsfd = 1.0f, zrsoft = 1.0f;
    const double dmaxl = dt1;
    double d = m.calc_de();
    for (int guard = 1;; guard++) {
        const double last_de = d;
        const double st = (double)fminf((float)(d * (double)p.z_step_div * (double)rsfd),
                                        fmaxf(m.ms_de_stop, 0.4f) * p.mh04zsd);
        dt1 -= st;
        add_w(m.it.c, hv, -st);
        zz2 += st * zz2mul;
        m.ms_de_stop = refl_de_stop(p, zz2);
        d = m.calc_de();
        if (zrs_mul > 0.0f) {
            const float r = (float)((dmaxl - dt1) / max_lhs);
            const float r8 = (r * r) * (r * r);
            zrsoft = fminf(zrsoft, __fadd_rn((float)((d - (double)m.ms_de_stop) * (double)zrs_mul / (dmaxl - dt1 + 0.11)),
                                             __fmul_rn(r8, r8)));
        }
        if (m.it.it_result >= m.max_its_result || d < (double)m.ms_de_stop) break;
        if (d > last_de + st) d = last_de + st;
        if (last_de > d + 1e-30) {
            const float t = (float)(st / (last_de - d));
            rsfd = t < 1.0f ? fmaxf(t, 0.5f) : 1.0f;
        } else {
            rsfd = 1.0f;
        }
        if (dt1 < 0.0 || guard > 1000000) break;
    }
    return zrsoft;
}

// calc_hs (src/reflect.rs:805-952), the scene's global shadow lights
template <int FM>
__device__ void refl_calc_hs(M64<FM> &m, G &si) {
    const DevParams &p = m.p;
    const float zz = (float)fabs(m.mzz);
    const double ic[3] = {m.it.c[0], m.it.c[1], m.it.c[2]};
    const float fov = fmaxf((float)p.fov_y, 0.0f);
    const double max_lhs = (double)((float)(p.width + p.height) * 0.6f *
                                    (1.0f + __fdiv_rn(0.5f * fminf(zz, (float)p.zend * 0.4f) * fov, (float)p.height)) *
                                    p.hs_max_len_mul);
    const double nrm[3] = {(double)si.n0 / 32767.0, (double)si.n1 / 32767.0, (double)si.n2 / 32767.0};
    double nvec[3];
    rot_rev(nrm, p.vgrads, nvec);
    if (p.shadow_soft) {
        if (p.n_lights < 1) return;
        const double *hv = p.light_vec[p.n_lights - 1];
        const float zrs_mul = __fdiv_rn(80.0f, fmaxf(p.soft_radius, 0.001f));
        si.shadow |= 0xFC00;
        double zz2 = m.mzz;
        m.ms_de_stop = refl_de_stop(p, (double)zz);
        const double dmaxl = max_lhs;
        const double zz2mul = -dot3d(hv, m.vfov) / sqrt(dot3d(hv, hv) * dot3d(m.vfov, m.vfov));
        if (dmaxl > 0.0) {
            if (dot3d(nvec, hv) > 0.0) {
                si.shadow &= 0x3FF;
                return;
            }
            double dt1 = dmaxl;
            const float zr = refl_hs_march<FM>(m, hv, dt1, zz2, zz2mul, zrs_mul, max_lhs);
            si.shadow = (unsigned short)((si.shadow & 0x3FF) |
                                         ((unsigned int)rintf(fminf(fmaxf(zr, 0.0f), 1.0f) * 63.4f) << 10));
            for (int k = 0; k < 3; k++) m.it.c[k] = ic[k];
        }
        return;
    }
    unsigned int mask = 0;
    for (int l = 0; l < p.n_lights; l++) mask |= 0x400u << p.light_idx[l];
    si.shadow &= (unsigned short)~mask;
    for (int l = 0; l < p.n_lights; l++) {
        const double *hv = p.light_vec[l];
        const unsigned int bit = 0x400u << p.light_idx[l];
        for (int k = 0; k < 3; k++) m.it.c[k] = ic[k];
        double zz2 = m.mzz;
        m.ms_de_stop = refl_de_stop(p, (double)zz);
        double dt1 = max_lhs;
        const double zz2mul = -dot3d(hv, m.vfov) / sqrt(dot3d(hv, hv) * dot3d(m.vfov, m.vfov));
        if (dt1 > 0.0) {
            if (dot3d(nvec, hv) > 0.0) {
                si.shadow |= (unsigned short)bit;
                continue;
            }
            refl_hs_march<FM>(m, hv, dt1, zz2, zz2mul, 0.0f, max_lhs);
            if (dt1 > 0.0) si.shadow |= (unsigned short)bit;
        }
    }
    for (int k = 0; k < 3; k++) m.it.c[k] = ic[k];
}

// CalcAmbShadowDEfor1pos (deao_1pos, src/reflect.rs:954-1090) at the
// marcher's position, the depth for the DE stop in m.mzz; the quality's
// directions and the pairs' angle terms come from the host's table
template <int FM>
__device__ void refl_deao(M64<FM> &m, G &si, const ReflAO &T, int q, float max_len) {
    si.amb_shadow = 0;
    if (si.zpos() >= 32768u || si.si_gradient >= 32768) return;
    const DevParams &p = m.p;
    m.it.calc_sit = false;
    const double s_max_d = (double)max_len * 0.5 * sqrt((double)p.height * (double)p.height + (double)p.width * (double)p.width);
    double ms_de_stop = (double)fminf(refl_de_stop(p, m.mzz), 1e6f);
    const double ic[3] = {m.it.c[0], m.it.c[1], m.it.c[2]};
    const double step_ao = ms_de_stop / (double)p.de_stop;
    const double max_dist = s_max_d * sqrt(step_ao);
    const double dsm = T.d_step_mul[q];
    if (p.de_stop_factor != 0.0f) ms_de_stop /= dsm * dsm;
    else ms_de_stop = (double)p.de_stop / (dsm * dsm);
    const int n = T.count[q], first = T.first[q];
    const double de_mul = sqrt((double)n * 0.5);
    const double md_d10 = 0.1 / (max_dist * de_mul);
    float nrm[3];
    {
        const float v[3] = {(float)si.n0, (float)si.n1, (float)si.n2};
        const float l = fmaxf(__fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(v[0], v[0]), __fmul_rn(v[1], v[1])), __fmul_rn(v[2], v[2]))), 1e-30f);
        nrm[0] = __fdiv_rn(v[0], l);
        nrm[1] = __fdiv_rn(v[1], l);
        nrm[2] = __fdiv_rn(v[2], l);
    }
    float rot_w[3][3];
    normal_matrix_d(nrm, rot_w);
    float min_ra[REFL_AO_MAX];
    for (int k = 0; k < n; k++) {
        const float *d = T.dirs[first + k];
        float v[3];
        for (int i = 0; i < 3; i++)
            v[i] = __fadd_rn(__fadd_rn(__fmul_rn(rot_w[i][0], d[0]), __fmul_rn(rot_w[i][1], d[1])), __fmul_rn(rot_w[i][2], d[2]));
        const double vd[3] = {(double)v[0], (double)v[1], (double)v[2]};
        double sv[3];
        rot_rev(vd, p.ao_rot, sv);
        double dt1 = step_ao * dsm, s = 1.0;
        bool end = false;
        for (int guard = 1;; guard++) {
            if (dt1 > max_dist) {
                dt1 = max_dist;
                end = true;
            }
            for (int i = 0; i < 3; i++) m.it.c[i] = ic[i];
            add_w(m.it.c, sv, dt1);
            const double d2 = m.calc_de();
            s = fmin(s, (d2 - ms_de_stop + dt1 * md_d10) / dt1);
            if (s < 0.02) break;
            dt1 += fmax(d2, dt1 * dsm);
            if (end || guard > 100000) break;
        }
        min_ra[k] = (float)(fmax(s, 0.0) * de_mul);
    }
    double amount = 0.0;
    for (int k = 0; k < n; k++) {
        float s_add = 0.0f;
        if (min_ra[k] < 1.0f) {
            const float max_add = __fsub_rn(1.0f, min_ra[k]);
            for (int k2 = 0; k2 < n; k2++) {
                if (k2 == k) continue;
                // (T.ang: acos(dot) * abr of the pair, or a huge value where the pair does not count)
                const float overlap = __fadd_rn(__fsub_rn(min_ra[k2], T.ang[q][k][k2]), 1.0f);
                if (overlap > 0.0f) s_add = __fadd_rn(s_add, __fmul_rn(fminf(max_add, overlap), T.corr_w[q]));
            }
        }
        amount += (double)fminf(__fadd_rn(s_add, min_ra[k]), 1.0f);
    }
    si.amb_shadow = sat_u16d(fmax(rint(16383.0 * (1.0 - amount / (double)n)), 0.0));
    for (int i = 0; i < 3; i++) m.it.c[i] = ic[i];
}

// march_ray (src/reflect.rs:1464-1675) for one ray
template <int FM>
__device__ void refl_march(const DevParams &p, const mb3d_cu_reflect_ray &r, int far_fog, const ReflAO &T,
                           mb3d_cu_reflect_hit &out) {
    M64<FM> m(p);
    const int x = (int)(r.pixel % (uint32_t)p.width), y = (int)(r.pixel / (uint32_t)p.width);
    double c0[3];
    pixel_ray(p, x, y, c0, m.vfov);
    const double nv[3] = {r.dir[0], r.dir[1], r.dir[2]};
    const double max_l = r.max_len > 0.0 ? r.max_len : p.zend;
    double zz = r.zz;
    for (int k = 0; k < 3; k++) m.it.c[k] = r.origin[k];
    const double zzplus = dot3d(m.vfov, nv) / sqrt(dot3d(m.vfov, m.vfov) * dot3d(nv, nv) + 1e-100);
    const float last_zz = (float)fabs(zz);
    double zz2 = fmin((double)p.de_stop * 0.25, 1.0);
    zz += zz2 * zzplus;
    add_w(m.it.c, nv, zz2);
    m.ms_de_stop = refl_de_stop(p, zz);
    bool open_air = false, de_limited = true;
    float step_count = 0.0f, rsfmul = 1.0f;
    double dtmp = m.calc_de();
    double rlast_sw = dtmp * (double)p.z_step_div;
    if (dtmp > 1e-10) {
        for (int guard = 1;; guard++) {
            const double rlast_de = dtmp;
            double dstep = fmax((dtmp - (double)p.ms_de_sub * (double)m.ms_de_stop) * (double)p.z_step_div * (double)rsfmul, 0.11);
            const double s = (double)(fmaxf(m.ms_de_stop, 0.4f) * p.mh04zsd);
            const bool count = p.dfog_on_it == 0 || m.it.it_result == p.dfog_on_it;
            if (s < dstep) {
                if (count) step_count = __fadd_rn(step_count, (float)(s / dstep));
                dstep = s;
            } else if (count) {
                step_count = __fadd_rn(step_count, 1.0f);
            }
            rlast_sw = dstep;
            zz2 += dstep;
            if (zz2 > max_l) {
                open_air = true;
                break;
            }
            add_w(m.it.c, nv, dstep);
            zz += dstep * zzplus;
            m.ms_de_stop = refl_de_stop(p, zz);
            dtmp = m.calc_de();
            if (m.it.it_result >= m.max_its_result) {
                de_limited = false;
                break;
            }
            if (dtmp < (double)m.ms_de_stop && m.it.it_result >= p.min_it) break;
            if (dtmp > rlast_de + rlast_sw) dtmp = rlast_de + rlast_sw;
            if (rlast_de > dtmp + 1e-10) {
                const double d = rlast_sw / (rlast_de - dtmp);
                rsfmul = d < 1.0 ? (float)fmax(d, 0.5) : 1.0f;
            } else {
                rsfmul = 1.0f;
            }
            if (guard > 1000000) {
                open_air = true;
                break;
            }
        }
    }
    const double zz2_paint = zz2;
    G si;
    si.clear();
    si.shadow = (unsigned short)rintf(fminf(fmaxf(step_count, 0.0f), 1023.0f));
    if (!open_air) {
        if (p.de_add_steps != 0) {
            if (de_limited) {
                int itmp = p.de_add_steps;
                double ds = rlast_sw * -0.5;
                double d = m.calc_de();
                while (fabs(d - (double)m.ms_de_stop) > 0.001) {
                    zz2 += ds;
                    zz += ds * zzplus;
                    add_w(m.it.c, nv, ds);
                    m.ms_de_stop = refl_de_stop(p, zz);
                    if (--itmp <= 0) break;
                    d = m.calc_de();
                    ds = d < (double)m.ms_de_stop ? fabs(ds) * -0.55 : fabs(ds) * 0.55;
                }
            } else {
                const double before = zz2;
                const double vf[3] = {m.vfov[0], m.vfov[1], m.vfov[2]};
                for (int k = 0; k < 3; k++) m.vfov[k] = nv[k];
                m.mzz = zz2;
                m.bin_search_it();
                zz2 = m.mzz;
                for (int k = 0; k < 3; k++) m.vfov[k] = vf[k];
                zz += (zz2 - before) * zzplus;
            }
        }
        m.mzz = fabs(zz);
        const float nn = p.normals_on_de ? m.calculate_normals(si) : m.calculate_normals_on_smooth_it(si);
        float v;
        if (de_limited) {
            const float l = (float)log((double)m.ms_de_stop * p.step_width);
            v = __fsub_rn(32767.0f, __fmul_rn(__fadd_rn(__fadd_rn(nn, p.d_col_plus), __fmul_rn(p.col_var, l)), p.mcts_m));
        } else {
            v = __fsub_rn(32767.0f, __fmul_rn(nn, p.mcts_m));
        }
        si.si_gradient = clip15(v);
        if (p.color_on_it != 0) m.do_color_on_it();
        m.do_color(si);
        double ds = zz2;
        if (far_fog) {
            const double a = zz2 + (double)last_zz;
            ds = sqrt(fmax(a * a - (double)last_zz + 1e-30, 0.0));
        }
        {
            const long long vz = sat_i64d(rint(p.zc_mul * (sqrt(fmax(ds, 0.0) * p.zcorr + 1.0) - 1.0)));
            long long z = 8388352LL - vz;
            z = z < 0 ? 0 : z > 8388352LL ? 8388352LL : z;
            unsigned int rr = (unsigned int)z << 8;
            if (p.sm_normals > 0) rr |= (unsigned int)sat_u16d(rint((double)__fmul_rn(m.s_roughness, 255.0f))) & 0xFFu;
            si.zpos_fine = rr;
        }
        const float saved = m.ms_de_stop;
        if (p.n_lights > 0) {
            m.mzz = fabs(zz);
            refl_calc_hs<FM>(m, si);
        }
        if (p.ao_quality >= 0) {
            const int q = r.rit == 1 ? 2 : r.rit == 2 ? 1 : 0;
            m.mzz = fabs(zz);
            refl_deao<FM>(m, si, T, q, p.ao_max_len);
            si.amb_shadow = (unsigned short)(((int)si.amb_shadow * 8) / (8 + (int)r.rit));
        } else {
            si.amb_shadow = 5000;
        }
        m.ms_de_stop = saved;
    } else {
        si.zpos_fine = 32768u << 16;
    }
    si.store(&out.si);
    out.hit = open_air ? 0 : 1;
    out.de_limited = de_limited ? 1 : 0;
    out.pad[0] = out.pad[1] = 0;
    for (int k = 0; k < 3; k++) out.pos[k] = m.it.c[k];
    out.zz = zz;
    out.zz2_paint = zz2_paint;
    out.zz2 = zz2;
}

// one thread per ray
template <int FM>
__global__ void __maxnreg__(168) k_reflect(const __grid_constant__ DevParams p, const mb3d_cu_reflect_ray *rays,
                                                 uint32_t n, int far_fog, const ReflAO *tab,
                                                 mb3d_cu_reflect_hit *hits) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const mb3d_cu_reflect_ray r = rays[i];
        mb3d_cu_reflect_hit h;
        refl_march<FM>(p, r, far_fog, *tab, h);
        hits[i] = h;
    }
}

// the first bounce of a pixel (start_pixel, src/reflect.rs:1686-1838, outside
// rendering, no water, no cutting plane: the surface found again from the
// stored depth, then step's mirror ray, :1286-1311) into tmp[i], valid[i]
// 1 where the pixel sends one
template <int FM>
__global__ void __maxnreg__(168) k_reflect_first(const __grid_constant__ DevParams p, const mb3d_cu_silight *g,
                                                       mb3d_cu_reflect_ray *tmp, unsigned char *valid) {
    const size_t npix = (size_t)p.width * p.height;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (size_t)gridDim.x * blockDim.x) {
        valid[i] = 0;
        G si;
        si.load(g[i]);
        if (si.zpos() >= 32768u || si.si_gradient >= 32768) continue;
        const int x = (int)(i % (size_t)p.width), y = (int)(i / (size_t)p.width);
        M64<FM> m(p);
        pixel_ray(p, x, y, m.it.c, m.vfov);
        m.it.calc_sit = false;
        const double zf = (double)(si.zpos_fine >> 8);
        auto zpos_of = [&](double iz) {
            const double q = (8388351.5 - iz) / p.zc_mul + 1.0;
            return (q * q - 1.0) / p.zcorr;
        };
        m.mzz = zpos_of(zf);
        add_w(m.it.c, m.vfov, m.mzz);
        m.update_de_stop();
        double d = m.calc_de();
        if (d < (double)m.ms_de_stop * 0.5) continue;
        const bool de_limited = m.it.it_result < m.max_its_result || d <= (double)m.ms_de_stop;
        if (de_limited) m.bin_search(d, m.mzz - zpos_of(zf - 1.0));
        else m.bin_search_it();
        const double n0[3] = {(double)si.n0 / 32767.0, (double)si.n1 / 32767.0, (double)si.n2 / 32767.0};
        double nrm[3];
        rot_rev(n0, p.vgrads, nrm);
        const double k = 2.0 * dot3d(nrm, m.vfov) / dot3d(nrm, nrm);
        mb3d_cu_reflect_ray r;
        for (int c = 0; c < 3; c++) {
            r.origin[c] = m.it.c[c];
            r.dir[c] = m.vfov[c] - nrm[c] * k;
        }
        r.zz = m.mzz;
        r.max_len = 0.0;
        r.pixel = (uint32_t)i;
        r.rit = 1;
        tmp[i] = r;
        valid[i] = 1;
    }
}

}  // namespace mb3dcu
