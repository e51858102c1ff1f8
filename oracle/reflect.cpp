// TEST INFRASTRUCTURE: the reflection pass's rays on the CPU (the march of a
// reflected ray to its hit with the hit's normal, colour, hard or soft
// shadow and DE ambient occlusion): SrTracer::march_ray
// (src/reflect.rs:1464-1675) with calc_hs (:805-952) and deao_1pos
// (:954-1090), the CPU side of gpu::reflect_batch (src/gpu.rs:2521), for
// the parity of the card's reflect batch.  Every ray gets a fresh marcher
// set up at its pixel (pixel_marcher, :1840-1845), as the card's batch
// treats its rays independently.  Outside rendering, no cutting planes, no
// ground plane, no volumetric light, the scene's global lights, no random
// first step of the ambient occlusion.
#include "oracle.hpp"
#include <algorithm>
#include <cstring>
#include <thread>
#include <vector>

namespace oracle {
namespace {

struct Ctx {
    const Params *p;
    std::vector<HsLight> lights;  // the shadow lights (soft: the last one)
    bool hs, soft, ao, far_fog;
    float soft_radius, hs_mul, ao_max_len;
};

// update_de_stop (src/reflect.rs:414-418)
inline void de_stop_at(Marcher &m, double zz) {
    m.ms_de_stop = (float)((double)m.p->de_stop * (1.0 + std::fabs(zz) * (double)m.p->de_stop_factor));
}

inline double sqr_len(const double v[3]) { return dot3(v, v); }

// the march toward a light (the closure of calc_hs, src/reflect.rs:815-848);
// returns the soft shadow's zrsoft when zrs_mul > 0
float hs_march(Marcher &m, const double hsvec[3], double &dt1, double &zz2, double zz2mul, float zrs_mul,
               double max_lhs) {
    const Params *p = m.p;
    float rsfd = 1.0f, zrsoft = 1.0f;
    const double dmaxl = dt1;
    double d = m.calc_de();
    for (int guard = 1;; guard++) {
        const double last_de = d;
        const double st = (double)rminf((float)(d * (double)p->z_step_div * (double)rsfd), rmaxf(m.ms_de_stop, 0.4f) * p->mh04zsd);
        dt1 -= st;
        add_weight(m.it.c, hsvec, -st);
        zz2 += st * zz2mul;
        de_stop_at(m, zz2);
        d = m.calc_de();
        if (zrs_mul > 0.0f) {
            const float r = (float)((dmaxl - dt1) / max_lhs);
            const float r8 = (r * r) * (r * r);
            zrsoft = rminf(zrsoft, (float)((d - (double)m.ms_de_stop) * (double)zrs_mul / (dmaxl - dt1 + 0.11)) + r8 * r8);
        }
        if (m.it.it_result >= m.max_its_result || d < (double)m.ms_de_stop) break;
        if (d > last_de + st) d = last_de + st;
        if (last_de > d + 1e-30) {
            const float t = (float)(st / (last_de - d));
            rsfd = t < 1.0f ? rmaxf(t, 0.5f) : 1.0f;
        } else {
            rsfd = 1.0f;
        }
        if (dt1 < 0.0 || guard > 1000000) break;
    }
    return zrsoft;
}

// calc_hs (src/reflect.rs:805-952), global lights only
void calc_hs(const Ctx &c, Marcher &m, SiLight &si) {
    const Params *p = c.p;
    const float zz = (float)std::fabs(m.mzz);
    const double ic[3] = {m.it.c[0], m.it.c[1], m.it.c[2]};
    const float fov = rmaxf((float)p->fov_y, 0.0f);
    const double max_lhs = (double)((float)(p->width + p->height) * 0.6f *
                                    (1.0f + 0.5f * rminf(zz, (float)p->zend * 0.4f) * fov / (float)p->height) * c.hs_mul);
    const double nrm[3] = {(double)si.normal[0] / 32767.0, (double)si.normal[1] / 32767.0, (double)si.normal[2] / 32767.0};
    double nvec[3];
    rotate_vector_reverse(nrm, p->vgrads, nvec);
    if (c.soft) {
        if (c.lights.empty()) return;
        const HsLight &l = c.lights.back();
        const float zrs_mul = 80.0f / c.soft_radius;
        si.shadow |= 0xFC00;
        double zz2 = m.mzz;
        de_stop_at(m, (double)zz);
        const double dmaxl = max_lhs;
        const double zz2mul = -dot3(l.vec, m.vfov) / std::sqrt(sqr_len(l.vec) * sqr_len(m.vfov));
        if (dmaxl > 0.0) {
            if (dot3(nvec, l.vec) > 0.0) {
                si.shadow &= 0x3FF;
                return;
            }
            double dt1 = dmaxl;
            const float zr = hs_march(m, l.vec, dt1, zz2, zz2mul, zrs_mul, max_lhs);
            si.shadow = (uint16_t)((si.shadow & 0x3FF) | ((uint16_t)rtef(rclampf(zr, 0.0f, 1.0f) * 63.4f) << 10));
            std::memcpy(m.it.c, ic, sizeof(ic));
        }
        return;
    }
    uint16_t mask = 0;
    for (const HsLight &l : c.lights) mask |= (uint16_t)(0x400 << l.idx);
    si.shadow &= (uint16_t)~mask;
    for (const HsLight &l : c.lights) {
        std::memcpy(m.it.c, ic, sizeof(ic));
        double zz2 = m.mzz;
        de_stop_at(m, (double)zz);
        double dt1 = max_lhs;
        const double zz2mul = -dot3(l.vec, m.vfov) / std::sqrt(sqr_len(l.vec) * sqr_len(m.vfov));
        if (dt1 > 0.0) {
            if (dot3(nvec, l.vec) > 0.0) {
                si.shadow |= (uint16_t)(0x400 << l.idx);
                continue;
            }
            hs_march(m, l.vec, dt1, zz2, zz2mul, 0.0f, max_lhs);
            if (dt1 > 0.0) si.shadow |= (uint16_t)(0x400 << l.idx);
        }
    }
    std::memcpy(m.it.c, ic, sizeof(ic));
}

// march_ray (src/reflect.rs:1464-1675)
void march_ray(const Ctx &c, const mb3d_cu_reflect_ray &r, mb3d_cu_reflect_hit &out) {
    const Params *p = c.p;
    const double sw = p->step_width;
    Marcher m(p, 0);
    const int x = (int)(r.pixel % (uint32_t)p->width), y = (int)(r.pixel / (uint32_t)p->width);
    m.cafy = ((double)y / (double)p->height - 0.5) * p->fov_y;
    m.calc_vgrads_fov(x + 1);
    m.calc_start_pos(x, y);
    const double *nv = r.dir;
    const double max_l = r.max_len > 0.0 ? r.max_len : p->zend;
    double zz = r.zz;
    std::memcpy(m.it.c, r.origin, sizeof(m.it.c));
    const double zzplus = dot3(m.vfov, nv) / std::sqrt(sqr_len(m.vfov) * sqr_len(nv) + 1e-100);
    const float last_zz = (float)std::fabs(zz);
    double zz2 = rmin((double)p->de_stop * 0.25, 1.0);
    zz += zz2 * zzplus;
    add_weight(m.it.c, nv, zz2);
    de_stop_at(m, zz);
    bool open_air = false, de_limited = true;
    float step_count = 0.0f, rsfmul = 1.0f;
    double dtmp = m.calc_de();
    double rlast_sw = dtmp * (double)p->z_step_div;
    if (dtmp > 1e-10) {
        for (int guard = 1;; guard++) {
            const double rlast_de = dtmp;
            double dstep = rmax((dtmp - (double)p->ms_de_sub * (double)m.ms_de_stop) * (double)p->z_step_div * (double)rsfmul, 0.11);
            const double s = (double)(rmaxf(m.ms_de_stop, 0.4f) * p->mh04zsd);
            const bool count = p->dfog_on_it == 0 || m.it.it_result == p->dfog_on_it;
            if (s < dstep) {
                if (count) step_count += (float)(s / dstep);
                dstep = s;
            } else if (count) {
                step_count += 1.0f;
            }
            rlast_sw = dstep;
            zz2 += dstep;
            if (zz2 > max_l) {
                open_air = true;
                break;
            }
            add_weight(m.it.c, nv, dstep);
            zz += dstep * zzplus;
            de_stop_at(m, zz);
            dtmp = m.calc_de();
            if (m.it.it_result >= m.max_its_result) {
                de_limited = false;
                break;
            }
            if (dtmp < (double)m.ms_de_stop && m.it.it_result >= p->min_it) break;
            if (dtmp > rlast_de + rlast_sw) dtmp = rlast_de + rlast_sw;
            if (rlast_de > dtmp + 1e-10) {
                const double d = rlast_sw / (rlast_de - dtmp);
                rsfmul = d < 1.0 ? (float)rmax(d, 0.5) : 1.0f;
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
    SiLight si;
    si.shadow = (uint16_t)rtef(rclampf(step_count, 0.0f, 1023.0f));
    if (!open_air) {
        if (p->de_add_steps != 0) {
            if (de_limited) {
                int itmp = p->de_add_steps;
                double ds = rlast_sw * -0.5;
                double d = m.calc_de();
                while (std::fabs(d - (double)m.ms_de_stop) > 0.001) {
                    zz2 += ds;
                    zz += ds * zzplus;
                    add_weight(m.it.c, nv, ds);
                    de_stop_at(m, zz);
                    if (--itmp <= 0) break;
                    d = m.calc_de();
                    ds = d < (double)m.ms_de_stop ? std::fabs(ds) * -0.55 : std::fabs(ds) * 0.55;
                }
            } else {
                const double before = zz2;
                double vf[3];
                std::memcpy(vf, m.vfov, sizeof(vf));
                std::memcpy(m.vfov, nv, sizeof(vf));
                m.mzz = zz2;
                m.bin_search_it();
                zz2 = m.mzz;
                std::memcpy(m.vfov, vf, sizeof(vf));
                zz += (zz2 - before) * zzplus;
            }
        }
        m.mzz = std::fabs(zz);
        const float nn = p->normals_on_de ? m.calculate_normals(si) : m.calculate_normals_on_smooth_it(si);
        float v;
        if (de_limited)
            v = 32767.0f - (nn + p->d_col_plus + p->col_var_de_stop_mul * (float)std::log((double)m.ms_de_stop * sw)) * p->mcts_m;
        else
            v = 32767.0f - nn * p->mcts_m;
        si.si_gradient = clip15(v);
        if (p->color_on_it != 0) m.do_color_on_it();
        m.do_color(si);
        double ds = zz2;
        if (c.far_fog) {
            const double a = zz2 + (double)last_zz;
            ds = std::sqrt(rmax(a * a - (double)last_zz + 1e-30, 0.0));
        }
        {
            const int64_t vz = sat_i64(rte(p->zc_mul * (std::sqrt(rmax(ds, 0.0) * p->zcorr + 1.0) - 1.0)));
            int64_t z = 8388352 - vz;
            z = z < 0 ? 0 : z > 8388352 ? 8388352 : z;
            uint32_t rr = (uint32_t)z << 8;
            if (p->sm_normals > 0) rr |= sat_u32(rte((double)(m.s_roughness * 255.0f))) & 0xFF;
            si.zpos_fine = rr;
        }
        const float saved = m.ms_de_stop;
        if (c.hs) {
            m.mzz = std::fabs(zz);
            calc_hs(c, m, si);
        }
        if (c.ao) {
            const int q = r.rit == 1 ? 2 : r.rit == 2 ? 1 : 0;
            m.mzz = std::fabs(zz);
            deao_1pos(m, si, q, c.ao_max_len);
            si.amb_shadow = (uint16_t)(((int32_t)si.amb_shadow * 8) / (8 + (int32_t)r.rit));
        } else {
            si.amb_shadow = 5000;
        }
        m.ms_de_stop = saved;
    } else {
        si.zpos_fine = 32768u << 16;
    }
    std::memset(&out, 0, sizeof(out));
    out.si.normal[0] = si.normal[0];
    out.si.normal[1] = si.normal[1];
    out.si.normal[2] = si.normal[2];
    out.si.zpos_fine = si.zpos_fine;
    out.si.shadow = si.shadow;
    out.si.amb_shadow = si.amb_shadow;
    out.si.si_gradient = si.si_gradient;
    out.si.otrap = si.otrap;
    out.hit = open_air ? 0 : 1;
    out.de_limited = de_limited ? 1 : 0;
    std::memcpy(out.pos, m.it.c, sizeof(out.pos));
    out.zz = zz;
    out.zz2_paint = zz2_paint;
    out.zz2 = zz2;
}

}  // namespace
}  // namespace oracle

extern "C" int oracle_reflect_batch(const mb3d_cu_scene *sc, const mb3d_cu_reflect_ray *rays, uint32_t n, int far_fog,
                                    mb3d_cu_reflect_hit *hits, int threads) {
    using namespace oracle;
    if (!sc || (n && (!rays || !hits))) return -1;
    Params p;
    std::string err;
    if (!make_params(*sc, p, err)) return -2;
    Ctx c;
    c.p = &p;
    shadow_lights(*sc, p, c.lights);
    c.hs = sc->shadow_lights != 0 && !c.lights.empty();
    c.soft = sc->shadow_soft != 0;
    c.soft_radius = rmaxf(sc->soft_radius, 0.001f);
    c.hs_mul = sc->hs_max_len_mul;
    c.ao = sc->deao_quality >= 0;
    c.ao_max_len = sc->deao_max_len;
    c.far_fog = far_fog != 0;
    for (uint32_t i = 0; i < n; i++)
        if (rays[i].pixel >= (uint32_t)(sc->width * sc->height)) return -3;
    int nt = threads > 0 ? threads : (int)std::max(1u, std::thread::hardware_concurrency());
    nt = (int)std::min<uint32_t>((uint32_t)nt, std::max<uint32_t>(n, 1));
    auto work = [&](int t) {
        for (uint32_t i = (uint32_t)t; i < n; i += (uint32_t)nt) march_ray(c, rays[i], hits[i]);
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < nt; t++) pool.emplace_back(work, t);
    work(0);
    for (auto &th : pool) th.join();
    return 0;
}

/* The first bounce of every object pixel of a G-buffer (start_pixel,
 * src/reflect.rs:1686-1838, outside rendering, no water, no cutting plane:
 * the surface found again from the stored depth, then step's mirror ray,
 * :1286-1311): the rays in pixel order into out (cap at most); returns the
 * count. */
extern "C" int oracle_reflect_first_rays(const mb3d_cu_scene *sc, const mb3d_cu_silight *gbuf, mb3d_cu_reflect_ray *out,
                                         uint32_t cap) {
    using namespace oracle;
    if (!sc || !gbuf || !out) return -1;
    Params p;
    std::string err;
    if (!make_params(*sc, p, err)) return -2;
    const int w = sc->width, h = sc->height;
    uint32_t n = 0;
    auto zpos_of = [&](double iz) {
        const double q = (8388351.5 - iz) / p.zc_mul + 1.0;
        return (q * q - 1.0) / p.zcorr;
    };
    for (int y = 0; y < h; y++)
        for (int x = 0; x < w; x++) {
            const mb3d_cu_silight &g = gbuf[(size_t)y * w + x];
            if ((g.zpos_fine >> 16) >= 32768u || g.si_gradient >= 32768) continue;
            Marcher m(&p, 0);
            m.cafy = ((double)y / (double)p.height - 0.5) * p.fov_y;
            m.calc_vgrads_fov(x + 1);
            m.calc_start_pos(x, y);
            m.it.calc_sit = false;
            const double zf = (double)(g.zpos_fine >> 8);
            m.mzz = zpos_of(zf);
            add_weight(m.it.c, m.vfov, m.mzz);
            m.update_de_stop();
            double d = m.calc_de();
            if (d < (double)m.ms_de_stop * 0.5) continue;
            const bool de_limited = m.it.it_result < m.max_its_result || d <= (double)m.ms_de_stop;
            if (de_limited) m.bin_search(d, m.mzz - zpos_of(zf - 1.0));
            else m.bin_search_it();
            const double nrm0[3] = {(double)g.normal[0] / 32767.0, (double)g.normal[1] / 32767.0, (double)g.normal[2] / 32767.0};
            double nrm[3];
            rotate_vector_reverse(nrm0, p.vgrads, nrm);
            const double k = 2.0 * dot3(nrm, m.vfov) / dot3(nrm, nrm);
            if (n >= cap) return -3;
            mb3d_cu_reflect_ray &r = out[n++];
            std::memset(&r, 0, sizeof(r));
            for (int i = 0; i < 3; i++) {
                r.origin[i] = m.it.c[i];
                r.dir[i] = m.vfov[i] - nrm[i] * k;
            }
            r.zz = m.mzz;
            r.max_len = 0.0;
            r.pixel = (uint32_t)(y * w + x);
            r.rit = 1;
        }
    return (int)n;
}
