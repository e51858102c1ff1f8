// Oracle (test infrastructure): depth of field on the painted picture, a
// C++ restatement of mb3d-rs's CPU path (src/dof.rs): focus (:49-78), the
// forward variant dof_forward (:125-223, its CPU loops) and the default
// sorted variant dof_sorted (:259-420, its CPU loops: the sources back to
// front in a counting sort over the fine depth, each band of rows walking the
// whole list).  8-bit pictures (Sample for u8, src/lighting.rs:33-50).
// Compiled with -ffp-contract=off: single precision arithmetic unfused, as
// Rust's.
#include "oracle.hpp"
#include <thread>
#include <vector>

namespace oracle {
namespace {

struct ZConv {
    double zc_mul_inv, zcorr_inv;
    float steps(double z) const {
        double a = z * zc_mul_inv + 1.0;
        return (float)((a * a - 1.0) * zcorr_inv);
    }
};

// (ap, de_stop_factor, z_sharp, r_sub) of a pass
void focus(const mb3d_cu_dof_opts &p, uint32_t pass, bool sorted, int width, int height, double fov_y_deg, float &ap,
           float &dsf, float &z_sharp, float &r_sub) {
    const float ap0 = rclampf(p.aperture, 0.0001f, 2.0f);
    const int lp = (int)(p.passes < 1 ? 1 : p.passes > 4 ? 4 : p.passes) - 1;
    if (lp == 0) {
        ap = ap0 * 0.5f;
    } else if (lp == 1) {
        ap = sorted ? ap0 * (0.25f + (float)pass * 0.58f) * 0.5f : ap0 * (0.3f + (float)pass * 0.55f) * 0.5f;
    } else {
        float p3 = 1.0f;
        for (uint32_t k = 0; k < pass; k++) p3 *= 3.0f;
        ap = sorted ? ap0 / 22.0f * p3 : ap0 / 12.0f * (float)(1u << pass);
    }
    dsf = (float)(rmax(fov_y_deg * (3.14159265358979323846 / 180.0), 0.0) / (double)height);  // (f64::to_radians)
    const float dw = rminf(p.z_sharp, p.z_sharp2) * (float)width;
    const float st = rmaxf(p.z_sharp, p.z_sharp2) * (float)width;
    const float w = (1.0f + dw * dsf) / (1.0f + st * dsf);
    z_sharp = (w * st + dw) / (1.0f + w);
    r_sub = std::fabs((dw - z_sharp) / (1.0f + dw * dsf) * ap);
}

inline uint8_t from_dof(float v) { return (uint8_t)rtef(rclampf(v, 0.0f, 255.0f)); }
inline float signumf(float v) { return std::isnan(v) ? v : (std::signbit(v) ? -1.0f : 1.0f); }

void dof_forward(std::vector<uint8_t> &rgb, const mb3d_cu_silight *gbuf, int width, int height, const ZConv &zc,
                 double fov, const mb3d_cu_dof_opts &p, uint32_t pass) {
    float ap, dsf, z_sharp, r_sub;
    focus(p, pass, false, width, height, fov, ap, dsf, z_sharp, r_sub);
    const float clip_r = rclampf(p.clip_r, 0.1f, 1000.0f);
    const size_t n = (size_t)width * height;
    const float bg = zc.steps(8388353.0);
    std::vector<float> rbuf(n);
    float max_r = 0.0f;
    for (size_t i = 0; i < n; i++) {
        const mb3d_cu_silight &s = gbuf[i];
        float w = (s.zpos_fine >> 16) > 32767 ? bg : zc.steps((double)(8388352 - (int64_t)(s.zpos_fine >> 8)));
        float v = (w - z_sharp) / (1.0f + w * dsf) * ap;
        v = rmaxf(std::fabs(v) - r_sub, 0.0f) * signumf(v);
        if (std::fabs(v) > clip_r) v = clip_r * signumf(v);
        max_r = rmaxf(max_r, std::fabs(v));
        rbuf[i] = v;
    }
    const float sm = 1.0f / (1.0f + max_r);
    std::vector<float> transp(n, 0.0f), col(n * 3, 0.0f);
    const int64_t wi = width, hi = height;
    for (int64_t y = 0; y < hi; y++)
        for (int64_t x = 0; x < wi; x++) {
            const size_t i = (size_t)(y * wi + x);
            const float rr = rbuf[i];
            const float a = std::fabs(rr) + 1.0f;
            const float s_ms = a * a;
            const float c[3] = {(float)rgb[i * 3], (float)rgb[i * 3 + 1], (float)rgb[i * 3 + 2]};
            const float sw = 0.5f / s_ms;
            const int64_t r = (int64_t)rtef(std::fabs(rr) + 0.5f);
            const int64_t xa = std::max(-r, -x), xe = std::min(r, wi - 1 - x);
            const int64_t ya = std::max(-r, -y), ye = std::min(r, hi - 1 - y);
            for (int64_t yy = ya; yy <= ye; yy++)
                for (int64_t xx = xa; xx <= xe; xx++) {
                    float w = s_ms - (float)(xx * xx) - (float)(yy * yy);
                    if (w > 0.0f) {
                        if (w > 1.0f) w = 1.0f;
                        const size_t j = (size_t)((y + yy) * wi + x + xx);
                        if (rbuf[j] >= rr) w *= sw;
                        else w *= sw * std::fabs(rbuf[j]) * sm;
                        transp[j] += w;
                        col[j * 3] += c[0] * w;
                        col[j * 3 + 1] += c[1] * w;
                        col[j * 3 + 2] += c[2] * w;
                    }
                }
        }
    for (size_t i = 0; i < n; i++) {
        const float m = transp[i] < 1e-10f ? 1e10f : 1.0f / transp[i];
        for (int k = 0; k < 3; k++) rgb[i * 3 + k] = from_dof(col[i * 3 + k] * m);
    }
}

struct SortedSrc {
    float s_ms, sw;
    int64_t ims, r;
    bool descale, bg;
};

SortedSrc sorted_src(int32_t iz, const ZConv &zc, float z_sharp, float ap, float dsf, float r_sub, float max_r) {
    const float w = zc.steps((double)(8388352 - (int64_t)iz));
    float s_radius = (w - z_sharp) * ap / (1.0f + w * dsf);
    SortedSrc t;
    t.descale = s_radius < 0.0f;
    s_radius = rclampf(std::fabs(s_radius) - r_sub, 0.0f, max_r);
    t.s_ms = s_radius + 1.0f;
    t.sw = 1.0f / (2.5f * s_radius * s_radius + 1.0f);
    t.ims = (int64_t)(t.s_ms * t.s_ms);
    t.r = (int64_t)rtef(std::fabs(s_radius) + 0.5f);
    t.bg = iz == -1;
    return t;
}

inline int32_t sort_depth(const mb3d_cu_silight &s) {
    const int32_t z = (int32_t)(s.zpos_fine >> 8);
    return (z > 8388352 || (s.zpos_fine >> 16) > 32767) ? -1 : z;
}

void dof_sorted(std::vector<uint8_t> &rgb, const mb3d_cu_silight *gbuf, int width, int height, const ZConv &zc,
                double fov, const mb3d_cu_dof_opts &p, uint32_t pass, int threads) {
    float ap, dsf, z_sharp, r_sub;
    focus(p, pass, true, width, height, fov, ap, dsf, z_sharp, r_sub);
    const float clip_r = rclampf(p.clip_r, 0.1f, 1000.0f);
    const size_t n = (size_t)width * height;
    int64_t zmin = 32768, zmax = 0;
    for (size_t i = 0; i < n; i++) {
        const int64_t z = gbuf[i].zpos_fine >> 16;
        if (z < 32768) {
            zmin = std::min(zmin, z);
            zmax = std::max(zmax, z);
        }
    }
    float w = zc.steps((double)((32768 - zmin) * 256));
    const float r0 = std::fabs((w - z_sharp) * ap / (1.0f + w * dsf));
    w = zc.steps((double)((32768 - zmax) * 256));
    const float max_r = rminf(clip_r, rmaxf(r0, std::fabs((w - z_sharp) / (1.0f + w * dsf) * ap)) * 1.5f);
    // back to front: ascending fine depth, the background first, equal
    // depths in pixel order (a stable counting sort)
    std::vector<size_t> start(8388355, 0);
    for (size_t i = 0; i < n; i++) start[(size_t)(sort_depth(gbuf[i]) + 2)]++;
    for (size_t k = 1; k < start.size(); k++) start[k] += start[k - 1];
    std::vector<uint32_t> order(n);
    for (size_t i = 0; i < n; i++) {
        const size_t k = (size_t)(sort_depth(gbuf[i]) + 1);
        order[start[k]++] = (uint32_t)i;
    }
    start.clear();
    start.shrink_to_fit();
    const int64_t wi = width, hi = height;
    const int64_t rmax_i = (int64_t)rtef(std::fabs(max_r) + 0.5f);
    if (threads < 1) threads = (int)std::thread::hardware_concurrency();
    if (threads < 1) threads = 1;
    const int band_rows = std::max(1, (height + threads * 4 - 1) / (threads * 4));
    const int n_bands = (height + band_rows - 1) / band_rows;
    std::vector<uint8_t> out(rgb.size());
    std::atomic<int> next{0};
    std::vector<std::thread> ts;
    for (int t = 0; t < std::min(threads, n_bands); t++)
        ts.emplace_back([&]() {
            for (;;) {
                const int b = next.fetch_add(1);
                if (b >= n_bands) break;
                const int64_t by0 = (int64_t)b * band_rows, by1 = std::min<int64_t>((int64_t)(b + 1) * band_rows, hi);
                const size_t bn = (size_t)(by1 - by0) * width;
                std::vector<float> transp(bn, 0.0f), col(bn * 3, 0.0f);
                const uint32_t lo = (uint32_t)(std::max<int64_t>(by0 - rmax_i, 0) * wi);
                const uint32_t hi_i = (uint32_t)(std::min<int64_t>(by1 + rmax_i, hi) * wi);
                for (uint32_t idx : order) {
                    if (idx < lo || idx >= hi_i) continue;
                    const size_t i = idx;
                    const int64_t x = (int64_t)(i % (size_t)width), y = (int64_t)(i / (size_t)width);
                    const float c[3] = {(float)rgb[i * 3], (float)rgb[i * 3 + 1], (float)rgb[i * 3 + 2]};
                    const SortedSrc s = sorted_src(sort_depth(gbuf[i]), zc, z_sharp, ap, dsf, r_sub, max_r);
                    const int64_t xa = std::max(-s.r, -x), xe = std::min(s.r, wi - 1 - x);
                    const int64_t ya = std::max(std::max(-s.r, -y), by0 - y), ye = std::min(std::min(s.r, hi - 1 - y), by1 - 1 - y);
                    for (int64_t yy = ya; yy <= ye; yy++) {
                        const int64_t iys = yy * yy;
                        for (int64_t xx = xa; xx <= xe; xx++) {
                            const int64_t ii = xx * xx + iys;
                            if (ii > s.ims) continue;
                            const size_t j = (size_t)((y + yy - by0) * wi + x + xx);
                            float wv = s.s_ms - std::sqrt((float)ii);
                            float dw = 0.0f;
                            if (s.descale) {
                                const float q = 0.8f * wv / s.s_ms;
                                dw = 1.0f - q * q;
                            }
                            wv = wv > 1.0f ? s.sw : wv * s.sw;
                            float *pc = &col[j * 3];
                            float &pt = transp[j];
                            if (s.descale && pt > dw) {
                                const float f = dw / pt;
                                for (int k = 0; k < 3; k++) pc[k] *= f;
                                pt *= f;
                            }
                            if (!s.bg && wv + pt > 1.01f) {
                                const float st = (1.01f - wv) / pt;
                                for (int k = 0; k < 3; k++) pc[k] = pc[k] * st + c[k] * wv;
                                pt = 1.01f;
                            } else {
                                for (int k = 0; k < 3; k++) pc[k] += c[k] * wv;
                                pt += wv;
                            }
                        }
                    }
                }
                for (size_t k = 0; k < bn * 3; k++) {
                    const float tt = transp[k / 3];
                    out[(size_t)by0 * width * 3 + k] = from_dof(col[k] * (tt < 1e-10f ? 1e10f : 1.0f / tt));
                }
            }
        });
    for (auto &t : ts) t.join();
    rgb.swap(out);
}

}  // namespace
}  // namespace oracle

extern "C" {

/* Depth of field (dof::apply, src/dof.rs:81-122) on an 8-bit picture in
 * place: all passes of the options' variant. */
int oracle_dof(uint8_t *rgb, const mb3d_cu_silight *gbuf, int width, int height, double zc_mul, double zcorr,
               double fov_y_deg, const mb3d_cu_dof_opts *opts, int threads) {
    using namespace oracle;
    if (!rgb || !gbuf || !opts || width < 1 || height < 1) return -22;
    const size_t n = (size_t)width * height;
    std::vector<uint8_t> pic(rgb, rgb + n * 3);
    ZConv zc{1.0 / zc_mul, 1.0 / zcorr};
    const uint32_t passes = opts->passes < 1 ? 1 : opts->passes > 4 ? 4 : opts->passes;
    for (uint32_t pass = 0; pass < passes; pass++) {
        if (opts->forward) dof_forward(pic, gbuf, width, height, zc, fov_y_deg, *opts, pass);
        else dof_sorted(pic, gbuf, width, height, zc, fov_y_deg, *opts, pass, threads);
    }
    std::copy(pic.begin(), pic.end(), rgb);
    return 0;
}

}  // extern "C"
