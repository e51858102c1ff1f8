// TEST INFRASTRUCTURE — C entry points of the parity oracle, for the tests
// (ctypes), the smoke check and the benchmark's CPU-baseline leg.  Threads
// take rows t, t+T, ... as the reference renderer does
// (src/render.rs:761-799); every row gets a fresh marcher and every pixel
// its `pixel_seed` (src/render.rs:777-784).
#include "oracle.hpp"
#include <thread>
#include <cstring>
#include <string>

using namespace oracle;

static thread_local std::string g_err;

static void to_c(const SiLight &s, mb3d_cu_silight &o) {
    o.normal[0] = s.normal[0];
    o.normal[1] = s.normal[1];
    o.normal[2] = s.normal[2];
    o.pad = 0;
    o.zpos_fine = s.zpos_fine;
    o.shadow = s.shadow;
    o.amb_shadow = s.amb_shadow;
    o.si_gradient = s.si_gradient;
    o.otrap = s.otrap;
}
static void from_c(const mb3d_cu_silight &o, SiLight &s) {
    s.normal[0] = o.normal[0];
    s.normal[1] = o.normal[1];
    s.normal[2] = o.normal[2];
    s.zpos_fine = o.zpos_fine;
    s.shadow = o.shadow;
    s.amb_shadow = o.amb_shadow;
    s.si_gradient = o.si_gradient;
    s.otrap = o.otrap;
}

template <class F>
static void rows_threaded(int threads, int rows, F f) {
    if (threads < 1) threads = (int)std::thread::hardware_concurrency();
    if (threads < 1) threads = 1;
    if (threads > rows) threads = rows > 0 ? rows : 1;
    std::vector<std::thread> ts;
    for (int t = 0; t < threads; t++)
        ts.emplace_back([=]() {
            for (int r = t; r < rows; r += threads) f(r);
        });
    for (auto &t : ts) t.join();
}

extern "C" {

const char *oracle_last_error(void) { return g_err.c_str(); }

/* The derived per-render values, for comparison with the product's own
 * parameter set-up: 40 doubles in a fixed order. */
int oracle_params(const mb3d_cu_scene *sc, double *out, int n) {
    Params p;
    if (!make_params(*sc, p, g_err)) return -22;
    double v[] = {(double)p.de_option,  (double)p.d_de_scale, (double)p.de_stop,   (double)p.z_step_div,
                  (double)p.mh04zsd,    (double)p.de_stop_factor, p.zcorr,         p.zc_mul,
                  p.zend,               p.step_width,          p.ystart[0],          p.ystart[1],
                  p.ystart[2],          p.d_rstop,             p.rstop3d,            (double)p.ln_rstop,
                  (double)p.de_offset,  (double)p.de_offset006, (double)p.mcts_m,   (double)p.d_col_plus,
                  (double)p.col_var_de_stop_mul, (double)p.fovx_off, (double)p.fovx_mul, p.fov_y,
                  (double)p.fhln[0],    (double)p.fhln[1],     (double)p.fhln[2],    (double)p.end_to,
                  (double)p.repeat_from, (double)p.is_custom_de, p.vgrads[0][0],     p.vgrads[0][1],
                  p.vgrads[0][2],       p.vgrads[1][0],        p.vgrads[1][1],       p.vgrads[1][2],
                  p.vgrads[2][0],       p.vgrads[2][1],        p.vgrads[2][2],       (double)p.min_it};
    int m = (int)(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < n && i < m; i++) out[i] = v[i];
    return m;
}

int32_t oracle_pixel_seed(int64_t y, int64_t x) { return pixel_seed(y, x); }

/* One formula step on v (x, y, z, w) and j (the constant). */
int oracle_formula_iterate(int formula, const double *options, double *v, double *j, double rout, int ade) {
    Formula f;
    mb3d_cu_slot s;
    std::memset(&s, 0, sizeof(s));
    s.formula = formula;
    s.iterations = 1;
    for (int k = 0; k < 16; k++) s.options[k] = options[k];
    if (!formula_from_slot(s, f, g_err)) return -22;
    f.iterate(v, j, rout, ade != 0);
    return 0;
}

/* calc::de_at (src/calc.rs:2695-2700): the DE in world units and the
 * iteration count at n points. */
int oracle_de_at(const mb3d_cu_scene *sc, const double *pos, int n, double *de, int32_t *its) {
    Params p;
    if (!make_params(*sc, p, g_err)) return -22;
    for (int i = 0; i < n; i++) {
        Marcher m(&p, 1);
        m.it.c[0] = pos[3 * i];
        m.it.c[1] = pos[3 * i + 1];
        m.it.c[2] = pos[3 * i + 2];
        double d = m.calc_de();
        de[i] = d * p.step_width;
        its[i] = m.it.it_result;
    }
    return 0;
}

/* The march of rows row0..row0+rows into out (rows * width records). */
int oracle_march(const mb3d_cu_scene *sc, int row0, int rows, mb3d_cu_silight *out, int threads, uint64_t *de_evals) {
    Params p;
    if (!make_params(*sc, p, g_err)) return -22;
    int w = p.width;
    g_de_evals.store(0);
    bool count = de_evals != nullptr;
    rows_threaded(threads, rows, [&](int r) {
        int y = row0 + r;
        Marcher m(&p, 0);
        m.count_de = count;
        for (int x = 0; x < w; x++) {
            m.seed = pixel_seed(y, x);
            SiLight s = m.march_pixel(x, y);
            to_c(s, out[(size_t)r * w + x]);
        }
    });
    if (de_evals) *de_evals = g_de_evals.load();
    return 0;
}

/* A list of pixels (x, y pairs) marched into out: a bounded sample for
 * timing and for spot checks of big pictures. */
int oracle_march_pixels(const mb3d_cu_scene *sc, const int32_t *xy, int n, mb3d_cu_silight *out, int threads) {
    Params p;
    if (!make_params(*sc, p, g_err)) return -22;
    int chunks = threads < 1 ? (int)std::thread::hardware_concurrency() : threads;
    if (chunks < 1) chunks = 1;
    rows_threaded(chunks, chunks, [&](int t) {
        Marcher m(&p, 0);
        for (int i = t; i < n; i += chunks) {
            int x = xy[2 * i], y = xy[2 * i + 1];
            m.seed = pixel_seed(y, x);
            SiLight s = m.march_pixel(x, y);
            to_c(s, out[i]);
        }
    });
    return 0;
}

/* The hard (or soft) shadow pass on the whole-picture G-buffer, in place
 * (src/render.rs:2430-2496; 8 binary search steps).  per_pixel = 1: without
 * the row-sequential open-air shortcut, as the reference's card pass. */
int oracle_shadows(const mb3d_cu_scene *sc, mb3d_cu_silight *gbuf, int threads, int per_pixel) {
    Params p;
    if (!make_params(*sc, p, g_err)) return -22;
    p.de_add_steps = 8;
    std::vector<HsLight> lights;
    shadow_lights(*sc, p, lights);
    if (lights.empty()) return 0;
    int w = p.width, h = p.height;
    rows_threaded(threads, h, [&](int y) {
        int32_t seed = (int32_t)((int64_t)0x24563487u + ((int64_t)y + 1) * (int64_t)0x324594A1);
        Marcher m(&p, seed);
        std::vector<SiLight> row(w);
        for (int x = 0; x < w; x++) from_c(gbuf[(size_t)y * w + x], row[x]);
        if (sc->shadow_soft)
            m.soft_shadow_row(y, row.data(), w, lights[0], sc->soft_radius, sc->hs_max_len_mul);
        else
            m.hard_shadow_row(y, row.data(), w, lights, sc->hs_max_len_mul, per_pixel != 0);
        for (int x = 0; x < w; x++) to_c(row[x], gbuf[(size_t)y * w + x]);
    });
    return 0;
}

/* The DE ambient occlusion pass in place (src/deao.rs:109-414; 5 binary
 * search steps). */
int oracle_deao(const mb3d_cu_scene *sc, mb3d_cu_silight *gbuf, int threads) {
    Params p;
    if (!make_params(*sc, p, g_err)) return -22;
    if (sc->deao_quality < 0) return 0;
    p.de_add_steps = 5;
    int w = p.width, h = p.height;
    rows_threaded(threads, h, [&](int y) {
        int32_t seed = (int32_t)((int64_t)0x24563487u + ((int64_t)y + 1) * (int64_t)0x324594A1);
        Marcher m(&p, seed);
        int32_t rnd = seed;
        std::vector<SiLight> row(w);
        for (int x = 0; x < w; x++) from_c(gbuf[(size_t)y * w + x], row[x]);
        deao_row(m, y, row.data(), w, sc->deao_quality, sc->deao_max_len, sc->deao_first_step_random != 0, rnd);
        for (int x = 0; x < w; x++) to_c(row[x], gbuf[(size_t)y * w + x]);
    });
    return 0;
}

/* The whole CPU render of a band of rows, as the reference's CPU path does
 * it (src/render.rs:459-799, then the post passes src/render.rs:2119-2496,
 * src/deao.rs:109): the march, the hard shadows with the row pass (with
 * its open-air shortcut) and the DE AO of the listed rows; threads take
 * rows t, t+T, ... of the list.  Used as the timed CPU baseline. */
int oracle_render_rows(const mb3d_cu_scene *sc, const int32_t *row_list, int rows, mb3d_cu_silight *out, int threads) {
    Params p;
    if (!make_params(*sc, p, g_err)) return -22;
    Params ps = p, pa = p;
    ps.de_add_steps = 8;
    pa.de_add_steps = 5;
    std::vector<HsLight> lights;
    shadow_lights(*sc, ps, lights);
    int w = p.width;
    rows_threaded(threads, rows, [&](int r) {
        int y = row_list[r];
        std::vector<SiLight> row(w);
        {
            Marcher m(&p, 0);
            for (int x = 0; x < w; x++) {
                m.seed = pixel_seed(y, x);
                row[x] = m.march_pixel(x, y);
            }
        }
        int32_t seed = (int32_t)((int64_t)0x24563487u + ((int64_t)y + 1) * (int64_t)0x324594A1);
        if (!lights.empty()) {
            Marcher m(&ps, seed);
            if (sc->shadow_soft)
                m.soft_shadow_row(y, row.data(), w, lights[0], sc->soft_radius, sc->hs_max_len_mul);
            else
                m.hard_shadow_row(y, row.data(), w, lights, sc->hs_max_len_mul, false);
        }
        if (sc->deao_quality >= 0) {
            Marcher m(&pa, seed);
            int32_t rnd = seed;
            deao_row(m, y, row.data(), w, sc->deao_quality, sc->deao_max_len, sc->deao_first_step_random != 0, rnd);
        }
        for (int x = 0; x < w; x++) to_c(row[x], out[(size_t)r * w + x]);
    });
    return 0;
}

/* The DE AO ray directions of a quality level (deao::build_rays,
 * src/deao.rs:75-104): their count, directions into dirs (3 floats each). */
int oracle_ao_rays(int quality, float *dirs, int cap) {
    SiLight dummy;
    (void)dummy;
    return oracle::ao_ray_table(quality, dirs, cap);
}

}  // extern "C"
