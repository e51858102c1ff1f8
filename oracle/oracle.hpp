// TEST INFRASTRUCTURE — the parity oracle.  A C++17 double precision
// restatement of mb3d-rs's CPU "Calculate 3D" path (the reference renderer,
// Rust, which cannot be compiled in this environment: no Rust toolchain).
// Only the tests, the smoke check and the benchmark's CPU-baseline leg use
// it; the product library never links or calls it.
//
// Parity pinning: the restatement is checked against every known-answer
// test the reference holds for this path (formula identities
// src/formulas.rs:860-967, the seed jump-ahead src/calc.rs:2986-2996, the DE
// sanity checks tests/render.rs:47-71, coverage/shadow/AO checks
// tests/render.rs:24-30,118-177, DE AO ray counts src/deao.rs:416-471).  The
// reference binary itself cannot run here, so image-level parity against
// the reference is pinned only through those tests.  The Menger IFS has no
// source in the reference (machine code in a .m3f file): parity unpinned.
//
// Each function cites the reference file:line it restates.  Rust semantics
// kept: round-half-even (`round_ties_even`), saturating float->int casts,
// f32 round trips where the reference stores singles, wrapping i32 LCGs,
// NaN-ignoring max/min (`f64::max`), no FMA contraction (build with
// -ffp-contract=off).
#pragma once
#include <cstdint>
#include <cmath>
#include <vector>
#include <string>
#include <atomic>
#include "../include/mb3d_cu.h"

namespace oracle {

typedef double Vec3[3];
typedef double Mat3[3][3];

// ---- Rust semantics helpers ----
inline double rmax(double a, double b) { return std::fmax(a, b); }
inline double rmin(double a, double b) { return std::fmin(a, b); }
inline float rmaxf(float a, float b) { return std::fmax(a, b); }
inline float rminf(float a, float b) { return std::fmin(a, b); }
// f64::clamp: NaN stays NaN
inline double rclamp(double x, double lo, double hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
inline float rclampf(float x, float lo, float hi) {
    if (x < lo) x = lo;
    if (x > hi) x = hi;
    return x;
}
inline double rte(double x) { return std::nearbyint(x); }  // round_ties_even
inline float rtef(float x) { return std::nearbyintf(x); }
// saturating `as` casts
inline int64_t sat_i64(double x) {
    if (std::isnan(x)) return 0;
    if (x >= 9.2233720368547758e18) return INT64_MAX;
    if (x <= -9.2233720368547758e18) return INT64_MIN;
    return (int64_t)x;
}
inline int32_t sat_i32(double x) {
    if (std::isnan(x)) return 0;
    if (x >= 2147483647.0) return INT32_MAX;
    if (x <= -2147483648.0) return INT32_MIN;
    return (int32_t)x;
}
inline uint16_t sat_u16(double x) {
    if (std::isnan(x) || x <= 0.0) return 0;
    if (x >= 65535.0) return 65535;
    return (uint16_t)x;
}
inline uint32_t sat_u32(double x) {
    if (std::isnan(x) || x <= 0.0) return 0;
    if (x >= 4294967295.0) return 4294967295u;
    return (uint32_t)x;
}
inline int16_t sat_i16(double x) {
    if (std::isnan(x)) return 0;
    if (x >= 32767.0) return 32767;
    if (x <= -32768.0) return -32768;
    return (int16_t)x;
}
inline int32_t wrap_lcg(int32_t s, uint32_t a, uint32_t c) { return (int32_t)((uint32_t)s * a + c); }

// ---- math helpers (src/math.rs:28-134) ----
inline void add_weight(double a[3], const double b[3], double w) {
    a[0] += b[0] * w;
    a[1] += b[1] * w;
    a[2] += b[2] * w;
}
inline double dot3(const double a[3], const double b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline void rotate_vector_reverse(const double v[3], const Mat3 m, double out[3]) {
    double r0 = v[0] * m[0][0] + v[1] * m[1][0] + v[2] * m[2][0];
    double r1 = v[0] * m[0][1] + v[1] * m[1][1] + v[2] * m[2][1];
    double r2 = v[0] * m[0][2] + v[1] * m[1][2] + v[2] * m[2][2];
    out[0] = r0;
    out[1] = r1;
    out[2] = r2;
}
inline void normalise_matrix_to(double n, const Mat3 m, Mat3 r) {
    for (int i = 0; i < 3; i++) {
        double d = n / std::sqrt(dot3(m[i], m[i]));
        for (int j = 0; j < 3; j++) r[i][j] = m[i][j] * d;
    }
}
// BuildViewVectorDFOV (src/math.rs:127-134)
inline void build_view_vector_dfov(double xa, double ya, double out[3]) {
    double sx = std::sin(xa), cx = std::cos(xa);
    double sy = std::sin(ya), cy = std::cos(ya);
    double v[3] = {-sy, sx, cx * cy};
    double n = 1.0 / std::sqrt(dot3(v, v));
    out[0] = v[0] * n;
    out[1] = v[1] * n;
    out[2] = v[2] * n;
}
// ---- formulas (src/formulas.rs) ----
enum FormulaKind { F_INTPOW = 0, F_REALPOWER = 1, F_QUATERNION = 2, F_TRICORN = 3, F_AMAZINGBOX = 4, F_BULBOX = 5, F_FOLDINGINTPOW = 6, F_AEXIONC = 9, F_MENGER = 100 };

struct Formula {
    int kind = F_INTPOW;
    double o[16] = {0};
    int power() const;  // integer power of IntPow / FoldingIntPow
    int de_option() const;
    double de_scale() const;
    double ade_scale() const { return 1.0; }
    double default_rstop() const;
    double si_pow() const;
    double first_option() const;
    bool first_option_double() const;
    bool julia_adds() const { return kind == F_MENGER; }
    void iterate(double v[4], double j[4], double rout, bool ade) const;
};

bool formula_from_slot(const mb3d_cu_slot &s, Formula &f, std::string &err);

struct Slot {
    Formula f;
    int iterations = 0;
    bool uncounted = false;
    bool ade = false;
    bool julia_add = false;
};

// ---- one part of a DE combination (HybridPart, src/calc.rs:210-220) ----
struct DeCombPart {
    int start = 0, end = 0, repeat = 0;
    int de_option = 0;
    bool is_custom_de = false;
    float d_de_scale = 1.f;
    int max_it = 0;
};

// ---- per-render parameters: CalcParams (src/calc.rs:21-134), built by
// CalcParams::new (src/calc.rs:375-891) for the alternating 3D hybrid ----
struct Params {
    std::vector<Slot> slots;
    int color_on_it = 0;
    bool is_custom_de = false;
    int de_option = 0;
    float d_de_scale = 1.f;
    int sm_normals = 0;
    float de_stop = 1.f;
    float z_step_div = 0.5f;
    int de_add_steps = 8;
    int width = 0, height = 0;
    double fov_y = 0;
    int max_it = 0, min_it = 0;
    int color_option = 0;
    float mct_color_mul = 512.f;
    double d_rstop = 0, rstop3d = 0;
    bool do_julia = false;
    double ju[4] = {0};
    Mat3 vgrads = {{0}};
    float pl_optic_z = 0;
    int dfog_on_it = 0;
    float fovx_off = 0, fovx_mul = 0;
    float d_col_plus = 0;
    double zcorr = 0, zc_mul = 0, zend = 0, step_width = 0;
    float col_var_de_stop_mul = 0.6f;
    bool first_step_random = true;
    float mh04zsd = 0;
    float de_stop_factor = 0;
    float ln_rstop = 0;
    bool normals_on_de = true;
    Vec3 ystart = {0};
    float de_offset = 0, de_offset006 = 0;
    float mcts_m = 0;
    float ms_de_sub = 0;
    float fhln[6];
    int end_to = 0, repeat_from = 0;
    bool ipol = false;              // an interpolation hybrid (HybridMode::Ipol3D)
    float ipol_w[2] = {1.f, 0.f};   // its normalised weights
    bool four_d = false;            // a 4D alternating hybrid (HybridMode::Alt4D)
    double smatrix4[4][4] = {{0}};  // its 4D rotation (BuildSMatrix4)
    // a DE combination (DeComb, src/calc.rs:224-236): kind 0 none, 1..5;
    // its second part, smoothing distance (steps) and part 2's place
    int dc_kind = 0;
    DeCombPart dc_part2;
    double dc_smooth = 0;
    bool dc_place = false;
    Mat3 dc_m = {{0}};
    Vec3 dc_offset = {0};
    double dc_scale = 1;
};

bool make_params(const mb3d_cu_scene &sc, Params &p, std::string &err);

// ---- the iteration record (src/iteration.rs:57-105, the 3D subset) ----
struct Iteration {
    double v[4] = {0}, c[3] = {0}, j[4] = {0}, ju[4] = {0};
    bool do_julia = false;
    double rout = 0, rold = 0, otrap = 0;
    int it_result = 0, max_it = 0;
    double rstop = 0;
    bool calc_sit = false;
    float smooth_it = 0;
    float ln_rstop = 0;
    int de_option = 0;
    int start_from = 0, end_to = 0, repeat_from = 0;
    float fhln[6];
    bool ipol = false;
    float ipol_w[2] = {1.f, 0.f};
    bool four_d = false;
    double smatrix4[4][4] = {{0}};
    void smooth_iterations(int n);
    void hybrid_4d(const std::vector<Slot> &slots);
    int run(const std::vector<Slot> &slots);
    void run_ipol(const std::vector<Slot> &slots, bool de);
    void hybrid_3d(const std::vector<Slot> &slots);
    double hybrid_3d_de(const std::vector<Slot> &slots);
};

struct SiLight {
    int16_t normal[3] = {0, 0, 0};
    uint32_t zpos_fine = 32768u << 16;
    uint16_t shadow = 0, amb_shadow = 0, si_gradient = 0, otrap = 0;
    uint32_t zpos() const { return zpos_fine >> 16; }
};

struct HsLight {
    int idx;
    Vec3 vec;
};

extern std::atomic<uint64_t> g_de_evals;

// ---- the marcher (src/calc.rs:1142-2980) ----
struct Marcher {
    const Params *p;
    Iteration it;
    float ms_de_stop;
    double mzz = 0;
    Vec3 vfov = {0, 0, 1};
    double cafy = 0;
    int max_its_result;
    float s_roughness = 0;
    int32_t seed;
    bool count_de = false;

    Marcher(const Params *pp, int32_t s);
    double calc_de();
    void set_part(int start, int end, int repeat, int max_it, int de_option);
    double calc_de_part(bool is_custom_de, float d_de_scale, bool invert);
    void calc_vgrads_fov(int ix);
    void calc_start_pos(int ix, int iy);
    void step(double d);
    void update_de_stop();
    void bin_search(double &de, double last_step_width);
    void bin_search_it();
    float calculate_normals(SiLight &si);
    float calculate_normals_on_smooth_it(SiLight &si);
    void do_color_on_it();
    void do_color(SiLight &si);
    void calc_zpos_and_rough(SiLight &si);
    bool surface_point(int x, int y, const SiLight &si, int steps, double thr);
    void surface_found(SiLight &si, double dtmp, double last_step);
    SiLight march_pixel(int x, int y);
    SiLight march_from(SiLight si, double dtmp, bool first_step, float step_count);
    bool hs_surface_start(int x, int y, const SiLight &si);
    double hs_max_len(int y, float mul);
    void hard_shadow_row(int y, SiLight *row, int n, const std::vector<HsLight> &lights, float mul, bool per_pixel);
    void soft_shadow_row(int y, SiLight *row, int n, const HsLight &light, float soft_radius, float mul);
};

int32_t pixel_seed(int64_t y, int64_t x);
void shadow_lights(const mb3d_cu_scene &sc, const Params &p, std::vector<HsLight> &out);
int ao_ray_table(int quality, float *dirs, int cap);
void deao_row(Marcher &m, int y, SiLight *row, int n, int quality, float max_len, bool first_step_random, int32_t &rnd);
void deao_1pos(Marcher &m, SiLight &si, int quality, float max_len);
uint16_t clip15(float s);  // MinMaxClip15bit

}  // namespace oracle
