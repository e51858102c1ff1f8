// TEST INFRASTRUCTURE — the parity oracle (see oracle.hpp for what it pins).
// C++17 FP64 restatement of mb3d-rs's CPU march, built with
// -O3 -ffp-contract=off so that it keeps the reference's unfused arithmetic.
#include "oracle.hpp"
#include <algorithm>
#include <array>
#include <cstring>

namespace oracle {

std::atomic<uint64_t> g_de_evals{0};

static const double PI = 3.14159265358979323846;
static const double TAU = 6.28318530717958647692;
// Rust's f64::to_radians: self * (PI / 180)
static inline double to_radians(double d) { return d * (PI / 180.0); }

// ---------------------------------------------------------------------------
// math helpers (src/math.rs:28-134, 218-246)
// create_xy_vecs_from_normals (src/math.rs:218-233)
static void create_xy_vecs_from_normals(const double n[3], double vx[3], double vy[3]) {
    double d = n[1] * n[1] + n[0] * n[0];
    if (d < 1e-50) {
        vx[0] = 1; vx[1] = 0; vx[2] = 0;
        vy[0] = 0; vy[1] = 1; vy[2] = 0;
        return;
    }
    double a = std::acos(rclamp(-n[2] / std::sqrt(d + n[2] * n[2] + 1e-100), -1.0, 1.0)) * 0.5;
    double sin_a = std::sin(a), cos_a = std::cos(a);
    sin_a /= std::sqrt(d);
    double dd = -n[1] * sin_a;
    double d1 = n[0] * sin_a;
    vx[0] = 1.0 - 2.0 * d1 * d1;
    vx[1] = 2.0 * dd * d1;
    vx[2] = 2.0 * d1 * cos_a;
    vy[0] = vx[1];
    vy[1] = 1.0 - 2.0 * dd * dd;
    vy[2] = -2.0 * dd * cos_a;
}
// MinMaxClip15bit (src/math.rs:246-255)
static inline uint16_t min_max_clip_15bit(float s) {
    if (std::isnan(s) || s < 0.0f) return 0;
    if (s > 32767.0f) return 32767;
    return (uint16_t)rtef(s);
}

// ---------------------------------------------------------------------------
// formulas (src/formulas.rs)
int Formula::power() const {
    int p = sat_i32(std::round(o[0]));
    return std::min(8, std::max(2, p));
}

// iDEoption (src/formulas.rs:492-499)
int Formula::de_option() const {
    switch (kind) {
        case F_AMAZINGBOX: return 11;
        case F_QUATERNION: return 4;  // the 4D numerical DE
        case F_MENGER: return 2;  // the .m3f header's .DEoption = 2
        default: return 0;
    }
}
// dDEscale (src/formulas.rs:502-509)
double Formula::de_scale() const {
    switch (kind) {
        case F_AMAZINGBOX: case F_BULBOX: case F_MENGER: return 0.2;
        case F_FOLDINGINTPOW: return 0.5;
        default: return 1.0;
    }
}
// dRstop (src/formulas.rs:520-528)
double Formula::default_rstop() const {
    switch (kind) {
        case F_AMAZINGBOX: case F_BULBOX: case F_FOLDINGINTPOW: case F_MENGER: return 1024.0;
        default: return 16.0;
    }
}
// dSIpow (src/formulas.rs:531-544); the Menger file has no .SIpower (0)
double Formula::si_pow() const {
    switch (kind) {
        case F_INTPOW: return (double)power();
        case F_REALPOWER: case F_AEXIONC: return o[0] == 0.0 ? 1e-40 : o[0];
        case F_MENGER: return 0.0;
        default: return 2.0;
    }
}
// first_option (src/formulas.rs:547-558)
double Formula::first_option() const {
    if (kind == F_INTPOW || kind == F_FOLDINGINTPOW) return o[1];
    return o[0];
}
bool Formula::first_option_double() const { return !(kind == F_INTPOW || kind == F_FOLDINGINTPOW); }

// box_fold (src/formulas.rs:707-709)
static inline double box_fold(double x, double fold) { return std::fabs(x + fold) - (std::fabs(x - fold) + x); }

// amazing_box (src/formulas.rs:713-735)
static void amazing_box(double scale, double min_r, double fold, double v[4], const double j[4], bool ade) {
    double x = box_fold(v[0], fold);
    double y = box_fold(v[1], fold);
    double z = box_fold(v[2], fold);
    double r = z * z + y * y + x * x;
    double m = rmax(min_r, 1e-40);
    double sqr_min_r = m * m;
    double mul;
    if (r < sqr_min_r) mul = scale / sqr_min_r;
    else if (1.0 < r) mul = scale;
    else mul = scale / r;
    if (ade) v[3] *= mul;
    v[2] = z * mul + j[2];
    v[1] = y * mul + j[1];
    v[0] = x * mul + j[0];
}

// int_pow2_scale (src/formulas.rs:739-751)
static void int_pow2_scale(double scaling, double v[4], const double j[4]) {
    double s = 1.0 / scaling;
    double x = v[0] * s, y = v[1] * s, z = v[2] * s;
    double xx = x * x, yy = y * y;
    double r = xx + yy;
    v[2] = -((std::sqrt(r) * z) * 2.0) * scaling + j[2];
    double a = (r - z * z) / r;
    v[0] = (xx - yy) * a * scaling + j[0];
    v[1] = (x * y * a) * 2.0 * scaling + j[1];
}

// real_power (src/formulas.rs:755-765)
static void real_power(double pw, double z_mul, double v[4], const double j[4], double rout) {
    double x = v[0], y = v[1], z = v[2];
    double theta = std::atan2(y, x) * pw;
    double sin_t = std::sin(theta), cos_t = std::cos(theta);
    double phi = std::atan2(z, std::sqrt(x * x + y * y)) * pw;
    double sin_p = std::sin(phi), cos_p = std::cos(phi);
    double r = std::pow(rout, pw * 0.5);
    v[0] = cos_t * cos_p * r + j[0];
    v[1] = sin_t * cos_p * r + j[1];
    v[2] = sin_p * r * z_mul + j[2];
}

// int_pow (src/formulas.rs:769-857)
static void int_pow(int power, double zmul, double v[4], const double j[4]) {
    double x = v[0], y = v[1], z = v[2];
    const double EPS = 1e-40;
    switch (power) {
        case 2: {
            double yy = y * y, xx = x * x;
            double r = xx + yy;
            v[2] = (std::sqrt(r) * zmul * z) * 2.0 + j[2];
            double a = (r - z * z) / r;
            v[0] = (xx - yy) * a + j[0];
            v[1] = (x * y * a) * 2.0 + j[1];
            break;
        }
        case 3: {
            double sy = y * y, sx = x * x;
            double r = sx + sy;
            double sz = z * z;
            double a = 1.0 - 3.0 * sz / (r + EPS);
            v[0] = (sx - 3.0 * sy) * a * x + j[0];
            v[2] = j[2] - (sz - 3.0 * r) * z * zmul;
            v[1] = a * (3.0 * sx - sy) * y + j[1];
            break;
        }
        case 4: {
            double sy = y * y, sx = x * x;
            double r = sx + sy;
            double sz = z * z;
            double a = 1.0 + sz * (sz - 6.0 * r) / (r * r + EPS);
            v[0] = (sx * (sx - 6.0 * sy) + sy * sy) * a + j[0];
            v[2] = std::sqrt(r) * (r - sz) * z * 4.0 * zmul + j[2];
            v[1] = a * x * (sx - sy) * 4.0 * y + j[1];
            break;
        }
        case 5: {
            double sy = y * y, sx = x * x;
            double r = sx + sy;
            double sz = z * z;
            double a = 1.0 + (sz * sz - sz * r * 2.0) * 5.0 / (r * r + EPS);
            v[1] = (5.0 * sx * sx - sy * (10.0 * sx - sy)) * a * y + j[1];
            v[2] = (sz * (sz - 10.0 * r) + 5.0 * r * r) * z * zmul + j[2];
            v[0] = a * x * (sx * (sx - 10.0 * sy) + 5.0 * sy * sy) + j[0];
            break;
        }
        case 6: {
            double sy = y * y, sx = x * x;
            double r = sx + sy;
            double sz = z * z;
            double rr = r * r;
            double a = 1.0 - sz * (15.0 * rr + sz * (sz - r * 15.0)) / (rr * r + EPS);
            v[1] = (3.0 * sy * sy + sx * (3.0 * sx - 10.0 * sy)) * a * y * x * 2.0 + j[1];
            v[2] = (sz * (3.0 * sz - 10.0 * r) + 3.0 * rr) * std::sqrt(r) * z * zmul * 2.0 + j[2];
            v[0] = (sy * sy * (15.0 * sx - sy) + sx * sx * (sx - 15.0 * sy)) * a + j[0];
            break;
        }
        case 7: {
            double sy = y * y, sx = x * x;
            double r = sx + sy;
            double sz = z * z;
            double rr = r * r;
            double a = 1.0 - 7.0 * (sz * (3.0 * rr + sz * (sz - 5.0 * r))) / (rr * r + EPS);
            v[1] = (sx * (21.0 * sy * sy + sx * (7.0 * sx - 35.0 * sy)) - sy * sy * sy) * a * y + j[1];
            v[2] = j[2] - (sz * sz * sz - 7.0 * r * (rr + sz * (3.0 * sz - 5.0 * r))) * z * zmul;
            v[0] = a * x * (sx * (35.0 * sy * sy + sx * (sx - 21.0 * sy)) - 7.0 * sy * sy * sy) + j[0];
            break;
        }
        default: {
            double xx = x * x, yy = y * y, zz = z * z;
            double r = xx + yy;
            double rr = r * r;
            double zzzz = zz * zz;
            double t = (zzzz - 6.0 * r * zz + rr) * (zz - r) * std::sqrt(r);
            v[2] = -(t * z * 8.0 * zmul) + j[2];
            double num = (rr * 70.0 + zzzz) * zzzz - 28.0 * zz * r * (zzzz + rr);
            double a = num / (rr * rr + EPS) + 1.0;
            double xxxx = xx * xx, yyyy = yy * yy;
            v[1] = (yyyy * (7.0 * xx - yy) + xxxx * (xx - 7.0 * yy)) * 8.0 * x * y * a + j[1];
            v[0] = a * (xxxx * xxxx + yyyy * (70.0 * xxxx + yyyy) - 28.0 * (xx * yy * (yyyy + xxxx))) + j[0];
            break;
        }
    }
}

// The Menger IFS: the published KIFS Menger sponge step (fold by the
// absolute values, sort the components descending, scale about the corner
// (CScale x, y) with the z condition); the reference runs it as machine code
// in MengerIFS_B_2v0.m3f, which is not restated here.  Analytic DE scales w.
static void menger_ifs(const double *o, double v[4], bool ade) {
    double x = std::fabs(v[0]), y = std::fabs(v[1]), z = std::fabs(v[2]);
    double t;
    if (x < y) { t = x; x = y; y = t; }
    if (x < z) { t = x; x = z; z = t; }
    if (y < z) { t = y; y = z; z = t; }
    double s = o[0];
    double s1 = s - 1.0;
    x = s * x - o[1] * s1;
    y = s * y - o[2] * s1;
    z = s * z;
    if (z > 0.5 * o[3] * s1) z -= o[3] * s1;
    if (ade) v[3] *= std::fabs(s);
    v[0] = x;
    v[1] = y;
    v[2] = z;
}

// aexion_c (src/formulas.rs:640-705): a real power bulb step with the angles
// as atan2 (theta from the y axis), then with "rotate C" the constant
// replaced by a power of its own angles.  Options: power, z_mul, rot_c,
// cond_phi, power_c, cz_mul, powc_dist, mode.
static void aexion_c(const double *o, double v[4], double j[4]) {
    const double power = o[0], z_mul = o[1], power_c = o[4], cz_mul = o[5];
    const bool rot_c = o[2] != 0.0, cond_phi = o[3] != 0.0, powc_dist = o[6] != 0.0;
    const int mode = (int)o[7];
    const double x = v[0], y = v[1], z = v[2];
    double r1 = x * x + y * y + z * z;
    const double th = std::atan2(std::sqrt(x * x + z * z), y) * power;
    const double ph = std::atan2(z, x) * power;
    r1 = std::exp(std::log(r1) * power * 0.5);
    const double st = std::sin(th), ct = std::cos(th), sp = std::sin(ph), cp = std::cos(ph);
    v[0] = cp * ct * r1 + j[0];
    v[2] = st * r1 * z_mul + j[2];
    v[1] = ct * sp * r1 + j[1];
    if (!rot_c) return;
    double pd = power_c;
    if (powc_dist) {
        const double d[3] = {v[0] - j[0], v[1] - j[1], v[2] - j[2]};
        pd *= std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    }
    const double r = std::sqrt(j[0] * j[0] + j[1] * j[1] + j[2] * j[2]);
    double a, b, c;
    if (mode & 16) {
        a = v[1] - j[1]; b = v[2] - j[2]; c = v[0] - j[0];
    } else {
        a = j[1]; b = j[2]; c = j[0];
    }
    int ofs = 0, ecx = 8;
    if (mode & 8) {
        std::swap(a, b);
        ecx = 16;
    }
    const double s = std::sqrt(b * b + c * c);
    double tha = (mode & 1) ? std::atan2(a, s) : std::atan2(s, a);
    double pha;
    if (mode & 2) {
        ofs = 24 - ecx;
        pha = std::atan2(c, b);
    } else {
        pha = std::atan2(b, c);
    }
    if (mode & 4) {
        std::swap(tha, pha);
        ofs = ecx;
    }
    if (cond_phi) {
        const double t = ofs == 0 ? v[0] : ofs == 8 ? v[1] : v[2];
        if (!std::signbit(t)) pha = -pha;
    }
    const double sa = std::sin(pha * pd), ca = std::cos(pha * pd), sb = std::sin(tha * pd), cb = std::cos(tha * pd);
    j[0] = ca * cb * r;
    j[2] = sb * r * cz_mul;
    j[1] = cb * sa * r;
}

// Formula::iterate (src/formulas.rs:576-637)
void Formula::iterate(double v[4], double j[4], double rout, bool ade) const {
    switch (kind) {
        case F_INTPOW: int_pow(power(), o[1], v, j); break;
        case F_REALPOWER: real_power(o[0], o[1], v, j, rout); break;
        case F_QUATERNION: {
            const double x = v[0], y = v[1], z = v[2], w = v[3];
            v[0] = x * x - y * y - z * z - w * w + j[0];
            v[1] = 2.0 * (y * x + z * w) + j[1];
            v[2] = 2.0 * (z * x + o[0] * y * w) + j[2];
            v[3] = 2.0 * (w * x + y * z) + o[1] + j[3];
            break;
        }
        case F_TRICORN: {
            double x = v[0], y = v[1], z = v[2];
            v[2] = z * x * o[0] + j[2] * o[1];
            v[0] = x * x - (y * y + z * z) + j[0];
            v[1] = 2.0 * (y * x) + j[1];
            break;
        }
        case F_AMAZINGBOX: amazing_box(o[0], o[1], o[2], v, j, ade); break;
        case F_BULBOX: {
            double scale = o[0], min_r = o[1], fold = o[2], bulb_scale = o[3], rt1o = o[4], rt2o = o[5];
            double rt1 = rt1o * rt1o, rt2 = rt2o * rt2o;
            if (rout < rt1) {
                if (rout < rt2) {
                    int_pow2_scale(bulb_scale, v, j);
                } else {
                    double m = (rout - rt2) / (rt1 - rt2);
                    double xyz_in[3] = {v[0], v[1], v[2]};
                    int_pow2_scale(bulb_scale, v, j);
                    double out[3] = {v[0], v[1], v[2]};
                    v[0] = xyz_in[0]; v[1] = xyz_in[1]; v[2] = xyz_in[2];
                    amazing_box(scale, min_r, fold, v, j, false);
                    double r1 = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                    double m2 = 1.0 - m;
                    double r2 = r1 * m + m2 * std::sqrt(out[0] * out[0] + out[1] * out[1] + out[2] * out[2]);
                    v[0] = v[0] * m + m2 * out[0];
                    v[1] = v[1] * m + m2 * out[1];
                    v[2] = v[2] * m + m2 * out[2];
                    double r1b = r2 / std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + 1e-40);
                    v[0] *= r1b; v[1] *= r1b; v[2] *= r1b;
                }
            } else {
                amazing_box(scale, min_r, fold, v, j, false);
            }
            break;
        }
        case F_FOLDINGINTPOW:
            for (int k = 0; k < 3; k++) v[k] = box_fold(v[k], o[2]);
            int_pow(power(), o[1], v, j);
            break;
        case F_MENGER: menger_ifs(o, v, ade); break;
        case F_AEXIONC: aexion_c(o, v, j); break;
        default: break;
    }
}

bool formula_from_slot(const mb3d_cu_slot &s, Formula &f, std::string &err) {
    switch (s.formula) {
        case F_INTPOW: case F_REALPOWER: case F_QUATERNION: case F_TRICORN: case F_AMAZINGBOX: case F_BULBOX:
        case F_FOLDINGINTPOW: case F_AEXIONC: case F_MENGER:
            f.kind = s.formula;
            for (int k = 0; k < 16; k++) f.o[k] = s.options[k];
            return true;
        default:
            err = "formula #" + std::to_string(s.formula) + " is not supported";
            return false;
    }
}

// ---------------------------------------------------------------------------
// CheckFormulaOptions (combine_de_options_range, src/calc.rs:311-372): the
// DE option of slots start..end_to
static int combine_de_options(const std::vector<Slot> &slots, int end_to, int start = 0) {
    int de_option = -1;
    for (int x = start; x <= end_to && x < (int)slots.size(); x++) {
        const Slot &s = slots[x];
        if (s.iterations == 0) continue;
        int de = s.f.de_option();
        if (de < 0 || de == de_option) continue;
        switch (de_option) {
            case -1: case 21: case 22: de_option = de; break;
            case 2: de_option = (de == 2 || de == 5 || de == 6 || de == 11) ? 2 : 0; break;
            case 4: de_option = (de == 5 || de == 6) ? 4 : 0; break;
            case 5:
                if (de == 4) de_option = 4;
                else if (de == 2 || de == 11) de_option = 2;
                else if (de != 6) de_option = 0;
                else de_option = 5;
                break;
            case 6: de_option = (de == 2 || de == 4 || de == 5 || de == 11) ? de : 0; break;
            case 11:
                if (de == 2 || de == 5) de_option = 2;
                else if (de != 6) de_option = 0;
                else de_option = 11;
                break;
            default: break;
        }
    }
    return de_option;
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
                double s = 0.0;
                for (int q = 0; q < 4; q++) s += a[i][q] * b[q][k];
                r[i][k] = s;
            }
    };
    double m[4][4], m2[4][4], m3[4][4], t[4][4];
    ini(m);
    m[0][0] = std::cos(xw); m[3][3] = std::cos(xw); m[0][3] = -std::sin(xw); m[3][0] = std::sin(xw);
    ini(m2);
    m2[1][1] = std::cos(yw); m2[3][3] = std::cos(yw); m2[1][3] = -std::sin(yw); m2[3][1] = std::sin(yw);
    mul(m2, m, t);
    ini(m3);
    m3[2][2] = std::cos(zw); m3[3][3] = std::cos(zw); m3[2][3] = -std::sin(zw); m3[3][2] = std::sin(zw);
    mul(m3, t, out);
    for (int i = 0; i < 4; i++)
        for (int k = 0; k < 4; k++) out[i][k] = (double)(float)out[i][k];
}

// ipol_de_option (src/calc.rs:255-308): CheckDEoption of the two weighted
// formulas (a weight counts when its bits as a signed integer are > 0)
static int ipol_de_option(const std::vector<Slot> &slots, const float raw[2]) {
    int de_option = -1;
    for (int x = 0; x < 2 && x < (int)slots.size(); x++) {
        int32_t bits;
        std::memcpy(&bits, &raw[x], 4);
        if (bits <= 0) continue;
        const int de = slots[x].f.de_option();
        if (de < 0 || de > 20 || de == de_option) continue;
        if ((de_option >= 0 && de_option < 20 && de > 19) || (de_option > 19 && de >= 0 && de < 20)) return -1;
        switch (de_option) {
            case -1: de_option = de; break;
            case 2: if (!(de == 2 || de == 5 || de == 6 || de == 11)) de_option = 0; break;
            case 4: if (!(de == 5 || de == 6)) de_option = 0; break;
            case 5:
                if (de == 4) de_option = 4;
                else if (de == 2 || de == 11) de_option = 2;
                else if (de != 6) de_option = 0;
                else de_option = 5;
                break;
            case 6: de_option = (de == 2 || de == 4 || de == 5 || de == 11) ? de : 0; break;
            case 11:
                if (de == 2 || de == 5) de_option = 2;
                else if (de != 6) de_option = 0;
                else de_option = 11;
                break;
            default: break;
        }
    }
    if (de_option > 19) de_option = 20;
    return de_option;
}

// CalcParams::new (src/calc.rs:375-891), the alternating 3D hybrid without
// DE combination, interpolation, dIFS, cutting planes, inside rendering,
// stereo or the ground.
bool make_params(const mb3d_cu_scene &sc, Params &p, std::string &err) {
    p = Params();
    if (sc.width <= 0 || sc.height <= 0) { err = "bad picture size"; return false; }
    int n = sc.n_slots;
    if (n < 1 || n > 6) { err = "n_slots must be 1..6"; return false; }
    // an interpolation hybrid: the two first formulas with their weights,
    // normalised to a sum of 1 (src/calc.rs:378-397)
    const bool ipol = sc.interpolation != 0;
    float ipw[2] = {1.f, 0.f};
    if (ipol) {
        if (n < 2) { err = "an interpolation hybrid needs two formulas"; return false; }
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
        n = 2;
    }
    bool any = ipol;
    for (int i = 0; i < n; i++) any = any || sc.slots[i].iterations != 0;
    if (!any) { err = "no formula with iterations > 0"; return false; }
    std::vector<Slot> slots;
    for (int i = 0; i < n; i++) {
        Slot s;
        if (sc.slots[i].iterations != 0 || ipol) {
            if (!formula_from_slot(sc.slots[i], s.f, err)) return false;
        } else {
            s.f.kind = F_INTPOW;  // an empty slot (src/m3p.rs:790-792)
            s.f.o[0] = 8; s.f.o[1] = -1;
        }
        s.iterations = ipol ? 1 : std::abs(sc.slots[i].iterations);
        s.uncounted = !ipol && sc.slots[i].iterations < 0;
        s.ade = false;
        s.julia_add = sc.julia && s.f.julia_adds();
        slots.push_back(s);
    }
    int last = (int)slots.size() - 1;
    while (last > 0 && slots[last].iterations == 0) last--;
    slots.resize(last + 1);
    // a DE combination (src/calc.rs:421-431): slots 0-based, clamped to 0..5
    // as the scene text's are; none in an interpolation hybrid
    if (sc.decomb < 0 || sc.decomb > 6) { err = "decomb must be 0..6"; return false; }
    auto slot_of = [](int v) { return std::min(std::max(v, 0), 5); };
    const bool dc = !ipol && sc.decomb != 0 && slot_of(sc.decomb_end1) < last && slot_of(sc.decomb_start2) <= last;
    int end_to = dc ? std::min(slot_of(sc.decomb_end1), last) : last;
    int repeat_from = std::min(std::max(sc.repeat_from, 0), end_to);
    while (repeat_from > 0 && slots[repeat_from].iterations <= 0) repeat_from--;
    int de_option = combine_de_options(slots, end_to);
    if (sc.disable_analytic_de) {
        if (de_option == 2 || de_option == 11) de_option = 0;
        else if (de_option == 5 || de_option == 6) de_option = 4;
    }
    if (de_option < 0 && !ipol) { err = "formula option is not valid"; return false; }
    if (ipol) {
        de_option = ipol_de_option(slots, sc.ipol_weights);
        if (de_option >= 20) { err = "dIFS formulas do not work in an interpolation hybrid"; return false; }
        if (de_option < 0) { err = "formula option is not valid"; return false; }
    }
    // a 4D hybrid (HybridMode::Alt4D): with the 4D numerical DE (option 4);
    // the analytic 4D DE (options 5, 6) is not restated
    const bool four_d = de_option >= 4 && de_option <= 6;
    if (four_d && de_option != 4) { err = "4D hybrids with the analytic DE are not supported"; return false; }

    bool is_custom_de = de_option == 2 || de_option == 5 || de_option == 6 || de_option == 11 || de_option == 20;
    // the second part of a DE combination (src/calc.rs:491-520); no formula
    // of this restatement is a dIFS one
    int start2 = 0, end2 = 0, rep2 = 0, de2 = -1;
    if (dc) {
        start2 = std::min(slot_of(sc.decomb_start2), last);
        end2 = std::min(std::max(slot_of(sc.decomb_end2), start2), last);
        de2 = combine_de_options(slots, end2, start2);
        if (sc.disable_analytic_de) {
            if (de2 == 2 || de2 == 11) de2 = 0;
            else if (de2 == 5 || de2 == 6) de2 = 4;
        }
        if (de2 < 0) { err = "DE combination: the second formula part has no valid DE option"; return false; }
        if (sc.decomb == 6 && de2 != 20) { err = "DE combination 'mix': the second hybrid part must be dIFS"; return false; }
        if (four_d || (de2 >= 4 && de2 <= 6)) { err = "4D hybrids in a DE combination are not restated"; return false; }
        rep2 = std::min(std::max(slot_of(sc.decomb_repeat2), start2), end2);
        while (rep2 > start2 && slots[rep2].iterations <= 0) rep2--;
    }
    const bool is_custom_de2 = dc && (de2 == 2 || de2 == 5 || de2 == 6 || de2 == 11 || de2 == 20);
    for (size_t x = 0; x < slots.size(); x++) {
        Slot &s = slots[x];
        s.ade = (dc && (int)x > end_to) ? is_custom_de2 : is_custom_de;
        int de = s.f.de_option();
        s.uncounted = s.uncounted || de < 0 || de > 20;
    }
    int max_it = sc.iterations;
    float fhln[6];
    for (int k = 0; k < 6; k++) fhln[k] = (float)(1.0 / std::log(2.0));
    double nn = 0, x1 = 0, y1 = 0, ii = 0;
    bool have_p1 = false;
    double p1_scale = 1.0;  // part 1's d_de_scale in a DE combination
    for (size_t x = 0; x < slots.size(); x++) {
        const Slot &s = slots[x];
        if (s.iterations == 0) continue;
        const bool second = dc && (int)x > end_to;
        if (second && !have_p1) {
            p1_scale = (nn > 0.0 && de_option != 20) ? x1 / nn : 1.0;
            have_p1 = true;
            nn = x1 = y1 = ii = 0.0;
        }
        const bool is_custom_de_x = second ? is_custom_de2 : is_custom_de;
        if (ipol || !s.uncounted) {
            double sip = s.f.si_pow();
            double z1 = sip > 1.0 ? sip : s.f.first_option();
            fhln[x] = (float)(1.0 / std::log(rmax(2.0, std::fabs(z1))));
        }
        // (an interpolation hybrid: weighted by the weights, counted once)
        double z1 = ipol ? (double)ipw[x] : (double)s.iterations, cnt = ipol ? 1.0 : (double)s.iterations;
        int j = s.f.de_option();
        if (is_custom_de_x && (ipol || !s.uncounted) && (j == 5 || j == 11)) {
            nn += cnt;
            ii += cnt;
            double x2 = s.f.first_option();
            if (x2 == 0.0) x2 = 1e-40;
            if (x2 < 0.0) x1 += 0.65 * z1;
            else x1 += (x2 * 1.2 + 1.0) / x2 * z1;
            y1 += std::fabs(x2) * z1;
        } else if (j >= 0 || ipol) {
            nn += cnt;
            x1 += (is_custom_de_x ? s.f.ade_scale() : s.f.de_scale()) * z1;
        }
    }
    float d_col_plus = 0.f;
    double d_de_scale = 1.0, d_de_scale2 = 1.0;
    if (have_p1) {
        d_de_scale = p1_scale;
        if (nn > 0.0 && de2 != 20) d_de_scale2 = x1 / nn;
    } else if (nn > 0.0 && de_option != 20) {
        d_de_scale = ipol ? x1 : x1 / nn;
    }
    if (nn > 0.0 && ii > 0.0) d_col_plus = (float)(std::pow(std::fabs(y1 / ii), 0.25) * 40.0 - 49.0);
    // mctColVarDEstopMul (src/calc.rs:591-652)
    float col_var = 0.6f;
    {
        double yy1 = 0, z1 = 0, z2 = 0;
        int ia = 0, itmp = 0;
        bool second = false;
        for (size_t x = 0; x < slots.size(); x++) {
            const Slot &s = slots[x];
            bool counted = ipol || (s.iterations > 0 && !s.uncounted);
            if (!counted) {
                if (!ipol && s.iterations > 0) {
                    if ((int)x > end_to) ia++;
                    else itmp++;
                }
                continue;
            }
            if ((int)x > end_to && !second) {
                second = true;
                col_var = z1 > 0.0 ? (float)(yy1 / z1) : 0.6f;
                z2 = z1;
                z1 = 0.0;
                yy1 = 0.0;
                if (!dc || de2 == 20) break;
            }
            double x2 = ipol ? (double)ipw[x] : (double)s.iterations;
            int de = s.f.de_option();
            if (de == 0 || de == 4) {
                yy1 += x2 * 0.6;
                z1 += x2;
            } else if ((de >= 1 && de <= 3) || (de >= 5 && de <= 40)) {
                if (s.f.first_option_double()) {
                    double v = s.f.first_option();
                    if (v > 1.0) {
                        if (v < 1.2) v = 1.1 + (v - 1.0) * (v - 1.0) * 2.5;
                        yy1 += x2 * 0.5 / (std::log(v) + 0.03);
                        z1 += x2;
                    } else if (v < -1.0) {
                        if (v > -1.2) v = -1.1 - (v + 1.0) * (v + 1.0) * 2.5;
                        yy1 += x2 * 0.5 / (std::log(-v) + 0.03);
                        z1 += x2;
                    }
                }
            }
        }
        if ((z1 >= z2 && z1 > 1e-3) || (ia > itmp && std::fabs(z1 - z2) < 1e-3 && z1 > 1e-3)) col_var = (float)(yy1 / z1);
        else if (z2 < 1e-3) col_var = 0.6f;
    }
    // effective_rstop (src/scene.rs:799-808)
    double rstop = sc.rstop;
    if (!(rstop > 0.0)) {
        rstop = 0.0;
        for (int i = 0; i < n; i++)
            if (sc.slots[i].iterations > 0) rstop = rmax(rstop, slots.size() > (size_t)i ? slots[i].f.default_rstop() : 16.0);
        rstop = rmax(rstop, 1.0001);
    }
    double width = sc.width, height = sc.height;
    double step_width = 2.1345 / (sc.zoom * width);
    double fov_y = to_radians(sc.fov_y);
    float z_step_div0 = (float)rmax(sc.z_step_div, 0.0001);
    float de_stop = (float)rmax(sc.de_stop, 0.001);
    double x1c = rclamp(fov_y * 0.5, 0.01, 1.5);
    float pl_optic_z = (float)(std::cos(x1c) * x1c / std::sin(x1c));
    float fovx_off = 0.5f * (float)sc.width;
    float fovx_mul = (float)(fov_y / height);
    double zcorr = std::sin(rmax(to_radians(sc.fov_y), 1.0) / height);
    double zc_mul = 32767.0 * 256.0 / (std::sqrt((sc.z_end - sc.z_start) * zcorr / step_width + 1.0) - 0.999999999);
    double zend = rmax(1e-10, (sc.z_end - sc.z_start) / step_width);
    float mh04zsd = (float)((double)std::max(sc.width, sc.height) * 0.5 * std::sqrt((double)z_step_div0 + 0.001) *
                            rmax(0.01, sc.raystep_limiter));
    float de_stop_factor = 0.f;
    if (sc.vary_de_stop_on_fov) {
        double ze = rmax(1e-16, (sc.z_end - sc.z_start) / step_width);
        double xx1 = 0.01 * height / (std::sin(0.01) * rmax(1.0 / 65535.0, to_radians(sc.fov_y)));
        double xx2 = step_width * (xx1 + ze) / xx1;
        de_stop_factor = (float)((xx2 - step_width) / (step_width * rmax(1e-6, ze)));
    }
    double xh = width * 0.5, yh = height * 0.5;
    double z1 = (sc.z_start - sc.mid[2]) / step_width;
    Mat3 vg;
    normalise_matrix_to(step_width, sc.vgrads, vg);
    for (int k = 0; k < 3; k++) p.ystart[k] = sc.mid[k] + z1 * vg[2][k] - yh * vg[1][k] - xh * vg[0][k];
    float de_offset = rminf(de_stop * 0.1f, 0.004f);
    float dds = is_custom_de ? (float)((double)(float)d_de_scale / step_width) : (float)d_de_scale * de_offset;
    float dds2 = is_custom_de2 ? (float)((double)(float)d_de_scale2 / step_width) : (float)d_de_scale2 * de_offset;
    float de_offset006 = de_offset * 0.06f;
    de_offset = (float)((double)de_offset * step_width);
    float z_step_div = z_step_div0, ms_de_sub = 0.f;
    if (sc.step_sub_de_stop) {
        float s = z_step_div0;
        s = s * s + (1.2f * s) * (1.0f - s);
        z_step_div = s;
        ms_de_sub = rminf(std::sqrt(s), 0.9f);
    }
    float ln_rstop = (float)std::log(std::log(rstop));
    double d_rstop = (double)(float)(rstop * rstop);
    double rstop3d = (double)(float)((d_rstop * d_rstop) * 64.0);
    // the iterations of both parts of a DE combination (iMaxitF2)
    const int iterations2 = sc.decomb_iterations2 > 0 ? sc.decomb_iterations2 : sc.iterations;
    int its = !dc ? max_it : sc.decomb > 5 ? max_it + iterations2 : std::max(max_it, iterations2);
    float mcts_m = 32767.0f / (float)std::max(its + 1, 1);
    d_col_plus = d_col_plus + (float)its * 0.1f;

    p.slots = slots;
    p.color_on_it = sc.color_on_it;
    p.is_custom_de = is_custom_de;
    p.de_option = de_option;
    p.d_de_scale = dds;
    p.sm_normals = std::min(8, std::max(0, sc.smooth_normals));
    p.de_stop = de_stop;
    p.z_step_div = z_step_div;
    p.de_add_steps = sc.bin_search_steps;
    p.width = sc.width;
    p.height = sc.height;
    p.fov_y = fov_y;
    p.max_it = max_it;
    p.min_it = std::min(sc.min_iterations, max_it);
    p.color_option = std::min(sc.color_option, 5);
    p.mct_color_mul = (float)(sc.color_mul * 512.0);
    p.d_rstop = d_rstop;
    p.rstop3d = rstop3d;
    p.do_julia = sc.julia != 0;
    for (int k = 0; k < 4; k++) p.ju[k] = sc.julia_c[k];
    std::memcpy(p.vgrads, vg, sizeof(vg));
    p.pl_optic_z = pl_optic_z;
    p.dfog_on_it = sc.dfog_on_it;
    p.fovx_off = fovx_off;
    p.fovx_mul = fovx_mul;
    p.d_col_plus = d_col_plus;
    p.zcorr = zcorr;
    p.zc_mul = zc_mul;
    p.zend = zend;
    p.step_width = step_width;
    p.col_var_de_stop_mul = col_var;
    p.first_step_random = sc.first_step_random != 0;
    p.mh04zsd = mh04zsd;
    p.de_stop_factor = de_stop_factor;
    p.ln_rstop = ln_rstop;
    p.normals_on_de = sc.normals_on_de || is_custom_de || dc;
    p.de_offset = de_offset;
    p.de_offset006 = de_offset006;
    p.mcts_m = mcts_m;
    p.ms_de_sub = ms_de_sub;
    for (int k = 0; k < 6; k++) p.fhln[k] = fhln[k];
    p.end_to = end_to;
    p.repeat_from = repeat_from;
    p.ipol = ipol;
    p.ipol_w[0] = ipw[0];
    p.ipol_w[1] = ipw[1];
    p.four_d = four_d;
    build_smatrix4(sc.rot_4d[0], sc.rot_4d[1], sc.rot_4d[2], p.smatrix4);
    // the DeComb (src/calc.rs:730-760) and its part 2's place: the rotation
    // (build_rot_matrix, src/math.rs:466-475) with rows 1 / scale long; a
    // placement of all defaults (part2_scale 0 reads as 1) is none
    p.dc_kind = dc ? sc.decomb : 0;
    if (dc) {
        DeCombPart &q = p.dc_part2;
        q.start = start2;
        q.end = end2;
        q.repeat = rep2;
        q.de_option = de2;
        q.is_custom_de = is_custom_de2;
        q.d_de_scale = dds2;
        q.max_it = std::max(iterations2, 1);
        p.dc_smooth = (double)rmaxf(sc.decomb_smooth, 1e-30f) / step_width;
        const double scale = sc.part2_scale > 0.0 ? sc.part2_scale : 1.0;
        const double *o = sc.part2_offset, *r = sc.part2_rotation;
        const bool placed = o[0] != 0.0 || o[1] != 0.0 || o[2] != 0.0 || r[0] != 0.0 || r[1] != 0.0 || r[2] != 0.0 ||
                            scale != 1.0;
        p.dc_place = placed && sc.decomb != 6;
        if (p.dc_place) {
            double sx = std::sin(to_radians(r[0])), cx = std::cos(to_radians(r[0]));
            double sy = std::sin(to_radians(r[1])), cy = std::cos(to_radians(r[1]));
            double sz = std::sin(to_radians(r[2])), cz = std::cos(to_radians(r[2]));
            Mat3 m = {{cy * cz, -cy * sz, sy},
                      {sx * sy * cz + cx * sz, cx * cz - sx * sy * sz, -sx * cy},
                      {sx * sz - cx * sy * cz, cx * sy * sz + sx * cz, cx * cy}};
            normalise_matrix_to(1.0 / rmax(scale, 1e-300), m, p.dc_m);
            for (int k = 0; k < 3; k++) p.dc_offset[k] = o[k];
            p.dc_scale = scale;
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// the hybrid loops (src/iteration.rs)

// CalcSmoothIterations (src/iteration.rs:140-152)
void Iteration::smooth_iterations(int n) {
    if (rout <= 1.0) {
        smooth_it = (float)it_result;
    } else if (rold < 1.0) {
        double d = std::log(std::log(rout) * 0.5) * (double)fhln[n];
        smooth_it = (float)((double)it_result + (double)ln_rstop - d);
    } else {
        double d = std::log(0.5 * std::log(rout));
        double e = d - std::log(0.5 * std::log(rold));
        smooth_it = (float)(((double)ln_rstop - d) / (e + 1e-100) + (double)it_result);
    }
}

// run_with (src/iteration.rs:268-313)
int Iteration::run(const std::vector<Slot> &slots) {
    int n = start_from;
    int btmp = std::max(slots[n].iterations, 0);
    it_result = 0;
    uint32_t uncounted_guard = 0;
    for (;;) {
        rold = rout;
        int guard = 0;
        while (btmp <= 0) {
            n += 1;
            if (n > end_to) n = repeat_from;
            btmp = std::max(slots[n].iterations, 0);
            guard++;
            if (guard > 64) return n;
        }
        const Slot &slot = slots[n];
        slot.f.iterate(v, j, rout, slot.ade);
        if (slot.julia_add) {
            for (int k = 0; k < 3; k++) v[k] += j[k];
        }
        btmp -= 1;
        if (slot.uncounted) {
            uncounted_guard++;
            if (uncounted_guard > 100000) return n;
            continue;
        }
        it_result += 1;
        double x = v[0], y = v[1], z = v[2], w = v[3];
        rout = four_d ? x * x + y * y + z * z + w * w : x * x + y * y + z * z;
        if (rout < otrap) otrap = rout;
        if (it_result >= max_it || rout > rstop) return n;
    }
}

// run_ipol (src/iteration.rs:347-401), 3D: both formulas on the same
// vector, the results and their lengths blended with the weights; `de`
// blends the running derivative (w) of the analytic-DE variant
void Iteration::run_ipol(const std::vector<Slot> &slots, bool de) {
    const bool fd = four_d;  // (doInterpolHybridPas4D: lengths and the blend's scale on four components)
    const double s1 = (double)ipol_w[0], s2 = (double)ipol_w[1];
    it_result = 0;
    for (;;) {
        rold = rout;
        const double y1[4] = {v[0], v[1], v[2], v[3]};
        slots[0].f.iterate(v, j, rout, slots[0].ade);
        if (slots[0].julia_add)
            for (int k = 0; k < 3; k++) v[k] += j[k];
        const double x1[4] = {v[0], v[1], v[2], v[3]};
        for (int k = 0; k < 4; k++) v[k] = y1[k];
        slots[1].f.iterate(v, j, rout, slots[1].ade);
        if (slots[1].julia_add)
            for (int k = 0; k < 3; k++) v[k] += j[k];
        const double x = v[0], y = v[1], z = v[2], w = v[3];
        double xx, yy0;
        if (fd) {
            xx = std::sqrt(x1[0] * x1[0] + x1[1] * x1[1] + x1[2] * x1[2] + x1[3] * x1[3]);
            yy0 = std::sqrt(x * x + y * y + z * z + w * w);
        } else {
            xx = std::sqrt(x1[0] * x1[0] + x1[1] * x1[1] + x1[2] * x1[2]);
            yy0 = std::sqrt(x * x + y * y + z * z);
        }
        xx = xx * s1 + yy0 * s2;
        double nv[4] = {x1[0] * s1 + x * s2, x1[1] * s1 + y * s2, x1[2] * s1 + z * s2, x1[3] * s1 + w * s2};
        if (de && !fd) nv[3] = std::fabs(x1[3]) * s1 + std::fabs(w) * s2;
        const double l2 = fd ? nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2] + nv[3] * nv[3]
                             : nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2];
        const double yy = xx / std::sqrt(l2 + 1e-40);
        nv[0] *= yy;
        nv[1] *= yy;
        nv[2] *= yy;
        if (fd) nv[3] *= yy;
        for (int k = 0; k < 4; k++) v[k] = nv[k];
        it_result += 1;
        rout = xx * xx;
        if (rout < otrap) otrap = rout;
        if (it_result >= max_it || rout > rstop) break;
    }
}

// doHybrid4DPas (src/iteration.rs:757-772): the 3D point turned into 4D
// (Rotate4Dex, src/math.rs:209-215), the hybrid on four components
void Iteration::hybrid_4d(const std::vector<Slot> &slots) {
    double v4[4];
    for (int i = 0; i < 4; i++) v4[i] = c[0] * smatrix4[i][0] + c[1] * smatrix4[i][1] + c[2] * smatrix4[i][2];
    for (int k = 0; k < 4; k++) {
        v[k] = v4[k];
        j[k] = do_julia ? ju[k] : v4[k];
    }
    rout = v4[0] * v4[0] + v4[1] * v4[1] + v4[2] * v4[2] + v4[3] * v4[3];
    otrap = rout;
    if (ipol) {  // doInterpolHybridPas4D (src/iteration.rs:457-464)
        run_ipol(slots, false);
        if (calc_sit) smooth_iterations(0);
        return;
    }
    int n = run(slots);
    if (calc_sit) smooth_iterations(n);
}

// doHybridPas (src/iteration.rs:521-535); an interpolation hybrid:
// doInterpolHybridPas (src/iteration.rs:403-439); a 4D hybrid: hybrid_4d
void Iteration::hybrid_3d(const std::vector<Slot> &slots) {
    if (four_d) {
        hybrid_4d(slots);
        return;
    }
    if (do_julia) { j[0] = ju[0]; j[1] = ju[1]; j[2] = ju[2]; }
    else { j[0] = c[0]; j[1] = c[1]; j[2] = c[2]; }
    v[0] = c[0]; v[1] = c[1]; v[2] = c[2]; v[3] = 0.0;
    rout = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
    otrap = rout;
    if (ipol) {
        run_ipol(slots, false);
        if (calc_sit) smooth_iterations(0);
        return;
    }
    int n = run(slots);
    if (calc_sit) smooth_iterations(n);
}

// doHybridPasDE (src/iteration.rs:539-574); an interpolation hybrid:
// doInterpolHybridPasDE (src/iteration.rs:441-455)
double Iteration::hybrid_3d_de(const std::vector<Slot> &slots) {
    if (ipol) {
        if (do_julia) { j[0] = ju[0]; j[1] = ju[1]; j[2] = ju[2]; }
        else { j[0] = c[0]; j[1] = c[1]; j[2] = c[2]; }
        v[0] = c[0]; v[1] = c[1]; v[2] = c[2];
        rout = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
        otrap = rout;
        v[3] = (de_option & 0x18) == 16 ? rout : 1.0;
        run_ipol(slots, true);
        const double w = v[3];
        const double r = (de_option & 7) == 4 ? std::fabs(v[2]) * std::log(std::fabs(v[2])) / w : std::sqrt(rout) / std::fabs(w);
        if (calc_sit) smooth_iterations(0);
        return r;
    }
    if (do_julia) { j[0] = ju[0]; j[1] = ju[1]; j[2] = ju[2]; }
    else { j[0] = c[0]; j[1] = c[1]; j[2] = c[2]; }
    v[0] = c[0]; v[1] = c[1]; v[2] = c[2];
    rout = c[0] * c[0] + c[1] * c[1] + c[2] * c[2];
    otrap = rout;
    if ((de_option & 0x38) == 16) v[3] = rout;
    else v[3] = 1.0;
    int n = run(slots);
    double w = v[3];
    double result;
    if ((de_option & 7) == 4) result = std::fabs(v[1]) * std::log(std::fabs(v[1])) / w;
    else result = std::sqrt(rout) / std::fabs(w);
    if (calc_sit) smooth_iterations(n);
    return result;
}

// ---------------------------------------------------------------------------
// the marcher

// pixel_seed (src/calc.rs:1125-1140)
int32_t pixel_seed(int64_t y, int64_t x) {
    uint32_t row = (uint32_t)(int32_t)((int64_t)0x24563487u + (y + 1) * (int64_t)0x324594A1);
    uint32_t a = 214013u, c = 2531011u, ra = 1u, rc = 0u;
    uint64_t n = (uint64_t)std::max<int64_t>(x, 0);
    while (n > 0) {
        if (n & 1) {
            rc = rc * a + c;
            ra = ra * a;
        }
        c = c * a + c;
        a = a * a;
        n >>= 1;
    }
    return (int32_t)(ra * row + rc);
}

Marcher::Marcher(const Params *pp, int32_t s) : p(pp), seed(s) {
    it.j[0] = p->ju[0]; it.j[1] = p->ju[1]; it.j[2] = p->ju[2]; it.j[3] = p->ju[3];
    for (int k = 0; k < 4; k++) it.ju[k] = p->ju[k];
    it.do_julia = p->do_julia;
    it.max_it = p->max_it;
    it.rstop = p->d_rstop;
    it.ln_rstop = p->ln_rstop;
    it.de_option = p->de_option;
    it.end_to = p->end_to;
    it.repeat_from = p->repeat_from;
    for (int k = 0; k < 6; k++) it.fhln[k] = p->fhln[k];
    it.ipol = p->ipol;
    it.ipol_w[0] = p->ipol_w[0];
    it.ipol_w[1] = p->ipol_w[1];
    it.four_d = p->four_d;
    std::memcpy(it.smatrix4, p->smatrix4, sizeof(it.smatrix4));
    ms_de_stop = p->de_stop;
    max_its_result = p->max_it;
}

// set_part (src/calc.rs:1476-1489): the slot range, iteration limit and DE
// option the iteration runs with
void Marcher::set_part(int start, int end, int repeat, int max_it, int de_option) {
    it.start_from = start;
    it.end_to = end;
    it.repeat_from = repeat;
    it.max_it = max_it;
    it.de_option = de_option;
}

// calc_de -> calc_de_fractal (src/calc.rs:1333-1455), outside rendering: one
// hybrid part, or a DE combination of two (CalcDEfull with FormulaType > 0)
double Marcher::calc_de() {
    if (count_de) g_de_evals.fetch_add(1, std::memory_order_relaxed);
    if (p->dc_kind == 0) return calc_de_part(p->is_custom_de, p->d_de_scale, false);
    const DeCombPart &q = p->dc_part2;
    double result = calc_de_part(p->is_custom_de, p->d_de_scale, false);
    // PrepareF1DEcomb
    const int b_it = it.it_result, b_max = max_its_result;
    const double b_otrap = it.otrap;
    const float b_sit = it.smooth_it;
    set_part(q.start, q.end, q.repeat, q.max_it, q.de_option);
    // the second part in its own place
    const Vec3 c0 = {it.c[0], it.c[1], it.c[2]};
    if (p->dc_place) {
        const double d[3] = {c0[0] - p->dc_offset[0], c0[1] - p->dc_offset[1], c0[2] - p->dc_offset[2]};
        for (int i = 0; i < 3; i++) it.c[i] = p->dc_m[i][0] * d[0] + p->dc_m[i][1] * d[1] + p->dc_m[i][2] * d[2];
    }
    double rst = calc_de_part(q.is_custom_de, q.d_de_scale, p->dc_kind == 3);
    if (p->dc_place) {
        rst *= p->dc_scale;
        for (int i = 0; i < 3; i++) it.c[i] = c0[i];
    }
    const double ms = (double)ms_de_stop;
    auto restore1 = [&]() {
        it.it_result = b_it;
        it.smooth_it = b_sit;
        it.otrap = b_otrap;
        max_its_result = b_max;
    };
    switch (p->dc_kind) {
        case 1:
            if (rst >= result) restore1();
            else result = rst;
            break;
        case 2:
        case 3:
            if (rst > result) result = rst;
            else restore1();
            break;
        default: {  // 4, 5: the smooth minima, colour values blended by distance
            if (!(rst < result)) {
                it.it_result = b_it;
                max_its_result = b_max;
            }
            const double sm = p->dc_smooth;
            if (p->dc_kind == 4) {
                result = std::fmin(rst - std::fmax(sm - result, 0.0), result - std::fmax(sm - rst, 0.0));
            } else {
                const double rd1 = std::fmax(sm - result - ms, 0.0);
                const double d2 = std::fmax(sm - rst - ms, 0.0);
                result = std::fmin(rst - rd1 * (sm - d2) / sm, result - d2 * (sm - rd1) / sm);
            }
            const double r2 = std::fabs(rst), w = std::fabs(result);
            const double f = 1.0 / (w + r2 + 1e-10);
            it.smooth_it = (float)(((double)it.smooth_it * w + (double)b_sit * r2) * f);
            it.otrap = (it.otrap * w + b_otrap * r2) * f;
            break;
        }
    }
    // RestoreF1DEcomb
    set_part(0, p->end_to, p->repeat_from, p->max_it, p->de_option);
    return result;
}

// calc_de_part (src/calc.rs:1495-1557) of the part the iteration is set to:
// the analytic DE or the numerical one; `invert` calculates the part as
// "inside" (the inverted max combination)
double Marcher::calc_de_part(bool is_custom_de, float d_de_scale, bool invert) {
    double result;
    if (is_custom_de) {
        result = it.hybrid_3d_de(p->slots) * (double)d_de_scale;
    } else {
        it.hybrid_3d(p->slots);
        if (it.rout < 1e-200) {
            result = 0.0;
        } else {
            bool buf_sit = it.calc_sit;
            int buf_max_it = it.max_it;
            double buf_rout = it.rout;
            it.calc_sit = false;
            it.max_it = it.it_result;
            it.rstop = p->rstop3d;
            double off = (double)p->de_offset;
            double g[3];
            for (int k = 0; k < 3; k++) {
                double bufd = it.c[k];
                it.c[k] = bufd + off;
                it.hybrid_3d(p->slots);
                g[k] = (buf_rout - it.rout) * (buf_rout - it.rout);
                it.c[k] = bufd;
            }
            result = buf_rout * std::log(buf_rout) * (double)d_de_scale /
                     (std::sqrt(g[0] + g[1] + g[2]) + (double)p->de_offset006);
            it.rout = buf_rout;
            it.it_result = it.max_it;
            it.max_it = buf_max_it;
            it.calc_sit = buf_sit;
            it.rstop = p->d_rstop;
        }
    }
    max_its_result = it.max_it;
    double mn = (double)ms_de_stop * 0.25;
    if (result < mn || std::isnan(result)) result = mn;
    if (invert) {
        result = (double)ms_de_stop * 4.0 - result * 3.0;
        if (result >= (double)ms_de_stop) it.it_result -= 1;
    }
    return result;
}

// RMCalculateVgradsFOV (src/calc.rs:1561-1573), the common camera
void Marcher::calc_vgrads_fov(int ix) {
    double cafx = (double)((p->fovx_off - (float)ix) * p->fovx_mul);
    double v[3];
    build_view_vector_dfov(cafy, cafx, v);
    rotate_vector_reverse(v, p->vgrads, vfov);
}

// RMCalculateStartPos (src/calc.rs:1673-1689)
void Marcher::calc_start_pos(int ix, int iy) {
    double x = ix, y = iy;
    for (int k = 0; k < 3; k++) it.c[k] = p->ystart[k] + p->vgrads[0][k] * x + p->vgrads[1][k] * y;
}

void Marcher::step(double d) { add_weight(it.c, vfov, d); }

// update_de_stop (src/calc.rs:1698-1701)
void Marcher::update_de_stop() { ms_de_stop = (float)((double)p->de_stop * (1.0 + mzz * (double)p->de_stop_factor)); }

// RMdoBinSearch (src/calc.rs:1706-1734), without the secant option
void Marcher::bin_search(double &de, double last_step_width) {
    int itmp = p->de_add_steps;
    double dt1 = last_step_width * -0.5;
    while (std::fabs(de - (double)ms_de_stop) > 0.001) {
        mzz += dt1;
        step(dt1);
        update_de_stop();
        itmp -= 1;
        if (itmp <= 0) break;
        de = calc_de();
        if (it.it_result >= max_its_result) {
            dt1 = -std::fabs(dt1);
            continue;
        }
        double f = de - (double)ms_de_stop;
        dt1 = f < 0.0 ? std::fabs(dt1) * -0.55 : std::fabs(dt1) * 0.55;
    }
}

// RMdoBinSearchIt (src/calc.rs:1737-1791)
void Marcher::bin_search_it() {
    float yp = (float)it.max_it - 0.99f;
    int saved_max = it.max_it;
    it.max_it += 1;
    int itmp = p->de_add_steps;
    it.calc_sit = true;
    double dt1 = 0.0, dmul = 1.0;
    bool first = true;
    float last_si = 0.f, last_dif = 0.f;
    for (;;) {
        mzz += dt1;
        step(dt1);
        calc_de();
        if (!first && last_dif < std::fabs(yp - it.smooth_it)) {
            mzz -= dt1;
            step(-dt1);
            it.smooth_it = last_si;
            if (dt1 > 0.0) dmul *= 0.5;
            else dmul *= 0.7;
        }
        last_dif = std::fabs(yp - it.smooth_it);
        last_si = it.smooth_it;
        if (it.smooth_it > (float)it.max_it - 0.1f) {
            dt1 = -3.0;
        } else {
            mzz -= 0.001;
            step(-0.001);
            calc_de();
            float r = last_si - it.smooth_it;
            if (std::fabs(r) < 1e-30f) dt1 = (last_si < it.smooth_it ? 1.0 : 0.0) - 0.5;
            else if (r < 0.0f) dt1 = (double)((yp - it.smooth_it) / (r * 500.0f));
            else dt1 = (double)((yp - it.smooth_it) / (r * 1000.0f));
            if (dt1 > 4.0) dt1 = std::sqrt(dt1) * 2.0;
            else if (dt1 < -9.0) dt1 = std::sqrt(-dt1) * -3.0;
            dt1 = dt1 * dmul + 0.0005;
        }
        first = false;
        itmp -= 1;
        if (itmp < 0) break;
    }
    it.max_it = saved_max;
}

// MakeWNormalsFromDVec (src/calc.rs:1794-1803)
static void store_normal(SiLight &si, const double n[3]) {
    double d = 32767.0 / std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2] + 1e-100);
    for (int k = 0; k < 3; k++) {
        double v = rte(n[k] * d);
        si.normal[k] = std::isnan(v) ? 0 : (int16_t)rclamp(v, -32767.0, 32767.0);
    }
    if (si.normal[0] == 0 && si.normal[1] == 0) si.normal[2] = si.normal[2] > 0 ? 32767 : -32767;
}

// RMCalcRoughness (src/calc.rs:1806-1809)
static float calc_roughness(const double n[3], double dt2, double dsg) {
    double a = (dsg * 7.0 * dt2 * dt2 + 1e-40) / (n[0] * n[0] + n[1] * n[1] + n[2] * n[2] + 1e-40);
    return (float)rclamp(std::sqrt(rmax(a, 0.0)) - 0.05, 0.0, 1.0);
}

// RMCalculateNormals (src/calc.rs:1813-1906)
float Marcher::calculate_normals(SiLight &si) {
    const Mat3 &vg = p->vgrads;
    it.calc_sit = true;
    double noffset = (double)rminf(p->de_stop, 1.0f) * (1.0 + mzz * (double)p->de_stop_factor) * 0.15;
    double ct1[3] = {it.c[0], it.c[1], it.c[2]};
    double dnn = calc_de();
    float nn = it.smooth_it;
    it.calc_sit = false;
    double n[3] = {0, 0, 0};
    if (p->sm_normals == 8) {
        double ssn = noffset * 1.3333;
        for (int a = -2; a <= 2; a++)
            for (int b = -2; b <= 2; b++)
                for (int c = -2; c <= 2; c++) {
                    if ((a | b | c) == 0) continue;
                    std::memcpy(it.c, ct1, sizeof(ct1));
                    add_weight(it.c, vg[2], a * ssn);
                    add_weight(it.c, vg[1], b * ssn);
                    add_weight(it.c, vg[0], c * ssn);
                    double d = calc_de();
                    if (a != 0) n[2] += d / a;
                    if (b != 0) n[1] += d / b;
                    if (c != 0) n[0] += d / c;
                }
        for (int k = 0; k < 3; k++) n[k] *= 0.0075;
    } else {
        const int ks[3] = {2, 0, 1};
        for (int q = 0; q < 3; q++) {
            int k = ks[q];
            std::memcpy(it.c, ct1, sizeof(ct1));
            add_weight(it.c, vg[k], noffset);
            double a = calc_de();
            add_weight(it.c, vg[k], -2.0 * noffset);
            n[k] = (a - calc_de()) * 0.5;
        }
    }
    if (p->sm_normals > 0) {
        noffset *= 2.0;
        if (p->sm_normals < 8) {
            std::memcpy(it.c, ct1, sizeof(ct1));
            add_weight(it.c, vg[0], -noffset);
            dnn += calc_de();
            add_weight(it.c, vg[0], 2.0 * noffset);
            dnn += calc_de();
            std::memcpy(it.c, ct1, sizeof(ct1));
            add_weight(it.c, vg[1], -noffset);
            dnn += calc_de();
            add_weight(it.c, vg[1], 2.0 * noffset);
            dnn = (dnn + calc_de()) * 0.2;
        }
        int sm = p->sm_normals;
        double ssn = noffset * 3.0 / ((double)sm + 0.5);
        double dm = (double)sm * 2.0;
        double vx0[3], vy0[3], vx[3], vy[3];
        create_xy_vecs_from_normals(n, vx0, vy0);
        rotate_vector_reverse(vx0, vg, vx);
        rotate_vector_reverse(vy0, vg, vy);
        auto sweep = [&](const double dir[3], double &nn1, double &ds) {
            std::memcpy(it.c, ct1, sizeof(ct1));
            add_weight(it.c, dir, -(double)sm * ssn);
            nn1 = 0; ds = 0;
            for (int k = -sm; k <= sm; k++) {
                if (k != 0) {
                    double d = (calc_de() - dnn) / (double)k;
                    nn1 += d;
                    ds += d * d;
                }
                add_weight(it.c, dir, ssn);
            }
        };
        double nn1, ds1, nn2, ds2;
        sweep(vx, nn1, ds1);
        sweep(vy, nn2, ds2);
        double dsg = ds1 * dm - nn1 * nn1 + ds2 * dm - nn2 * nn2;
        double dt2 = noffset * 0.5 / (dm * ssn);
        s_roughness = calc_roughness(n, dt2, dsg);
        if (p->sm_normals < 8) {
            n[0] += nn1 * dt2;
            n[1] += nn2 * dt2;
        }
    }
    std::memcpy(it.c, ct1, sizeof(ct1));
    store_normal(si, n);
    return nn;
}

// RMCalculateNormalsOnSmoothIt (src/calc.rs:1910-2006), without smoothing
float Marcher::calculate_normals_on_smooth_it(SiLight &si) {
    const Mat3 &vg = p->vgrads;
    double noffset = (double)rminf(p->de_stop, 1.0f) * (1.0 + mzz * (double)p->de_stop_factor) * 0.15;
    it.calc_sit = true;
    double ct1[3] = {it.c[0], it.c[1], it.c[2]};
    it.hybrid_3d(p->slots);
    float nn = it.smooth_it;
    double n[3] = {0, 0, 0};
    const int ks[3] = {2, 0, 1};
    for (int q = 0; q < 3; q++) {
        int k = ks[q];
        std::memcpy(it.c, ct1, sizeof(ct1));
        add_weight(it.c, vg[k], noffset);
        it.hybrid_3d(p->slots);
        double a = (double)it.smooth_it;
        add_weight(it.c, vg[k], -2.0 * noffset);
        it.hybrid_3d(p->slots);
        n[k] = ((double)it.smooth_it - a) * 0.5;
    }
    std::memcpy(it.c, ct1, sizeof(ct1));
    store_normal(si, n);
    return nn;
}

// doColorOnIt (src/calc.rs:2010-2024)
void Marcher::do_color_on_it() {
    if (p->color_on_it == 1) {
        it.v[0] = it.c[0]; it.v[1] = it.c[1]; it.v[2] = it.c[2];
    } else {
        int i = it.max_it;
        it.max_it = p->color_on_it - 1;
        it.rstop = p->rstop3d;
        calc_de();
        it.max_it = i;
        it.rstop = p->d_rstop;
    }
}

// RMdoColor (src/calc.rs:2068-2088)
void Marcher::do_color(SiLight &si) {
    double x = it.v[0], y = it.v[1], z = it.v[2];
    const double *c = it.c;
    double s;
    switch (p->color_option) {
        case 1: s = std::log(it.rout / (it.rold + 1.0)) * (double)p->mct_color_mul; break;
        case 2: s = (std::atan2(y - c[1], x - c[0]) + PI) * 5200.0; break;
        case 3: s = (std::atan2(z - c[2], x - c[0]) + PI) * 5200.0; break;
        case 4: s = (std::atan2(z - c[2], y - c[1]) + PI) * 5200.0; break;
        case 5: {
            s = (std::atan2(x, y) + PI) * 5215.0;
            double r = std::sqrt(x * x + y * y + 1e-100 + z * z);
            double s2 = (PI + std::asin(rclamp(z / r, -1.0, 1.0)) * 2.0) * 5215.0;
            si.si_gradient = min_max_clip_15bit((float)s2);
            break;
        }
        default: s = it.otrap * 4096.0; break;
    }
    si.otrap = min_max_clip_15bit((float)s);
}

// CalcZposAndRough (src/calc.rs:2194-2204)
void Marcher::calc_zpos_and_rough(SiLight &si) {
    double zz = rmax(mzz, 0.0);
    int64_t v = sat_i64(rte(p->zc_mul * (std::sqrt(zz * p->zcorr + 1.0) - 1.0)));
    int64_t d = 8388352 - v;
    if (d < 0) d = 0;
    if (d > 8388352) d = 8388352;
    uint32_t r = (uint32_t)d << 8;
    if (p->sm_normals > 0) r |= sat_u32(rte((double)(s_roughness * 255.0f))) & 0xFF;
    si.zpos_fine = r;
}

// surface_point (src/calc.rs:2157-2191)
bool Marcher::surface_point(int x, int y, const SiLight &si, int steps, double thr) {
    if (si.zpos() >= 32768 || si.si_gradient >= 32768) return false;
    cafy = ((double)y / (double)p->height - 0.5) * p->fov_y;
    calc_vgrads_fov(x + 1);
    calc_start_pos(x, y);
    it.calc_sit = false;
    double zf = (double)(si.zpos_fine >> 8);
    double q = (8388351.5 - zf) / p->zc_mul + 1.0;
    mzz = (q * q - 1.0) / p->zcorr;
    add_weight(it.c, vfov, mzz);
    update_de_stop();
    double d = rmin(calc_de(), (double)ms_de_stop * 2.0);
    if (it.it_result < max_its_result || d < (double)ms_de_stop) {
        double q2 = (8388351.9 - zf) / p->zc_mul + 1.0;
        double dt1 = (q2 * q2 - 1.0) / p->zcorr - mzz;
        int itmp = steps;
        while (itmp > 0 && std::fabs(d - (double)ms_de_stop) > thr) {
            mzz += dt1;
            add_weight(it.c, vfov, dt1);
            update_de_stop();
            itmp -= 1;
            if (itmp > 0) {
                d = calc_de();
                dt1 = d < (double)ms_de_stop ? std::fabs(dt1) * -0.55 : std::fabs(dt1) * 0.55;
            }
        }
    } else {
        bin_search_it();
        ms_de_stop = (float)((double)p->de_stop * (1.0 + std::fabs(mzz) * (double)p->de_stop_factor));
    }
    return true;
}

// surface_found (src/calc.rs:2471-2511)
void Marcher::surface_found(SiLight &si, double dtmp, double last_step) {
    bool de_limited = it.it_result < max_its_result || dtmp < (double)ms_de_stop;
    if (p->de_add_steps != 0) {
        if (de_limited) bin_search(dtmp, last_step);
        else bin_search_it();
    }
    float nn = p->normals_on_de ? calculate_normals(si) : calculate_normals_on_smooth_it(si);
    float v;
    if (de_limited) {
        float l = (float)std::log((double)rmaxf(p->de_stop, ms_de_stop) * p->step_width);
        v = 32767.0f - (nn + p->d_col_plus + p->col_var_de_stop_mul * l) * p->mcts_m;
    } else {
        v = 32767.0f - nn * p->mcts_m;
    }
    si.si_gradient = min_max_clip_15bit(v);
    if (p->color_on_it != 0) do_color_on_it();
    do_color(si);
    calc_zpos_and_rough(si);
}

// march_pixel / march_pixel_from (src/calc.rs:2207-2318), outside rendering,
// no cutting planes, no cone march
SiLight Marcher::march_pixel(int x, int y) {
    SiLight si;
    si.amb_shadow = 5000;
    cafy = ((double)y / (double)p->height - 0.5) * p->fov_y;
    calc_vgrads_fov(x + 1);
    calc_start_pos(x, y);
    it.calc_sit = false;
    float step_count = 0.f;
    mzz = 0.0;
    ms_de_stop = p->de_stop;
    bool first_step = p->first_step_random;
    double dtmp = calc_de();
    if (it.it_result >= max_its_result || dtmp < (double)ms_de_stop) {
        if (p->color_on_it != 0) do_color_on_it();
        si.zpos_fine = 0x7FFF0000u;
        si.normal[0] = 0; si.normal[1] = 0; si.normal[2] = -32767;
        do_color(si);
        if (p->color_option > 4) {
            si.si_gradient |= 32768;
        } else {
            double t = rclamp(it.rout / p->d_rstop, 0.0, 1.0);
            si.si_gradient = (uint16_t)(32768 + sat_u16(rte(32767.0 * t)));
        }
        return si;
    }
    return march_from(si, dtmp, first_step, step_count);
}

// march_from (src/calc.rs:2533-2655), without the volumetric light and the
// experimental relaxed steps
SiLight Marcher::march_from(SiLight si, double dtmp, bool first_step, float step_count) {
    float rsf_mul = 1.0f;
    double last_step = dtmp * (double)p->z_step_div;
    double last_de;
    uint32_t guard = 0;
    for (;;) {
        guard++;
        if (guard > 2000000) break;
        if (it.it_result >= max_its_result) {
            double dt1 = -0.5 * last_step;
            mzz += dt1;
            step(dt1);
            update_de_stop();
            dtmp = calc_de();
            last_step = -dt1;
        }
        if (it.it_result < p->min_it || (it.it_result < max_its_result && dtmp >= (double)ms_de_stop)) {
            last_de = dtmp;
            double d = rmax(0.11, (dtmp - (double)p->ms_de_sub * (double)ms_de_stop) * (double)p->z_step_div * (double)rsf_mul);
            double s1 = (double)(rmaxf(ms_de_stop, 0.4f) * p->mh04zsd);
            bool count = p->dfog_on_it == 0 || it.it_result == p->dfog_on_it;
            if (s1 < d) {
                if (count) step_count += (float)(s1 / d);
                d = s1;
            } else if (count) {
                step_count += 1.0f;
            }
            if (first_step) {
                first_step = false;
                seed = wrap_lcg(seed, 214013u, 2531011u);
                d *= (double)(seed & 0x7FFFFFFF) * (1.0 / 2147483647.0);
            }
            mzz += d;
            if (mzz > p->zend) break;
            last_step = d;
            step(d);
            update_de_stop();
            dtmp = calc_de();
            if (dtmp > last_de + last_step) dtmp = last_de + last_step;
            if (last_de > dtmp + 1e-30) {
                double t = last_step / (last_de - dtmp);
                rsf_mul = t < 1.0 ? (float)rmax(0.5, t) : 1.0f;
            } else {
                rsf_mul = 1.0f;
            }
        } else {
            surface_found(si, dtmp, last_step);
            break;
        }
    }
    si.shadow = sat_u16(rtef(rclampf(step_count, 0.0f, 1023.0f)));
    return si;
}

// ---------------------------------------------------------------------------
// hard and soft shadows (src/calc.rs:2705-2979, src/render.rs:2383-2415)

static inline double dot_normalize(const double a[3], const double b[3]) {
    return dot3(a, b) / rmax(std::sqrt(dot3(a, a) * dot3(b, b)), 1e-300);
}

// shadow_job (src/render.rs:2383-2415) for global (directional) lights:
// HSvecs = RotateVectorReverse(-StepWidth * LN, M), LN from the light
// angles as LightVals::new has it (src/lighting.rs:998-1004)
void shadow_lights(const mb3d_cu_scene &sc, const Params &p, std::vector<HsLight> &out) {
    out.clear();
    Mat3 m;
    normalise_matrix_to(1.0, p.vgrads, m);
    for (int idx = 0; idx < 6; idx++) {
        const mb3d_cu_light &li = sc.lights[idx];
        if (!li.on || !((sc.shadow_lights >> idx) & 1)) continue;
        double dtmp = -li.x_angle, dtmp2 = li.y_angle;
        double v[3] = {-std::sin(dtmp), std::sin(dtmp2), std::cos(dtmp2) * std::cos(dtmp)};
        double nrm = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        float ln[3] = {(float)(-v[0] / nrm), (float)(-v[1] / nrm), (float)(-v[2] / nrm)};
        double l[3] = {(double)ln[0], (double)ln[1], (double)ln[2]};
        double ll = std::sqrt(dot3(l, l));
        double u[3] = {l[0], l[1], l[2]};
        if (ll > 0.0) { u[0] = l[0] * (1.0 / ll); u[1] = l[1] * (1.0 / ll); u[2] = l[2] * (1.0 / ll); }
        double w[3] = {-u[0] * p.step_width, -u[1] * p.step_width, -u[2] * p.step_width};
        HsLight h;
        h.idx = idx;
        rotate_vector_reverse(w, m, h.vec);
        out.push_back(h);
    }
    if (sc.shadow_soft && !out.empty()) {
        HsLight last = out.back();
        out.clear();
        out.push_back(last);
    }
}

// hs_surface_start (src/calc.rs:2741-2764)
bool Marcher::hs_surface_start(int x, int y, const SiLight &si) {
    if (si.zpos() >= 32768 || si.si_gradient >= 32768) return false;
    cafy = ((double)y / (double)p->height - 0.5) * p->fov_y;
    calc_vgrads_fov(x + 1);
    calc_start_pos(x, y);
    double zf = (double)(si.zpos_fine >> 8);
    double q = (8388351.5 - zf) / p->zc_mul + 1.0;
    mzz = (q * q - 1.0) / p->zcorr;
    add_weight(it.c, vfov, mzz);
    update_de_stop();
    double d = calc_de();
    bool de_limited = it.it_result < max_its_result || d < (double)ms_de_stop;
    if (de_limited) {
        double q2 = (8388351.9 - zf) / p->zc_mul + 1.0;
        double dt1 = (q2 * q2 - 1.0) / p->zcorr - mzz;
        bin_search(d, dt1);
    } else {
        bin_search_it();
    }
    return true;
}

// MaxLHS (src/calc.rs:2767-2773)
double Marcher::hs_max_len(int y, float mul) {
    return (double)((float)(p->width + y) * 0.6f *
                    (1.0f + 0.5f * (float)rmin(mzz, p->zend * 0.4) * (float)rmax(p->fov_y, 0.0) / (float)p->height) * mul);
}

// THardShadowCalcThread.Execute for one row (src/calc.rs:2777-2898).
// per_pixel: without the row's "open air" shortcut (b_zz_oathr), as the
// reference's card shadow pass has it (src/gpu_march.wgsl:3343-3500), so
// that every pixel is independent of its row neighbours.
void Marcher::hard_shadow_row(int y, SiLight *row, int n, const std::vector<HsLight> &lights, float max_len_mul,
                              bool per_pixel) {
    int b_zz_oathr[6] = {0, 0, 0, 0, 0, 0};
    double d_last_found[6] = {0, 0, 0, 0, 0, 0};
    double d_last_z = 0.0;
    uint16_t clear_mask = 0;
    for (const auto &l : lights) clear_mask |= (uint16_t)(0x400 << l.idx);
    for (int x = 0; x < n; x++) {
        SiLight &si = row[x];
        for (int k = 0; k < 6; k++)
            if (b_zz_oathr[k] > 0) b_zz_oathr[k] -= 1;
        if (per_pixel) {
            for (int k = 0; k < 6; k++) { b_zz_oathr[k] = 0; d_last_found[k] = 0; }
        }
        si.shadow &= (uint16_t)~clear_mask;
        double nv0[3] = {si.normal[0] / 32767.0, si.normal[1] / 32767.0, si.normal[2] / 32767.0};
        double nvec[3];
        rotate_vector_reverse(nv0, p->vgrads, nvec);
        if (!hs_surface_start(x, y, si)) continue;
        mzz = rmax(mzz - 0.1, 0.0);
        add_weight(it.c, vfov, -0.1);
        update_de_stop();
        double ic[3] = {it.c[0], it.c[1], it.c[2]};
        double max_lhs = hs_max_len(y, max_len_mul);
        double oa_thr = (1.0 + (mzz + max_lhs) * (double)p->de_stop_factor) * 3.3 / (double)p->z_step_div;
        for (const auto &l : lights) {
            int li = l.idx;
            bool b_thr = b_zz_oathr[li] > 0;
            if (b_thr) {
                b_zz_oathr[li] -= sat_i32(rte(std::fabs(d_last_z - mzz) * 3.3 / oa_thr));
                if (b_zz_oathr[li] <= 0) {
                    b_thr = false;
                    b_zz_oathr[li] = 0;
                } else {
                    d_last_found[li] -= std::fabs(d_last_z - mzz) + (1.0 + mzz * (double)p->de_stop_factor);
                    if (d_last_found[li] <= 0.0) {
                        b_thr = false;
                        b_zz_oathr[li] = 0;
                    }
                }
            }
            std::memcpy(it.c, ic, sizeof(ic));
            double zz2 = mzz;
            const double *lvec = l.vec;
            double zz2mul = -dot_normalize(lvec, vfov);
            if (dot3(nvec, lvec) > 0.0) {
                si.shadow |= (uint16_t)(0x400 << li);
                b_zz_oathr[li] = 0;
                continue;
            }
            double dt1 = max_lhs;
            if (dt1 > 0.0) {
                ms_de_stop = (float)((double)p->de_stop * (1.0 + std::fabs(zz2) * (double)p->de_stop_factor));
                float rsf = 2.0f;
                double d = calc_de();
                int guard = 0;
                for (;;) {
                    guard++;
                    if (guard > 1000000) break;
                    if (b_thr && d_last_found[li] > dt1) {
                        dt1 = -1.0;
                        break;
                    }
                    double last_de = d;
                    double st = (double)rminf(
                        rmaxf(0.11f, (float)((d - (double)p->ms_de_sub * (double)ms_de_stop) * (double)p->z_step_div * (double)rsf)),
                        rmaxf(ms_de_stop, 0.4f) * p->mh04zsd);
                    dt1 -= st;
                    add_weight(it.c, lvec, -st);
                    zz2 += st * zz2mul;
                    ms_de_stop = (float)((double)p->de_stop * (1.0 + std::fabs(zz2) * (double)p->de_stop_factor));
                    d = calc_de();
                    if (it.it_result >= max_its_result || d <= (double)ms_de_stop) break;
                    if (d > last_de + st) d = last_de + st;
                    if (!b_thr) {
                        if (d > oa_thr) {
                            if (b_zz_oathr[li] < 3) {
                                d_last_found[li] = dt1;
                                b_zz_oathr[li] = 3;
                            }
                        } else {
                            b_zz_oathr[li] = 0;
                        }
                    }
                    if (last_de > d + 1e-30) {
                        float t = (float)(st / (last_de - d));
                        rsf = t < 1.0f ? rmaxf(t, 0.5f) : 1.0f;
                    } else {
                        rsf = 1.0f;
                    }
                    if (dt1 < 0.0) break;
                }
            }
            if (dt1 > 0.0) {
                si.shadow |= (uint16_t)(0x400 << li);
                b_zz_oathr[li] = 0;
            }
        }
        d_last_z = mzz;
    }
}

// calcHSsoft (src/calc.rs:2901-2979), directional light
void Marcher::soft_shadow_row(int y, SiLight *row, int n, const HsLight &light, float soft_radius, float max_len_mul) {
    float zrs_mul = 80.0f / rmaxf(soft_radius, 0.001f);
    for (int x = 0; x < n; x++) {
        SiLight &si = row[x];
        si.shadow |= 0xFC00;
        double nv0[3] = {si.normal[0] / 32767.0, si.normal[1] / 32767.0, si.normal[2] / 32767.0};
        double nvec[3];
        rotate_vector_reverse(nv0, p->vgrads, nvec);
        if (!hs_surface_start(x, y, si)) continue;
        mzz -= 0.1;
        add_weight(it.c, vfov, -0.1);
        double max_lhs = hs_max_len(y, max_len_mul);
        double zz2 = mzz;
        update_de_stop();
        const double *lvec = light.vec;
        double d_max_l = max_lhs;
        double zz2mul = -dot_normalize(lvec, vfov);
        if (dot3(nvec, lvec) > 0.0) {
            si.shadow &= 0x3FF;
            continue;
        }
        float zr_soft = 1.0f;
        double dt1 = d_max_l;
        if (dt1 > 0.0) {
            ms_de_stop = (float)((double)p->de_stop * (1.0 + std::fabs(zz2) * (double)p->de_stop_factor));
            float rsf = 2.0f;
            double d = calc_de();
            int guard = 0;
            for (;;) {
                guard++;
                if (guard > 1000000) break;
                double last_de = d;
                double st = (double)rminf(
                    rmaxf(0.11f, (float)((d - (double)p->ms_de_sub * (double)ms_de_stop) * (double)p->z_step_div * (double)rsf)),
                    rmaxf(ms_de_stop, 0.4f) * p->mh04zsd);
                dt1 -= st;
                add_weight(it.c, lvec, -st);
                zz2 += st * zz2mul;
                ms_de_stop = (float)((double)p->de_stop * (1.0 + std::fabs(zz2) * (double)p->de_stop_factor));
                d = calc_de();
                double r = (d_max_l - dt1) / max_lhs;
                double r8 = (r * r) * (r * r);
                zr_soft = rminf(zr_soft, (float)((d - (double)ms_de_stop) * (double)zrs_mul / (d_max_l - dt1 + 0.11) + r8 * r8));
                if (it.it_result >= max_its_result || d <= (double)ms_de_stop) break;
                if (d > last_de + st) d = last_de + st;
                if (last_de > d + 1e-30) {
                    float t = (float)(st / (last_de - d));
                    rsf = t < 1.0f ? rmaxf(t, 0.5f) : 1.0f;
                } else {
                    rsf = 1.0f;
                }
                if (dt1 < 0.0) break;
            }
        }
        si.shadow = (uint16_t)((si.shadow & 0x3FF) | (sat_u16(rtef(rclampf(zr_soft, 0.0f, 1.0f) * 63.4f)) << 10));
    }
}

// ---------------------------------------------------------------------------
// DE ambient occlusion (src/deao.rs:35-414), without dithering

typedef float SVec[3];

// ray_dir (src/deao.rs:38-42)
static void ray_dir(double ya, double za, SVec out) {
    double sy = std::sin(ya), cy = std::cos(ya);
    double sz = std::sin(za), cz = std::cos(za);
    out[0] = (float)(sy * cz);
    out[1] = (float)(-sy * sz);
    out[2] = (float)(-cy);
}

// normal_matrix (src/deao.rs:45-62)
static void normal_matrix(const SVec n, float m[3][3]) {
    double a = std::acos(rclamp((double)-n[2], -1.0, 1.0)) * 0.5;
    double sa = std::sin(a), ca = std::cos(a);
    double nn = std::sqrt((double)(n[1] * n[1] + n[0] * n[0]));
    double q[4];
    if (nn < 1e-25) {
        q[0] = 0; q[1] = 0; q[2] = 0; q[3] = ca;
    } else {
        sa /= nn;
        q[0] = -(double)n[1] * sa; q[1] = (double)n[0] * sa; q[2] = 0; q[3] = ca;
    }
    double mm[3][3] = {
        {1.0 - 2.0 * (q[1] * q[1] + q[2] * q[2]), 2.0 * (q[0] * q[1] + q[2] * q[3]), 2.0 * (q[0] * q[2] - q[1] * q[3])},
        {2.0 * (q[0] * q[1] - q[2] * q[3]), 1.0 - 2.0 * (q[0] * q[0] + q[2] * q[2]), 2.0 * (q[2] * q[1] + q[0] * q[3])},
        {2.0 * (q[0] * q[2] + q[1] * q[3]), 2.0 * (q[1] * q[2] - q[0] * q[3]), 1.0 - 2.0 * (q[0] * q[0] + q[1] * q[1])},
    };
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) m[i][j] = (float)mm[i][j];
}

static inline float sdot(const SVec a, const SVec b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

struct Rays {
    std::vector<std::array<float, 3>> dirs;
    int row_count[4] = {0, 0, 0, 0};
    float d_step_mul, d_min_a_dif, correction_weight;
};

// build_rays (src/deao.rs:75-104)
static Rays build_rays(int quality) {
    Rays r;
    int q = std::min(std::max(quality, 0), 3);
    SVec d;
    if (q == 0) {
        double abr = to_radians(60.0);
        for (int x = 0; x < 3; x++) {
            ray_dir(0.5 * abr, (double)x * TAU / 3.0, d);
            r.dirs.push_back({d[0], d[1], d[2]});
        }
        r.d_step_mul = 1.8f;
        r.d_min_a_dif = -1.0f;
        r.correction_weight = 0.3f;
    } else {
        ray_dir(0.0, 0.0, d);
        r.dirs.push_back({d[0], d[1], d[2]});
        double abr = (PI / 2.0) / ((double)q + 0.9);
        for (int y = 1; y <= q; y++) {
            double dt1 = (double)y * abr;
            int n = (int)rte(std::sin(dt1) * TAU / abr);
            r.row_count[y] = n;
            for (int x = 0; x < n; x++) {
                ray_dir(dt1, (double)x * TAU / (double)n, d);
                r.dirs.push_back({d[0], d[1], d[2]});
            }
        }
        r.d_step_mul = (float)(1.0 + std::sin(abr));
        r.d_min_a_dif = (float)std::cos(abr * 1.2);
        r.correction_weight = q == 1 ? 0.2f : 0.1666f;
    }
    return r;
}

int ao_ray_table(int quality, float *dirs, int cap) {
    Rays r = build_rays(quality);
    int n = (int)r.dirs.size();
    for (int k = 0; k < n && k < cap; k++)
        for (int i = 0; i < 3; i++) dirs[3 * k + i] = r.dirs[k][i];
    return n;
}

// get_rand (src/deao.rs:263-266)
static double get_rand(int32_t &seed) {
    seed = wrap_lcg(seed, 0x343FDu, 0x269EC3u);
    return (double)(((uint32_t)seed >> 8) & 0x7FFFFF) / (double)0x7FFFFF;
}

// deao_row (src/deao.rs:268-414), outside rendering, no dithering, no cutting planes
void deao_row(Marcher &m, int y, SiLight *row, int n, int quality, float max_len, bool first_step_random, int32_t &rnd) {
    const Params *p = m.p;
    Rays base = build_rays(quality);
    double sw = p->step_width;
    Mat3 rot_v;
    normalise_matrix_to(sw, p->vgrads, rot_v);
    double s_max_d = (double)max_len * 0.5 * std::sqrt((double)p->height * (double)p->height + (double)p->width * (double)p->width);
    double de_stop = (double)p->de_stop;
    for (int x = 0; x < n; x++) {
        SiLight &si = row[x];
        si.amb_shadow = 0;
        if (si.zpos() >= 32768 || si.si_gradient >= 32768) continue;
        if (!m.surface_point(x, y, si, 5, 0.004)) continue;
        double ms_de_stop = rmin((double)m.ms_de_stop, 1e6);
        double ic[3] = {m.it.c[0], m.it.c[1], m.it.c[2]};
        double step_ao = ms_de_stop / de_stop;
        double max_dist = s_max_d * std::sqrt(step_ao);
        double d_step_mul = (double)base.d_step_mul;
        if (p->de_stop_factor == 0.0f) ms_de_stop = de_stop / (d_step_mul * d_step_mul);
        else ms_de_stop = ms_de_stop / (d_step_mul * d_step_mul);
        const auto &dirs = base.dirs;
        int ray_count = (int)dirs.size();
        double de_mul = std::sqrt((double)ray_count * 0.5);
        double abr = 1.2 / std::asin(rclamp(1.0 / de_mul, -1.0, 1.0));
        double md_d10 = 0.1 / (max_dist * de_mul);
        float nrm[3];
        {
            float v[3] = {(float)si.normal[0], (float)si.normal[1], (float)si.normal[2]};
            float l = rmaxf(std::sqrt(sdot(v, v)), 1e-30f);
            nrm[0] = v[0] / l; nrm[1] = v[1] / l; nrm[2] = v[2] / l;
        }
        float rot_w[3][3];
        normal_matrix(nrm, rot_w);
        std::vector<float> min_ra(ray_count, 0.f);
        for (int k = 0; k < ray_count; k++) {
            const float *d = dirs[k].data();
            float v[3] = {sdot(rot_w[0], d), sdot(rot_w[1], d), sdot(rot_w[2], d)};
            double vd[3] = {(double)v[0], (double)v[1], (double)v[2]};
            double sv[3];
            rotate_vector_reverse(vd, rot_v, sv);
            double dt1 = step_ao * d_step_mul;
            double s_tmp = 1.0;
            bool b_end = false;
            bool b_first = first_step_random;
            for (;;) {
                if (b_first) {
                    b_first = false;
                    dt1 *= get_rand(rnd) * 1.5 + 0.5;
                } else if (dt1 > max_dist) {
                    dt1 = max_dist;
                    b_end = true;
                }
                std::memcpy(m.it.c, ic, sizeof(ic));
                add_weight(m.it.c, sv, dt1);
                double dt2 = m.calc_de();
                s_tmp = rmin(s_tmp, (dt2 - ms_de_stop + dt1 * md_d10) / dt1);
                if (s_tmp < 0.02) break;
                dt1 += rmax(dt2, dt1 * d_step_mul);
                if (b_end) break;
            }
            min_ra[k] = (float)(rmax(s_tmp, 0.0) * de_mul);
        }
        double amount = 0.0;
        for (int k = 0; k < ray_count; k++) {
            float s_add = 0.f;
            if (min_ra[k] < 1.0f) {
                float max_add = 1.0f - min_ra[k];
                for (int k2 = 0; k2 < ray_count; k2++) {
                    if (k2 == k) continue;
                    float dt = sdot(dirs[k].data(), dirs[k2].data());
                    if (dt > base.d_min_a_dif) {
                        float overlap = min_ra[k2] - (float)((double)std::acos(rclampf(dt, -1.0f, 1.0f)) * abr) + 1.0f;
                        if (overlap > 0.0f) s_add += rminf(max_add, overlap) * base.correction_weight;
                    }
                }
            }
            amount += (double)rminf(s_add + min_ra[k], 1.0f);
        }
        si.amb_shadow = sat_u16(rmax(rte(16383.0 * (1.0 - amount / (double)ray_count)), 0.0));
    }
}

// CalcAmbShadowDEfor1pos (deao_1pos, src/reflect.rs:954-1090): the DE
// ambient occlusion at the marcher's position (the reflection pass's hits),
// outside rendering, no cutting planes, no random first step; the depth
// for the DE stop is m.mzz
void deao_1pos(Marcher &m, SiLight &si, int quality, float max_len) {
    si.amb_shadow = 0;
    if (si.zpos() >= 32768 || si.si_gradient >= 32768) return;
    const Params *p = m.p;
    const double sw = p->step_width;
    m.it.calc_sit = false;
    Mat3 rot_v;
    normalise_matrix_to(sw, p->vgrads, rot_v);
    const double s_max_d = (double)max_len * 0.5 * std::sqrt((double)p->height * (double)p->height + (double)p->width * (double)p->width);
    double ms_de_stop = (double)rminf((float)((double)p->de_stop * (1.0 + std::fabs(m.mzz) * (double)p->de_stop_factor)), 1e6f);
    const double ic[3] = {m.it.c[0], m.it.c[1], m.it.c[2]};
    const double step_ao = ms_de_stop / (double)p->de_stop;
    const double max_dist = s_max_d * std::sqrt(step_ao);
    // the directions (src/reflect.rs:973-998): not deao.rs's table -- every
    // ring has the same number of rays, round(sin(0.25) * tau / abr); the
    // step multiplier in double precision
    Rays base;
    double d_step_mul;
    {
        const int q = std::min(std::max(quality, 0), 3);
        SVec d;
        if (q == 0) {
            const double abr = to_radians(60.0);
            for (int i = 0; i < 3; i++) {
                ray_dir(0.5 * abr, (double)i * TAU / 3.0, d);
                base.dirs.push_back({d[0], d[1], d[2]});
            }
            d_step_mul = 1.8;
            base.d_min_a_dif = -1.0f;
            base.correction_weight = 0.3f;
        } else {
            const double abr = (PI / 2.0) / ((double)q + 0.9);
            ray_dir(0.0, 0.0, d);
            base.dirs.push_back({d[0], d[1], d[2]});
            for (int iy = 1; iy <= q; iy++) {
                const int n = (int)rte(std::sin(0.25) * TAU / abr);
                for (int ix = 0; ix < n; ix++) {
                    ray_dir(abr * (double)iy, (double)ix * TAU / (double)n, d);
                    base.dirs.push_back({d[0], d[1], d[2]});
                }
            }
            d_step_mul = 1.0 + std::sin(abr);
            base.d_min_a_dif = (float)std::cos(abr * 1.2);
            base.correction_weight = q == 1 ? 0.2f : 0.1666f;
        }
    }
    if (p->de_stop_factor != 0.0f) ms_de_stop /= d_step_mul * d_step_mul;
    else ms_de_stop = (double)p->de_stop / (d_step_mul * d_step_mul);
    const auto &dirs = base.dirs;
    const int ray_count = (int)dirs.size();
    const double de_mul = std::sqrt((double)ray_count * 0.5);
    const double abr = 1.2 / std::asin(rclamp(1.0 / de_mul, -1.0, 1.0));
    const double md_d10 = 0.1 / (max_dist * de_mul);
    float nrm[3];
    {
        float v[3] = {(float)si.normal[0], (float)si.normal[1], (float)si.normal[2]};
        float l = rmaxf(std::sqrt(sdot(v, v)), 1e-30f);
        nrm[0] = v[0] / l; nrm[1] = v[1] / l; nrm[2] = v[2] / l;
    }
    float rot_w[3][3];
    normal_matrix(nrm, rot_w);
    std::vector<float> min_ra(ray_count, 0.f);
    for (int k = 0; k < ray_count; k++) {
        const float *d = dirs[k].data();
        float v[3] = {sdot(rot_w[0], d), sdot(rot_w[1], d), sdot(rot_w[2], d)};
        double vd[3] = {(double)v[0], (double)v[1], (double)v[2]};
        double sv[3];
        rotate_vector_reverse(vd, rot_v, sv);
        double dt1 = step_ao * d_step_mul;
        double s = 1.0;
        bool end = false;
        for (int guard = 1;; guard++) {
            if (dt1 > max_dist) {
                dt1 = max_dist;
                end = true;
            }
            std::memcpy(m.it.c, ic, sizeof(ic));
            add_weight(m.it.c, sv, dt1);
            const double d2 = m.calc_de();
            s = rmin(s, (d2 - ms_de_stop + dt1 * md_d10) / dt1);
            if (s < 0.02) break;
            dt1 += rmax(d2, dt1 * d_step_mul);
            if (end || guard > 100000) break;
        }
        min_ra[k] = (float)(rmax(s, 0.0) * de_mul);
    }
    double amount = 0.0;
    for (int k = 0; k < ray_count; k++) {
        float s_add = 0.f;
        if (min_ra[k] < 1.0f) {
            const float max_add = 1.0f - min_ra[k];
            for (int k2 = 0; k2 < ray_count; k2++) {
                if (k2 == k) continue;
                const float dt = sdot(dirs[k].data(), dirs[k2].data());
                if (dt > base.d_min_a_dif) {
                    const float overlap = min_ra[k2] - (float)((double)std::acos(rclampf(dt, -1.0f, 1.0f)) * abr) + 1.0f;
                    if (overlap > 0.0f) s_add += rminf(max_add, overlap) * base.correction_weight;
                }
            }
        }
        amount += (double)rminf(s_add + min_ra[k], 1.0f);
    }
    si.amb_shadow = sat_u16(rmax(rte(16383.0 * (1.0 - amount / (double)ray_count)), 0.0));
    std::memcpy(m.it.c, ic, sizeof(ic));
}

uint16_t clip15(float s) { return min_max_clip_15bit(s); }

}  // namespace oracle
