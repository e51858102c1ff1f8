// The built-in formulas as inlined device functions, one template for the
// double precision march and the single precision bulk march.  Each is one
// iteration on v (x, y, z, w) with the constant j added, as in mb3d-rs's
// Formula::iterate (src/formulas.rs:576-857); the Menger IFS is the
// published KIFS Menger step (the reference runs it as .m3f machine code).
// The formula of a slot is chosen by its number (`DevSlot::formula`), the
// same for every lane of a warp at a given iteration, so the switch does not
// diverge.
#pragma once
#include "devparams.h"
#include "../../include/mb3d_cu.h"

namespace mb3dcu {

template <typename R> struct Num;
template <> struct Num<double> {
    static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
    static __device__ __forceinline__ double div_(double a, double b) { return a / b; }
    static __device__ __forceinline__ double eps() { return 1e-40; }
    static __device__ __forceinline__ double opt(const DevSlot &s, int k) { return s.o[k]; }
    static __device__ __forceinline__ double atan2_(double y, double x) { return atan2(y, x); }
    static __device__ __forceinline__ void sincos_(double a, double *s, double *c) { sincos(a, s, c); }
    static __device__ __forceinline__ double pow_(double a, double b) { return pow(a, b); }
};
// single precision: 1e-40 is a denormal, flushed to zero in the bulk march;
// the smallest normal single keeps the division defined on the z axis
template <> struct Num<float> {
    static __device__ __forceinline__ float sqrt_(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }
    static __device__ __forceinline__ float div_(float a, float b) { return __fdividef(a, b); }
    static __device__ __forceinline__ float eps() { return 1.2e-38f; }
    static __device__ __forceinline__ float opt(const DevSlot &s, int k) { return s.of[k]; }
    static __device__ __forceinline__ float atan2_(float y, float x) { return atan2f(y, x); }
    static __device__ __forceinline__ void sincos_(float a, float *s, float *c) { __sincosf(a, s, c); }
    static __device__ __forceinline__ float pow_(float a, float b) { return __powf(a, b); }
};

template <typename R>
__device__ __forceinline__ R box_fold(R x, R fold) {
    return fabs(x + fold) - (fabs(x - fold) + x);
}

// Amazing Box (HybridCube / HybridCubeDE)
template <typename R>
__device__ __forceinline__ void f_amazing_box(R scale, R min_r, R fold, R v[4], const R j[3], bool ade) {
    R x = box_fold(v[0], fold);
    R y = box_fold(v[1], fold);
    R z = box_fold(v[2], fold);
    R r = z * z + y * y + x * x;
    R m = fmax(min_r, Num<R>::eps());
    R sqr_min_r = m * m;
    R mul;
    if (sizeof(R) == 4) {
        // (branch-free in the single precision bulk: the quotient is formed
        // for the chosen divisor, then selected)
        const bool below = r < sqr_min_r;
        R q = Num<R>::div_(scale, below ? sqr_min_r : r);
        mul = (!below && R(1) < r) ? scale : q;
    } else {
        if (r < sqr_min_r) mul = Num<R>::div_(scale, sqr_min_r);
        else if (R(1) < r) mul = scale;
        else mul = Num<R>::div_(scale, r);
    }
    v[3] = ade ? v[3] * mul : v[3];
    v[2] = z * mul + j[2];
    v[1] = y * mul + j[1];
    v[0] = x * mul + j[0];
}

// sine bulb power 2 with scaling (HybridItIntPow2scale, for the Bulbox)
template <typename R>
__device__ __forceinline__ void f_int_pow2_scale(R scaling, R v[4], const R j[3]) {
    R s = Num<R>::div_(R(1), scaling);
    R x = v[0] * s, y = v[1] * s, z = v[2] * s;
    R xx = x * x, yy = y * y;
    R r = xx + yy;
    v[2] = -((Num<R>::sqrt_(r) * z) * R(2)) * scaling + j[2];
    R a = Num<R>::div_(r - z * z, r);
    v[0] = (xx - yy) * a * scaling + j[0];
    v[1] = (x * y * a) * R(2) * scaling + j[1];
}

// the integer power triplex formulas (fHIntFunctions)
template <typename R>
__device__ __forceinline__ void f_int_pow(int power, R zmul, R v[4], const R j[3]) {
    const R x = v[0], y = v[1], z = v[2];
    const R EPS = Num<R>::eps();
    if (power == 8) {
        // White's / Nylander's power 8 without trigonometry (HybridIntP8)
        R xx = x * x, yy = y * y, zz = z * z;
        R r = xx + yy;
        R rr = r * r;
        R zzzz = zz * zz;
        R t = (zzzz - R(6) * r * zz + rr) * (zz - r) * Num<R>::sqrt_(r);
        v[2] = -(t * z * R(8) * zmul) + j[2];
        R num = (rr * R(70) + zzzz) * zzzz - R(28) * zz * r * (zzzz + rr);
        R a = Num<R>::div_(num, rr * rr + EPS) + R(1);
        R xxxx = xx * xx, yyyy = yy * yy;
        v[1] = (yyyy * (R(7) * xx - yy) + xxxx * (xx - R(7) * yy)) * R(8) * x * y * a + j[1];
        v[0] = a * (xxxx * xxxx + yyyy * (R(70) * xxxx + yyyy) - R(28) * (xx * yy * (yyyy + xxxx))) + j[0];
        return;
    }
    switch (power) {
        case 2: {
            R yy = y * y, xx = x * x;
            R r = xx + yy;
            v[2] = (Num<R>::sqrt_(r) * zmul * z) * R(2) + j[2];
            R a = Num<R>::div_(r - z * z, r);
            v[0] = (xx - yy) * a + j[0];
            v[1] = (x * y * a) * R(2) + j[1];
            break;
        }
        case 3: {
            R sy = y * y, sx = x * x;
            R r = sx + sy;
            R sz = z * z;
            R a = R(1) - Num<R>::div_(R(3) * sz, r + EPS);
            v[0] = (sx - R(3) * sy) * a * x + j[0];
            v[2] = j[2] - (sz - R(3) * r) * z * zmul;
            v[1] = a * (R(3) * sx - sy) * y + j[1];
            break;
        }
        case 4: {
            R sy = y * y, sx = x * x;
            R r = sx + sy;
            R sz = z * z;
            R a = R(1) + Num<R>::div_(sz * (sz - R(6) * r), r * r + EPS);
            v[0] = (sx * (sx - R(6) * sy) + sy * sy) * a + j[0];
            v[2] = Num<R>::sqrt_(r) * (r - sz) * z * R(4) * zmul + j[2];
            v[1] = a * x * (sx - sy) * R(4) * y + j[1];
            break;
        }
        case 5: {
            R sy = y * y, sx = x * x;
            R r = sx + sy;
            R sz = z * z;
            R a = R(1) + Num<R>::div_((sz * sz - sz * r * R(2)) * R(5), r * r + EPS);
            v[1] = (R(5) * sx * sx - sy * (R(10) * sx - sy)) * a * y + j[1];
            v[2] = (sz * (sz - R(10) * r) + R(5) * r * r) * z * zmul + j[2];
            v[0] = a * x * (sx * (sx - R(10) * sy) + R(5) * sy * sy) + j[0];
            break;
        }
        case 6: {
            R sy = y * y, sx = x * x;
            R r = sx + sy;
            R sz = z * z;
            R rr = r * r;
            R a = R(1) - Num<R>::div_(sz * (R(15) * rr + sz * (sz - r * R(15))), rr * r + EPS);
            v[1] = (R(3) * sy * sy + sx * (R(3) * sx - R(10) * sy)) * a * y * x * R(2) + j[1];
            v[2] = (sz * (R(3) * sz - R(10) * r) + R(3) * rr) * Num<R>::sqrt_(r) * z * zmul * R(2) + j[2];
            v[0] = (sy * sy * (R(15) * sx - sy) + sx * sx * (sx - R(15) * sy)) * a + j[0];
            break;
        }
        default: {  // 7
            R sy = y * y, sx = x * x;
            R r = sx + sy;
            R sz = z * z;
            R rr = r * r;
            R a = R(1) - Num<R>::div_(R(7) * (sz * (R(3) * rr + sz * (sz - R(5) * r))), rr * r + EPS);
            v[1] = (sx * (R(21) * sy * sy + sx * (R(7) * sx - R(35) * sy)) - sy * sy * sy) * a * y + j[1];
            v[2] = j[2] - (sz * sz * sz - R(7) * r * (rr + sz * (R(3) * sz - R(5) * r))) * z * zmul;
            v[0] = a * x * (sx * (R(35) * sy * sy + sx * (sx - R(21) * sy)) - R(7) * sy * sy * sy) + j[0];
            break;
        }
    }
}

// Real Power (HybridFloatPow), uses the squared radius of the last iteration
template <typename R>
__device__ __forceinline__ void f_real_power(R pw, R z_mul, R v[4], const R j[3], R rout) {
    R x = v[0], y = v[1], z = v[2];
    R st, ct, sp, cp;
    Num<R>::sincos_(Num<R>::atan2_(y, x) * pw, &st, &ct);
    Num<R>::sincos_(Num<R>::atan2_(z, Num<R>::sqrt_(x * x + y * y)) * pw, &sp, &cp);
    R r = Num<R>::pow_(rout, pw * R(0.5));
    v[0] = ct * cp * r + j[0];
    v[1] = st * cp * r + j[1];
    v[2] = sp * r * z_mul + j[2];
}

// the KIFS Menger sponge step
template <typename R>
__device__ __forceinline__ void f_menger(R s, R cx, R cy, R cz, R v[4], bool ade) {
    R x = fabs(v[0]), y = fabs(v[1]), z = fabs(v[2]);
    R t;
    if (x < y) { t = x; x = y; y = t; }
    if (x < z) { t = x; x = z; z = t; }
    if (y < z) { t = y; y = z; z = t; }
    R s1 = s - R(1);
    x = s * x - cx * s1;
    y = s * y - cy * s1;
    z = s * z;
    if (z > R(0.5) * cz * s1) z -= cz * s1;
    v[3] = ade ? v[3] * fabs(s) : v[3];
    v[0] = x;
    v[1] = y;
    v[2] = z;
}

// The formula set a kernel is compiled for (FKIND_* bits): the kernels are
// built for a few sets (the scene's set must be inside the kernel's), so
// that a kernel holds only the formulas its scenes use and its loop fits
// the instruction cache.  FKIND_ALL holds every built-in formula.
#define FKIND_IP8 1
#define FKIND_IPN 2
#define FKIND_BOX 4
#define FKIND_MENGER 8
#define FKIND_REAL 16
#define FKIND_TRI 32
#define FKIND_BULBOX 64
#define FKIND_FIP 128
#define FKIND_ALL 255
#define FKIND_QUAT 256  // (only in the all-formula kernels' switch: a 4-component j)
#define FKIND_AEXION 512  // (likewise: it writes j)

// J4: j has four components (the sequential FP64 iteration's record); only
// then is the Quaternion (4D, it reads j's fourth) on the switch -- the
// lock-step DE's j has three, and scenes with a Quaternion never reach it
// aexion_c (src/formulas.rs:640-705), double precision: a real power bulb
// step with the angles as atan2 (theta from the y axis), then with "rotate
// C" the constant replaced by a power of its own angles (it writes j).
// Options: power, z_mul, rot_c, cond_phi, power_c, cz_mul, powc_dist, mode.
__device__ __forceinline__ void f_aexion_c(const DevSlot &s, double v[4], double *j) {
    const double power = s.o[0], z_mul = s.o[1], power_c = s.o[4], cz_mul = s.o[5];
    const bool rot_c = s.o[2] != 0.0, cond_phi = s.o[3] != 0.0, powc_dist = s.o[6] != 0.0;
    const int mode = (int)s.o[7];
    const double x = v[0], y = v[1], z = v[2];
    double r1 = x * x + y * y + z * z;
    const double th = atan2(sqrt(x * x + z * z), y) * power;
    const double ph = atan2(z, x) * power;
    r1 = exp(log(r1) * power * 0.5);
    double st, ct, sp, cp;
    sincos(th, &st, &ct);
    sincos(ph, &sp, &cp);
    v[0] = cp * ct * r1 + j[0];
    v[2] = st * r1 * z_mul + j[2];
    v[1] = ct * sp * r1 + j[1];
    if (!rot_c) return;
    double pd = power_c;
    if (powc_dist) {
        const double d0 = v[0] - j[0], d1 = v[1] - j[1], d2 = v[2] - j[2];
        pd *= sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    }
    const double r = sqrt(j[0] * j[0] + j[1] * j[1] + j[2] * j[2]);
    double a = j[1], b = j[2], c = j[0];
    if (mode & 16) {
        a = v[1] - j[1];
        b = v[2] - j[2];
        c = v[0] - j[0];
    }
    int ofs = 0, ecx = 8;
    if (mode & 8) {
        const double t = a;
        a = b;
        b = t;
        ecx = 16;
    }
    const double sb2 = sqrt(b * b + c * c);
    double tha = (mode & 1) ? atan2(a, sb2) : atan2(sb2, a);
    double pha;
    if (mode & 2) {
        ofs = 24 - ecx;
        pha = atan2(c, b);
    } else {
        pha = atan2(b, c);
    }
    if (mode & 4) {
        const double t = tha;
        tha = pha;
        pha = t;
        ofs = ecx;
    }
    if (cond_phi) {
        const double t = ofs == 0 ? v[0] : ofs == 8 ? v[1] : v[2];
        if (!signbit(t)) pha = -pha;
    }
    double sa, ca, sb, cb;
    sincos(pha * pd, &sa, &ca);
    sincos(tha * pd, &sb, &cb);
    j[0] = ca * cb * r;
    j[2] = sb * r * cz_mul;
    j[1] = cb * sa * r;
}

template <typename R, int FM = FKIND_ALL, bool J4 = false>
__device__ __forceinline__ void formula_iterate(const DevSlot &s, R v[4], R *j, R rout) {
    const bool ade = s.ade != 0;
    if (FM == FKIND_IP8) {
        f_int_pow<R>(8, Num<R>::opt(s, 1), v, j);
        return;
    }
    if ((FM & FKIND_IP8) && s.kind == FKIND_IP8) {
        f_int_pow<R>(8, Num<R>::opt(s, 1), v, j);
        return;
    }
    if ((FM & FKIND_BOX) && s.kind == FKIND_BOX) {
        f_amazing_box<R>(Num<R>::opt(s, 0), Num<R>::opt(s, 1), Num<R>::opt(s, 2), v, j, ade);
        return;
    }
    if ((FM & FKIND_MENGER) && s.kind == FKIND_MENGER) {
        f_menger<R>(Num<R>::opt(s, 0), Num<R>::opt(s, 1), Num<R>::opt(s, 2), Num<R>::opt(s, 3), v, ade);
        return;
    }
    if (FM != FKIND_ALL) return;
    switch (s.formula) {
        case MB3D_CU_F_INTPOW: f_int_pow<R>(s.ipow, Num<R>::opt(s, 1), v, j); break;
        case MB3D_CU_F_AMAZINGBOX:
            f_amazing_box<R>(Num<R>::opt(s, 0), Num<R>::opt(s, 1), Num<R>::opt(s, 2), v, j, ade);
            break;
        case MB3D_CU_F_MENGERIFS:
            f_menger<R>(Num<R>::opt(s, 0), Num<R>::opt(s, 1), Num<R>::opt(s, 2), Num<R>::opt(s, 3), v, ade);
            break;
        case MB3D_CU_F_REALPOWER: f_real_power<R>(Num<R>::opt(s, 0), Num<R>::opt(s, 1), v, j, rout); break;
        case MB3D_CU_F_AEXIONC:
            if constexpr (J4 && sizeof(R) == 8) f_aexion_c(s, v, j);
            break;
        case MB3D_CU_F_QUATERNION:  // src/formulas.rs:580-586
            if constexpr (J4) {
                const R x = v[0], y = v[1], z = v[2], w = v[3];
                v[0] = x * x - y * y - z * z - w * w + j[0];
                v[1] = R(2) * (y * x + z * w) + j[1];
                v[2] = R(2) * (z * x + Num<R>::opt(s, 0) * y * w) + j[2];
                v[3] = R(2) * (w * x + y * z) + Num<R>::opt(s, 1) + j[3];
            }
            break;
        case MB3D_CU_F_TRICORN: {
            R x = v[0], y = v[1], z = v[2];
            v[2] = z * x * Num<R>::opt(s, 0) + j[2] * Num<R>::opt(s, 1);
            v[0] = x * x - (y * y + z * z) + j[0];
            v[1] = R(2) * (y * x) + j[1];
            break;
        }
        case MB3D_CU_F_FOLDINGINTPOW: {
            R fold = Num<R>::opt(s, 2);
            v[0] = box_fold(v[0], fold);
            v[1] = box_fold(v[1], fold);
            v[2] = box_fold(v[2], fold);
            f_int_pow<R>(s.ipow, Num<R>::opt(s, 1), v, j);
            break;
        }
        case MB3D_CU_F_BULBOX: {
            R scale = Num<R>::opt(s, 0), min_r = Num<R>::opt(s, 1), fold = Num<R>::opt(s, 2);
            R bulb = Num<R>::opt(s, 3), t1 = Num<R>::opt(s, 4), t2 = Num<R>::opt(s, 5);
            R rt1 = t1 * t1, rt2 = t2 * t2;
            if (rout < rt1) {
                if (rout < rt2) {
                    f_int_pow2_scale<R>(bulb, v, j);
                } else {
                    R m = Num<R>::div_(rout - rt2, rt1 - rt2);
                    R in0 = v[0], in1 = v[1], in2 = v[2];
                    f_int_pow2_scale<R>(bulb, v, j);
                    R o0 = v[0], o1 = v[1], o2 = v[2];
                    v[0] = in0; v[1] = in1; v[2] = in2;
                    f_amazing_box<R>(scale, min_r, fold, v, j, false);
                    R r1 = Num<R>::sqrt_(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
                    R m2 = R(1) - m;
                    R r2 = r1 * m + m2 * Num<R>::sqrt_(o0 * o0 + o1 * o1 + o2 * o2);
                    v[0] = v[0] * m + m2 * o0;
                    v[1] = v[1] * m + m2 * o1;
                    v[2] = v[2] * m + m2 * o2;
                    R rb = Num<R>::div_(r2, Num<R>::sqrt_(v[0] * v[0] + v[1] * v[1] + v[2] * v[2] + Num<R>::eps()));
                    v[0] *= rb; v[1] *= rb; v[2] *= rb;
                }
            } else {
                f_amazing_box<R>(scale, min_r, fold, v, j, false);
            }
            break;
        }
        default: break;
    }
}

// ---------------------------------------------------------------------------
// Pairs of single precision orbits in the packed FP32 instructions of sm_100
// (FFMA2 / FMUL2 / FADD2: two lanes of arithmetic per instruction).  The
// numeric DE iterates its four orbits in lock-step, so orbits (0, 1) and
// (2, 3) go through the formulas as two float2; the multiply-adds are
// packed, the reciprocals, square roots, absolute values and choices stay
// per orbit.  Each lane is an IEEE single precision operation, as in the
// scalar single precision formulas above (whose contraction the compiler
// chooses).
__device__ __forceinline__ float2 p2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
// a - b (b times -1 is exact: one rounding, as a scalar subtraction)
__device__ __forceinline__ float2 psub(float2 a, float2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ float2 pabs(float2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
__device__ __forceinline__ float2 psq3(const float2 v[3]) { return pfma(v[0], v[0], pfma(v[1], v[1], pmul(v[2], v[2]))); }

// the integer power 8 of f_int_pow (HybridIntP8) on a pair of orbits
__device__ __forceinline__ void f_int_pow8_x2(float zmul, float2 v[3], const float2 j[3]) {
    const float2 x = v[0], y = v[1], z = v[2];
    const float2 xx = pmul(x, x), yy = pmul(y, y), zz = pmul(z, z);
    const float2 r = padd(xx, yy);
    const float2 rr = pmul(r, r);
    const float2 zzzz = pmul(zz, zz);
    float2 sr;  // sqrt(r): r * rsqrt(r), 0 where r is 0 (r * rsqrt(1e-30))
    sr.x = rsqrtf(fmaxf(r.x, 1e-30f));
    sr.y = rsqrtf(fmaxf(r.y, 1e-30f));
    sr = pmul(r, sr);
    // t = (zzzz - 6 r zz + rr) (zz - r) sqrt(r)
    const float2 t = pmul(pmul(padd(pfma(pmul(p2(-6.0f), r), zz, zzzz), rr), psub(zz, r)), sr);
    v[2] = pfma(pmul(pmul(t, z), p2(-8.0f)), p2(zmul), j[2]);
    // a = ((rr 70 + zzzz) zzzz - 28 zz r (zzzz + rr)) / (rr rr + eps) + 1
    const float2 num = pfma(pmul(pmul(p2(-28.0f), zz), r), padd(zzzz, rr), pmul(pfma(rr, p2(70.0f), zzzz), zzzz));
    const float2 den = pfma(rr, rr, p2(1.2e-38f));
    const float2 a = pfma(num, make_float2(__fdividef(1.0f, den.x), __fdividef(1.0f, den.y)), p2(1.0f));
    const float2 xxxx = pmul(xx, xx), yyyy = pmul(yy, yy);
    // v1 = (yyyy (7 xx - yy) + xxxx (xx - 7 yy)) 8 x y a + j1
    const float2 s1 = pfma(yyyy, psub(pmul(p2(7.0f), xx), yy), pmul(xxxx, pfma(p2(-7.0f), yy, xx)));
    v[1] = pfma(pmul(pmul(pmul(s1, p2(8.0f)), x), y), a, j[1]);
    // v0 = a (xxxx xxxx + yyyy (70 xxxx + yyyy) - 28 xx yy (yyyy + xxxx)) + j0
    const float2 s0 = pfma(xxxx, xxxx, pmul(yyyy, pfma(p2(70.0f), xxxx, yyyy)));
    v[0] = pfma(a, pfma(p2(-28.0f), pmul(pmul(xx, yy), padd(yyyy, xxxx)), s0), j[0]);
}

// box_fold on a pair, |x + f| - (|x - f| + x), in the equal form
// t clamp(x, -a, a) - x with a = |f|, t = 2 sign(f) (for f >= 0: x inside the
// fold, 2f - x above, -2f - x below; the sign of f flips |x + f| - |x - f|),
// which has no rounding of its own inside the fold and needs no absolute
// values (the packed instructions take no operand modifiers)
__device__ __forceinline__ float2 box_fold_x2(float2 x, float a, float t) {
    const float2 c = make_float2(fminf(fmaxf(x.x, -a), a), fminf(fmaxf(x.y, -a), a));
    return pfma(c, p2(t), pmul(x, p2(-1.0f)));
}

// the Amazing Box (HybridCube) on a pair of orbits; the numeric DE does not
// use the derivative w, which is left out
__device__ __forceinline__ void f_amazing_box_x2(float scale, float min_r, float fold, float2 v[3], const float2 j[3]) {
    const float fa = fabsf(fold), ft = copysignf(2.0f, fold);
    const float2 x = box_fold_x2(v[0], fa, ft), y = box_fold_x2(v[1], fa, ft), z = box_fold_x2(v[2], fa, ft);
    const float2 r = pfma(x, x, pfma(y, y, pmul(z, z)));
    const float m = fmaxf(min_r, 1.2e-38f), sqr_min_r = m * m;
    // scale / minR^2 below minR^2, scale / r up to 1, scale above: scale /
    // clamp(r, minR^2, 1) (when minR >= 1 the first branch rules, as there)
    float2 mul;
    mul.x = __fdividef(scale, r.x < sqr_min_r ? sqr_min_r : fminf(r.x, 1.0f));
    mul.y = __fdividef(scale, r.y < sqr_min_r ? sqr_min_r : fminf(r.y, 1.0f));
    v[2] = pfma(z, mul, j[2]);
    v[1] = pfma(y, mul, j[1]);
    v[0] = pfma(x, mul, j[0]);
}

// The interpolation hybrid's loop (run_ipol, src/iteration.rs:347-401, 3D):
// both of the first two slots' formulas on the same vector, the results and
// their lengths blended with the normalised weights, the blend scaled to the
// blended length; `de` blends the running derivative (w) of the analytic-DE
// variant.  Every iteration counts; returns the count.
template <typename R, int FM>
__device__ __forceinline__ int ipol_run(const DevParams &p, R v[4], R j[4], R &rout, R &rold, R &otrap, int max_it,
                                        R rstop, bool de) {
    const R s1 = (R)p.ipol_w[0], s2 = (R)p.ipol_w[1];
    const DevSlot &a = p.slots[0], &b = p.slots[1];
    int it = 0;
    for (int guard = 0; guard < (1 << 20); guard++) {
        rold = rout;
        const R y1[4] = {v[0], v[1], v[2], v[3]};
        formula_iterate<R, FM, true>(a, v, j, rout);
        if (a.julia_add) {
            v[0] += j[0];
            v[1] += j[1];
            v[2] += j[2];
        }
        const R x1[4] = {v[0], v[1], v[2], v[3]};
        v[0] = y1[0];
        v[1] = y1[1];
        v[2] = y1[2];
        v[3] = y1[3];
        formula_iterate<R, FM, true>(b, v, j, rout);
        if (b.julia_add) {
            v[0] += j[0];
            v[1] += j[1];
            v[2] += j[2];
        }
        const R x = v[0], y = v[1], z = v[2], w = v[3];
        const bool fd = p.four_d != 0;  // (doInterpolHybridPas4D: four components)
        R xx = fd ? sqrt(x1[0] * x1[0] + x1[1] * x1[1] + x1[2] * x1[2] + x1[3] * x1[3])
                  : sqrt(x1[0] * x1[0] + x1[1] * x1[1] + x1[2] * x1[2]);
        const R yy0 = fd ? sqrt(x * x + y * y + z * z + w * w) : sqrt(x * x + y * y + z * z);
        xx = xx * s1 + yy0 * s2;
        R nv[4] = {x1[0] * s1 + x * s2, x1[1] * s1 + y * s2, x1[2] * s1 + z * s2, x1[3] * s1 + w * s2};
        if (de && !fd) nv[3] = fabs(x1[3]) * s1 + fabs(w) * s2;
        const R l2 = fd ? nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2] + nv[3] * nv[3]
                        : nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2];
        const R q = xx / sqrt(l2 + (R)1e-40);
        v[0] = nv[0] * q;
        v[1] = nv[1] * q;
        v[2] = nv[2] * q;
        v[3] = fd ? nv[3] * q : nv[3];
        it += 1;
        rout = xx * xx;
        if (rout < otrap) otrap = rout;
        if (it >= max_it || rout > rstop) break;
    }
    return it;
}

}  // namespace mb3dcu
