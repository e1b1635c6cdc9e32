// fmath.h -- deterministic single-precision elementary functions, usable in
// host and device code.
//
// The path's shaders call sin, cos, atan2, acos, exp, log, log2 and pow
// (sampling warps, env-map coordinates, vMF lobes, LogLuv, Fresnel, MIS).
// HLSL leaves their accuracy to the platform, so the reference defines no
// bit pattern for them.  The kernels and the CPU restatement both evaluate
// them through this header: every step is an IEEE single-precision operation
// (explicit fmaf where a fused multiply-add is meant, no contraction
// elsewhere), so the same input gives the same bits on the GPU and on the host,
// and a path that takes a branch on one side takes it on the other.
//
// Methods (textbook, no platform library code):
//  * sin/cos: Cody and Waite's additive range reduction by pi/2 with a
//    four-part constant (W. J. Cody, W. Waite, "Software Manual for the
//    Elementary Functions", 1980), then the Taylor series of sin and cos on
//    [-pi/4, pi/4] (terms to x^11 and x^12).
//  * atan2: reduction to [0, 1] by min/max of |x|, |y|, to [0, tan(pi/12)]
//    by atan(a) = pi/6 + atan((sqrt(3) a - 1) / (a + sqrt(3))), Taylor series of
//    atan to a^15; quadrant by the signs.  acos(x) = atan2(sqrt((1-x)(1+x)), x).
//  * log, log2: x = m 2^e with m in [sqrt(1/2), sqrt(2)), ln m = 2 atanh(s),
//    s = (m - 1) / (m + 1), series to s^11; ln 2 split in two parts.
//  * exp, exp2: k = rint(x log2 e) (Cody-Waite with a two-part ln 2), Taylor
//    series of e^r on |r| <= ln(2)/2 to r^9; 2^f = sum (f ln 2)^n / n!.
//  * pow: small integer exponents by repeated multiplication, otherwise
//    2^(y log2 x) with y log2 x carried in two floats.
// Accuracy: within 3 ulp of the correctly rounded result over the ranges the
// path uses (|x| <= 2^12 pi/2 for sin/cos); checked against the host C library
// and against CUDA's functions by the tests.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#if defined(__CUDACC__)
#define FM_HD __host__ __device__ __forceinline__
#else
#define FM_HD inline
#endif

namespace fm {

FM_HD float ffma(float a, float b, float c) {
#if defined(__CUDA_ARCH__)
    return __fmaf_rn(a, b, c);
#else
    return std::fma(a, b, c);
#endif
}
FM_HD uint32_t bits(float x) {
#if defined(__CUDA_ARCH__)
    return __float_as_uint(x);
#else
    uint32_t u;
    std::memcpy(&u, &x, 4);
    return u;
#endif
}
FM_HD float from_bits(uint32_t u) {
#if defined(__CUDA_ARCH__)
    return __uint_as_float(u);
#else
    float x;
    std::memcpy(&x, &u, 4);
    return x;
#endif
}
FM_HD float rint_(float x) {
#if defined(__CUDA_ARCH__)
    return rintf(x);
#else
    return std::rint(x);
#endif
}
FM_HD float fabs_(float x) { return from_bits(bits(x) & 0x7fffffffu); }
FM_HD float copysign_(float x, float s) { return from_bits((bits(x) & 0x7fffffffu) | (bits(s) & 0x80000000u)); }
FM_HD bool isnan_(float x) { return (bits(x) & 0x7fffffffu) > 0x7f800000u; }
FM_HD float qnan() { return from_bits(0x7fc00000u); }
FM_HD float inf() { return from_bits(0x7f800000u); }

// x * 2^k for integer k in [-300, 300] (two exact power-of-two scalings).
FM_HD float ldexp_(float x, int k) {
    if (k > 127) { x = x * from_bits(uint32_t(127 + 127) << 23); k -= 127; if (k > 127) k = 127; }
    if (k < -126) { x = x * from_bits(uint32_t(1) << 23); k += 126; if (k < -126) k = -126; }
    return x * from_bits(uint32_t(k + 127) << 23);
}

// ---------------------------------------------------------------------------
// sin / cos
// ---------------------------------------------------------------------------
constexpr float kTwoOverPi = 0.6366197466850281f;
constexpr float kPio2A = 1.5703125f;                // pi/2, 12 significant bits
constexpr float kPio2B = 0.0004837512969970703f;    // next 12 bits
constexpr float kPio2C = 7.549790126404332e-08f;    // next 24 bits
constexpr float kPio2D = -1.7151245100058819e-15f;  // remainder, rounded

FM_HD float sin_poly(float r) {  // sin(r), |r| <= pi/4
    const float r2 = r * r;
    float p = ffma(r2, -2.5052107943679403e-08f, 2.7557318844628753e-06f);
    p = ffma(r2, p, -0.00019841270113829523f);
    p = ffma(r2, p, 0.008333333767950535f);
    p = ffma(r2, p, -0.1666666716337204f);
    return ffma(r * r2, p, r);
}
FM_HD float cos_poly(float r) {  // cos(r), |r| <= pi/4
    const float r2 = r * r;
    float p = ffma(r2, 2.0876755879584152e-09f, -2.755731998149713e-07f);
    p = ffma(r2, p, 2.4801587642286904e-05f);
    p = ffma(r2, p, -0.0013888889225199819f);
    p = ffma(r2, p, 0.0416666679084301f);
    p = ffma(r2, p, -0.5f);
    return ffma(r2, p, 1.f);
}
// Reduces x to r in [-pi/4, pi/4] and returns the quadrant (0..3).
FM_HD int reduce_pio2(float x, float& r) {
    const float k = rint_(x * kTwoOverPi);
    float t = ffma(-k, kPio2A, x);
    t = ffma(-k, kPio2B, t);
    t = ffma(-k, kPio2C, t);
    r = ffma(-k, kPio2D, t);
    return int(int64_t(k) & 3);
}
FM_HD void sincos(float x, float& s, float& c) {
    if (isnan_(x) || fabs_(x) == inf()) { s = c = qnan(); return; }
    float r;
    const int q = reduce_pio2(x, r);
    const float sr = sin_poly(r), cr = cos_poly(r);
    switch (q) {
        case 0: s = sr; c = cr; break;
        case 1: s = cr; c = -sr; break;
        case 2: s = -sr; c = -cr; break;
        default: s = -cr; c = sr; break;
    }
}
FM_HD float sin(float x) { float s, c; sincos(x, s, c); return s; }
FM_HD float cos(float x) { float s, c; sincos(x, s, c); return c; }

// ---------------------------------------------------------------------------
// atan2 / acos
// ---------------------------------------------------------------------------
constexpr float kPi = 3.1415927410125732f;
constexpr float kPio2 = 1.5707963705062866f;
constexpr float kPio6 = 0.5235987901687622f;
constexpr float kSqrt3 = 1.7320507764816284f;
constexpr float kTanPio12 = 0.2679491937160492f;

FM_HD float atan_poly(float a) {  // atan(a), |a| <= tan(pi/12)
    const float a2 = a * a;
    float p = ffma(a2, -0.06666667014360428f, 0.07692307978868484f);
    p = ffma(a2, p, -0.09090909361839294f);
    p = ffma(a2, p, 0.1111111119389534f);
    p = ffma(a2, p, -0.1428571492433548f);
    p = ffma(a2, p, 0.20000000298023224f);
    p = ffma(a2, p, -0.3333333432674408f);
    return ffma(a * a2, p, a);
}
FM_HD float atan2(float y, float x) {
    if (isnan_(x) || isnan_(y)) return qnan();
    const float ax = fabs_(x), ay = fabs_(y);
    const float mx = ax > ay ? ax : ay, mn = ax > ay ? ay : ax;
    float r;
    if (mx == 0.f) {
        r = 0.f;
    } else if (mx == inf()) {
        r = mn == inf() ? kPio2 * 0.5f : 0.f;
    } else {
        float a = mn / mx;
        float off = 0.f;
        if (a > kTanPio12) {
            a = (a * kSqrt3 - 1.f) / (a + kSqrt3);
            off = kPio6;
        }
        r = off + atan_poly(a);
    }
    if (ay > ax) r = kPio2 - r;
    if (bits(x) & 0x80000000u) r = kPi - r;
    return copysign_(r, y);
}
FM_HD float acos(float x) {
    if (isnan_(x) || fabs_(x) > 1.f) return qnan();
    const float s2 = (1.f - x) * (1.f + x);
#if defined(__CUDA_ARCH__)
    const float s = __fsqrt_rn(s2);
#else
    const float s = std::sqrt(s2);
#endif
    return atan2(s, x);
}

// ---------------------------------------------------------------------------
// log / log2
// ---------------------------------------------------------------------------
constexpr float kLn2Hi = 0.693145751953125f;
constexpr float kLn2Lo = 1.428606765330187e-06f;
constexpr float kLog2eHi = 1.4426950216293335f;
constexpr float kLog2eLo = 1.925963033500011e-08f;
constexpr float kSqrt2 = 1.4142135381698608f;

// x > 0 finite: m in [sqrt(1/2), sqrt(2)) and e with x = m 2^e; returns ln m.
FM_HD float log_reduce(float x, int& e) {
    uint32_t u = bits(x);
    e = 0;
    if (u < 0x00800000u) {  // subnormal
        x = x * 8388608.f;
        u = bits(x);
        e = -23;
    }
    e += int(u >> 23) - 127;
    float m = from_bits((u & 0x007fffffu) | 0x3f800000u);
    if (m > kSqrt2) {
        m = m * 0.5f;
        e += 1;
    }
    const float f = m - 1.f;
    const float s = f / (2.f + f);
    const float s2 = s * s;
    float p = ffma(s2, 0.09090909361839294f, 0.1111111119389534f);
    p = ffma(s2, p, 0.1428571492433548f);
    p = ffma(s2, p, 0.20000000298023224f);
    p = ffma(s2, p, 0.3333333432674408f);
    const float t = s + s;
    return ffma(t * s2, p, t);
}
FM_HD float log(float x) {
    if (isnan_(x) || x < 0.f) return qnan();
    if (x == 0.f) return -inf();
    if (x == inf()) return x;
    int e;
    const float lm = log_reduce(x, e);
    const float fe = float(e);
    return ffma(fe, kLn2Hi, ffma(fe, kLn2Lo, lm));
}
// log2 x as an unevaluated sum hi + lo (x > 0 finite).
FM_HD float log2_ext(float x, float& lo) {
    int e;
    const float lm = log_reduce(x, e);
    const float t = ffma(lm, kLog2eHi, lm * kLog2eLo);
    const float fe = float(e);
    const float hi = fe + t;
    lo = t - (hi - fe);  // exact remainder: |t| < 1 <= |e| or e == 0
    return hi;
}
FM_HD float log2(float x) {
    if (isnan_(x) || x < 0.f) return qnan();
    if (x == 0.f) return -inf();
    if (x == inf()) return x;
    float lo;
    return log2_ext(x, lo);
}

// ---------------------------------------------------------------------------
// exp / exp2 / pow
// ---------------------------------------------------------------------------
FM_HD float exp(float x) {
    if (isnan_(x)) return x;
    if (x > 88.72284f) return inf();
    if (x < -103.97208f) return 0.f;
    const float k = rint_(x * kLog2eHi);
    float r = ffma(-k, kLn2Hi, x);
    r = ffma(-k, kLn2Lo, r);
    float p = ffma(r, 2.7557318844628753e-06f, 2.4801587642286904e-05f);
    p = ffma(r, p, 0.00019841270113829523f);
    p = ffma(r, p, 0.0013888889225199819f);
    p = ffma(r, p, 0.008333333767950535f);
    p = ffma(r, p, 0.0416666679084301f);
    p = ffma(r, p, 0.1666666716337204f);
    p = ffma(r, p, 0.5f);
    p = ffma(r, p, 1.f);
    p = ffma(r, p, 1.f);
    return ldexp_(p, int(k));
}
// 2^(k + f), |f| <= ~1/2.
FM_HD float exp2_kf(float k, float f) {
    float p = ffma(f, 1.0178086284895471e-07f, 1.3215486660556053e-06f);
    p = ffma(f, p, 1.5252733646775596e-05f);
    p = ffma(f, p, 0.0001540352968731895f);
    p = ffma(f, p, 0.0013333557872101665f);
    p = ffma(f, p, 0.009618128649890423f);
    p = ffma(f, p, 0.05550410971045494f);
    p = ffma(f, p, 0.24022650718688965f);
    p = ffma(f, p, 0.6931471824645996f);
    p = ffma(f, p, 1.f);
    return ldexp_(p, int(k));
}
FM_HD float exp2(float x) {
    if (isnan_(x)) return x;
    if (x >= 128.f) return inf();
    if (x < -150.f) return 0.f;
    const float k = rint_(x);
    return exp2_kf(k, x - k);  // x - k exact
}
// x^n for an integer 1 <= n <= 8, multiplied left to right.
FM_HD float ipow(float x, int n) {
    float r = x;
    for (int i = 1; i < n; i++) r = r * x;
    return r;
}
// x^y for finite x > 0 and y not handled by the integer path.
FM_HD float pow_pos(float x, float y) {
    if (x == 1.f) return 1.f;
    if (x == inf()) return y > 0.f ? inf() : 0.f;
    // y log2 x carried as hi + lo so that the exponent keeps its low bits.
    float lo;
    const float hi = log2_ext(x, lo);
    const float zh = y * hi;
    const float zl = ffma(y, hi, -zh) + y * lo;
    if (zh >= 128.f) return inf();
    if (zh < -150.f) return 0.f;
    const float k = rint_(zh);
    return exp2_kf(k, (zh - k) + zl);
}
FM_HD float pow(float x, float y) {
    if (y == 0.f) return 1.f;
    if (isnan_(x) || isnan_(y)) return qnan();
    const bool yInt = rint_(y) == y;
    if (yInt && y >= 1.f && y <= 8.f) return ipow(x, int(y));
    if (x == 0.f) return y > 0.f ? 0.f : inf();
    if (x < 0.f) {
        if (!yInt) return qnan();
        const float a = pow_pos(-x, y);
        const bool odd = fabs_(y) < 16777216.f && (int64_t(y) & 1) != 0;
        return odd ? -a : a;
    }
    return pow_pos(x, y);
}

}  // namespace fm
