// oracle_math.h -- CPU restatement of the Slang math, sampling, RNG and BSDF
// code on Falcor's path-tracing hot path.
//
// TEST INFRASTRUCTURE ONLY.  This is the correctness oracle: it is used by the
// tests, by smoke() as a checker and by bench.py's cpu_baseline leg.  It is
// never part of the product path.
//
// Every function restates the reference Slang function named in its comment
// (paths relative to the Falcor source tree).  Everything is templated on the
// real type R: R = float is the FP32 parity oracle (compiled with
// -ffp-contract=off so that no multiply-add is contracted, matching the
// uncontracted GPU build), R = double is the FP64 "truth" used for converged
// RMSE.  Integer code (RNG, hashing, packing) is exact.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <algorithm>
#include <limits>

#include "oracle_dual.h"
#include "../falcor_b200/csrc/fmath.h"

namespace orc {
// Elementary functions of the restatement.  Single precision goes through the
// deterministic functions the kernels use (falcor_b200/csrc/fmath.h: HLSL
// leaves their last bits to the platform, so both sides fix one definition);
// double and the derivative types use the C library.
template <class R> inline R el_sin(const R& x) { return std::sin(x); }
template <class R> inline R el_cos(const R& x) { return std::cos(x); }
template <class R> inline R el_exp(const R& x) { return std::exp(x); }
template <class R> inline R el_log(const R& x) { return std::log(x); }
template <class R> inline R el_log2(const R& x) { return std::log2(x); }
template <class R> inline R el_atan2(const R& y, const R& x) { return std::atan2(y, x); }
template <class R> inline R el_acos(const R& x) { return std::acos(x); }
template <class R> inline R el_pow(const R& x, const R& y) { return std::pow(x, y); }
inline float el_sin(float x) { return fm::sin(x); }
inline float el_cos(float x) { return fm::cos(x); }
inline float el_exp(float x) { return fm::exp(x); }
inline float el_log(float x) { return fm::log(x); }
inline float el_log2(float x) { return fm::log2(x); }
inline float el_atan2(float y, float x) { return fm::atan2(y, x); }
inline float el_acos(float x) { return fm::acos(x); }
inline float el_pow(float x, float y) { return fm::pow(x, y); }
}  // namespace orc

namespace orc {

// ---------------------------------------------------------------------------
// Vector types with HLSL/Slang semantics: component-wise, left-to-right
// evaluation, no contraction.
// ---------------------------------------------------------------------------
template <class R> struct V2 {
    R x, y;
    V2() : x(0), y(0) {}
    V2(R a, R b) : x(a), y(b) {}
    explicit V2(R a) : x(a), y(a) {}
};
template <class R> struct V3 {
    R x, y, z;
    V3() : x(0), y(0), z(0) {}
    V3(R a, R b, R c) : x(a), y(b), z(c) {}
    explicit V3(R a) : x(a), y(a), z(a) {}
    R operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    R& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};
template <class R> struct V4 {
    R x, y, z, w;
    V4() : x(0), y(0), z(0), w(0) {}
    V4(R a, R b, R c, R d) : x(a), y(b), z(c), w(d) {}
};

#define ORC_V3_BINOP(op)                                                                   \
    template <class R> inline V3<R> operator op(const V3<R>& a, const V3<R>& b) {         \
        return V3<R>(a.x op b.x, a.y op b.y, a.z op b.z);                                  \
    }                                                                                      \
    template <class R> inline V3<R> operator op(const V3<R>& a, R s) {                    \
        return V3<R>(a.x op s, a.y op s, a.z op s);                                        \
    }                                                                                      \
    template <class R> inline V3<R> operator op(R s, const V3<R>& a) {                    \
        return V3<R>(s op a.x, s op a.y, s op a.z);                                        \
    }
ORC_V3_BINOP(+)
ORC_V3_BINOP(-)
ORC_V3_BINOP(*)
ORC_V3_BINOP(/)
#undef ORC_V3_BINOP
template <class R> inline V3<R> operator-(const V3<R>& a) { return V3<R>(-a.x, -a.y, -a.z); }
template <class R> inline V3<R>& operator+=(V3<R>& a, const V3<R>& b) { a = a + b; return a; }
template <class R> inline V3<R>& operator*=(V3<R>& a, const V3<R>& b) { a = a * b; return a; }
template <class R> inline V3<R>& operator*=(V3<R>& a, R s) { a = a * s; return a; }
template <class R> inline V3<R>& operator/=(V3<R>& a, R s) { a = a / s; return a; }

template <class R> inline V2<R> operator+(const V2<R>& a, const V2<R>& b) { return V2<R>(a.x + b.x, a.y + b.y); }
template <class R> inline V2<R> operator-(const V2<R>& a, const V2<R>& b) { return V2<R>(a.x - b.x, a.y - b.y); }
template <class R> inline V2<R> operator*(const V2<R>& a, R s) { return V2<R>(a.x * s, a.y * s); }
template <class R> inline V2<R> operator*(R s, const V2<R>& a) { return V2<R>(s * a.x, s * a.y); }

template <class R> inline R dot(const V3<R>& a, const V3<R>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline R dot(const V2<R>& a, const V2<R>& b) { return a.x * b.x + a.y * b.y; }
template <class R> inline V3<R> cross(const V3<R>& a, const V3<R>& b) {
    return V3<R>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <class R> inline R length(const V3<R>& a) { return std::sqrt(dot(a, a)); }
// normalize(v) = v / length(v).  Defined with an IEEE divide and square root
// so that the FP32 result is bit-identical on CPU and GPU.
template <class R> inline V3<R> normalize(const V3<R>& a) { R l = std::sqrt(dot(a, a)); return a / l; }
template <class R> inline V3<R> vabs(const V3<R>& a) { return V3<R>(std::fabs(a.x), std::fabs(a.y), std::fabs(a.z)); }
template <class R> inline R vmin(R a, R b) { return a < b ? a : b; }   // HLSL min (NaN-agnostic)
template <class R> inline R vmax(R a, R b) { return a > b ? a : b; }
template <class R> inline V3<R> vmax(const V3<R>& a, R b) { return V3<R>(vmax(a.x, b), vmax(a.y, b), vmax(a.z, b)); }
template <class R> inline R saturate(R v) { return v < R(0) ? R(0) : (v > R(1) ? R(1) : v); }
template <class R> inline R sgn(R v) { return v > R(0) ? R(1) : (v < R(0) ? R(-1) : R(0)); }
// HLSL lerp(a, b, t) = a + t * (b - a).
template <class R> inline R lerp(R a, R b, R t) { return a + t * (b - a); }
template <class R> inline V3<R> lerp(const V3<R>& a, const V3<R>& b, R t) { return a + t * (b - a); }
template <class R> inline bool any_pos(const V3<R>& a) { return a.x > R(0) || a.y > R(0) || a.z > R(0); }
template <class R> inline bool any_nan(const V3<R>& a) { return std::isnan(a.x) || std::isnan(a.y) || std::isnan(a.z); }
template <class R> inline V3<R> cvt3(const V3<float>& a) { return V3<R>(R(a.x), R(a.y), R(a.z)); }
inline V3<float> tof(const V3<float>& a) { return a; }
inline V3<float> tof(const V3<double>& a) { return V3<float>(float(a.x), float(a.y), float(a.z)); }

// Constants as Slang sees them: unsuffixed literals take the precision of the
// other operand (Utils/Math/MathConstants.slangh:56-117).
template <class R> struct K {
    static constexpr R pi = R(3.14159265358979323846);
    static constexpr R pi_2 = R(1.57079632679489661923);
    static constexpr R pi_4 = R(0.785398163397448309616);
    static constexpr R inv_pi = R(0.318309886183790671538);
    static constexpr R two_pi = R(6.28318530717958647693);
    static constexpr R inv_2pi = R(0.159154943091895335769);
    static constexpr R two_over_pi = R(0.636619772367581343076);
    static constexpr R four_pi = R(12.5663706143591729539);
    static constexpr R inv_4pi = R(0.079577471545947667884);
};

inline uint32_t asuint(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float asfloat(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }
inline int32_t asint(float f) { int32_t i; std::memcpy(&i, &f, 4); return i; }
inline float asfloat_i(int32_t i) { float f; std::memcpy(&f, &i, 4); return f; }

// ---------------------------------------------------------------------------
// fp16 conversions.
// Host-side quantisation (material and vertex packing on the CPU) follows
// Falcor's float32ToFloat16 (Utils/Math/Float16.cpp:56-169): round to nearest,
// ties away from zero on the magnitude bits.  Device f16tof32 is exact.
// ---------------------------------------------------------------------------
inline uint16_t f32tof16_host(float value) {
    const uint32_t bits = asuint(value);
    const int32_t sign = int32_t((bits >> 16) & 0x8000u);
    int32_t exp = int32_t((bits >> 23) & 0xffu) - (127 - 15);
    int32_t man = int32_t(bits & 0x007fffffu);
    if (exp <= 0) {
        if (exp < -10) return uint16_t(sign);
        man = (man | 0x00800000) >> (1 - exp);
        if (man & 0x00001000) man += 0x00002000;
        return uint16_t(sign | (man >> 13));
    }
    if (exp == 0xff - (127 - 15)) {
        if (man == 0) return uint16_t(sign | 0x7c00);
        man >>= 13;
        return uint16_t(sign | 0x7c00 | man | (man == 0));
    }
    if (man & 0x00001000) {
        man += 0x00002000;
        if (man & 0x00800000) { man = 0; exp += 1; }
    }
    if (exp > 30) return uint16_t(sign | 0x7c00);
    return uint16_t(sign | (exp << 10) | (man >> 13));
}
inline float f16tof32(uint32_t h) {
    h &= 0xffffu;
    const uint32_t sign = (h & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1fu;
    uint32_t man = h & 0x3ffu;
    uint32_t out;
    if (exp == 0) {
        if (man == 0) {
            out = sign;
        } else {  // subnormal half -> normal float
            int e = -1;
            do { e++; man <<= 1; } while ((man & 0x400u) == 0);
            man &= 0x3ffu;
            out = sign | (uint32_t(127 - 15 - e) << 23) | (man << 13);
        }
    } else if (exp == 31) {
        out = sign | 0x7f800000u | (man << 13);
    } else {
        out = sign | ((exp + (127 - 15)) << 23) | (man << 13);
    }
    return asfloat(out);
}
inline float quantize_f16(float v) { return f16tof32(f32tof16_host(v)); }

// ---------------------------------------------------------------------------
// Snorm / octahedral normal packing (Utils/Math/FormatConversion.h:45-90,
// Utils/Math/PackedFormats.slang:53-66, Utils/Math/MathHelpers.slang:156-194).
// ---------------------------------------------------------------------------
inline int32_t float_to_snorm16(float v) {
    v = std::isnan(v) ? 0.f : std::min(std::max(v, -1.f), 1.f);
    return int32_t(std::trunc(v * 32767.f + (v >= 0.f ? 0.5f : -0.5f)));
}
inline uint32_t pack_snorm2x16(float x, float y) {
    return (uint32_t(float_to_snorm16(x)) & 0xffffu) | (uint32_t(float_to_snorm16(y)) << 16);
}
inline V2<float> unpack_snorm2x16(uint32_t p) {
    int32_t bx = int32_t(p << 16) >> 16;
    int32_t by = int32_t(p) >> 16;
    return V2<float>(std::max(float(bx) / 32767.f, -1.f), std::max(float(by) / 32767.f, -1.f));
}
inline V2<float> oct_wrap(V2<float> v) {
    return V2<float>((1.f - std::fabs(v.y)) * (v.x >= 0.f ? 1.f : -1.f),
                     (1.f - std::fabs(v.x)) * (v.y >= 0.f ? 1.f : -1.f));
}
inline V2<float> ndir_to_oct_snorm(V3<float> n) {
    float s = 1.f / (std::fabs(n.x) + std::fabs(n.y) + std::fabs(n.z));
    V2<float> p(n.x * s, n.y * s);
    return (n.z < 0.f) ? oct_wrap(p) : p;
}
inline V3<float> oct_to_ndir_snorm(V2<float> p) {
    V3<float> n(p.x, p.y, 1.f - std::fabs(p.x) - std::fabs(p.y));
    if (n.z < 0.f) { V2<float> w = oct_wrap(V2<float>(n.x, n.y)); n.x = w.x; n.y = w.y; }
    return normalize(n);
}
inline uint32_t encode_normal2x16(V3<float> n) { V2<float> o = ndir_to_oct_snorm(n); return pack_snorm2x16(o.x, o.y); }
inline V3<float> decode_normal2x16(uint32_t p) { return oct_to_ndir_snorm(unpack_snorm2x16(p)); }

// ---------------------------------------------------------------------------
// Bit tricks and hashes (Utils/Math/BitTricks.slang:47-110,
// Utils/Math/HashUtils.slang:39-74).
// ---------------------------------------------------------------------------
inline uint32_t interleave_32bit(uint32_t vx, uint32_t vy) {
    uint32_t x = vx & 0x0000ffffu;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    uint32_t y = vy & 0x0000ffffu;
    y = (y | (y << 8)) & 0x00FF00FFu;
    y = (y | (y << 4)) & 0x0F0F0F0Fu;
    y = (y | (y << 2)) & 0x33333333u;
    y = (y | (y << 1)) & 0x55555555u;
    return x | (y << 1);
}
inline uint32_t interleave_16bit(uint32_t vx, uint32_t vy) {
    vx &= 0xffu; vy &= 0xffu;
    uint32_t j = (vy << 16) | vx;
    j = (j ^ (j << 4)) & 0x0f0f0f0fu;
    j = (j ^ (j << 2)) & 0x33333333u;
    j = (j ^ (j << 1)) & 0x55555555u;
    return (j >> 15) | (j & 0xffffu);
}
inline void deinterleave_16bit(uint32_t i, uint32_t& x, uint32_t& y) {
    uint32_t j = ((i >> 1) << 16) | i;
    j &= 0x55555555u;
    j = (j ^ (j >> 1)) & 0x33333333u;
    j = (j ^ (j >> 2)) & 0x0f0f0f0fu;
    j = (j ^ (j >> 4)) & 0x00ff00ffu;
    x = j & 0xffu; y = j >> 16;
}
inline void deinterleave_8bit(uint32_t i, uint32_t& x, uint32_t& y) {
    uint32_t j = ((i >> 1) << 8) | i;
    j &= 0x00005555u;
    j = (j ^ (j >> 1)) & 0x33333333u;
    j = (j ^ (j >> 2)) & 0x0f0f0f0fu;
    x = j & 0xfu; y = j >> 8;
}
inline void deinterleave_2x8bit(uint32_t i, uint32_t& x, uint32_t& y) {
    uint32_t j = ((i & ~0x00010001u) << 7) | i;
    j &= 0x55555555u;
    j = (j ^ (j >> 1)) & 0x33333333u;
    j = (j ^ (j >> 2)) & 0x0f0f0f0fu;
    x = j & 0x000f000fu; y = (j >> 8) & 0x000f000fu;
}
inline uint32_t jenkins_hash(uint32_t a) {
    a = (a + 0x7ed55d16u) + (a << 12);
    a = (a ^ 0xc761c23cu) ^ (a >> 19);
    a = (a + 0x165667b1u) + (a << 5);
    a = (a + 0xd3a2646cu) ^ (a << 9);
    a = (a + 0xfd7046c5u) + (a << 3);
    a = (a ^ 0xb55a4f09u) ^ (a >> 16);
    return a;
}
inline void block_cipher_tea(uint32_t v0, uint32_t v1, uint32_t& o0, uint32_t& o1, uint32_t iterations = 16) {
    uint32_t sum = 0;
    const uint32_t delta = 0x9e3779b9u;
    const uint32_t k0 = 0xa341316cu, k1 = 0xc8013ea4u, k2 = 0xad90777du, k3 = 0x7e95761eu;
    for (uint32_t i = 0; i < iterations; i++) {
        sum += delta;
        v0 += ((v1 << 4) + k0) ^ (v1 + sum) ^ ((v1 >> 5) + k1);
        v1 += ((v0 << 4) + k2) ^ (v0 + sum) ^ ((v0 >> 5) + k3);
    }
    o0 = v0; o1 = v1;
}

// ---------------------------------------------------------------------------
// Pseudorandom generators (Utils/Sampling/Pseudorandom/{Xoshiro,SplitMix64,
// LCG}.slang) and the two sample generators
// (UniformSampleGenerator.slang:53-78, TinyUniformSampleGenerator.slang:51-71).
// ---------------------------------------------------------------------------
struct SplitMix64 {
    uint64_t state;
    uint64_t next64() {
        uint64_t z = (state += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    static SplitMix64 create(uint32_t s0, uint32_t s1) { return SplitMix64{(uint64_t(s1) << 32) | uint64_t(s0)}; }
};
struct Xoshiro128 {
    uint32_t s[4];
    static uint32_t rotl(uint32_t x, int k) { return (x << k) | (x >> (32 - k)); }
    uint32_t next() {
        const uint32_t result = rotl(s[0] * 5u, 7) * 9u;
        const uint32_t t = s[1] << 9;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 11);
        return result;
    }
};
struct LCG {
    uint32_t state;
    uint32_t next() { state = 1664525u * state + 1013904223u; return state; }
};

// SAMPLE_GENERATOR_UNIFORM: SplitMix64(interleave(pixel), sampleNumber) -> xoshiro128**.
struct UniformSG {
    Xoshiro128 rng;
    UniformSG(uint32_t px, uint32_t py, uint32_t sampleNumber) {
        SplitMix64 sm = SplitMix64::create(interleave_32bit(px, py), sampleNumber);
        uint64_t s0 = sm.next64();
        uint64_t s1 = sm.next64();
        rng.s[0] = uint32_t(s0); rng.s[1] = uint32_t(s0 >> 32);
        rng.s[2] = uint32_t(s1); rng.s[3] = uint32_t(s1 >> 32);
    }
    uint32_t next() { return rng.next(); }
};
// SAMPLE_GENERATOR_TINY_UNIFORM: LCG seeded with blockCipherTEA(interleave(pixel), sampleNumber).x.
struct TinyUniformSG {
    LCG rng;
    TinyUniformSG(uint32_t px, uint32_t py, uint32_t sampleNumber) {
        uint32_t a, b;
        block_cipher_tea(interleave_32bit(px, py), sampleNumber, a, b);
        rng.state = a;
    }
    uint32_t next() { return rng.next(); }
};

// sampleNext1D/2D (SampleGeneratorInterface.slang:50-65): upper 24 bits * 2^-24,
// x drawn before y.
template <class R, class SG> inline R next1D(SG& sg) { uint32_t bits = sg.next(); return R(float(bits >> 8) * 0x1p-24f); }
template <class R, class SG> inline V2<R> next2D(SG& sg) { V2<R> s; s.x = next1D<R>(sg); s.y = next1D<R>(sg); return s; }

// ---------------------------------------------------------------------------
// Color (Utils/Color/ColorHelpers.slang:42-81) and LogLuv
// (Utils/Math/PackedFormats.slang:125-200).
// ---------------------------------------------------------------------------
template <class R> inline R luminance(const V3<R>& c) { return dot(c, V3<R>(R(0.2126f), R(0.7152f), R(0.0722f))); }

inline uint32_t encode_logluv_hdr(V3<float> c) {
    const float X = 0.4123907992659595f * c.x + 0.3575843393838780f * c.y + 0.1804807884018343f * c.z;
    const float Y = 0.2126390058715104f * c.x + 0.7151686787677559f * c.y + 0.0721923153607337f * c.z;
    const float Z = 0.0193308187155918f * c.x + 0.1191947797946259f * c.y + 0.9505321522496608f * c.z;
    float logY = 409.6f * (el_log2(Y) + 20.f);
    float cl = std::min(std::max(logY, 0.f), 16383.f);
    if (std::isnan(logY)) cl = 0.f;
    uint32_t Le = uint32_t(cl);
    if (Le == 0) return 0;
    float invDenom = 1.f / (-2.f * X + 12.f * Y + 3.f * (X + Y + Z));
    float u = 4.f * X * invDenom;
    float v = 9.f * Y * invDenom;
    uint32_t ue = uint32_t(std::min(std::max(820.f * u, 0.f), 511.f));
    uint32_t ve = uint32_t(std::min(std::max(820.f * v, 0.f), 511.f));
    return (Le << 18) | (ue << 9) | ve;
}
inline V3<float> decode_logluv_hdr(uint32_t p) {
    uint32_t Le = p >> 18;
    if (Le == 0) return V3<float>(0.f);
    float logY = (float(Le) + 0.5f) / 409.6f - 20.f;
    float Y = el_pow(2.f, logY);
    float u = (float((p >> 9) & 0x1ffu) + 0.5f) / 820.f;
    float v = (float(p & 0x1ffu) + 0.5f) / 820.f;
    float invDenom = 1.f / (6.f * u - 16.f * v + 12.f);
    float x = 9.f * u * invDenom;
    float y = 4.f * v * invDenom;
    float s = Y / y;
    float X = s * x, Z = s * (1.f - x - y);
    V3<float> rgb(3.240969941904522f * X + -1.537383177570094f * Y + -0.4986107602930032f * Z,
                  -0.9692436362808803f * X + 1.875967501507721f * Y + 0.04155505740717569f * Z,
                  0.05563007969699373f * X + -0.2039769588889765f * Y + 1.056971514242878f * Z);
    return vmax(rgb, 0.f);
}

// ---------------------------------------------------------------------------
// Sampling warps (Utils/Math/MathHelpers.slang:111-411).
// ---------------------------------------------------------------------------
template <class R> inline V2<R> sample_disk_concentric(V2<R> u) {
    u = V2<R>(R(2) * u.x - R(1), R(2) * u.y - R(1));
    if (u.x == R(0) && u.y == R(0)) return u;
    R phi, r;
    if (std::fabs(u.x) > std::fabs(u.y)) {
        r = u.x;
        phi = (u.y / u.x) * K<R>::pi_4;
    } else {
        r = u.y;
        phi = K<R>::pi_2 - (u.x / u.y) * K<R>::pi_4;
    }
    return V2<R>(r * el_cos(phi), r * el_sin(phi));
}
template <class R> inline V3<R> sample_cosine_hemisphere_concentric(V2<R> u, R& pdf) {
    V2<R> d = sample_disk_concentric(u);
    R z = std::sqrt(vmax(R(0), R(1) - dot(d, d)));
    pdf = z * K<R>::inv_pi;
    return V3<R>(d.x, d.y, z);
}
template <class R> inline V3<R> sample_triangle(V2<R> u) {
    R su = std::sqrt(u.x);
    R bx = R(1) - su, by = u.y * su;
    return V3<R>(R(1) - bx - by, bx, by);
}
template <class R> inline V3<R> sample_von_mises_fisher(V2<R> u, R kappa) {
    R sy = vmax(R(1) - u.y, R(1e-6f));
    R phi = K<R>::two_pi * u.x;
    R cosTheta = R(1) + el_log(el_exp(R(-2) * kappa) * (R(1) - sy) + sy) / kappa;
    R sinTheta = std::sqrt(R(1) - cosTheta * cosTheta);
    return V3<R>(el_cos(phi) * sinTheta, el_sin(phi) * sinTheta, cosTheta);
}
template <class R> inline V2<R> world_to_latlong_map(V3<R> dir) {
    V3<R> p = normalize(dir);
    V2<R> uv;
    uv.x = el_atan2(p.x, -p.z) * K<R>::inv_2pi + R(0.5f);
    uv.y = el_acos(p.y) * K<R>::inv_pi;
    return uv;
}
template <class R> inline V2<R> ndir_to_oct_equal_area_unorm(V3<R> n) {
    R r = std::sqrt(R(1) - std::fabs(n.z));
    R phi = el_atan2(R(std::fabs(n.y)), R(std::fabs(n.x)));
    V2<R> p;
    p.y = r * phi * K<R>::two_over_pi;
    p.x = r - p.y;
    if (n.z < R(0)) p = V2<R>(R(1) - p.y, R(1) - p.x);
    p.x *= sgn(n.x);
    p.y *= sgn(n.y);
    return V2<R>(p.x * R(0.5f) + R(0.5f), p.y * R(0.5f) + R(0.5f));
}
template <class R> inline V3<R> oct_to_ndir_equal_area_unorm(V2<R> p) {
    p = V2<R>(p.x * R(2) - R(1), p.y * R(2) - R(1));
    R d = R(1) - (std::fabs(p.x) + std::fabs(p.y));
    R r = R(1) - std::fabs(d);
    R phi = (r > R(0)) ? ((std::fabs(p.y) - std::fabs(p.x)) / r + R(1)) * K<R>::pi_4 : R(0);
    R f = r * std::sqrt(R(2) - r * r);
    R x = f * sgn(p.x) * el_cos(phi);
    R y = f * sgn(p.y) * el_sin(phi);
    R z = sgn(d) * (R(1) - r * r);
    return V3<R>(x, y, z);
}
// perp_stark (Utils/Math/MathHelpers.slang:540-551).
template <class R> inline V3<R> perp_stark(V3<R> u) {
    V3<R> a = vabs(u);
    uint32_t uyx = (a.x - a.y) < R(0) ? 1u : 0u;
    uint32_t uzx = (a.x - a.z) < R(0) ? 1u : 0u;
    uint32_t uzy = (a.y - a.z) < R(0) ? 1u : 0u;
    uint32_t xm = uyx & uzx;
    uint32_t ym = (1u ^ xm) & uzy;
    uint32_t zm = 1u ^ (xm | ym);
    return normalize(cross(u, V3<R>(R(xm), R(ym), R(zm))));
}

// ---------------------------------------------------------------------------
// Ray origin offset (Utils/Geometry/GeometryHelpers.slang:51-68), FP32 only:
// the integer ULP offset is defined on the fp32 bit pattern.
// ---------------------------------------------------------------------------
inline V3<float> compute_ray_origin(V3<float> pos, V3<float> normal) {
    const float origin = 1.f / 16.f;
    const float fScale = 3.f / 65536.f;
    const float iScale = 3 * 256.f;
    V3<float> out;
    for (int i = 0; i < 3; i++) {
        int32_t iOff = int32_t(normal[i] * iScale);
        float iPos = asfloat_i(asint(pos[i]) + (pos[i] < 0.f ? -iOff : iOff));
        float fOff = normal[i] * fScale;
        out[i] = std::fabs(pos[i]) < origin ? pos[i] + fOff : iPos;
    }
    return out;
}
inline V3<double> compute_ray_origin(V3<double> pos, V3<double> normal) {
    V3<float> r = compute_ray_origin(tof(pos), tof(normal));
    return V3<double>(r.x, r.y, r.z);
}

// ---------------------------------------------------------------------------
// Watertight ray/triangle test (Utils/Geometry/IntersectionHelpers.slang:118-189).
// Vertices and ray are fp32 scene data; the arithmetic is done in R.
// ---------------------------------------------------------------------------
template <class R>
inline bool intersect_ray_triangle(const V3<R>& ro, const V3<R>& rd, const V3<R> v[3], V3<R>& bary, R& t) {
    bary = V3<R>(0); t = R(0);
    const V3<R> ad = vabs(rd);
    uint32_t axis = 0;
    if (ad.y > ad.x && ad.y > ad.z) axis = 1;
    if (ad.z > ad.x && ad.z > ad.y) axis = 2;
    uint32_t kz = axis, kx = (kz + 1) % 3, ky = (kx + 1) % 3;
    if (rd[kz] < R(0)) std::swap(kx, ky);
    R Sx = rd[kx] / rd[kz];
    R Sy = rd[ky] / rd[kz];
    R Sz = R(1) / rd[kz];
    const V3<R> A = v[0] - ro, B = v[1] - ro, C = v[2] - ro;
    const R Ax = A[kx] - Sx * A[kz];
    const R Ay = A[ky] - Sy * A[kz];
    const R Bx = B[kx] - Sx * B[kz];
    const R By = B[ky] - Sy * B[kz];
    const R Cx = C[kx] - Sx * C[kz];
    const R Cy = C[ky] - Sy * C[kz];
    R U = Cx * By - Cy * Bx;
    R V = Ax * Cy - Ay * Cx;
    R W = Bx * Ay - By * Ax;
    if (U == R(0) || V == R(0) || W == R(0)) {
        double CxBy = double(Cx) * double(By), CyBx = double(Cy) * double(Bx);
        U = R(CxBy - CyBx);
        double AxCy = double(Ax) * double(Cy), AyCx = double(Ay) * double(Cx);
        V = R(AxCy - AyCx);
        double BxAy = double(Bx) * double(Ay), ByAx = double(By) * double(Ax);
        W = R(BxAy - ByAx);
    }
    if ((U < R(0) || V < R(0) || W < R(0)) && (U > R(0) || V > R(0) || W > R(0))) return false;
    R det = U + V + W;
    if (det == R(0)) return false;
    const R Az = Sz * A[kz], Bz = Sz * B[kz], Cz = Sz * C[kz];
    const R T = U * Az + V * Bz + W * Cz;
    const R rcpDet = R(1) / det;
    t = T * rcpDet;
    bary = V3<R>(U * rcpDet, V * rcpDet, W * rcpDet);
    return true;
}

// ---------------------------------------------------------------------------
// GGX microfacet model (Rendering/Materials/IsotropicGGX.slang:46-206) and
// Fresnel (Rendering/Materials/Fresnel.slang:42-51).
// ---------------------------------------------------------------------------
template <class R> inline R pw(R a, R b) { return el_pow(a, b); }

template <class R> inline R eval_ndf_ggx(R alpha, R cosTheta) {
    R a2 = alpha * alpha;
    R d = ((cosTheta * a2 - cosTheta) * cosTheta + R(1));
    return a2 / (d * d * K<R>::pi);
}
template <class R> inline R eval_g1_ggx(R alphaSqr, R cosTheta) {
    if (cosTheta <= R(0)) return R(0);
    R c2 = cosTheta * cosTheta;
    R tan2 = vmax(R(1) - c2, R(0)) / c2;
    return R(2) / (R(1) + std::sqrt(R(1) + alphaSqr * tan2));
}
template <class R> inline R eval_lambda_ggx(R alphaSqr, R cosTheta) {
    if (cosTheta <= R(0)) return R(0);
    R c2 = cosTheta * cosTheta;
    R tan2 = vmax(R(1) - c2, R(0)) / c2;
    return R(0.5f) * (R(-1) + std::sqrt(R(1) + alphaSqr * tan2));
}
template <class R> inline R eval_masking_smith_ggx_correlated(R alpha, R cosI, R cosO) {
    R a2 = alpha * alpha;
    R li = eval_lambda_ggx(a2, cosI);
    R lo = eval_lambda_ggx(a2, cosO);
    return R(1) / (R(1) + li + lo);
}
template <class R> inline R eval_pdf_ggx_vndf(R alpha, V3<R> wi, V3<R> h) {
    R G1 = eval_g1_ggx(alpha * alpha, wi.z);
    R D = eval_ndf_ggx(alpha, h.z);
    return G1 * D * vmax(R(0), dot(wi, h)) / wi.z;
}
template <class R> inline V3<R> sample_vndf_hemisphere(V2<R> u, V3<R> Vh) {
    R phi = R(2) * K<R>::pi * u.x;
    R z = std::fma((R(1) - u.y), (R(1) + Vh.z), -Vh.z);
    R sinTheta = std::sqrt(saturate(R(1) - z * z));
    R x = sinTheta * el_cos(phi);
    R y = sinTheta * el_sin(phi);
    return V3<R>(x, y, z) + Vh;
}
template <class R> inline V3<R> sample_ggx_vndf(R alpha, V3<R> wi, V2<R> u, R& pdf) {
    V3<R> Vh = normalize(V3<R>(alpha * wi.x, alpha * wi.y, wi.z));
    V3<R> Nh = sample_vndf_hemisphere(u, Vh);
    V3<R> h = normalize(V3<R>(alpha * Nh.x, alpha * Nh.y, Nh.z));
    pdf = eval_pdf_ggx_vndf(alpha, wi, h);
    return h;
}
// evalFresnelSchlick (Rendering/Materials/Fresnel.slang:42-51): pow(1 - cosTheta, 5),
// evaluated as x^2, x^4, x^4 * x (the library does the same, so FP32 results
// stay bit-identical).
template <class R> inline R pow5(R x) {
    R x2 = x * x;
    R x4 = x2 * x2;
    return x4 * x;
}
template <class R> inline V3<R> fresnel_schlick(V3<R> f0, V3<R> f90, R cosTheta) {
    R p = pow5(vmax(R(1) - cosTheta, R(0)));
    return f0 + (f90 - f0) * p;
}
template <class R> inline R fresnel_schlick(R f0, R f90, R cosTheta) {
    return f0 + (f90 - f0) * pow5(vmax(R(1) - cosTheta, R(0)));
}
template <class R> inline R fresnel_dielectric(R eta, R cosThetaI, R& cosThetaT) {
    if (cosThetaI < R(0)) { eta = R(1) / eta; cosThetaI = -cosThetaI; }
    R sinThetaTSq = eta * eta * (R(1) - cosThetaI * cosThetaI);
    if (sinThetaTSq > R(1)) { cosThetaT = R(0); return R(1); }
    cosThetaT = std::sqrt(R(1) - sinThetaTSq);
    R Rs = (eta * cosThetaI - cosThetaT) / (eta * cosThetaI + cosThetaT);
    R Rp = (eta * cosThetaT - cosThetaI) / (eta * cosThetaT + cosThetaI);
    return R(0.5f) * (Rs * Rs + Rp * Rp);
}

// ---------------------------------------------------------------------------
// Lobe types (Rendering/Materials/LobeType.slang).
// ---------------------------------------------------------------------------
enum LobeType : uint32_t {
    LOBE_NONE = 0x00,
    LOBE_DIFFUSE_REFLECTION = 0x01,
    LOBE_SPECULAR_REFLECTION = 0x02,
    LOBE_DELTA_REFLECTION = 0x04,
    LOBE_DIFFUSE_TRANSMISSION = 0x10,
    LOBE_SPECULAR_TRANSMISSION = 0x20,
    LOBE_DELTA_TRANSMISSION = 0x40,
    LOBE_DIFFUSE = 0x11,
    LOBE_SPECULAR = 0x22,
    LOBE_DELTA = 0x44,
    LOBE_NON_DELTA = 0x33,
    LOBE_REFLECTION = 0x0f,
    LOBE_TRANSMISSION = 0xf0,
    LOBE_NON_DELTA_REFLECTION = 0x03,
    LOBE_NON_DELTA_TRANSMISSION = 0x30,
    LOBE_ALL = 0xff,
};

constexpr float kMinCosTheta = 1e-6f;   // Rendering/Materials/IBSDF.slang:35
constexpr float kMinGGXAlpha = 0.0064f; // Rendering/Materials/BSDFs/StandardBSDF.slang:53

// StandardBSDFData (StandardBSDF.slang:58-89), restricted to the surface fields.
template <class R> struct BSDFData {
    V3<R> diffuse, specular, transmission;
    R roughness, metallic, eta, diffuseTransmission, specularTransmission;
};

template <class R> struct BSDFSampleOut {
    V3<R> wo, weight;
    R pdf;
    uint32_t lobe;
};

// StandardBSDF (StandardBSDF.slang:95-327) with the FrostbiteDiffuseBRDF
// (default, BSDFConfig.slangh:41-43) or LambertDiffuseBRDF diffuse lobe,
// height-correlated Smith masking (BSDFConfig.slangh:45-50), the
// SpecularMicrofacetBRDF (SpecularMicrofacet.slang:49-201), the
// LambertDiffuseBTDF and the SpecularMicrofacetBSDF transmission lobes.
template <class R> struct StandardBSDF {
    bool lambert;
    // lobes
    V3<R> diffAlbedo; R diffRoughness;
    V3<R> transAlbedo;
    V3<R> specAlbedo; R alpha; uint32_t activeLobes;
    R stAlpha, stEta;
    R diffTrans, specTrans;
    R pDiffuseReflection, pDiffuseTransmission, pSpecularReflection, pSpecularTransmission;

    StandardBSDF() = default;  // lobes set field by field (single-lobe unit tests)
    StandardBSDF(const V3<R>& wi, const BSDFData<R>& d, bool thinSurface, uint32_t lobes, bool lambertDiffuse) {
        lambert = lambertDiffuse;
        V3<R> transmissionAlbedo = thinSurface ? d.transmission
                                               : V3<R>(std::sqrt(d.transmission.x), std::sqrt(d.transmission.y), std::sqrt(d.transmission.z));
        diffAlbedo = d.diffuse;
        diffRoughness = d.roughness;
        transAlbedo = transmissionAlbedo;
        R a = d.roughness * d.roughness;
        if (a < R(kMinGGXAlpha)) a = R(0);
        activeLobes = lobes;
        specAlbedo = d.specular;
        alpha = a;
        stAlpha = d.eta == R(1) ? R(0) : a;
        stEta = d.eta;
        diffTrans = d.diffuseTransmission;
        specTrans = d.specularTransmission;
        R metallicBRDF = d.metallic * (R(1) - specTrans);
        R dielectricBSDF = (R(1) - d.metallic) * (R(1) - specTrans);
        R specularBSDF = specTrans;
        R diffuseWeight = luminance(d.diffuse);
        R specularWeight = luminance(fresnel_schlick(d.specular, V3<R>(R(1)), wi.z));
        pDiffuseReflection = (lobes & LOBE_DIFFUSE_REFLECTION) ? diffuseWeight * dielectricBSDF * (R(1) - diffTrans) : R(0);
        pDiffuseTransmission = (lobes & LOBE_DIFFUSE_TRANSMISSION) ? diffuseWeight * dielectricBSDF * diffTrans : R(0);
        pSpecularReflection = (lobes & (LOBE_SPECULAR_REFLECTION | LOBE_DELTA_REFLECTION)) ? specularWeight * (metallicBRDF + dielectricBSDF) : R(0);
        pSpecularTransmission = (lobes & (LOBE_SPECULAR_REFLECTION | LOBE_DELTA_REFLECTION | LOBE_SPECULAR_TRANSMISSION | LOBE_DELTA_TRANSMISSION)) ? specularBSDF : R(0);
        R norm = pDiffuseReflection + pDiffuseTransmission + pSpecularReflection + pSpecularTransmission;
        if (norm > R(0)) {
            norm = R(1) / norm;
            pDiffuseReflection *= norm;
            pDiffuseTransmission *= norm;
            pSpecularReflection *= norm;
            pSpecularTransmission *= norm;
        }
    }

    static uint32_t lobe_types(const BSDFData<R>& d) {
        R a = d.roughness * d.roughness;
        bool isDelta = a < R(kMinGGXAlpha);
        uint32_t t = isDelta ? LOBE_DELTA_REFLECTION : LOBE_SPECULAR_REFLECTION;
        if ((d.diffuse.x > R(0) || d.diffuse.y > R(0) || d.diffuse.z > R(0)) && d.specularTransmission < R(1)) {
            if (d.diffuseTransmission < R(1)) t |= LOBE_DIFFUSE_REFLECTION;
            if (d.diffuseTransmission > R(0)) t |= LOBE_DIFFUSE_TRANSMISSION;
        }
        if (d.specularTransmission > R(0)) t |= (isDelta ? LOBE_DELTA_TRANSMISSION : LOBE_SPECULAR_TRANSMISSION);
        return t;
    }

    // --- diffuse reflection (FrostbiteDiffuseBRDF.slang:43-91 / LambertDiffuseBRDF.slang:44-80)
    V3<R> frostbite_weight(V3<R> wi, V3<R> wo) const {
        V3<R> h = normalize(wi + wo);
        R woDotH = dot(wo, h);
        R energyBias = lerp(R(0), R(0.5f), diffRoughness);
        R energyFactor = lerp(R(1), R(1) / R(1.51f), diffRoughness);
        R fd90 = energyBias + R(2) * woDotH * woDotH * diffRoughness;
        R fd0 = R(1);
        R wiScatter = fresnel_schlick(fd0, fd90, wi.z);
        R woScatter = fresnel_schlick(fd0, fd90, wo.z);
        return diffAlbedo * wiScatter * woScatter * energyFactor;
    }
    V3<R> diffuse_eval(V3<R> wi, V3<R> wo) const {
        if (vmin(wi.z, wo.z) < R(kMinCosTheta)) return V3<R>(0);
        if (lambert) return K<R>::inv_pi * diffAlbedo * wo.z;
        return frostbite_weight(wi, wo) * K<R>::inv_pi * wo.z;
    }
    R diffuse_pdf(V3<R> wi, V3<R> wo) const {
        if (vmin(wi.z, wo.z) < R(kMinCosTheta)) return R(0);
        return K<R>::inv_pi * wo.z;
    }
    template <class SG> bool diffuse_sample(V3<R> wi, V3<R>& wo, R& pdf, V3<R>& weight, uint32_t& lobe, SG& sg) const {
        wo = sample_cosine_hemisphere_concentric(next2D<R>(sg), pdf);
        lobe = LOBE_DIFFUSE_REFLECTION;
        if (vmin(wi.z, wo.z) < R(kMinCosTheta)) { weight = V3<R>(0); return false; }
        weight = lambert ? diffAlbedo : frostbite_weight(wi, wo);
        return true;
    }
    // --- diffuse transmission (LambertDiffuseBTDF.slang)
    V3<R> difftrans_eval(V3<R> wi, V3<R> wo) const {
        if (vmin(wi.z, -wo.z) < R(kMinCosTheta)) return V3<R>(0);
        return K<R>::inv_pi * transAlbedo * -wo.z;
    }
    R difftrans_pdf(V3<R> wi, V3<R> wo) const {
        if (vmin(wi.z, -wo.z) < R(kMinCosTheta)) return R(0);
        return K<R>::inv_pi * -wo.z;
    }
    template <class SG> bool difftrans_sample(V3<R> wi, V3<R>& wo, R& pdf, V3<R>& weight, uint32_t& lobe, SG& sg) const {
        wo = sample_cosine_hemisphere_concentric(next2D<R>(sg), pdf);
        wo.z = -wo.z;
        lobe = LOBE_DIFFUSE_TRANSMISSION;
        if (vmin(wi.z, -wo.z) < R(kMinCosTheta)) { weight = V3<R>(0); return false; }
        weight = transAlbedo;
        return true;
    }
    // --- specular reflection (SpecularMicrofacetBRDF)
    bool spec_has(uint32_t l) const { return (activeLobes & l) != 0; }
    V3<R> spec_eval(V3<R> wi, V3<R> wo) const {
        if (vmin(wi.z, wo.z) < R(kMinCosTheta)) return V3<R>(0);
        if (alpha == R(0)) return V3<R>(0);
        if (!spec_has(LOBE_SPECULAR_REFLECTION)) return V3<R>(0);
        V3<R> h = normalize(wi + wo);
        R wiDotH = dot(wi, h);
        R D = eval_ndf_ggx(alpha, h.z);
        R G = eval_masking_smith_ggx_correlated(alpha, wi.z, wo.z);
        V3<R> F = fresnel_schlick(specAlbedo, V3<R>(R(1)), wiDotH);
        return F * D * G * R(0.25f) / wi.z;
    }
    R spec_pdf(V3<R> wi, V3<R> wo) const {
        if (vmin(wi.z, wo.z) < R(kMinCosTheta)) return R(0);
        if (alpha == R(0)) return R(0);
        if (!spec_has(LOBE_SPECULAR_REFLECTION)) return R(0);
        V3<R> h = normalize(wi + wo);
        R wiDotH = dot(wi, h);
        R pdf = eval_pdf_ggx_vndf(alpha, wi, h);
        return pdf / (R(4) * wiDotH);
    }
    template <class SG> bool spec_sample(V3<R> wi, V3<R>& wo, R& pdf, V3<R>& weight, uint32_t& lobe, SG& sg) const {
        wo = V3<R>(0); weight = V3<R>(0); pdf = R(0); lobe = LOBE_SPECULAR_REFLECTION;
        if (wi.z < R(kMinCosTheta)) return false;
        if (alpha == R(0)) {
            if (!spec_has(LOBE_DELTA_REFLECTION)) return false;
            wo = V3<R>(-wi.x, -wi.y, wi.z);
            pdf = R(0);
            weight = fresnel_schlick(specAlbedo, V3<R>(R(1)), wi.z);
            lobe = LOBE_DELTA_REFLECTION;
            return true;
        }
        if (!spec_has(LOBE_SPECULAR_REFLECTION)) return false;
        V3<R> h = sample_ggx_vndf(alpha, wi, next2D<R>(sg), pdf);
        R wiDotH = dot(wi, h);
        wo = R(2) * wiDotH * h - wi;
        if (wo.z < R(kMinCosTheta)) return false;
        R G = eval_masking_smith_ggx_correlated(alpha, wi.z, wo.z);
        R GOverG1wo = G * (R(1) + eval_lambda_ggx(alpha * alpha, wi.z));
        V3<R> F = fresnel_schlick(specAlbedo, V3<R>(R(1)), wiDotH);
        pdf /= (R(4) * wiDotH);
        weight = F * GOverG1wo;
        lobe = LOBE_SPECULAR_REFLECTION;
        return true;
    }
    // --- specular transmission (SpecularMicrofacetBSDF, SpecularMicrofacet.slang:206-471)
    V3<R> st_eval(V3<R> wi, V3<R> wo) const;
    R st_pdf(V3<R> wi, V3<R> wo) const;
    template <class SG> bool st_sample(V3<R> wi, V3<R>& wo, R& pdf, V3<R>& weight, uint32_t& lobe, SG& sg) const;

    // --- mixture (StandardBSDF.slang:226-327)
    V3<R> eval(V3<R> wi, V3<R> wo) const {
        V3<R> r(0);
        if (pDiffuseReflection > R(0)) r += (R(1) - specTrans) * (R(1) - diffTrans) * diffuse_eval(wi, wo);
        if (pDiffuseTransmission > R(0)) r += (R(1) - specTrans) * diffTrans * difftrans_eval(wi, wo);
        if (pSpecularReflection > R(0)) r += (R(1) - specTrans) * spec_eval(wi, wo);
        if (pSpecularTransmission > R(0)) r += specTrans * (st_eval(wi, wo));
        return r;
    }
    R eval_pdf(V3<R> wi, V3<R> wo) const {
        R pdf = R(0);
        if (pDiffuseReflection > R(0)) pdf += pDiffuseReflection * diffuse_pdf(wi, wo);
        if (pDiffuseTransmission > R(0)) pdf += pDiffuseTransmission * difftrans_pdf(wi, wo);
        if (pSpecularReflection > R(0)) pdf += pSpecularReflection * spec_pdf(wi, wo);
        if (pSpecularTransmission > R(0)) pdf += pSpecularTransmission * st_pdf(wi, wo);
        return pdf;
    }
    template <class SG> bool sample(V3<R> wi, V3<R>& wo, R& pdf, V3<R>& weight, uint32_t& lobe, SG& sg) const {
        wo = V3<R>(0); weight = V3<R>(0); pdf = R(0); lobe = LOBE_DIFFUSE_REFLECTION;
        bool valid = false;
        R uSelect = next1D<R>(sg);
        if (uSelect < pDiffuseReflection) {
            valid = diffuse_sample(wi, wo, pdf, weight, lobe, sg);
            weight /= pDiffuseReflection;
            weight *= (R(1) - specTrans) * (R(1) - diffTrans);
            pdf *= pDiffuseReflection;
            if (pSpecularReflection > R(0)) pdf += pSpecularReflection * spec_pdf(wi, wo);
            if (pSpecularTransmission > R(0)) pdf += pSpecularTransmission * st_pdf(wi, wo);
        } else if (uSelect < pDiffuseReflection + pDiffuseTransmission) {
            valid = difftrans_sample(wi, wo, pdf, weight, lobe, sg);
            weight /= pDiffuseTransmission;
            weight *= (R(1) - specTrans) * diffTrans;
            pdf *= pDiffuseTransmission;
            if (pSpecularTransmission > R(0)) pdf += pSpecularTransmission * st_pdf(wi, wo);
        } else if (uSelect < pDiffuseReflection + pDiffuseTransmission + pSpecularReflection) {
            valid = spec_sample(wi, wo, pdf, weight, lobe, sg);
            weight /= pSpecularReflection;
            weight *= (R(1) - specTrans);
            pdf *= pSpecularReflection;
            if (pDiffuseReflection > R(0)) pdf += pDiffuseReflection * diffuse_pdf(wi, wo);
            if (pSpecularTransmission > R(0)) pdf += pSpecularTransmission * st_pdf(wi, wo);
        } else if (pSpecularTransmission > R(0)) {
            valid = st_sample(wi, wo, pdf, weight, lobe, sg);
            weight /= pSpecularTransmission;
            weight *= specTrans;
            pdf *= pSpecularTransmission;
            if (pDiffuseReflection > R(0)) pdf += pDiffuseReflection * diffuse_pdf(wi, wo);
            if (pDiffuseTransmission > R(0)) pdf += pDiffuseTransmission * difftrans_pdf(wi, wo);
            if (pSpecularReflection > R(0)) pdf += pSpecularReflection * spec_pdf(wi, wo);
        }
        return valid;
    }
};

// SpecularMicrofacetBSDF (SpecularMicrofacet.slang:206-471): rough and delta
// dielectric transmission.  Only reached when specularTransmission > 0.
template <class R> V3<R> StandardBSDF<R>::st_eval(V3<R> wi, V3<R> wo) const {
    if (vmin(wi.z, std::fabs(wo.z)) < R(kMinCosTheta)) return V3<R>(0);
    if (stAlpha == R(0)) return V3<R>(0);
    const bool hasReflection = spec_has(LOBE_SPECULAR_REFLECTION);
    const bool hasTransmission = spec_has(LOBE_SPECULAR_TRANSMISSION);
    const bool isReflection = wo.z > R(0);
    if ((isReflection && !hasReflection) || (!isReflection && !hasTransmission)) return V3<R>(0);
    const R eta = stEta;
    V3<R> h = normalize(wo + wi * (isReflection ? R(1) : eta));
    h *= sgn(h.z);
    R wiDotH = dot(wi, h), woDotH = dot(wo, h);
    R D = eval_ndf_ggx(stAlpha, h.z);
    R G = eval_masking_smith_ggx_correlated(stAlpha, wi.z, std::fabs(wo.z));
    R cosThetaT;
    R F = fresnel_dielectric(eta, wiDotH, cosThetaT);
    if (isReflection) return V3<R>(F * D * G * R(0.25f) / wi.z);
    R sqrtDenom = woDotH + eta * wiDotH;
    R t = eta * eta * wiDotH * woDotH / (wi.z * sqrtDenom * sqrtDenom);
    return transAlbedo * (R(1) - F) * D * G * std::fabs(t);
}
template <class R> R StandardBSDF<R>::st_pdf(V3<R> wi, V3<R> wo) const {
    if (vmin(wi.z, std::fabs(wo.z)) < R(kMinCosTheta)) return R(0);
    if (stAlpha == R(0)) return R(0);
    const bool isReflection = wo.z > R(0);
    const bool hasReflection = spec_has(LOBE_SPECULAR_REFLECTION);
    const bool hasTransmission = spec_has(LOBE_SPECULAR_TRANSMISSION);
    if ((isReflection && !hasReflection) || (!isReflection && !hasTransmission)) return R(0);
    const R eta = stEta;
    V3<R> h = normalize(wo + wi * (isReflection ? R(1) : eta));
    h *= sgn(h.z);
    R wiDotH = dot(wi, h), woDotH = dot(wo, h);
    R cosThetaT;
    R F = fresnel_dielectric(eta, wiDotH, cosThetaT);
    R pdf = eval_pdf_ggx_vndf(stAlpha, wi, h);
    if (isReflection) {
        pdf /= R(4) * woDotH;
    } else {
        if (woDotH > R(0)) return R(0);
        R sqrtDenom = woDotH + eta * wiDotH;
        R denom = sqrtDenom * sqrtDenom;
        pdf = (denom > R(0)) ? pdf * std::fabs(woDotH) / denom : std::numeric_limits<R>::max();
    }
    if (hasReflection && hasTransmission) pdf *= isReflection ? F : R(1) - F;
    return pdf;
}
template <class R> template <class SG>
bool StandardBSDF<R>::st_sample(V3<R> wi, V3<R>& wo, R& pdf, V3<R>& weight, uint32_t& lobe, SG& sg) const {
    wo = V3<R>(0); weight = V3<R>(0); pdf = R(0); lobe = LOBE_SPECULAR_REFLECTION;
    if (wi.z < R(kMinCosTheta)) return false;
    R lobeSample = next1D<R>(sg);
    const R eta = stEta;
    if (stAlpha == R(0)) {
        const bool hasReflection = spec_has(LOBE_DELTA_REFLECTION);
        const bool hasTransmission = spec_has(LOBE_DELTA_TRANSMISSION);
        if (!(hasReflection || hasTransmission)) return false;
        R cosThetaT;
        R F = fresnel_dielectric(eta, wi.z, cosThetaT);
        bool isReflection = hasReflection;
        if (hasReflection && hasTransmission) isReflection = lobeSample < F;
        else if (hasTransmission && F == R(1)) return false;
        pdf = R(0);
        weight = isReflection ? V3<R>(R(1)) : transAlbedo;
        if (!(hasReflection && hasTransmission)) weight *= V3<R>(isReflection ? F : R(1) - F);
        wo = isReflection ? V3<R>(-wi.x, -wi.y, wi.z) : V3<R>(-wi.x * eta, -wi.y * eta, -cosThetaT);
        lobe = isReflection ? LOBE_DELTA_REFLECTION : LOBE_DELTA_TRANSMISSION;
        if (std::fabs(wo.z) < R(kMinCosTheta) || ((wo.z > R(0)) != isReflection)) return false;
        return true;
    }
    const bool hasReflection = spec_has(LOBE_SPECULAR_REFLECTION);
    const bool hasTransmission = spec_has(LOBE_SPECULAR_TRANSMISSION);
    if (!(hasReflection || hasTransmission)) return false;
    V3<R> h = sample_ggx_vndf(stAlpha, wi, next2D<R>(sg), pdf);
    R wiDotH = dot(wi, h);
    R cosThetaT;
    R F = fresnel_dielectric(eta, wiDotH, cosThetaT);
    bool isReflection = hasReflection;
    if (hasReflection && hasTransmission) isReflection = lobeSample < F;
    else if (hasTransmission && F == R(1)) return false;
    wo = isReflection ? (R(2) * wiDotH * h - wi) : ((eta * wiDotH - cosThetaT) * h - eta * wi);
    if (std::fabs(wo.z) < R(kMinCosTheta) || ((wo.z > R(0)) != isReflection)) return false;
    R woDotH = dot(wo, h);
    lobe = isReflection ? LOBE_SPECULAR_REFLECTION : LOBE_SPECULAR_TRANSMISSION;
    R G = eval_masking_smith_ggx_correlated(stAlpha, wi.z, std::fabs(wo.z));
    R GOverG1wo = G * (R(1) + eval_lambda_ggx(stAlpha * stAlpha, wi.z));
    weight = V3<R>(GOverG1wo);
    if (isReflection) {
        pdf /= R(4) * woDotH;
    } else {
        R sqrtDenom = woDotH + eta * wiDotH;
        R denom = sqrtDenom * sqrtDenom;
        pdf = (denom > R(0)) ? pdf * std::fabs(woDotH) / denom : std::numeric_limits<R>::max();
        weight *= transAlbedo * eta * eta;
    }
    if (hasReflection && hasTransmission) pdf *= isReflection ? F : R(1) - F;
    else weight *= isReflection ? F : R(1) - F;
    return true;
}

}  // namespace orc
