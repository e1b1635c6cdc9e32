// device_math.cuh -- device-side vector math, pseudorandom generators, sample
// warps, packing helpers and the StandardMaterial BSDF for sm_100a.
//
// Every translation unit that includes this file is compiled with
// -fmad=false: no multiply-add is contracted unless written as fmaf(), which is
// where the reference writes fma().  Together with IEEE division and square
// root this keeps FP32 results bit-identical to the uncontracted reference
// arithmetic; only transcendental functions (sinf, cosf, powf, ...) may differ
// from a CPU libm in the last ulp.
#pragma once

#include "fmath.h"
#include <cstdint>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "common.h"

namespace fpt {
namespace dev {

#define FPT_D __device__ __forceinline__

// ---------------------------------------------------------------------------
// float3 arithmetic (component-wise, left to right).
// ---------------------------------------------------------------------------
FPT_D float3 f3(float a) { return make_float3(a, a, a); }
FPT_D float3 operator+(float3 a, float3 b) { return make_float3(a.x + b.x, a.y + b.y, a.z + b.z); }
FPT_D float3 operator-(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
FPT_D float3 operator*(float3 a, float3 b) { return make_float3(a.x * b.x, a.y * b.y, a.z * b.z); }
FPT_D float3 operator/(float3 a, float3 b) { return make_float3(a.x / b.x, a.y / b.y, a.z / b.z); }
FPT_D float3 operator*(float3 a, float s) { return make_float3(a.x * s, a.y * s, a.z * s); }
FPT_D float3 operator*(float s, float3 a) { return make_float3(s * a.x, s * a.y, s * a.z); }
FPT_D float3 operator/(float3 a, float s) { return make_float3(a.x / s, a.y / s, a.z / s); }
FPT_D float3 operator-(float3 a) { return make_float3(-a.x, -a.y, -a.z); }
FPT_D float3& operator+=(float3& a, float3 b) { a = a + b; return a; }
FPT_D float3& operator-=(float3& a, float3 b) { a = a - b; return a; }
FPT_D float3& operator*=(float3& a, float3 b) { a = a * b; return a; }
FPT_D float3& operator*=(float3& a, float s) { a = a * s; return a; }
FPT_D float3& operator/=(float3& a, float s) { a = a / s; return a; }
FPT_D float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
FPT_D float3 cross(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
FPT_D float length(float3 a) { return sqrtf(dot(a, a)); }
FPT_D float3 normalize(float3 a) { float l = sqrtf(dot(a, a)); return a / l; }
FPT_D float comp(float3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
FPT_D float hmin(float a, float b) { return a < b ? a : b; }
FPT_D float hmax(float a, float b) { return a > b ? a : b; }
FPT_D float saturate(float v) { return v < 0.f ? 0.f : (v > 1.f ? 1.f : v); }
FPT_D float sgn(float v) { return v > 0.f ? 1.f : (v < 0.f ? -1.f : 0.f); }
FPT_D float lerp(float a, float b, float t) { return a + t * (b - a); }
FPT_D float3 lerp(float3 a, float3 b, float t) { return a + t * (b - a); }
FPT_D bool any_pos(float3 a) { return a.x > 0.f || a.y > 0.f || a.z > 0.f; }
FPT_D float3 load3(const float* p) { return make_float3(p[0], p[1], p[2]); }

constexpr float kPi = 3.14159265358979323846f;
constexpr float kPi_2 = 1.57079632679489661923f;
constexpr float kPi_4 = 0.785398163397448309616f;
constexpr float kInvPi = 0.318309886183790671538f;
constexpr float k2Pi = 6.28318530717958647693f;
constexpr float kInv2Pi = 0.159154943091895335769f;
constexpr float k2OverPi = 0.636619772367581343076f;
constexpr float k4Pi = 12.5663706143591729539f;
constexpr float kInv4Pi = 0.079577471545947667884f;
constexpr float kFltMin = 1.175494351e-38f;
constexpr float kMinCosTheta = 1e-6f;   // IBSDF.slang:35
constexpr float kMinGGXAlpha = 0.0064f; // StandardBSDF.slang:53

// ---------------------------------------------------------------------------
// Packing (Utils/Math/FormatConversion.slang, PackedFormats.slang).
// ---------------------------------------------------------------------------
FPT_D float f16(uint32_t h) { return __half2float(__ushort_as_half((unsigned short)(h & 0xffffu))); }
FPT_D float2 unpack_snorm2x16(uint32_t p) {
    int bx = int(p << 16) >> 16, by = int(p) >> 16;
    return make_float2(hmax(float(bx) / 32767.f, -1.f), hmax(float(by) / 32767.f, -1.f));
}
FPT_D float3 oct_to_ndir_snorm(float2 p) {
    float3 n = make_float3(p.x, p.y, 1.f - fabsf(p.x) - fabsf(p.y));
    if (n.z < 0.f) {
        float wx = (1.f - fabsf(n.y)) * (n.x >= 0.f ? 1.f : -1.f);
        float wy = (1.f - fabsf(n.x)) * (n.y >= 0.f ? 1.f : -1.f);
        n.x = wx;
        n.y = wy;
    }
    return normalize(n);
}
FPT_D float3 decode_normal2x16(uint32_t p) { return oct_to_ndir_snorm(unpack_snorm2x16(p)); }

// ---------------------------------------------------------------------------
// Pseudorandom generators and sample generators (Utils/Sampling/...).
// ---------------------------------------------------------------------------
// jenkinsHash (Utils/Math/HashUtils.slang:41-50): Bob Jenkins' 32-bit integer hash.
FPT_D uint32_t jenkins_hash(uint32_t a) {
    a = (a + 0x7ed55d16u) + (a << 12);
    a = (a ^ 0xc761c23cu) ^ (a >> 19);
    a = (a + 0x165667b1u) + (a << 5);
    a = (a + 0xd3a2646cu) ^ (a << 9);
    a = (a + 0xfd7046c5u) + (a << 3);
    a = (a ^ 0xb55a4f09u) ^ (a >> 16);
    return a;
}
FPT_D uint32_t interleave_32bit(uint32_t vx, uint32_t vy) {
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

// SAMPLE_GENERATOR_UNIFORM: SplitMix64 -> xoshiro128** (UniformSampleGenerator.slang:53-78).
struct UniformSG {
    uint32_t s0, s1, s2, s3;
    FPT_D void init(uint32_t px, uint32_t py, uint32_t sampleNumber) {
        uint64_t st = (uint64_t(sampleNumber) << 32) | uint64_t(interleave_32bit(px, py));
        uint64_t v[2];
#pragma unroll
        for (int i = 0; i < 2; i++) {
            uint64_t z = (st += 0x9E3779B97F4A7C15ull);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            v[i] = z ^ (z >> 31);
        }
        s0 = uint32_t(v[0]); s1 = uint32_t(v[0] >> 32); s2 = uint32_t(v[1]); s3 = uint32_t(v[1] >> 32);
    }
    FPT_D uint32_t next() {
        const uint32_t result = __funnelshift_l(s0 * 5u, s0 * 5u, 7) * 9u;
        const uint32_t t = s1 << 9;
        s2 ^= s0;
        s3 ^= s1;
        s1 ^= s2;
        s0 ^= s3;
        s2 ^= t;
        s3 = __funnelshift_l(s3, s3, 11);
        return result;
    }
};

// SAMPLE_GENERATOR_TINY_UNIFORM: TEA-seeded LCG (TinyUniformSampleGenerator.slang:51-71).
struct TinyUniformSG {
    uint32_t state;
    FPT_D void init(uint32_t px, uint32_t py, uint32_t sampleNumber) {
        uint32_t v0 = interleave_32bit(px, py), v1 = sampleNumber, sum = 0;
#pragma unroll
        for (int i = 0; i < 16; i++) {
            sum += 0x9e3779b9u;
            v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + sum) ^ ((v1 >> 5) + 0xc8013ea4u);
            v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + sum) ^ ((v0 >> 5) + 0x7e95761eu);
        }
        state = v0;
    }
    FPT_D uint32_t next() { state = 1664525u * state + 1013904223u; return state; }
};

template <class SG> FPT_D float next1D(SG& sg) { return float(sg.next() >> 8) * 0x1p-24f; }
template <class SG> FPT_D float2 next2D(SG& sg) { float2 s; s.x = next1D(sg); s.y = next1D(sg); return s; }

// ---------------------------------------------------------------------------
// Warps (Utils/Math/MathHelpers.slang:111-411).
// ---------------------------------------------------------------------------
FPT_D float2 sample_disk_concentric(float2 u) {
    u = make_float2(2.f * u.x - 1.f, 2.f * u.y - 1.f);
    if (u.x == 0.f && u.y == 0.f) return u;
    float phi, r;
    if (fabsf(u.x) > fabsf(u.y)) { r = u.x; phi = (u.y / u.x) * kPi_4; }
    else { r = u.y; phi = kPi_2 - (u.x / u.y) * kPi_4; }
    float sp, cp;
    fm::sincos(phi, sp, cp);
    return make_float2(r * cp, r * sp);
}
FPT_D float3 sample_cosine_hemisphere_concentric(float2 u, float& pdf) {
    float2 d = sample_disk_concentric(u);
    float z = sqrtf(hmax(0.f, 1.f - (d.x * d.x + d.y * d.y)));
    pdf = z * kInvPi;
    return make_float3(d.x, d.y, z);
}
FPT_D float3 sample_triangle_bary(float2 u) {
    float su = sqrtf(u.x);
    float bx = 1.f - su, by = u.y * su;
    return make_float3(1.f - bx - by, bx, by);
}
FPT_D float2 world_to_latlong_map(float3 dir) {
    float3 p = normalize(dir);
    float2 uv;
    uv.x = fm::atan2(p.x, -p.z) * kInv2Pi + 0.5f;
    uv.y = fm::acos(p.y) * kInvPi;
    return uv;
}
FPT_D float2 ndir_to_oct_equal_area_unorm(float3 n) {
    float r = sqrtf(1.f - fabsf(n.z));
    float phi = fm::atan2(fabsf(n.y), fabsf(n.x));
    float2 p;
    p.y = r * phi * k2OverPi;
    p.x = r - p.y;
    if (n.z < 0.f) p = make_float2(1.f - p.y, 1.f - p.x);
    p.x *= sgn(n.x);
    p.y *= sgn(n.y);
    return make_float2(p.x * 0.5f + 0.5f, p.y * 0.5f + 0.5f);
}
FPT_D float3 oct_to_ndir_equal_area_unorm(float2 p) {
    p = make_float2(p.x * 2.f - 1.f, p.y * 2.f - 1.f);
    float d = 1.f - (fabsf(p.x) + fabsf(p.y));
    float r = 1.f - fabsf(d);
    float phi = (r > 0.f) ? ((fabsf(p.y) - fabsf(p.x)) / r + 1.f) * kPi_4 : 0.f;
    float f = r * sqrtf(2.f - r * r);
    float sp, cp;
    fm::sincos(phi, sp, cp);
    float x = f * sgn(p.x) * cp;
    float y = f * sgn(p.y) * sp;
    float z = sgn(d) * (1.f - r * r);
    return make_float3(x, y, z);
}
FPT_D float3 perp_stark(float3 u) {
    float ax = fabsf(u.x), ay = fabsf(u.y), az = fabsf(u.z);
    uint32_t uyx = (ax - ay) < 0.f ? 1u : 0u;
    uint32_t uzx = (ax - az) < 0.f ? 1u : 0u;
    uint32_t uzy = (ay - az) < 0.f ? 1u : 0u;
    uint32_t xm = uyx & uzx;
    uint32_t ym = (1u ^ xm) & uzy;
    uint32_t zm = 1u ^ (xm | ym);
    return normalize(cross(u, make_float3(float(xm), float(ym), float(zm))));
}
// sampleVonMisesFisher (Utils/Math/MathHelpers.slang:403-411): direction around +z.
FPT_D float3 sample_von_mises_fisher(float2 u, float kappa) {
    const float sy = fmaxf(1.f - u.y, 1e-6f);
    const float phi = 6.28318530717958647692f * u.x;
    const float cosTheta = 1.f + fm::log(fm::exp(-2.f * kappa) * (1.f - sy) + sy) / kappa;
    const float sinTheta = sqrtf(1.f - cosTheta * cosTheta);
    float sp, cp;
    fm::sincos(phi, sp, cp);
    return make_float3(cp * sinTheta, sp * sinTheta, cosTheta);
}
// computeRayOrigin (Utils/Geometry/GeometryHelpers.slang:51-68).
FPT_D float ray_origin_1(float p, float n) {
    const float origin = 1.f / 16.f, fScale = 3.f / 65536.f, iScale = 3 * 256.f;
    int iOff = int(n * iScale);
    float iPos = __int_as_float(__float_as_int(p) + (p < 0.f ? -iOff : iOff));
    float fOff = n * fScale;
    return fabsf(p) < origin ? p + fOff : iPos;
}
FPT_D float3 compute_ray_origin(float3 p, float3 n) {
    return make_float3(ray_origin_1(p.x, n.x), ray_origin_1(p.y, n.y), ray_origin_1(p.z, n.z));
}
FPT_D float luminance(float3 c) { return dot(c, make_float3(0.2126f, 0.7152f, 0.0722f)); }

// LogLuv HDR (Utils/Math/PackedFormats.slang:125-200).
FPT_D uint32_t encode_logluv_hdr(float3 c) {
    const float X = 0.4123907992659595f * c.x + 0.3575843393838780f * c.y + 0.1804807884018343f * c.z;
    const float Y = 0.2126390058715104f * c.x + 0.7151686787677559f * c.y + 0.0721923153607337f * c.z;
    const float Z = 0.0193308187155918f * c.x + 0.1191947797946259f * c.y + 0.9505321522496608f * c.z;
    float logY = 409.6f * (fm::log2(Y) + 20.f);
    float cl = fminf(fmaxf(logY, 0.f), 16383.f);
    uint32_t Le = uint32_t(cl);
    if (Le == 0) return 0;
    float invDenom = 1.f / (-2.f * X + 12.f * Y + 3.f * (X + Y + Z));
    float u = 4.f * X * invDenom, v = 9.f * Y * invDenom;
    uint32_t ue = uint32_t(fminf(fmaxf(820.f * u, 0.f), 511.f));
    uint32_t ve = uint32_t(fminf(fmaxf(820.f * v, 0.f), 511.f));
    return (Le << 18) | (ue << 9) | ve;
}
FPT_D float3 decode_logluv_hdr(uint32_t p) {
    uint32_t Le = p >> 18;
    if (Le == 0) return f3(0.f);
    float logY = (float(Le) + 0.5f) / 409.6f - 20.f;
    float Y = fm::pow(2.f, logY);
    float u = (float((p >> 9) & 0x1ffu) + 0.5f) / 820.f, v = (float(p & 0x1ffu) + 0.5f) / 820.f;
    float invDenom = 1.f / (6.f * u - 16.f * v + 12.f);
    float x = 9.f * u * invDenom, y = 4.f * v * invDenom;
    float s = Y / y;
    float X = s * x, Z = s * (1.f - x - y);
    float3 rgb = make_float3(3.240969941904522f * X + -1.537383177570094f * Y + -0.4986107602930032f * Z,
                             -0.9692436362808803f * X + 1.875967501507721f * Y + 0.04155505740717569f * Z,
                             0.05563007969699373f * X + -0.2039769588889765f * Y + 1.056971514242878f * Z);
    return make_float3(hmax(rgb.x, 0.f), hmax(rgb.y, 0.f), hmax(rgb.z, 0.f));
}

// ---------------------------------------------------------------------------
// GGX, Fresnel (Rendering/Materials/IsotropicGGX.slang, Fresnel.slang).
// ---------------------------------------------------------------------------
FPT_D float eval_ndf_ggx(float alpha, float c) {
    float a2 = alpha * alpha;
    float d = ((c * a2 - c) * c + 1.f);
    return a2 / (d * d * kPi);
}
FPT_D float eval_g1_ggx(float a2, float c) {
    if (c <= 0.f) return 0.f;
    float c2 = c * c;
    float t2 = hmax(1.f - c2, 0.f) / c2;
    return 2.f / (1.f + sqrtf(1.f + a2 * t2));
}
FPT_D float eval_lambda_ggx(float a2, float c) {
    if (c <= 0.f) return 0.f;
    float c2 = c * c;
    float t2 = hmax(1.f - c2, 0.f) / c2;
    return 0.5f * (-1.f + sqrtf(1.f + a2 * t2));
}
FPT_D float eval_masking_correlated(float alpha, float ci, float co) {
    float a2 = alpha * alpha;
    return 1.f / (1.f + eval_lambda_ggx(a2, ci) + eval_lambda_ggx(a2, co));
}
FPT_D float eval_pdf_ggx_vndf(float alpha, float3 wi, float3 h) {
    float G1 = eval_g1_ggx(alpha * alpha, wi.z);
    float D = eval_ndf_ggx(alpha, h.z);
    return G1 * D * hmax(0.f, dot(wi, h)) / wi.z;
}
FPT_D float3 sample_ggx_vndf(float alpha, float3 wi, float2 u, float& pdf) {
    float3 Vh = normalize(make_float3(alpha * wi.x, alpha * wi.y, wi.z));
    float phi = 2.f * kPi * u.x;
    float z = fmaf((1.f - u.y), (1.f + Vh.z), -Vh.z);
    float sinTheta = sqrtf(saturate(1.f - z * z));
    float sp, cp;
    fm::sincos(phi, sp, cp);
    float3 Nh = make_float3(sinTheta * cp, sinTheta * sp, z) + Vh;
    float3 h = normalize(make_float3(alpha * Nh.x, alpha * Nh.y, Nh.z));
    pdf = eval_pdf_ggx_vndf(alpha, wi, h);
    return h;
}
// Schlick's (1 - cos)^5 (Rendering/Materials/Fresnel.slang:42-51, evalFresnelSchlick
// writes pow(1 - cosTheta, 5)) as three products, x^2, x^4 and x^4 * x: the
// same operations in the oracle and in the adjoint's dual numbers.
FPT_D float pow5(float x) {
    const float x2 = x * x, x4 = x2 * x2;
    return x4 * x;
}
FPT_D float fresnel_schlick(float f0, float f90, float c) { return f0 + (f90 - f0) * pow5(hmax(1.f - c, 0.f)); }
FPT_D float3 fresnel_schlick(float3 f0, float c) {
    float p = pow5(hmax(1.f - c, 0.f));
    return f0 + (f3(1.f) - f0) * p;
}
FPT_D float fresnel_dielectric(float eta, float ci, float& ct) {
    if (ci < 0.f) { eta = 1.f / eta; ci = -ci; }
    float s2 = eta * eta * (1.f - ci * ci);
    if (s2 > 1.f) { ct = 0.f; return 1.f; }
    ct = sqrtf(1.f - s2);
    float Rs = (eta * ci - ct) / (eta * ci + ct);
    float Rp = (eta * ct - ci) / (eta * ct + ci);
    return 0.5f * (Rs * Rs + Rp * Rp);
}

// Lobe types (Rendering/Materials/LobeType.slang).
constexpr uint32_t L_DIFF_R = 0x01, L_SPEC_R = 0x02, L_DELTA_R = 0x04, L_DIFF_T = 0x10, L_SPEC_T = 0x20, L_DELTA_T = 0x40;
constexpr uint32_t L_DELTA = 0x44, L_NON_DELTA = 0x33, L_REFLECTION = 0x0f, L_TRANSMISSION = 0xf0;
constexpr uint32_t L_NON_DELTA_R = 0x03, L_NON_DELTA_T = 0x30, L_ALL = 0xff;

struct BSDFData {
    float3 diffuse, specular, transmission;
    float roughness, metallic, eta, diffTrans, specTrans;
};

FPT_D uint32_t bsdf_lobe_types(const BSDFData& d) {
    bool isDelta = d.roughness * d.roughness < kMinGGXAlpha;
    uint32_t t = isDelta ? L_DELTA_R : L_SPEC_R;
    if ((d.diffuse.x > 0.f || d.diffuse.y > 0.f || d.diffuse.z > 0.f) && d.specTrans < 1.f) {
        if (d.diffTrans < 1.f) t |= L_DIFF_R;
        if (d.diffTrans > 0.f) t |= L_DIFF_T;
    }
    if (d.specTrans > 0.f) t |= isDelta ? L_DELTA_T : L_SPEC_T;
    return t;
}

// StandardBSDF (Rendering/Materials/BSDFs/StandardBSDF.slang:124-327) with the
// Frostbite (default) or Lambert diffuse lobe, the GGX reflection lobe and,
// when HAS_TRANSMISSION, the LambertDiffuseBTDF and SpecularMicrofacetBSDF.
template <bool HAS_TRANSMISSION>
struct StandardBSDF {
    float3 diffAlbedo, transAlbedo, specAlbedo;
    float diffRoughness, alpha, stAlpha, eta, diffTrans, specTrans;
    float pDR, pDT, pSR, pST;
    uint32_t activeLobes;
    bool lambert;

    FPT_D void init(float3 wi, const BSDFData& d, bool thin, uint32_t lobes, bool lambertDiffuse) {
        lambert = lambertDiffuse;
        transAlbedo = thin ? d.transmission : make_float3(sqrtf(d.transmission.x), sqrtf(d.transmission.y), sqrtf(d.transmission.z));
        diffAlbedo = d.diffuse;
        diffRoughness = d.roughness;
        float a = d.roughness * d.roughness;
        if (a < kMinGGXAlpha) a = 0.f;
        activeLobes = lobes;
        specAlbedo = d.specular;
        alpha = a;
        stAlpha = d.eta == 1.f ? 0.f : a;
        eta = d.eta;
        diffTrans = d.diffTrans;
        specTrans = d.specTrans;
        float metallicBRDF = d.metallic * (1.f - specTrans);
        float dielectricBSDF = (1.f - d.metallic) * (1.f - specTrans);
        float specularBSDF = specTrans;
        float diffuseWeight = luminance(d.diffuse);
        float specularWeight = luminance(fresnel_schlick(d.specular, wi.z));
        pDR = (lobes & L_DIFF_R) ? diffuseWeight * dielectricBSDF * (1.f - diffTrans) : 0.f;
        pDT = (lobes & L_DIFF_T) ? diffuseWeight * dielectricBSDF * diffTrans : 0.f;
        pSR = (lobes & (L_SPEC_R | L_DELTA_R)) ? specularWeight * (metallicBRDF + dielectricBSDF) : 0.f;
        pST = (lobes & (L_SPEC_R | L_DELTA_R | L_SPEC_T | L_DELTA_T)) ? specularBSDF : 0.f;
        float norm = pDR + pDT + pSR + pST;
        if (norm > 0.f) {
            norm = 1.f / norm;
            pDR *= norm; pDT *= norm; pSR *= norm; pST *= norm;
        }
    }

    FPT_D float3 frostbite(float3 wi, float3 wo) const {
        float3 h = normalize(wi + wo);
        float woDotH = dot(wo, h);
        float energyBias = lerp(0.f, 0.5f, diffRoughness);
        float energyFactor = lerp(1.f, 1.f / 1.51f, diffRoughness);
        float fd90 = energyBias + 2.f * woDotH * woDotH * diffRoughness;
        float wiScatter = fresnel_schlick(1.f, fd90, wi.z);
        float woScatter = fresnel_schlick(1.f, fd90, wo.z);
        return diffAlbedo * wiScatter * woScatter * energyFactor;
    }
    FPT_D float3 diffuse_eval(float3 wi, float3 wo) const {
        if (hmin(wi.z, wo.z) < kMinCosTheta) return f3(0.f);
        if (lambert) return kInvPi * diffAlbedo * wo.z;
        return frostbite(wi, wo) * kInvPi * wo.z;
    }
    FPT_D float diffuse_pdf(float3 wi, float3 wo) const {
        if (hmin(wi.z, wo.z) < kMinCosTheta) return 0.f;
        return kInvPi * wo.z;
    }
    FPT_D float3 difftrans_eval(float3 wi, float3 wo) const {
        if (hmin(wi.z, -wo.z) < kMinCosTheta) return f3(0.f);
        return kInvPi * transAlbedo * -wo.z;
    }
    FPT_D float difftrans_pdf(float3 wi, float3 wo) const {
        if (hmin(wi.z, -wo.z) < kMinCosTheta) return 0.f;
        return kInvPi * -wo.z;
    }
    FPT_D bool has(uint32_t l) const { return (activeLobes & l) != 0; }
    FPT_D float3 spec_eval(float3 wi, float3 wo) const {
        if (hmin(wi.z, wo.z) < kMinCosTheta) return f3(0.f);
        if (alpha == 0.f) return f3(0.f);
        if (!has(L_SPEC_R)) return f3(0.f);
        float3 h = normalize(wi + wo);
        float wiDotH = dot(wi, h);
        float D = eval_ndf_ggx(alpha, h.z);
        float G = eval_masking_correlated(alpha, wi.z, wo.z);
        float3 F = fresnel_schlick(specAlbedo, wiDotH);
        return F * D * G * 0.25f / wi.z;
    }
    FPT_D float spec_pdf(float3 wi, float3 wo) const {
        if (hmin(wi.z, wo.z) < kMinCosTheta) return 0.f;
        if (alpha == 0.f) return 0.f;
        if (!has(L_SPEC_R)) return 0.f;
        float3 h = normalize(wi + wo);
        float wiDotH = dot(wi, h);
        return eval_pdf_ggx_vndf(alpha, wi, h) / (4.f * wiDotH);
    }
    // spec_eval and spec_pdf together: the half vector and the NDF are
    // evaluated once (the same operations, so the same values).
    FPT_D void spec_eval_pdf(float3 wi, float3 wo, float3& f, float& pdf) const {
        f = f3(0.f);
        pdf = 0.f;
        if (hmin(wi.z, wo.z) < kMinCosTheta) return;
        if (alpha == 0.f) return;
        if (!has(L_SPEC_R)) return;
        float3 h = normalize(wi + wo);
        float wiDotH = dot(wi, h);
        float D = eval_ndf_ggx(alpha, h.z);
        float G = eval_masking_correlated(alpha, wi.z, wo.z);
        float3 F = fresnel_schlick(specAlbedo, wiDotH);
        f = F * D * G * 0.25f / wi.z;
        float G1 = eval_g1_ggx(alpha * alpha, wi.z);
        pdf = (G1 * D * hmax(0.f, wiDotH) / wi.z) / (4.f * wiDotH);
    }
    FPT_D float3 st_eval(float3 wi, float3 wo) const {
        if (hmin(wi.z, fabsf(wo.z)) < kMinCosTheta) return f3(0.f);
        if (stAlpha == 0.f) return f3(0.f);
        const bool hasR = has(L_SPEC_R), hasT = has(L_SPEC_T), isR = wo.z > 0.f;
        if ((isR && !hasR) || (!isR && !hasT)) return f3(0.f);
        float3 h = normalize(wo + wi * (isR ? 1.f : eta));
        h *= sgn(h.z);
        float wiDotH = dot(wi, h), woDotH = dot(wo, h);
        float D = eval_ndf_ggx(stAlpha, h.z);
        float G = eval_masking_correlated(stAlpha, wi.z, fabsf(wo.z));
        float ct;
        float F = fresnel_dielectric(eta, wiDotH, ct);
        if (isR) return f3(F * D * G * 0.25f / wi.z);
        float sd = woDotH + eta * wiDotH;
        float t = eta * eta * wiDotH * woDotH / (wi.z * sd * sd);
        return transAlbedo * (1.f - F) * D * G * fabsf(t);
    }
    FPT_D float st_pdf(float3 wi, float3 wo) const {
        if (hmin(wi.z, fabsf(wo.z)) < kMinCosTheta) return 0.f;
        if (stAlpha == 0.f) return 0.f;
        const bool isR = wo.z > 0.f, hasR = has(L_SPEC_R), hasT = has(L_SPEC_T);
        if ((isR && !hasR) || (!isR && !hasT)) return 0.f;
        float3 h = normalize(wo + wi * (isR ? 1.f : eta));
        h *= sgn(h.z);
        float wiDotH = dot(wi, h), woDotH = dot(wo, h);
        float ct;
        float F = fresnel_dielectric(eta, wiDotH, ct);
        float pdf = eval_pdf_ggx_vndf(stAlpha, wi, h);
        if (isR) pdf /= 4.f * woDotH;
        else {
            if (woDotH > 0.f) return 0.f;
            float sd = woDotH + eta * wiDotH;
            float den = sd * sd;
            pdf = (den > 0.f) ? pdf * fabsf(woDotH) / den : 3.402823466e+38f;
        }
        if (hasR && hasT) pdf *= isR ? F : 1.f - F;
        return pdf;
    }

    FPT_D float3 eval(float3 wi, float3 wo) const {
        float3 r = f3(0.f);
        if (pDR > 0.f) r += (1.f - specTrans) * (1.f - diffTrans) * diffuse_eval(wi, wo);
        if (HAS_TRANSMISSION && pDT > 0.f) r += (1.f - specTrans) * diffTrans * difftrans_eval(wi, wo);
        if (pSR > 0.f) r += (1.f - specTrans) * spec_eval(wi, wo);
        if (HAS_TRANSMISSION && pST > 0.f) r += specTrans * (st_eval(wi, wo));
        return r;
    }
    FPT_D float eval_pdf(float3 wi, float3 wo) const {
        float pdf = 0.f;
        if (pDR > 0.f) pdf += pDR * diffuse_pdf(wi, wo);
        if (HAS_TRANSMISSION && pDT > 0.f) pdf += pDT * difftrans_pdf(wi, wo);
        if (pSR > 0.f) pdf += pSR * spec_pdf(wi, wo);
        if (HAS_TRANSMISSION && pST > 0.f) pdf += pST * st_pdf(wi, wo);
        return pdf;
    }

    // eval and eval_pdf in one pass (each sum in its own order, as above).
    FPT_D void eval_with_pdf(float3 wi, float3 wo, float3& r, float& pdf) const {
        r = f3(0.f);
        pdf = 0.f;
        if (pDR > 0.f) {
            r += (1.f - specTrans) * (1.f - diffTrans) * diffuse_eval(wi, wo);
            pdf += pDR * diffuse_pdf(wi, wo);
        }
        if (HAS_TRANSMISSION && pDT > 0.f) {
            r += (1.f - specTrans) * diffTrans * difftrans_eval(wi, wo);
            pdf += pDT * difftrans_pdf(wi, wo);
        }
        if (pSR > 0.f) {
            float3 f;
            float q;
            spec_eval_pdf(wi, wo, f, q);
            r += (1.f - specTrans) * f;
            pdf += pSR * q;
        }
        if (HAS_TRANSMISSION && pST > 0.f) {
            r += specTrans * (st_eval(wi, wo));
            pdf += pST * st_pdf(wi, wo);
        }
    }

    template <class SG>
    FPT_D bool spec_sample(float3 wi, float3& wo, float& pdf, float3& weight, uint32_t& lobe, SG& sg) const {
        wo = f3(0.f); weight = f3(0.f); pdf = 0.f; lobe = L_SPEC_R;
        if (wi.z < kMinCosTheta) return false;
        if (alpha == 0.f) {
            if (!has(L_DELTA_R)) return false;
            wo = make_float3(-wi.x, -wi.y, wi.z);
            pdf = 0.f;
            weight = fresnel_schlick(specAlbedo, wi.z);
            lobe = L_DELTA_R;
            return true;
        }
        if (!has(L_SPEC_R)) return false;
        float3 h = sample_ggx_vndf(alpha, wi, next2D(sg), pdf);
        float wiDotH = dot(wi, h);
        wo = 2.f * wiDotH * h - wi;
        if (wo.z < kMinCosTheta) return false;
        float G = eval_masking_correlated(alpha, wi.z, wo.z);
        float GOverG1wo = G * (1.f + eval_lambda_ggx(alpha * alpha, wi.z));
        float3 F = fresnel_schlick(specAlbedo, wiDotH);
        pdf /= (4.f * wiDotH);
        weight = F * GOverG1wo;
        lobe = L_SPEC_R;
        return true;
    }
    template <class SG>
    FPT_D bool st_sample(float3 wi, float3& wo, float& pdf, float3& weight, uint32_t& lobe, SG& sg) const {
        wo = f3(0.f); weight = f3(0.f); pdf = 0.f; lobe = L_SPEC_R;
        if (wi.z < kMinCosTheta) return false;
        float lobeSample = next1D(sg);
        if (stAlpha == 0.f) {
            const bool hasR = has(L_DELTA_R), hasT = has(L_DELTA_T);
            if (!(hasR || hasT)) return false;
            float ct;
            float F = fresnel_dielectric(eta, wi.z, ct);
            bool isR = hasR;
            if (hasR && hasT) isR = lobeSample < F;
            else if (hasT && F == 1.f) return false;
            pdf = 0.f;
            weight = isR ? f3(1.f) : transAlbedo;
            if (!(hasR && hasT)) weight *= f3(isR ? F : 1.f - F);
            wo = isR ? make_float3(-wi.x, -wi.y, wi.z) : make_float3(-wi.x * eta, -wi.y * eta, -ct);
            lobe = isR ? L_DELTA_R : L_DELTA_T;
            if (fabsf(wo.z) < kMinCosTheta || ((wo.z > 0.f) != isR)) return false;
            return true;
        }
        const bool hasR = has(L_SPEC_R), hasT = has(L_SPEC_T);
        if (!(hasR || hasT)) return false;
        float3 h = sample_ggx_vndf(stAlpha, wi, next2D(sg), pdf);
        float wiDotH = dot(wi, h);
        float ct;
        float F = fresnel_dielectric(eta, wiDotH, ct);
        bool isR = hasR;
        if (hasR && hasT) isR = lobeSample < F;
        else if (hasT && F == 1.f) return false;
        wo = isR ? (2.f * wiDotH * h - wi) : ((eta * wiDotH - ct) * h - eta * wi);
        if (fabsf(wo.z) < kMinCosTheta || ((wo.z > 0.f) != isR)) return false;
        float woDotH = dot(wo, h);
        lobe = isR ? L_SPEC_R : L_SPEC_T;
        float G = eval_masking_correlated(stAlpha, wi.z, fabsf(wo.z));
        float GOverG1wo = G * (1.f + eval_lambda_ggx(stAlpha * stAlpha, wi.z));
        weight = f3(GOverG1wo);
        if (isR) pdf /= 4.f * woDotH;
        else {
            float sd = woDotH + eta * wiDotH;
            float den = sd * sd;
            pdf = (den > 0.f) ? pdf * fabsf(woDotH) / den : 3.402823466e+38f;
            weight *= transAlbedo * eta * eta;
        }
        if (hasR && hasT) pdf *= isR ? F : 1.f - F;
        else weight *= isR ? F : 1.f - F;
        return true;
    }

    template <class SG>
    FPT_D bool sample(float3 wi, float3& wo, float& pdf, float3& weight, uint32_t& lobe, SG& sg) const {
        wo = f3(0.f); weight = f3(0.f); pdf = 0.f; lobe = L_DIFF_R;
        bool valid = false;
        float u = next1D(sg);
        if (u < pDR) {
            wo = sample_cosine_hemisphere_concentric(next2D(sg), pdf);
            lobe = L_DIFF_R;
            if (hmin(wi.z, wo.z) < kMinCosTheta) { weight = f3(0.f); valid = false; }
            else { weight = lambert ? diffAlbedo : frostbite(wi, wo); valid = true; }
            weight /= pDR;
            weight *= (1.f - specTrans) * (1.f - diffTrans);
            pdf *= pDR;
            if (pSR > 0.f) pdf += pSR * spec_pdf(wi, wo);
            if (HAS_TRANSMISSION && pST > 0.f) pdf += pST * st_pdf(wi, wo);
        } else if (HAS_TRANSMISSION && u < pDR + pDT) {
            wo = sample_cosine_hemisphere_concentric(next2D(sg), pdf);
            wo.z = -wo.z;
            lobe = L_DIFF_T;
            if (hmin(wi.z, -wo.z) < kMinCosTheta) { weight = f3(0.f); valid = false; }
            else { weight = transAlbedo; valid = true; }
            weight /= pDT;
            weight *= (1.f - specTrans) * diffTrans;
            pdf *= pDT;
            if (pST > 0.f) pdf += pST * st_pdf(wi, wo);
        } else if (u < pDR + pDT + pSR) {
            valid = spec_sample(wi, wo, pdf, weight, lobe, sg);
            weight /= pSR;
            weight *= (1.f - specTrans);
            pdf *= pSR;
            if (pDR > 0.f) pdf += pDR * diffuse_pdf(wi, wo);
            if (HAS_TRANSMISSION && pST > 0.f) pdf += pST * st_pdf(wi, wo);
        } else if (HAS_TRANSMISSION && pST > 0.f) {
            valid = st_sample(wi, wo, pdf, weight, lobe, sg);
            weight /= pST;
            weight *= specTrans;
            pdf *= pST;
            if (pDR > 0.f) pdf += pDR * diffuse_pdf(wi, wo);
            if (pDT > 0.f) pdf += pDT * difftrans_pdf(wi, wo);
            if (pSR > 0.f) pdf += pSR * spec_pdf(wi, wo);
        }
        return valid;
    }
};

}  // namespace dev
}  // namespace fpt
