// diff_bsdf.cuh -- forward-mode derivatives of the StandardBSDF evaluation
// for the WARDiffPathTracer adjoint.
//
// StandardMaterialInstance.evalAD (Rendering/Materials/StandardMaterialInstance.slang:75-89)
// is differentiable in the StandardBSDFData fields, which
// StandardMaterial.setupDiffMaterialInstance (StandardMaterial.slang:135-250)
// derives from the material parameters read through GradientIOWrapper, and in
// the local directions.  The lobe probabilities are detached
// (BSDFs/StandardBSDF.slang:174-184) and only gate the lobes.  The adjoint
// needs the 3 x P Jacobian of one evaluation with respect to P = 11 material
// parameters (StandardMaterialParamLayout offsets 0-10) and, for the NEE term,
// the 3 local components of the outgoing direction: the evaluation is run
// once on a small dual-number type carrying those tangents.
#pragma once

#include "device_math.cuh"

namespace fpt {
namespace dev {

template <int N>
struct DF {
    float v;
    float d[N];
};

template <int N> FPT_D DF<N> dconst(float x) {
    DF<N> r;
    r.v = x;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = 0.f;
    return r;
}
template <int N> FPT_D DF<N> dvar(float x, int slot) {
    DF<N> r = dconst<N>(x);
    if (slot >= 0 && slot < N) r.d[slot] = 1.f;
    return r;
}
template <int N> FPT_D DF<N> operator+(const DF<N>& a, const DF<N>& b) {
    DF<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N> FPT_D DF<N> operator-(const DF<N>& a, const DF<N>& b) {
    DF<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N> FPT_D DF<N> operator-(const DF<N>& a) {
    DF<N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = -a.d[i];
    return r;
}
template <int N> FPT_D DF<N> operator*(const DF<N>& a, const DF<N>& b) {
    DF<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N> FPT_D DF<N> operator/(const DF<N>& a, const DF<N>& b) {
    DF<N> r;
    r.v = a.v / b.v;
    const float inv = 1.f / b.v;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
    return r;
}
template <int N> FPT_D DF<N> operator*(const DF<N>& a, float s) {
    DF<N> r;
    r.v = a.v * s;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * s;
    return r;
}
template <int N> FPT_D DF<N> operator*(float s, const DF<N>& a) { return a * s; }
template <int N> FPT_D DF<N> operator+(const DF<N>& a, float s) {
    DF<N> r = a;
    r.v = a.v + s;
    return r;
}
template <int N> FPT_D DF<N> operator+(float s, const DF<N>& a) { return a + s; }
template <int N> FPT_D DF<N> operator-(float s, const DF<N>& a) { return (-a) + s; }
template <int N> FPT_D DF<N> operator-(const DF<N>& a, float s) { return a + (-s); }
template <int N> FPT_D DF<N> operator/(const DF<N>& a, float s) { return a * (1.f / s); }
template <int N> FPT_D DF<N> chain(const DF<N>& a, float fa, float fp) {
    DF<N> r;
    r.v = fa;
#pragma unroll
    for (int i = 0; i < N; i++) r.d[i] = a.d[i] * fp;
    return r;
}
template <int N> FPT_D DF<N> dsqrt(const DF<N>& a) {
    const float s = sqrtf(a.v);
    return chain(a, s, 0.5f / s);
}
template <int N> FPT_D DF<N> dabs(const DF<N>& a) { return a.v < 0.f ? -a : a; }
template <int N> FPT_D DF<N> dmax(const DF<N>& a, float b) { return a.v > b ? a : dconst<N>(b); }
template <int N> FPT_D DF<N> dmin(const DF<N>& a, const DF<N>& b) { return a.v < b.v ? a : b; }
// pow(x, 5) with derivative 5 x^4 (Schlick's exponent).
template <int N> FPT_D DF<N> dpow5(const DF<N>& a) {
    const float x2 = a.v * a.v, x4 = x2 * x2;
    return chain(a, x4 * a.v, 5.f * x4);
}

template <int N> struct DV3 {
    DF<N> x, y, z;
};
template <int N> FPT_D DV3<N> dv3(const DF<N>& x, const DF<N>& y, const DF<N>& z) { return DV3<N>{x, y, z}; }
template <int N> FPT_D DV3<N> dv3c(float3 a) { return DV3<N>{dconst<N>(a.x), dconst<N>(a.y), dconst<N>(a.z)}; }
template <int N> FPT_D DV3<N> dv3s(const DF<N>& s) { return DV3<N>{s, s, s}; }
template <int N> FPT_D DV3<N> operator+(const DV3<N>& a, const DV3<N>& b) { return DV3<N>{a.x + b.x, a.y + b.y, a.z + b.z}; }
template <int N> FPT_D DV3<N> operator-(const DV3<N>& a, const DV3<N>& b) { return DV3<N>{a.x - b.x, a.y - b.y, a.z - b.z}; }
template <int N> FPT_D DV3<N> operator*(const DV3<N>& a, const DV3<N>& b) { return DV3<N>{a.x * b.x, a.y * b.y, a.z * b.z}; }
template <int N> FPT_D DV3<N> operator*(const DV3<N>& a, const DF<N>& s) { return DV3<N>{a.x * s, a.y * s, a.z * s}; }
template <int N> FPT_D DV3<N> operator*(const DV3<N>& a, float s) { return DV3<N>{a.x * s, a.y * s, a.z * s}; }
template <int N> FPT_D DF<N> ddot(const DV3<N>& a, const DV3<N>& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <int N> FPT_D DV3<N> dnormalize(const DV3<N>& a) {
    const DF<N> l = dsqrt(ddot(a, a));
    return DV3<N>{a.x / l, a.y / l, a.z / l};
}
template <int N> FPT_D DF<N> dluminance(const DV3<N>& c) { return c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f; }

// StandardBSDFData (Rendering/Materials/BSDFs/StandardBSDF.slang:59-93).
template <int N> struct DBSDFData {
    DV3<N> diffuse, specular, transmission;
    DF<N> roughness, metallic, eta, diffTrans, specTrans;
};

// Material parameters -> StandardBSDFData (StandardMaterial.slang:146-196),
// tangents in slots 0-10 = StandardMaterialParamLayout offsets 0-10:
// baseColor rgb, metallic, roughness, ior, transmissionColor rgb,
// diffuseTransmission, specularTransmission.
template <int N>
FPT_D DBSDFData<N> diff_bsdf_data(float3 baseColor, float metallic, float roughness, float ior, float3 transmission,
                                  float diffTrans, float specTrans, bool frontFacing) {
    DBSDFData<N> d;
    const DF<N> IoR = dvar<N>(ior, 5);
    d.eta = frontFacing ? (dconst<N>(1.f) / IoR) : (IoR / dconst<N>(1.f));
    d.diffTrans = dvar<N>(diffTrans, 9);
    d.specTrans = dvar<N>(specTrans, 10);
    d.transmission = dv3c<N>(make_float3(0.f, 0.f, 0.f));
    if (diffTrans > 0.f || specTrans > 0.f) d.transmission = dv3(dvar<N>(transmission.x, 6), dvar<N>(transmission.y, 7), dvar<N>(transmission.z, 8));
    const DF<N> f = (IoR - 1.f) / (IoR + 1.f);
    const DF<N> F0 = f * f;
    const DV3<N> bc = dv3(dvar<N>(baseColor.x, 0), dvar<N>(baseColor.y, 1), dvar<N>(baseColor.z, 2));
    const DF<N> m = dvar<N>(metallic, 3);
    // lerp(a, b, t) = a + t * (b - a)
    d.diffuse = bc + (dv3c<N>(make_float3(0.f, 0.f, 0.f)) - bc) * m;
    d.specular = dv3s(F0) + (bc - dv3s(F0)) * m;
    d.roughness = dvar<N>(roughness, 4);
    d.metallic = m;
    return d;
}

template <int N> FPT_D DF<N> d_ndf_ggx(const DF<N>& alpha, const DF<N>& c) {
    const DF<N> a2 = alpha * alpha;
    const DF<N> d = (c * a2 - c) * c + 1.f;
    return a2 / (d * d * kPi);
}
template <int N> FPT_D DF<N> d_lambda_ggx(const DF<N>& a2, const DF<N>& c) {
    if (c.v <= 0.f) return dconst<N>(0.f);
    const DF<N> c2 = c * c;
    const DF<N> t2 = dmax(1.f - c2, 0.f) / c2;
    return 0.5f * (dsqrt(1.f + a2 * t2) - 1.f);
}
template <int N> FPT_D DF<N> d_masking_correlated(const DF<N>& alpha, const DF<N>& ci, const DF<N>& co) {
    const DF<N> a2 = alpha * alpha;
    return dconst<N>(1.f) / (1.f + d_lambda_ggx(a2, ci) + d_lambda_ggx(a2, co));
}
template <int N> FPT_D DF<N> d_schlick(const DF<N>& f0, const DF<N>& f90, const DF<N>& c) {
    return f0 + (f90 - f0) * dpow5(dmax(1.f - c, 0.f));
}
template <int N> FPT_D DV3<N> d_schlick3(const DV3<N>& f0, const DF<N>& c) {
    const DF<N> p = dpow5(dmax(1.f - c, 0.f));
    const DF<N> one = dconst<N>(1.f);
    return DV3<N>{f0.x + (one - f0.x) * p, f0.y + (one - f0.y) * p, f0.z + (one - f0.z) * p};
}
template <int N> FPT_D DF<N> d_fresnel_dielectric(DF<N> eta, DF<N> ci) {
    if (ci.v < 0.f) { eta = dconst<N>(1.f) / eta; ci = -ci; }
    const DF<N> s2 = eta * eta * (1.f - ci * ci);
    if (s2.v > 1.f) return dconst<N>(1.f);
    const DF<N> ct = dsqrt(1.f - s2);
    const DF<N> Rs = (eta * ci - ct) / (eta * ci + ct);
    const DF<N> Rp = (eta * ct - ci) / (eta * ct + ci);
    return 0.5f * (Rs * Rs + Rp * Rp);
}

// StandardBSDF.eval (StandardBSDF.slang:227-249) with its lobes
// (FrostbiteDiffuseBRDF.slang:44-64, LambertDiffuseBRDF.slang:41-50,
// LambertDiffuseBTDF.slang:40-50, SpecularMicrofacet.slang:57-96,215-283).
// pDR/pDT/pSR/pST are the (detached) lobe probabilities of the float BSDF.
template <int N>
FPT_D DV3<N> diff_bsdf_eval(const DBSDFData<N>& d, const DV3<N>& wi, const DV3<N>& wo, bool thin, uint32_t lobes, bool lambert,
                            float pDR, float pDT, float pSR, float pST) {
    const DV3<N> zero = dv3c<N>(make_float3(0.f, 0.f, 0.f));
    const DV3<N> transAlbedo = thin ? d.transmission : DV3<N>{dsqrt(d.transmission.x), dsqrt(d.transmission.y), dsqrt(d.transmission.z)};
    DF<N> alpha = d.roughness * d.roughness;
    if (alpha.v < kMinGGXAlpha) alpha = dconst<N>(0.f);
    const DF<N> stAlpha = d.eta.v == 1.f ? dconst<N>(0.f) : alpha;
    const DF<N> one = dconst<N>(1.f);
    DV3<N> r = zero;
    if (pDR > 0.f) {
        DV3<N> v = zero;
        if (fminf(wi.z.v, wo.z.v) >= kMinCosTheta) {
            if (lambert) {
                v = d.diffuse * (wo.z * kInvPi);
            } else {
                const DV3<N> h = dnormalize(wi + wo);
                const DF<N> woDotH = ddot(wo, h);
                const DF<N> energyBias = 0.5f * d.roughness;             // lerp(0, 0.5, r)
                const DF<N> energyFactor = 1.f + d.roughness * (1.f / 1.51f - 1.f);  // lerp(1, 1/1.51, r)
                const DF<N> fd90 = energyBias + 2.f * woDotH * woDotH * d.roughness;
                const DF<N> wiScatter = d_schlick(one, fd90, wi.z);
                const DF<N> woScatter = d_schlick(one, fd90, wo.z);
                v = d.diffuse * (wiScatter * woScatter * energyFactor) * (wo.z * kInvPi);
            }
        }
        r = r + v * ((one - d.specTrans) * (one - d.diffTrans));
    }
    if (pDT > 0.f && fminf(wi.z.v, -wo.z.v) >= kMinCosTheta) {
        r = r + transAlbedo * ((-wo.z) * kInvPi) * ((one - d.specTrans) * d.diffTrans);
    }
    if (pSR > 0.f && fminf(wi.z.v, wo.z.v) >= kMinCosTheta && alpha.v != 0.f && (lobes & L_SPEC_R)) {
        const DV3<N> h = dnormalize(wi + wo);
        const DF<N> wiDotH = ddot(wi, h);
        const DF<N> D = d_ndf_ggx(alpha, h.z);
        const DF<N> G = d_masking_correlated(alpha, wi.z, wo.z);
        const DV3<N> F = d_schlick3(d.specular, wiDotH);
        r = r + F * (D * G * 0.25f / wi.z) * (one - d.specTrans);
    }
    if (pST > 0.f && fminf(wi.z.v, fabsf(wo.z.v)) >= kMinCosTheta && stAlpha.v != 0.f) {
        const bool isR = wo.z.v > 0.f;
        const bool hasR = (lobes & L_SPEC_R) != 0, hasT = (lobes & L_SPEC_T) != 0;
        if ((isR && hasR) || (!isR && hasT)) {
            DV3<N> h = dnormalize(wo + wi * (isR ? one : d.eta));
            const float sg = h.z.v > 0.f ? 1.f : (h.z.v < 0.f ? -1.f : 0.f);
            h = h * sg;
            const DF<N> wiDotH = ddot(wi, h), woDotH = ddot(wo, h);
            const DF<N> D = d_ndf_ggx(stAlpha, h.z);
            const DF<N> G = d_masking_correlated(stAlpha, wi.z, dabs(wo.z));
            const DF<N> F = d_fresnel_dielectric(d.eta, wiDotH);
            DV3<N> v;
            if (isR) {
                v = dv3s(F * D * G * 0.25f / wi.z);
            } else {
                const DF<N> sd = woDotH + d.eta * wiDotH;
                const DF<N> t = d.eta * d.eta * wiDotH * woDotH / (wi.z * sd * sd);
                v = transAlbedo * ((one - F) * D * G * dabs(t));
            }
            r = r + v * d.specTrans;
        }
    }
    return r;
}

}  // namespace dev
}  // namespace fpt
