// oracle_render.cpp -- CPU restatement of the reference render passes:
// VBufferRT primary hits, MinimalPathTracer and PathTracer (NEE + MIS,
// emissive Uniform/Power samplers, env-map importance sampling, LogLuv
// per-sample colour, resolve), templated on the real type for the FP32
// parity oracle and the FP64 truth renderer.
//
// TEST INFRASTRUCTURE ONLY (see oracle_math.h).
#include "oracle_render.h"

#include <atomic>
#include <functional>
#include <thread>
#include <type_traits>

namespace orc {

// ---------------------------------------------------------------------------
// Camera (Scene/Camera/Camera.slang:46-78).
// ---------------------------------------------------------------------------
template <class R> struct Ray { V3<R> origin, dir; R tMin, tMax; };

template <class R> static V3<R> cam_vec(const float v[3]) { return V3<R>(R(v[0]), R(v[1]), R(v[2])); }

template <class R>
static V3<R> camera_nonnormalized_dir(const fpt_camera_data& c, uint32_t px, uint32_t py, uint32_t W, uint32_t H, bool jitter = true) {
    V2<R> p((R(float(px)) + R(0.5f)) / R(float(W)), (R(float(py)) + R(0.5f)) / R(float(H)));
    if (jitter) p = p + V2<R>(-R(c.jitterX), R(c.jitterY));
    V2<R> ndc(R(2) * p.x + R(-1), R(-2) * p.y + R(1));
    return ndc.x * cam_vec<R>(c.cameraU) + ndc.y * cam_vec<R>(c.cameraV) + cam_vec<R>(c.cameraW);
}
template <class R>
static Ray<R> camera_ray_pinhole(const fpt_camera_data& c, uint32_t px, uint32_t py, uint32_t W, uint32_t H) {
    Ray<R> r;
    r.origin = cam_vec<R>(c.posW);
    r.dir = normalize(camera_nonnormalized_dir<R>(c, px, py, W, H));
    R invCos = R(1) / dot(normalize(cam_vec<R>(c.cameraW)), r.dir);
    r.tMin = R(c.nearZ) * invCos;
    r.tMax = R(c.farZ) * invCos;
    return r;
}

// ---------------------------------------------------------------------------
// HitInfo packing (Scene/HitInfo.slang:109-122,457-487), uncompressed uint4.
// ---------------------------------------------------------------------------
void pack_hit(const fpt_hitinfo_bits& b, const Hit& h, uint32_t out[4]) {
    out[0] = out[1] = out[2] = out[3] = 0;
    if (!h.valid) return;
    const uint32_t header = b.type_bits + b.instance_id_bits + b.primitive_index_bits;
    const uint32_t typeOffset = 32u - b.type_bits;
    if (header <= 32) {
        out[0] = (1u << typeOffset) | (h.instanceID << b.primitive_index_bits) | h.primitiveIndex;
    } else {
        out[0] = (1u << typeOffset) | h.instanceID;
        out[1] = h.primitiveIndex;
    }
    out[2] = asuint(h.baryX);
    out[3] = asuint(h.baryY);
}
Hit unpack_hit(const fpt_hitinfo_bits& b, const uint32_t in[4]) {
    Hit h;
    const uint32_t typeOffset = 32u - b.type_bits;
    uint32_t type = in[0] >> typeOffset;
    if (type != 1u) return h;  // HitType::Triangle
    const uint32_t header = b.type_bits + b.instance_id_bits + b.primitive_index_bits;
    if (header <= 32) {
        h.instanceID = (in[0] >> b.primitive_index_bits) & ((1u << b.instance_id_bits) - 1u);
        h.primitiveIndex = in[0] & ((b.primitive_index_bits >= 32) ? 0xffffffffu : ((1u << b.primitive_index_bits) - 1u));
    } else {
        h.instanceID = in[0] & ((1u << b.instance_id_bits) - 1u);
        h.primitiveIndex = in[1];
    }
    h.baryX = asfloat(in[2]);
    h.baryY = asfloat(in[3]);
    h.valid = true;
    return h;
}

// ---------------------------------------------------------------------------
// Shading data (Scene/Scene.slang:440-526, MaterialFactory.slang:78-106,
// ShadingFrame.slang:76-150, ShadingData.slang:77-88).
// ---------------------------------------------------------------------------
template <class R> struct ShadingData {
    V3<R> posW, V, T, B, N, faceN;
    V2<R> uv;
    R tangentW[4];
    bool frontFacing;
    uint32_t materialID;
    R IoR;
    V3<R> computeRayOrigin(bool viewside = true) const {
        return compute_ray_origin(posW, (frontFacing == viewside) ? faceN : -faceN);
    }
    V3<R> orientedFaceN() const { return frontFacing ? faceN : -faceN; }
};

template <class R>
static ShadingData<R> load_shading_data(const Scene& s, const Hit& hit, V3<R> rayDir) {
    uint32_t idx[3];
    s.getTriangleVertexIndices(hit.instanceID, hit.primitiveIndex, idx);
    StaticVertex v[3] = {s.getVertex(idx[0]), s.getVertex(idx[1]), s.getVertex(idx[2])};
    // TriangleHit::getBarycentricWeights.
    R bx = R(hit.baryX), by = R(hit.baryY);
    R b[3] = {R(1) - bx - by, bx, by};
    V3<R> posW = cvt3<R>(v[0].position) * b[0];
    posW += cvt3<R>(v[1].position) * b[1];
    posW += cvt3<R>(v[2].position) * b[2];
    V3<R> normalW = cvt3<R>(v[0].normal) * b[0];
    normalW += cvt3<R>(v[1].normal) * b[1];
    normalW += cvt3<R>(v[2].normal) * b[2];
    R tan[4];
    for (int k = 0; k < 4; k++) {
        tan[k] = R(v[0].tangent[k]) * b[0];
        tan[k] += R(v[1].tangent[k]) * b[1];
        tan[k] += R(v[2].tangent[k]) * b[2];
    }
    tan[3] = sgn(tan[3]);
    V2<R> uv(R(v[0].uv.x) * b[0], R(v[0].uv.y) * b[0]);
    uv = uv + V2<R>(R(v[1].uv.x) * b[1], R(v[1].uv.y) * b[1]);
    uv = uv + V2<R>(R(v[2].uv.x) * b[2], R(v[2].uv.y) * b[2]);
    // getFaceNormalInObjectSpace (Scene.slang:348-355).
    V3<R> p0 = cvt3<R>(v[0].position), p1 = cvt3<R>(v[1].position), p2 = cvt3<R>(v[2].position);
    V3<R> faceN = normalize(cross(p1 - p0, p2 - p0));
    const fpt_geometry_instance& inst = s.instances[hit.instanceID];
    if (inst.flags & FPT_INSTANCE_FRONT_FACE_CW) faceN = -faceN;
    // Static geometry: identity world matrices.
    normalW = normalize(normalW);
    faceN = normalize(faceN);
    V3<R> tW = normalize(V3<R>(tan[0], tan[1], tan[2]));

    ShadingData<R> sd;
    sd.posW = posW;
    sd.uv = uv;
    sd.V = -rayDir;
    // ShadingFrame::createSafe / orthonormalizeSafe.
    sd.N = normalize(normalW);
    R NdotT = dot(tW, sd.N);
    bool nonParallel = std::fabs(NdotT) < R(0.9999f);
    bool nonZero = dot(tW, tW) > R(0);
    bool valid = std::fabs(tan[3]) == R(1) && nonZero && nonParallel;
    if (valid) {
        sd.T = normalize(tW - sd.N * NdotT);
        sd.B = cross(sd.N, sd.T) * tan[3];
        sd.tangentW[0] = tW.x; sd.tangentW[1] = tW.y; sd.tangentW[2] = tW.z; sd.tangentW[3] = tan[3];
    } else {
        sd.T = perp_stark(sd.N);
        sd.B = cross(sd.N, sd.T);
        sd.tangentW[0] = sd.T.x; sd.tangentW[1] = sd.T.y; sd.tangentW[2] = sd.T.z; sd.tangentW[3] = R(1);
    }
    sd.faceN = faceN;
    sd.frontFacing = dot(sd.V, sd.faceN) >= R(0);
    sd.materialID = inst.material_id;
    sd.IoR = R(1);
    return sd;
}

// StandardMaterial::setupMaterialInstance (Rendering/Materials/StandardMaterial.slang:50-133)
// and StandardMaterialInstance (StandardMaterialInstance.slang:63-160).
template <class R> struct MaterialInstance {
    V3<R> T, B, N;     // final shading frame
    BSDFData<R> data;
    V3<R> emission;
    bool thin;
    uint32_t activeLobes;
    bool lambert;

    V3<R> toLocal(V3<R> v) const { return V3<R>(dot(v, T), dot(v, B), dot(v, N)); }
    V3<R> fromLocal(V3<R> v) const { return T * v.x + B * v.y + N * v.z; }

    static bool valid_hemisphere(const ShadingData<R>& sd, V3<R> sfN, V3<R> wiL, V3<R> woL, V3<R> wo) {
        // isValidHemisphereReflectionOrTransmission (Scene/Material/ShadingUtils.slang:216-245).
        const bool isTransmission = wiL.z * woL.z < R(0);
        R cosThetaI = wiL.z;
        if (vmin(cosThetaI, std::fabs(woL.z)) < R(kMinCosTheta)) return false;
        bool wiTop = sd.frontFacing;
        bool woTop = dot(wo, sd.faceN) >= R(0);
        if (isTransmission) { if (wiTop == woTop) return false; }
        else { if (wiTop != woTop) return false; }
        bool shadingTop = dot(sfN, sd.faceN) >= R(0);
        if (wiTop != shadingTop) return false;
        return true;
    }
    StandardBSDF<R> bsdf(V3<R> wiL) const { return StandardBSDF<R>(wiL, data, thin, activeLobes, lambert); }

    V3<R> eval(const ShadingData<R>& sd, V3<R> wo) const {
        V3<R> wiL = toLocal(sd.V), woL = toLocal(wo);
        if (!valid_hemisphere(sd, N, wiL, woL, wo)) return V3<R>(0);
        return bsdf(wiL).eval(wiL, woL);
    }
    R evalPdf(const ShadingData<R>& sd, V3<R> wo, bool useIS) const {
        V3<R> wiL = toLocal(sd.V), woL = toLocal(wo);
        if (!valid_hemisphere(sd, N, wiL, woL, wo)) return R(0);
        if (!useIS) {
            if (lobeTypes() & LOBE_TRANSMISSION) {
                if (vmin(std::fabs(wiL.z), std::fabs(woL.z)) < R(kMinCosTheta)) return R(0);
                return R(0.5f) * woL.z * K<R>::inv_pi;
            }
            if (vmin(wiL.z, woL.z) < R(kMinCosTheta)) return R(0);
            return woL.z * K<R>::inv_pi;
        }
        return bsdf(wiL).eval_pdf(wiL, woL);
    }
    template <class SG> bool sample(const ShadingData<R>& sd, SG& sg, BSDFSampleOut<R>& out, bool useIS) const {
        V3<R> wiL = toLocal(sd.V), woL(0);
        if (!useIS) {
            // sampleReference (StandardMaterialInstance.slang:202-230).
            out.weight = V3<R>(0); out.lobe = 0;
            const bool isTransmissive = (lobeTypes() & LOBE_TRANSMISSION) != 0;
            woL = sample_cosine_hemisphere_concentric(next2D<R>(sg), out.pdf);
            if (isTransmissive) {
                if (next1D<R>(sg) < R(0.5f)) woL.z = -woL.z;
                out.pdf *= R(0.5f);
                if (vmin(std::fabs(wiL.z), std::fabs(woL.z)) < R(kMinCosTheta) || out.pdf == R(0)) return false;
            } else {
                if (vmin(wiL.z, woL.z) < R(kMinCosTheta) || out.pdf == R(0)) return false;
            }
            out.weight = bsdf(wiL).eval(wiL, woL) / out.pdf;
            out.lobe = woL.z > R(0) ? LOBE_DIFFUSE_REFLECTION : LOBE_DIFFUSE_TRANSMISSION;
        } else {
            StandardBSDF<R> b = bsdf(wiL);
            if (!b.sample(wiL, woL, out.pdf, out.weight, out.lobe, sg)) return false;
        }
        out.wo = fromLocal(woL);
        if (!valid_hemisphere(sd, N, wiL, woL, out.wo)) return false;
        return true;
    }
    uint32_t lobeTypes() const { return StandardBSDF<R>::lobe_types(data); }
    R propRoughness() const {
        R alpha = data.roughness * data.roughness;
        return alpha < R(kMinGGXAlpha) ? R(0) : data.roughness;
    }
};

template <class R>
static MaterialInstance<R> material_instance(const Scene& s, const ShadingData<R>& sd, bool lambert) {
    const Material& m = s.materials[sd.materialID];
    MaterialInstance<R> mi;
    mi.lambert = lambert;
    mi.thin = m.thinSurface;
    mi.activeLobes = m.activeLobes;
    BSDFData<R>& d = mi.data;
    R IoR = R(m.ior);
    d.eta = sd.frontFacing ? (sd.IoR / IoR) : (IoR / sd.IoR);
    d.diffuseTransmission = R(m.diffTrans);
    d.specularTransmission = R(m.specTrans);
    d.transmission = V3<R>(R(1));
    if (d.diffuseTransmission > R(0) || d.specularTransmission > R(0))
        d.transmission = V3<R>(R(m.transmission[0]), R(m.transmission[1]), R(m.transmission[2]));
    R f = (IoR - R(1)) / (IoR + R(1));
    R F0 = f * f;
    V3<R> baseColor(R(m.baseColor[0]), R(m.baseColor[1]), R(m.baseColor[2]));
    if (m.baseColorTexture >= 0) baseColor = tex_sample<R>(s, uint32_t(m.baseColorTexture), float(sd.uv.x), float(sd.uv.y));
    R specG = R(m.specular[1]), specB = R(m.specular[2]);
    d.diffuse = lerp(baseColor, V3<R>(R(0)), specB);
    d.specular = lerp(V3<R>(F0), baseColor, specB);
    d.roughness = specG;
    d.metallic = specB;
    mi.T = sd.T; mi.B = sd.B; mi.N = sd.N;
    if (!sd.frontFacing && m.doubleSided) mi.N = -mi.N;  // flipShadingNormal
    mi.emission = V3<R>(0);
    if (sd.frontFacing)
        mi.emission = V3<R>(R(m.emissive[0]), R(m.emissive[1]), R(m.emissive[2])) * R(m.emissiveFactor);
    return mi;
}

// ---------------------------------------------------------------------------
// Lights.
// ---------------------------------------------------------------------------
template <class R> struct TriLightSample {
    uint32_t triangleIndex;
    V3<R> posW, normalW, dir, Le;
    R distance, pdf;
};

// sampleTriangle (Rendering/Lights/EmissiveLightSamplerHelpers.slang:54-99).
template <class R>
static bool sample_triangle_light(const Scene& s, V3<R> posW, uint32_t tri, V2<R> u, TriLightSample<R>& ls) {
    ls = TriLightSample<R>();
    ls.triangleIndex = tri;
    const EmissiveTri& t = s.emissive[tri];
    V3<R> b = sample_triangle(u);
    ls.posW = cvt3<R>(t.posW[0]) * b.x + cvt3<R>(t.posW[1]) * b.y + cvt3<R>(t.posW[2]) * b.z;
    V3<R> toLight = ls.posW - posW;
    const R distSqr = vmax(R(std::numeric_limits<float>::min()), dot(toLight, toLight));
    ls.distance = std::sqrt(distSqr);
    ls.dir = toLight / ls.distance;
    ls.normalW = cvt3<R>(t.normal);
    R cosTheta = dot(ls.normalW, -ls.dir);
    if (cosTheta <= R(0)) return false;
    const Material& m = s.materials[t.materialID];
    ls.Le = V3<R>(R(m.emissive[0]), R(m.emissive[1]), R(m.emissive[2])) * R(m.emissiveFactor);
    R denom = vmax(R(std::numeric_limits<float>::min()), cosTheta * R(t.area));
    ls.pdf = distSqr / denom;
    return true;
}
// evalTrianglePdf (EmissiveLightSamplerHelpers.slang:106-124).
template <class R>
static R eval_triangle_pdf(const Scene& s, V3<R> posW, uint32_t tri, V3<R> hitPos, V3<R> hitN) {
    V3<R> toLight = hitPos - posW;
    const R distSqr = dot(toLight, toLight);
    if (distSqr <= R(std::numeric_limits<float>::min())) return R(0);
    V3<R> L = toLight / std::sqrt(distSqr);
    R cosTheta = dot(hitN, -L);
    if (cosTheta <= R(0)) return R(0);
    R denom = vmax(R(std::numeric_limits<float>::min()), cosTheta * R(s.emissive[tri].area));
    return distSqr / denom;
}

// LightBVHSampler (Rendering/Lights/LightBVHSampler.slang:70-534), default
// options: bounding cone, lighting cone, node flux, uniform leaf selection,
// SolidAngleBoundMethod::Sphere (GeometryHelpers.slang:222-240).
template <class R> struct LbvhNodeR { uint32_t w0; V3<R> origin, extent, coneDir; R cosCone, flux; };
template <class R> static LbvhNodeR<R> lbvh_node(const Scene& s, uint32_t i) {
    const uint32_t* w = &s.lightBvh.nodes[8 * size_t(i)];
    LbvhNodeR<R> n;
    n.w0 = w[0];
    float o[3], fl;
    std::memcpy(o, &w[1], 12);
    std::memcpy(&fl, &w[7], 4);
    n.origin = V3<R>(R(o[0]), R(o[1]), R(o[2]));
    n.extent = V3<R>(R(f16tof32(w[4] & 0xffffu)), R(f16tof32(w[4] >> 16)), R(f16tof32(w[5] & 0xffffu)));
    n.cosCone = R(float(w[5] >> 16) * (1.f / 32767.f) - 1.f);
    const V3<float> cd = decode_normal2x16(w[6]);
    n.coneDir = V3<R>(R(cd.x), R(cd.y), R(cd.z));
    n.flux = R(fl);
    return n;
}
template <class R> static R cos_sub_clamped(R sinA, R cosA, R sinB, R cosB) { return cosA > cosB ? R(1) : cosA * cosB + sinA * sinB; }
template <class R> static R sin_sub_clamped(R sinA, R cosA, R sinB, R cosB) { return cosA > cosB ? R(0) : sinA * cosB - cosA * sinB; }
// computeImportance (LightBVHSampler.slang:206-259).
template <class R> static R lbvh_importance(const Scene& s, V3<R> posW, V3<R> normalW, bool upper, uint32_t i) {
    const LbvhNodeR<R> n = lbvh_node<R>(s, i);
    R distance = length(n.origin - posW);
    // boundCosineTerm with the bounding sphere of the box.
    const R sqrRadius = dot(n.extent, n.extent);
    const V3<R> c = n.origin - posW;
    const R d2 = dot(c, c);
    R sinCone, cosCone;
    if (d2 < sqrRadius) { sinCone = R(0); cosCone = R(-1); }
    else { R s2 = sqrRadius / d2; cosCone = std::sqrt(R(1) - s2); sinCone = std::sqrt(s2); }
    const V3<R> L = normalize(n.origin - posW);
    R cosL = dot(normalW, L);
    cosL = cosL < R(-1) ? R(-1) : (cosL > R(1) ? R(1) : cosL);
    const R sinL = std::sqrt(R(1) - cosL * cosL);
    R NdotL = cos_sub_clamped(sinL, cosL, sinCone, cosCone);
    NdotL = NdotL < R(0) ? R(0) : (NdotL > R(1) ? R(1) : NdotL);
    if (!upper) NdotL = R(1);
    R orient = R(1);
    const V3<R> toBox = (n.origin - posW) / distance;
    if (n.cosCone != R(-1) && n.cosCone > R(0)) {
        const R sinConeAngle = std::sqrt(vmax(R(0), R(1) - n.cosCone * n.cosCone));
        const R cosT = dot(n.coneDir, -toBox);
        const R sinT = std::sqrt(vmax(R(0), R(1) - cosT * cosT));
        const R sinB = std::sqrt(vmax(R(0), R(1) - cosCone * cosCone));
        const R c0 = cos_sub_clamped(sinT, cosT, sinConeAngle, n.cosCone);
        const R s0 = sin_sub_clamped(sinT, cosT, sinConeAngle, n.cosCone);
        orient = vmax(R(0), cos_sub_clamped(s0, c0, sinB, cosCone));
    }
    const R half = vmax(n.extent.x, vmax(n.extent.y, n.extent.z));
    distance = vmax(half, distance);
    return (n.flux * NdotL) * orient / (distance * distance);
}
// traverseTree + pickTriangle (uniform) (LightBVHSampler.slang:262-392).
template <class R> static bool lbvh_select(const Scene& s, V3<R> posW, V3<R> normalW, bool upper, R u, R& pdf, uint32_t& tri) {
    pdf = R(1);
    uint32_t node = 0;
    uint32_t w0 = s.lightBvh.nodes[0];
    while (!(w0 >> 31)) {
        const uint32_t left = node + 1, right = w0;
        const R il = lbvh_importance<R>(s, posW, normalW, upper, left), ir = lbvh_importance<R>(s, posW, normalW, upper, right);
        const R total = il + ir;
        if (total == R(0)) return false;
        const R pLeft = il / total, pRight = R(1) - pLeft;
        if (u < pLeft) { u = u / pLeft; pdf *= pLeft; node = left; }
        else { u = (u - pLeft) / pRight; pdf *= pRight; node = right; }
        w0 = s.lightBvh.nodes[8 * size_t(node)];
    }
    const uint32_t count = (w0 >> 27) & 15u, offset = w0 & ((1u << 27) - 1u);
    const uint32_t idx = std::min(uint32_t(u * R(float(count))), count - 1);
    tri = s.lightBvh.triIndices[offset + idx];
    pdf *= R(1) / R(float(count));
    return true;
}
// evalTriangleSelectionPdf (LightBVHSampler.slang:95-125, 418-458).
template <class R> static R lbvh_selection_pdf(const Scene& s, V3<R> posW, V3<R> normalW, bool upper, uint32_t tri) {
    uint64_t mask = s.lightBvh.bitmasks[tri];
    R pdf = R(1);
    uint32_t node = 0;
    uint32_t w0 = s.lightBvh.nodes[0];
    while (!(w0 >> 31)) {
        const uint32_t left = node + 1, right = w0;
        const R il = lbvh_importance<R>(s, posW, normalW, upper, left), ir = lbvh_importance<R>(s, posW, normalW, upper, right);
        const R total = il + ir;
        if (total == R(0)) return R(0);
        const R pLeft = il / total, pRight = R(1) - pLeft;
        if ((mask & 1ull) == 0) { pdf *= pLeft; node = left; }
        else { pdf *= pRight; node = right; }
        mask >>= 1;
        w0 = s.lightBvh.nodes[8 * size_t(node)];
    }
    const uint32_t count = (w0 >> 27) & 15u;
    return pdf * (R(1) / R(float(count)));
}

// EmissiveUniformSampler.sampleLight (EmissiveUniformSampler.slang:55-76),
// LightBVHSampler.sampleLight (LightBVHSampler.slang:70-90) and
// EmissivePowerSampler.sampleLight (EmissivePowerSampler.slang:61-91).
template <class R, class SG>
static bool emissive_sample_light(const Scene& s, int samplerType, V3<R> posW, SG& sg, TriLightSample<R>& ls,
                                  V3<R> normalW = V3<R>(R(0)), bool upperHemisphere = false) {
    if (samplerType == 1) {
        if (s.emissive.empty() || s.lightBvh.nodes.empty()) return false;
        R uLight = next1D<R>(sg);
        R selPdf;
        uint32_t tri;
        if (!lbvh_select<R>(s, posW, normalW, upperHemisphere, uLight, selPdf, tri)) return false;
        V2<R> u = next2D<R>(sg);
        if (!sample_triangle_light(s, posW, tri, u, ls)) return false;
        ls.pdf *= selPdf;
        return true;
    }
    if (samplerType == 0) {
        if (s.activeTriangles.empty()) return false;
        R uLight = next1D<R>(sg);
        uint32_t n = uint32_t(s.activeTriangles.size());
        uint32_t idx = std::min(uint32_t(uLight * R(float(n))), n - 1);
        uint32_t tri = s.activeTriangles[idx];
        R selPdf = R(1) / R(float(n));
        V2<R> u = next2D<R>(sg);
        if (!sample_triangle_light(s, posW, tri, u, ls)) return false;
        ls.pdf *= selPdf;
        return true;
    }
    if (s.emissive.empty()) return false;
    R uLight = next1D<R>(sg);
    uint32_t n = uint32_t(s.emissive.size());
    uint32_t tri = std::min(uint32_t(uLight * R(float(n))), n - 1);
    uint32_t px = s.aliasTable[2 * tri], py = s.aliasTable[2 * tri + 1];
    R threshold = R(f16tof32(px >> 16u));
    uint32_t selectAbove = ((px & 0xFFFFu) << 8u) | ((py >> 24u) & 0xFFu);
    uint32_t selectBelow = py & 0xFFFFFFu;
    tri = (next1D<R>(sg) >= threshold) ? selectAbove : selectBelow;
    R selPdf = R(s.emissive[tri].flux) * R(1.0f / s.aliasWeightSum);
    V2<R> u = next2D<R>(sg);
    if (!sample_triangle_light(s, posW, tri, u, ls)) return false;
    ls.pdf *= selPdf;
    return true;
}
template <class R>
static R emissive_eval_pdf(const Scene& s, int samplerType, V3<R> posW, uint32_t tri, V3<R> hitPos, V3<R> hitN,
                           V3<R> normalW = V3<R>(R(0)), bool upperHemisphere = false) {
    if (tri == 0xffffffffu) return R(0);
    R sel;
    if (samplerType == 1) {
        if (s.lightBvh.nodes.empty()) return R(0);
        sel = lbvh_selection_pdf<R>(s, posW, normalW, upperHemisphere, tri);
        if (sel == R(0)) return R(0);
    } else if (samplerType == 0) {
        uint32_t n = uint32_t(s.activeTriangles.size());
        sel = n > 0 ? R(1) / R(float(n)) : R(0);
    } else {
        sel = R(s.emissive[tri].flux) * R(1.0f / s.aliasWeightSum);
    }
    return sel * eval_triangle_pdf(s, posW, tri, hitPos, hitN);
}

// EnvMapSampler.sample / evalPdf (Rendering/Lights/EnvMapSampler.slang:75-164).
template <class R> struct EnvSample { V3<R> dir, Le; R pdf; };
template <class R>
static bool env_sample(const Scene& s, V2<R> rnd, EnvSample<R>& res) {
    V2<R> p = rnd;
    uint32_t posx = 0, posy = 0;
    for (int mip = int(s.impBaseMip) - 1; mip >= 0; mip--) {
        posx *= 2; posy *= 2;
        const std::vector<float>& M = s.impMips[size_t(mip)];
        uint32_t d = s.impDim >> mip;
        R w0 = R(M[size_t(posy) * d + posx]), w1 = R(M[size_t(posy) * d + posx + 1]);
        R w2 = R(M[size_t(posy + 1) * d + posx]), w3 = R(M[size_t(posy + 1) * d + posx + 1]);
        R q0 = w0 + w2, q1 = w1 + w3;
        uint32_t offx, offy;
        R dd = q0 / (q0 + q1);
        if (p.x < dd) { offx = 0; p.x = p.x / dd; }
        else { offx = 1; p.x = (p.x - dd) / (R(1) - dd); }
        R e = offx == 0 ? (w0 / q0) : (w1 / q1);
        if (p.y < e) { offy = 0; p.y = p.y / e; }
        else { offy = 1; p.y = (p.y - e) / (R(1) - e); }
        posx += offx; posy += offy;
    }
    R inv = R(1.f / float(s.impDim));
    V2<R> uv((R(float(posx)) + p.x) * inv, (R(float(posy)) + p.y) * inv);
    V3<R> dir = oct_to_ndir_equal_area_unorm(uv);
    R avg_w = R(s.impMips[s.impBaseMip][0]);
    R pdf = R(s.impMips[0][size_t(posy) * s.impDim + posx]) / avg_w;
    res.dir = dir;
    res.pdf = pdf * K<R>::inv_4pi;
    if constexpr (std::is_same<R, float>::value) res.Le = s.envEval(res.dir);
    else res.Le = s.envEvalD(res.dir);
    return true;
}
template <class R>
static R env_eval_pdf(const Scene& s, V3<R> dir) {
    V2<R> uv = ndir_to_oct_equal_area_unorm(dir);
    R avg_w = R(s.impMips[s.impBaseMip][0]);
    int x = int(std::floor(uv.x * R(float(s.impDim)))), y = int(std::floor(uv.y * R(float(s.impDim))));
    x = std::min(std::max(x, 0), int(s.impDim) - 1);
    y = std::min(std::max(y, 0), int(s.impDim) - 1);
    R pdf = R(s.impMips[0][size_t(y) * s.impDim + x]) / avg_w;
    return pdf * (R(1) / K<R>::four_pi);
}

template <class R> static V3<R> env_eval(const Scene& s, V3<R> dir) {
    if constexpr (std::is_same<R, float>::value) return s.envEval(dir);
    else return s.envEvalD(dir);
}
template <class R> static Hit trace_closest(const Scene& s, V3<R> o, V3<R> d, R tMin, R tMax, TraceCounters* c) {
    if constexpr (std::is_same<R, float>::value) return s.traceClosest(o, d, tMin, tMax, c);
    else return s.traceClosestD(o, d, tMin, tMax);
}
template <class R> static bool trace_visibility(const Scene& s, V3<R> o, V3<R> d, R tMin, R tMax, TraceCounters* c) {
    if constexpr (std::is_same<R, float>::value) return s.traceVisibility(o, d, tMin, tMax, c);
    else return s.traceVisibilityD(o, d, tMin, tMax);
}

// ---------------------------------------------------------------------------
// VBufferRT: primary closest hit per pixel (VBufferRT.rt.slang:47-86,
// VBufferRT.slang:57-66, Center sample pattern).
// ---------------------------------------------------------------------------
void render_vbuffer_pixel(const Scene& s, uint32_t W, uint32_t H, uint32_t x, uint32_t y, uint32_t* out) {
    Ray<float> r = camera_ray_pinhole<float>(s.camera, x, y, W, H);
    Hit h = s.traceClosest(r.origin, r.dir, r.tMin, r.tMax, nullptr);
    pack_hit(s.hitBits, h, out + (size_t(y) * W + x) * 4);
}
void render_vbuffer(const Scene& s, uint32_t W, uint32_t H, uint32_t* out, uint32_t y0, uint32_t y1, TraceCounters* c) {
    for (uint32_t y = y0; y < y1; y++)
        for (uint32_t x = 0; x < W; x++) {
            Ray<float> r = camera_ray_pinhole<float>(s.camera, x, y, W, H);
            Hit h = s.traceClosest(r.origin, r.dir, r.tMin, r.tMax, c);
            pack_hit(s.hitBits, h, out + (size_t(y) * W + x) * 4);
        }
}

// ---------------------------------------------------------------------------
// MinimalPathTracer (RenderPasses/MinimalPathTracer/MinimalPathTracer.rt.slang:297-468).
// ---------------------------------------------------------------------------
template <class R, class SG> struct ScatterRayData {
    V3<R> radiance, thp, origin, direction;
    bool terminated;
    uint32_t pathLength;
    SG sg;
    ScatterRayData(const SG& g) : radiance(R(0)), thp(R(1)), origin(R(0)), direction(R(0)), terminated(false), pathLength(0), sg(g) {}
};

template <class R, class SG>
static bool mpt_generate_scatter_ray(const ShadingData<R>& sd, const MaterialInstance<R>& mi, V3<R> rayOrigin,
                                     ScatterRayData<R, SG>& rd, bool useIS) {
    BSDFSampleOut<R> bs;
    if (mi.sample(sd, rd.sg, bs, useIS)) {
        rd.origin = rayOrigin;
        if (bs.lobe & LOBE_TRANSMISSION) rd.origin = sd.computeRayOrigin(false);
        rd.direction = bs.wo;
        rd.thp *= bs.weight;
        return any_pos(rd.thp);
    }
    return false;
}

// One entry of a per-vertex hit record (see oracle_render.h).
static void record_hit(uint32_t* trace, uint32_t perSample, uint32_t vertexIndex, const Hit& h) {
    if (!trace || vertexIndex == 0 || vertexIndex > perSample) return;
    uint32_t* e = trace + 4 * size_t(vertexIndex - 1);
    if (!h.valid) { e[0] = e[1] = e[2] = e[3] = 0; return; }
    e[0] = h.instanceID + 1;
    e[1] = h.primitiveIndex;
    std::memcpy(&e[2], &h.baryX, 4);
    std::memcpy(&e[3], &h.baryY, 4);
}

template <class R>
V3<R> minimal_pt_pixel(const Scene& s, const MinimalPTParams& p, uint32_t x, uint32_t y, const uint32_t* vbufferPixel,
                       uint32_t* rays, uint32_t* trace) {
    const uint32_t traceLen = p.maxBounces + 2;
    const bool useEmissive = !s.emissive.empty();
    const bool useEnvLight = s.hasEnv, useEnvBg = s.hasEnv;
    V3<R> outColor(R(0));
    Ray<R> pr = camera_ray_pinhole<R>(s.camera, x, y, p.width, p.height);
    const V3<R> primaryDir = pr.dir;
    Hit hit = unpack_hit(s.hitBits, vbufferPixel);
    uint32_t nrays = 0;
    if (hit.valid) {
        record_hit(trace, traceLen, 1, hit);
        ShadingData<R> sd = load_shading_data<R>(s, hit, primaryDir);
        MaterialInstance<R> mi = material_instance<R>(s, sd, p.lambert != 0);
        UniformSG sg(x, y, p.frameCount);
        for (uint32_t i = 0; i < p.prngDimension; i++) next1D<R>(sg);
        V3<R> rayOrigin = sd.computeRayOrigin();
        if (p.computeDirect) outColor += mi.emission;
        ScatterRayData<R, UniformSG> rd(sg);
        if (!mpt_generate_scatter_ray(sd, mi, rayOrigin, rd, p.useImportanceSampling != 0)) rd.terminated = true;
        for (uint32_t depth = 0; depth <= p.maxBounces && !rd.terminated; depth++) {
            // traceScatterRay (.rt.slang:233-243): TMin 0, TMax FLT_MAX.
            nrays++;
            Hit h = trace_closest<R>(s, rd.origin, rd.direction, R(0), R(std::numeric_limits<float>::max()), nullptr);
            record_hit(trace, traceLen, depth + 2, h);
            if (!h.valid) {
                // scatterMiss (.rt.slang:475-486)
                rd.terminated = true;
                if (useEnvLight && (p.computeDirect || rd.pathLength > 0)) rd.radiance += rd.thp * env_eval<R>(s, rd.direction);
                continue;
            }
            // handleHit (.rt.slang:324-376)
            ShadingData<R> hsd = load_shading_data<R>(s, h, rd.direction);
            MaterialInstance<R> hmi = material_instance<R>(s, hsd, p.lambert != 0);
            if (useEmissive && (p.computeDirect || rd.pathLength > 0)) rd.radiance += rd.thp * hmi.emission;
            if (rd.pathLength >= p.maxBounces) { rd.terminated = true; continue; }
            V3<R> ro = hsd.computeRayOrigin();
            if (!mpt_generate_scatter_ray(hsd, hmi, ro, rd, p.useImportanceSampling != 0)) { rd.terminated = true; continue; }
            rd.pathLength++;
        }
        outColor += rd.radiance;
    } else {
        outColor = useEnvBg ? env_eval<R>(s, primaryDir) : V3<R>(R(0));
    }
    if (rays) *rays = nrays;
    return outColor;
}

// ---------------------------------------------------------------------------
// PathTracer (RenderPasses/PathTracer/PathTracer.slang:241-1202,
// TracePass.rt.slang:385-507, GeneratePaths.cs.slang:93-256,
// ResolvePass.cs.slang:80-101).
// ---------------------------------------------------------------------------
enum PathFlag : uint32_t {
    PF_ACTIVE = 0x1, PF_HIT = 0x2, PF_TRANSMISSION = 0x4, PF_SPECULAR = 0x8, PF_DELTA = 0x10,
    PF_INSIDE_DIELECTRIC = 0x20, PF_LIGHT_UPPER = 0x40, PF_LIGHT_LOWER = 0x80,
};

template <class R, class SG> struct PTPath {
    uint32_t flags = 0, vertexIndex = 0, bounces = 0;
    V3<R> origin, dir, normal, thp, L;
    R pdf = R(0);
    Hit hit;
    SG sg;
    explicit PTPath(const SG& g) : sg(g) {}
    bool has(uint32_t f) const { return (flags & f) != 0; }
    void set(uint32_t f, bool v = true) { if (v) flags |= f; else flags &= ~f; }
    uint32_t getBounces(int type) const { return (bounces >> (type * 8)) & 0xffu; }
    void incBounces(int type) { bounces += (1u << (type * 8)); }
    bool isLightSampled() const { return has(PF_LIGHT_UPPER | PF_LIGHT_LOWER); }
    bool isLightSamplable() const { return !has(PF_DELTA); }
};

template <class R> static R eval_mis(const PathTracerParams& p, R n0, R p0, R n1, R p1) {
    if (p.misHeuristic == 0) { R q0 = n0 * p0, q1 = n1 * p1; return q0 / (q0 + q1); }
    if (p.misHeuristic == 1) { R q0 = (n0 * p0) * (n0 * p0), q1 = (n1 * p1) * (n1 * p1); return q0 / (q0 + q1); }
    R q0 = el_pow(R(n0 * p0), R(p.misPowerExponent)), q1 = el_pow(R(n1 * p1), R(p.misPowerExponent));
    return q0 / (q0 + q1);
}

template <class R> struct LightSample { V3<R> Li, origin, dir; R pdf, distance; uint32_t lightType; };

template <class R>
static V3<R> vertex_ray_origin(V3<R> pos, V3<R> faceN, V3<R> rayDir) {
    return compute_ray_origin(pos, dot(faceN, rayDir) >= R(0) ? faceN : -faceN);
}

template <class R, class SG>
static bool generate_light_sample(const Scene& s, const PathTracerParams& p, V3<R> vpos, V3<R> vfaceN, bool vfront,
                                  bool upper, bool lower, SG& sg, LightSample<R>& ls) {
    ls = LightSample<R>();
    const bool useEnv = s.hasEnv, useEmissive = !s.emissive.empty();
    R pr[3] = {useEnv ? R(1) : R(0), useEmissive ? R(1) : R(0), R(0)};
    R sum = pr[0] + pr[1] + pr[2];
    if (sum != R(0)) { R inv = R(1) / sum; pr[0] *= inv; pr[1] *= inv; pr[2] *= inv; }
    // selectLightType (PathTracer.slang:671-693)
    R u = next1D<R>(sg);
    uint32_t lightType = 3;
    R selPdf = R(0);
    for (uint32_t t = 0; t < 3; t++) {
        if (u < pr[t]) { lightType = t; selPdf = pr[t]; break; }
        u -= pr[t];
    }
    if (lightType == 3) return false;
    V3<R> orientedN = vfront ? vfaceN : -vfaceN;
    bool valid = false;
    if (useEnv && lightType == 0) {
        EnvSample<R> es;
        if (env_sample<R>(s, next2D<R>(sg), es)) {
            ls.Li = es.pdf > R(0) ? es.Le / es.pdf : V3<R>(R(0));
            ls.pdf = es.pdf;
            ls.origin = vertex_ray_origin(vpos, vfaceN, es.dir);
            ls.distance = R(1e30f);
            ls.dir = es.dir;
            valid = any_pos(ls.Li);
        }
    }
    if (useEmissive && lightType == 1) {
        TriLightSample<R> tls;
        if (emissive_sample_light<R>(s, p.emissiveSampler, vpos, sg, tls, orientedN, upper && !lower)) {
            ls.Li = tls.pdf > R(0) ? tls.Le / tls.pdf : V3<R>(R(0));
            ls.pdf = tls.pdf;
            V3<R> lightPos = compute_ray_origin(tls.posW, tls.normalW);
            ls.origin = vertex_ray_origin(vpos, vfaceN, lightPos - vpos);
            V3<R> toLight = lightPos - ls.origin;
            ls.distance = length(toLight);
            ls.dir = normalize(toLight);
            valid = any_pos(ls.Li);
        }
    }
    if (!valid) return false;
    R NdotL = dot(orientedN, ls.dir);
    if ((!upper && NdotL >= -R(kMinCosTheta)) || (!lower && NdotL <= R(kMinCosTheta))) return false;
    ls.lightType = lightType;
    ls.pdf *= selPdf;
    ls.Li = ls.Li / selPdf;
    return true;
}

template <class R, class SG>
static void pt_handle_hit(const Scene& s, const PathTracerParams& p, PTPath<R, SG>& path, PathCounters* pc) {
    const bool isPrimaryHit = path.vertexIndex == 1;
    const bool useEnv = s.hasEnv, useEmissive = !s.emissive.empty();
    ShadingData<R> sd = load_shading_data<R>(s, path.hit, path.dir);
    MaterialInstance<R> mi = material_instance<R>(s, sd, p.lambert != 0);
    V3<R> emission = mi.emission;
    R roughness = mi.propRoughness();
    const bool isLightSamplable = path.isLightSamplable();
    bool computeEmissive = isPrimaryHit || (useEmissive && (!p.useNEE || p.useMIS || !path.isLightSampled() || !isLightSamplable));
    if (computeEmissive && any_pos(emission)) {
        R misWeight = R(1);
        if (useEmissive && p.useNEE && p.useMIS && !isPrimaryHit && path.isLightSampled() && isLightSamplable) {
            uint32_t triIdx = s.emissiveIndex(path.hit.instanceID, path.hit.primitiveIndex);
            bool upperHemisphere = path.has(PF_LIGHT_UPPER) && !path.has(PF_LIGHT_LOWER);
            R emissiveSel = (useEnv && useEmissive) ? R(0.5f) : R(1);
            R lightPdf = emissiveSel * emissive_eval_pdf<R>(s, p.emissiveSampler, path.origin, triIdx, sd.posW, sd.orientedFaceN(),
                                                            path.normal, upperHemisphere);
            misWeight = eval_mis<R>(p, R(1), path.pdf, R(1), lightPdf);
        }
        path.L += path.thp * (misWeight * emission);
    }
    auto finished = [&]() {
        uint32_t d = path.getBounces(0), sp = path.getBounces(1), tr = path.getBounces(2);
        return (d + sp + tr > p.maxSurfaceBounces) || (d > p.maxDiffuseBounces) || (sp > p.maxSpecularBounces) ||
               (tr > p.maxTransmissionBounces);
    };
    if (finished()) { path.set(PF_ACTIVE, false); return; }
    path.origin = sd.computeRayOrigin();
    const uint32_t lobeTypes = mi.lobeTypes();
    const bool hasNonDeltaLobes = (lobeTypes & LOBE_NON_DELTA) != 0;
    const bool applyNEE = p.useNEE && hasNonDeltaLobes;
    path.set(PF_LIGHT_UPPER, false);
    path.set(PF_LIGHT_LOWER, false);
    if (applyNEE) {
        bool upper = (lobeTypes & LOBE_NON_DELTA_REFLECTION) != 0;
        bool lower = (lobeTypes & LOBE_NON_DELTA_TRANSMISSION) != 0;
        LightSample<R> ls;
        bool validSample = generate_light_sample<R>(s, p, sd.posW, sd.faceN, sd.frontFacing, upper, lower, path.sg, ls);
        path.set(PF_LIGHT_UPPER, upper);
        path.set(PF_LIGHT_LOWER, lower);
        if (validSample) {
            if (p.useMIS) {
                R scatterPdf = mi.evalPdf(sd, ls.dir, p.useBSDFSampling != 0);
                ls.Li *= eval_mis<R>(p, R(1), ls.pdf, R(1), scatterPdf);
            }
            V3<R> weight = mi.eval(sd, ls.dir);
            V3<R> Lr = weight * ls.Li;
            if (any_pos(Lr)) {
                if (pc) pc->rays++;
                bool visible = trace_visibility<R>(s, ls.origin, ls.dir, R(0), ls.distance, pc ? &pc->tc : nullptr);
                if (visible) path.L += path.thp * Lr;
            }
        }
    }
    // generateScatterRay (PathTracer.slang:385-513)
    BSDFSampleOut<R> bs;
    bool valid = mi.sample(sd, path.sg, bs, p.useBSDFSampling != 0);
    if (valid) {
        path.dir = bs.wo;
        path.thp *= bs.weight;
        path.pdf = bs.pdf;
        path.set(PF_TRANSMISSION | PF_SPECULAR | PF_DELTA, false);
        if (bs.lobe & LOBE_REFLECTION) {
            bool isDiffuse = (bs.lobe & LOBE_DIFFUSE_REFLECTION) || roughness > R(p.specularRoughnessThreshold);
            if (isDiffuse) path.incBounces(0);
            else { path.incBounces(1); path.set(PF_SPECULAR); }
        }
        if (bs.lobe & LOBE_DELTA) path.set(PF_DELTA);
        if (bs.lobe & LOBE_TRANSMISSION) {
            path.incBounces(2);
            path.set(PF_TRANSMISSION);
            path.origin = sd.computeRayOrigin(false);
        }
        path.normal = sd.orientedFaceN();
        valid = any_pos(path.thp);
    }
    const bool isLastVertex = finished();
    if (p.useNEE && !p.useMIS && isLastVertex && path.isLightSamplable()) valid = false;
    if (!valid) path.set(PF_ACTIVE, false);
}

template <class R, class SG>
static void pt_handle_miss(const Scene& s, const PathTracerParams& p, PTPath<R, SG>& path) {
    const bool useEnv = s.hasEnv, useEmissive = !s.emissive.empty();
    const bool isLightSamplable = path.isLightSamplable();
    bool computeEnv = useEnv && (!p.useNEE || p.useMIS || !path.isLightSampled() || !isLightSamplable);
    if (computeEnv) {
        R misWeight = R(1);
        if (p.useNEE && p.useMIS && path.isLightSampled() && isLightSamplable) {
            R envSel = (useEnv && useEmissive) ? R(0.5f) : R(1);
            R lightPdf = envSel * env_eval_pdf<R>(s, path.dir);
            misWeight = eval_mis<R>(p, R(1), path.pdf, R(1), lightPdf);
        }
        V3<R> Le = env_eval<R>(s, path.dir);
        path.L += path.thp * (misWeight * Le);
    }
    path.set(PF_ACTIVE, false);
}

template <class R, class SG>
static V3<R> pt_trace_path(const Scene& s, const PathTracerParams& p, uint32_t x, uint32_t y, uint32_t sampleIdx,
                           const uint32_t* vbufferPixel, PathCounters* pc, uint32_t* trace) {
    const uint32_t traceLen = p.maxSurfaceBounces + 2;
    // generatePath (PathTracer.slang:273-301)
    const uint32_t maxSpp = p.samplesPerPixel;
    SG sg(x, y, p.seed * maxSpp + sampleIdx);
    PTPath<R, SG> path(sg);
    path.set(PF_ACTIVE);
    path.thp = V3<R>(R(1));
    Ray<R> cr = camera_ray_pinhole<R>(s.camera, x, y, p.width, p.height);
    path.origin = cr.origin;
    path.dir = cr.dir;
    Hit hit = unpack_hit(s.hitBits, vbufferPixel);
    if (!hit.valid) return V3<R>(R(0));  // background handled by generatePaths
    if (hit.valid) {
        hit.globalTri = s.instanceTriOffset[hit.instanceID] + hit.primitiveIndex;
        path.hit = hit;
        path.set(PF_HIT);
        path.vertexIndex = 1;
    }
    record_hit(trace, traceLen, 1, hit);
    pt_handle_hit<R, SG>(s, p, path, pc);
    while (path.has(PF_ACTIVE)) {
        path.vertexIndex++;
        if (pc) pc->rays++;
        Hit h = trace_closest<R>(s, path.origin, path.dir, R(0), R(1e30f), pc ? &pc->tc : nullptr);
        record_hit(trace, traceLen, path.vertexIndex, h);
        if (h.valid) {
            path.hit = h;
            path.set(PF_HIT);
            pt_handle_hit<R, SG>(s, p, path, pc);
        } else {
            path.set(PF_HIT, false);
            pt_handle_miss<R, SG>(s, p, path);
        }
    }
    if (pc) pc->paths++;
    return path.L;
}

template <class R>
void path_tracer_pixel(const Scene& s, const PathTracerParams& p, uint32_t x, uint32_t y, const uint32_t* vbufferPixel,
                       float* sampleOut, float* colorOut, PathCounters* pc, uint32_t* trace) {
    Hit hit = unpack_hit(s.hitBits, vbufferPixel);
    const uint32_t spp = p.samplesPerPixel;
    V3<R> color(R(0));
    if (!hit.valid) {
        // GeneratePaths::writeBackground (GeneratePaths.cs.slang:208-245)
        Ray<R> cr = camera_ray_pinhole<R>(s.camera, x, y, p.width, p.height);
        V3<R> bg = s.hasEnv ? env_eval<R>(s, cr.dir) : V3<R>(R(0));
        for (uint32_t i = 0; i < spp; i++) {
            if (sampleOut) { float* o = sampleOut + (size_t(i)) * 3; o[0] = float(bg.x); o[1] = float(bg.y); o[2] = float(bg.z); }
            V3<R> stored = bg;
            if (spp != 1 && p.colorFormat == 1) stored = cvt3<R>(decode_logluv_hdr(encode_logluv_hdr(tof(bg))));
            color += stored;
        }
    } else {
        for (uint32_t i = 0; i < spp; i++) {
            uint32_t* tr = trace ? trace + size_t(i) * (p.maxSurfaceBounces + 2) * 4 : nullptr;
            V3<R> L = (p.sampleGenerator == 0) ? pt_trace_path<R, TinyUniformSG>(s, p, x, y, i, vbufferPixel, pc, tr)
                                               : pt_trace_path<R, UniformSG>(s, p, x, y, i, vbufferPixel, pc, tr);
            if (sampleOut) { float* o = sampleOut + size_t(i) * 3; o[0] = float(L.x); o[1] = float(L.y); o[2] = float(L.z); }
            V3<R> stored = L;
            if (spp != 1 && p.colorFormat == 1) stored = cvt3<R>(decode_logluv_hdr(encode_logluv_hdr(tof(L))));
            color += stored;
        }
    }
    R invSpp = R(1) / R(float(spp));
    if (spp == 1) invSpp = R(1);
    V3<R> out = spp == 1 ? color : color * invSpp;
    colorOut[0] = float(out.x); colorOut[1] = float(out.y); colorOut[2] = float(out.z); colorOut[3] = 1.f;
}

float lbvh_selection_pdf_f(const Scene& s, const float posW[3], const float n[3], bool upper, uint32_t tri) {
    if (s.lightBvh.nodes.empty() || tri >= s.lightBvh.bitmasks.size()) return 0.f;
    return lbvh_selection_pdf<float>(s, V3<float>(posW[0], posW[1], posW[2]), V3<float>(n[0], n[1], n[2]), upper, tri);
}
bool lbvh_select_f(const Scene& s, const float posW[3], const float n[3], bool upper, float u, uint32_t* tri, float* pdf) {
    if (s.lightBvh.nodes.empty()) return false;
    return lbvh_select<float>(s, V3<float>(posW[0], posW[1], posW[2]), V3<float>(n[0], n[1], n[2]), upper, u, *pdf, *tri);
}

#include "oracle_wardiff.inl"

template V3<float> minimal_pt_pixel<float>(const Scene&, const MinimalPTParams&, uint32_t, uint32_t, const uint32_t*, uint32_t*,
                                           uint32_t*);
template V3<double> minimal_pt_pixel<double>(const Scene&, const MinimalPTParams&, uint32_t, uint32_t, const uint32_t*, uint32_t*,
                                             uint32_t*);
template void path_tracer_pixel<float>(const Scene&, const PathTracerParams&, uint32_t, uint32_t, const uint32_t*, float*, float*,
                                       PathCounters*, uint32_t*);
template void path_tracer_pixel<double>(const Scene&, const PathTracerParams&, uint32_t, uint32_t, const uint32_t*, float*, float*,
                                        PathCounters*, uint32_t*);

// Runs fn(x, y) over the pixels of [x0,x1)x[y0,y1) in 16x16 tiles on `threads` threads.
void parallel_tiles(uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1, uint32_t threads,
                    const std::function<void(uint32_t, uint32_t, uint32_t)>& fn) {
    const uint32_t tw = (x1 - x0 + 15) / 16, th = (y1 - y0 + 15) / 16;
    const uint32_t ntiles = tw * th;
    std::atomic<uint32_t> next(0);
    if (threads == 0) threads = std::max(1u, std::thread::hardware_concurrency());
    auto worker = [&](uint32_t tid) {
        for (;;) {
            uint32_t t = next.fetch_add(1);
            if (t >= ntiles) break;
            uint32_t bx = x0 + (t % tw) * 16, by = y0 + (t / tw) * 16;
            for (uint32_t y = by; y < std::min(by + 16, y1); y++)
                for (uint32_t x = bx; x < std::min(bx + 16, x1); x++) fn(x, y, tid);
        }
    };
    std::vector<std::thread> pool;
    for (uint32_t i = 1; i < threads; i++) pool.emplace_back(worker, i);
    worker(0);
    for (auto& t : pool) t.join();
}

}  // namespace orc
