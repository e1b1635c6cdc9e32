// device_scene.cuh -- device view of a scene and the per-hit operations of the
// hot path: compressed 8-wide BVH traversal with a shared-memory stack, the
// watertight ray/triangle test, shading-data load, StandardMaterial set-up,
// emissive and environment light sampling.
#pragma once

#include "device_math.cuh"

namespace fpt {

// Kernel-parameter view of a device scene (all pointers are device memory).
struct DevScene {
    const uint4* nodes;               // BVH8Node, 5 x uint4 each
    const float4* tris;               // TriRecord, 3 x float4 each
    const PackedVertex* vertices;
    const uint32_t* indices;
    const DevInstance* instances;
    const DevMaterial* materials;
    const DevEmissiveTri* emissive;
    const float* flux;
    const uint2* alias;
    const uint32_t* instEmissiveOffset;
    const uint32_t* activeTris;
    const float4* env;                // envW x envH texels (rgb, 0)
    const float* impMips;             // importance mips, concatenated
    uint32_t emissiveCount, activeCount;
    float invWeightSum;
    uint32_t envW, envH;
    float envScale[3];
    uint32_t impDim, impBaseMip;
    uint32_t impMipOffset[16];
    fpt_camera_data camera;
    fpt_hitinfo_bits bits;
    uint32_t hasEnv, hasEmissive, hasTransmission;
    uint32_t nodeCount, triCount;
    uint32_t* errorWord;              // device error word (FPT_DEVERR_*)
};

namespace dev {

constexpr int kStackSize = 32;  // entries per thread; the host checks BVH depth <= kStackSize

struct HitRec {
    uint32_t instanceID, primIndex, globalTri;
    float baryX, baryY, t;
    bool valid;
};

// Watertight ray/triangle test (Utils/Geometry/IntersectionHelpers.slang:118-189).
// kx/ky/kz and the shear constants depend on the ray only.
struct RayShear {
    int kx, ky, kz;
    float Sx, Sy, Sz;
};
FPT_D RayShear make_shear(float3 d) {
    RayShear s;
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int axis = 0;
    if (ay > ax && ay > az) axis = 1;
    if (az > ax && az > ay) axis = 2;
    s.kz = axis;
    s.kx = (s.kz + 1) % 3;
    s.ky = (s.kx + 1) % 3;
    if (comp(d, s.kz) < 0.f) { int t = s.kx; s.kx = s.ky; s.ky = t; }
    s.Sx = comp(d, s.kx) / comp(d, s.kz);
    s.Sy = comp(d, s.ky) / comp(d, s.kz);
    s.Sz = 1.f / comp(d, s.kz);
    return s;
}
FPT_D bool intersect_triangle(const RayShear& rs, float3 o, float3 v0, float3 v1, float3 v2, float& t, float& bu, float& bv) {
    const float3 A = v0 - o, B = v1 - o, C = v2 - o;
    const float Akx = comp(A, rs.kx), Aky = comp(A, rs.ky), Akz = comp(A, rs.kz);
    const float Bkx = comp(B, rs.kx), Bky = comp(B, rs.ky), Bkz = comp(B, rs.kz);
    const float Ckx = comp(C, rs.kx), Cky = comp(C, rs.ky), Ckz = comp(C, rs.kz);
    const float Ax = Akx - rs.Sx * Akz, Ay = Aky - rs.Sy * Akz;
    const float Bx = Bkx - rs.Sx * Bkz, By = Bky - rs.Sy * Bkz;
    const float Cx = Ckx - rs.Sx * Ckz, Cy = Cky - rs.Sy * Ckz;
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.f || V == 0.f || W == 0.f) {
        double CxBy = double(Cx) * double(By), CyBx = double(Cy) * double(Bx);
        U = float(CxBy - CyBx);
        double AxCy = double(Ax) * double(Cy), AyCx = double(Ay) * double(Cx);
        V = float(AxCy - AyCx);
        double BxAy = double(Bx) * double(Ay), ByAx = double(By) * double(Ax);
        W = float(BxAy - ByAx);
    }
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
    float det = U + V + W;
    if (det == 0.f) return false;
    const float Az = rs.Sz * Akz, Bz = rs.Sz * Bkz, Cz = rs.Sz * Ckz;
    const float T = U * Az + V * Bz + W * Cz;
    const float rcpDet = 1.f / det;
    t = T * rcpDet;
    bu = V * rcpDet;
    bv = W * rcpDet;
    return true;
}

// Conservative ray/box slab test: the computed entry/exit distances carry a
// relative error of a few ulps, so the interval is widened by 2^-19 of its
// magnitude before it is compared; no box that the ray touches is culled.
FPT_D float widen_lo(float t) { return t - fabsf(t) * 1.9073486e-6f; }
FPT_D float widen_hi(float t) { return t + fabsf(t) * 1.9073486e-6f; }

// Traces one ray through the compressed 8-wide BVH.
//   ANY = false: closest hit in [tMin, tMax]; ties on t resolve to the
//                smaller global triangle index.
//   ANY = true : first hit in [tMin, tMax] (visibility rays).
// `stack` is this thread's slice of the block's shared-memory stack, strided
// by `stride` entries.  Returns false and sets FPT_DEVERR_STACK_OVERFLOW if the
// stack would overflow (the ray is then treated as a miss).
struct TraceStats {
    uint32_t nodes = 0, tris = 0;
};

template <bool ANY>
FPT_D bool trace_bvh(const DevScene& s, float3 o, float3 d, float tMin, float tMax, HitRec& hit, uint2* stack,
                     uint32_t stride, TraceStats* ts = nullptr) {
    hit.valid = false;
    if (s.nodeCount == 0) return true;
    const RayShear rs = make_shear(d);
    const float ix = 1.f / (fabsf(d.x) > 1e-20f ? d.x : copysignf(1e-20f, d.x));
    const float iy = 1.f / (fabsf(d.y) > 1e-20f ? d.y : copysignf(1e-20f, d.y));
    const float iz = 1.f / (fabsf(d.z) > 1e-20f ? d.z : copysignf(1e-20f, d.z));
    const uint32_t octinv = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
    float tBest = tMax;
    uint32_t bestTri = 0xffffffffu, bestInst = 0, bestPrim = 0;
    float bestU = 0.f, bestV = 0.f;

    int sp = 0;
    uint32_t nodeIdx = 0;
    bool haveNode = true;
    uint32_t gBase = 0, gHits = 0, gImask = 0;
    uint32_t visits = 0, triTests = 0;
    for (;;) {
        uint32_t tBase = 0, tHits = 0;
        if (haveNode) {
            haveNode = false;
            visits++;
            // A well-formed tree visits each node at most once per ray; guard
            // against corrupted input so that the loop always terminates.
            if (nodeIdx >= s.nodeCount || visits > s.nodeCount) {
                atomicOr(s.errorWord, FPT_DEVERR_BAD_INDEX);
                break;
            }
            const uint4* np = s.nodes + size_t(nodeIdx) * 5;
            const uint4 w0 = __ldg(np + 0), w1 = __ldg(np + 1), w2 = __ldg(np + 2), w3 = __ldg(np + 3), w4 = __ldg(np + 4);
            const float px = __uint_as_float(w0.x), py = __uint_as_float(w0.y), pz = __uint_as_float(w0.z);
            const uint32_t ew = w0.w;
            const float sx = __uint_as_float((ew & 0xffu) << 23);
            const float sy = __uint_as_float(((ew >> 8) & 0xffu) << 23);
            const float sz = __uint_as_float(((ew >> 16) & 0xffu) << 23);
            const uint32_t imask = ew >> 24;
            const uint32_t childBase = w1.x, triBase = w1.y;
            const uint32_t meta[2] = {w1.z, w1.w};
            const uint32_t qlx[2] = {w2.x, w2.y}, qly[2] = {w2.z, w2.w}, qlz[2] = {w3.x, w3.y};
            const uint32_t qhx[2] = {w3.z, w3.w}, qhy[2] = {w4.x, w4.y}, qhz[2] = {w4.z, w4.w};
            uint32_t innerHits = 0;
#pragma unroll
            for (int k = 0; k < 8; k++) {
                const int wi = k >> 2, sh = (k & 3) * 8;
                const uint32_t m = (meta[wi] >> sh) & 0xffu;
                const bool internal = (imask >> k) & 1u;
                if (!internal && m == 0u) continue;
                const float lox = fmaf(float((qlx[wi] >> sh) & 0xffu), sx, px);
                const float loy = fmaf(float((qly[wi] >> sh) & 0xffu), sy, py);
                const float loz = fmaf(float((qlz[wi] >> sh) & 0xffu), sz, pz);
                const float hix = fmaf(float((qhx[wi] >> sh) & 0xffu), sx, px);
                const float hiy = fmaf(float((qhy[wi] >> sh) & 0xffu), sy, py);
                const float hiz = fmaf(float((qhz[wi] >> sh) & 0xffu), sz, pz);
                const float t0x = ((octinv & 1u) ? hix : lox) - o.x, t1x = ((octinv & 1u) ? lox : hix) - o.x;
                const float t0y = ((octinv & 2u) ? hiy : loy) - o.y, t1y = ((octinv & 2u) ? loy : hiy) - o.y;
                const float t0z = ((octinv & 4u) ? hiz : loz) - o.z, t1z = ((octinv & 4u) ? loz : hiz) - o.z;
                const float tn = fmaxf(fmaxf(t0x * ix, t0y * iy), fmaxf(t0z * iz, tMin));
                const float tf = fminf(fminf(t1x * ix, t1y * iy), fminf(t1z * iz, tBest));
                if (!(widen_lo(tn) <= widen_hi(tf))) continue;
                if (internal) {
                    innerHits |= 1u << (k ^ octinv);
                } else {
                    const uint32_t cnt = m >> 5, off = m & 31u;
                    tHits |= ((1u << cnt) - 1u) << off;
                }
            }
            tBase = triBase;
            if (gHits) {
                if (sp >= kStackSize) {
                    atomicOr(s.errorWord, FPT_DEVERR_STACK_OVERFLOW);
                    if (ts) { ts->nodes += visits; ts->tris += triTests; }
                    return false;
                }
                stack[size_t(sp) * stride] = make_uint2(gBase, gHits | (gImask << 8));
                sp++;
            }
            gBase = childBase;
            gHits = innerHits;
            gImask = imask;
        }
        // Leaf triangles of the node just visited.
        while (tHits) {
            const int b = __ffs(tHits) - 1;
            tHits &= tHits - 1u;
            if (tBase + uint32_t(b) >= s.triCount) {
                atomicOr(s.errorWord, FPT_DEVERR_BAD_INDEX);
                continue;
            }
            const float4* tp = s.tris + size_t(tBase + uint32_t(b)) * 3;
            const float4 a = __ldg(tp), bb = __ldg(tp + 1), c = __ldg(tp + 2);
            triTests++;
            float t, u, v;
            if (!intersect_triangle(rs, o, make_float3(a.x, a.y, a.z), make_float3(bb.x, bb.y, bb.z), make_float3(c.x, c.y, c.z), t, u, v))
                continue;
            if (!(t >= tMin && t <= tBest)) continue;
            const uint32_t g = __float_as_uint(a.w);
            if (t == tBest && g > bestTri) continue;
            if (ANY) {
                hit.valid = true;
                if (ts) { ts->nodes += visits; ts->tris += triTests; }
                return true;
            }
            tBest = t;
            bestTri = g;
            bestInst = __float_as_uint(bb.w);
            bestPrim = __float_as_uint(c.w);
            bestU = u;
            bestV = v;
        }
        // Next node: nearest remaining child of the current group, else pop.
        if (gHits == 0) {
            if (sp == 0) break;
            sp--;
            const uint2 e = stack[size_t(sp) * stride];
            gBase = e.x;
            gHits = e.y & 0xffu;
            gImask = e.y >> 8;
        }
        const int i = __ffs(gHits) - 1;
        gHits &= gHits - 1u;
        const uint32_t slot = uint32_t(i) ^ octinv;
        nodeIdx = gBase + __popc(gImask & ((1u << slot) - 1u));
        haveNode = true;
    }
    if (ts) { ts->nodes += visits; ts->tris += triTests; }
    if (bestTri != 0xffffffffu) {
        hit.valid = true;
        hit.globalTri = bestTri;
        hit.instanceID = bestInst;
        hit.primIndex = bestPrim;
        hit.baryX = bestU;
        hit.baryY = bestV;
        hit.t = tBest;
    }
    return true;
}

// ---------------------------------------------------------------------------
// HitInfo packing (Scene/HitInfo.slang:457-487), uncompressed uint4.
// ---------------------------------------------------------------------------
FPT_D uint4 pack_hit(const fpt_hitinfo_bits& b, const HitRec& h) {
    if (!h.valid) return make_uint4(0, 0, 0, 0);
    const uint32_t header = b.type_bits + b.instance_id_bits + b.primitive_index_bits;
    const uint32_t typeOffset = 32u - b.type_bits;
    uint4 o;
    if (header <= 32) { o.x = (1u << typeOffset) | (h.instanceID << b.primitive_index_bits) | h.primIndex; o.y = 0; }
    else { o.x = (1u << typeOffset) | h.instanceID; o.y = h.primIndex; }
    o.z = __float_as_uint(h.baryX);
    o.w = __float_as_uint(h.baryY);
    return o;
}
FPT_D bool unpack_hit(const fpt_hitinfo_bits& b, uint4 in, HitRec& h) {
    h.valid = false;
    if ((in.x >> (32u - b.type_bits)) != 1u) return false;
    const uint32_t header = b.type_bits + b.instance_id_bits + b.primitive_index_bits;
    if (header <= 32) {
        h.instanceID = (in.x >> b.primitive_index_bits) & ((1u << b.instance_id_bits) - 1u);
        h.primIndex = in.x & ((1u << b.primitive_index_bits) - 1u);
    } else {
        h.instanceID = in.x & ((1u << b.instance_id_bits) - 1u);
        h.primIndex = in.y;
    }
    h.baryX = __uint_as_float(in.z);
    h.baryY = __uint_as_float(in.w);
    h.valid = true;
    return true;
}

// ---------------------------------------------------------------------------
// Camera (Scene/Camera/Camera.slang:46-78).
// ---------------------------------------------------------------------------
FPT_D float3 camera_ray_dir(const fpt_camera_data& c, uint32_t px, uint32_t py, uint32_t W, uint32_t H, float& tMin, float& tMax) {
    float2 p = make_float2((float(px) + 0.5f) / float(W), (float(py) + 0.5f) / float(H));
    p = make_float2(p.x + -c.jitterX, p.y + c.jitterY);
    const float ndcx = 2.f * p.x + -1.f, ndcy = -2.f * p.y + 1.f;
    const float3 U = load3(c.cameraU), V = load3(c.cameraV), Wv = load3(c.cameraW);
    const float3 dir = normalize(ndcx * U + ndcy * V + Wv);
    const float invCos = 1.f / dot(normalize(Wv), dir);
    tMin = c.nearZ * invCos;
    tMax = c.farZ * invCos;
    return dir;
}

// ---------------------------------------------------------------------------
// Shading data (Scene/Scene.slang:440-526, MaterialFactory.slang:78-106,
// ShadingFrame.slang:76-150) and StandardMaterial set-up
// (StandardMaterial.slang:50-133).
// ---------------------------------------------------------------------------
struct ShadingData {
    float3 posW, V, T, B, N, faceN;
    bool frontFacing;
    uint32_t materialID;
};

FPT_D void unpack_vertex(const PackedVertex& pv, float3& pos, float3& n) {
    pos = make_float3(pv.pos[0], pv.pos[1], pv.pos[2]);
    n = normalize(make_float3(f16(pv.nxy & 0xffffu), f16(pv.nxy >> 16), f16(pv.nz_tw & 0xffffu)));
}

// Reads one packed vertex as two 16-byte loads.
FPT_D PackedVertex load_vertex(const PackedVertex* vb, uint32_t i) {
    const uint4* p = reinterpret_cast<const uint4*>(vb + i);
    const uint4 a = __ldg(p), b = __ldg(p + 1);
    PackedVertex v;
    v.pos[0] = __uint_as_float(a.x); v.pos[1] = __uint_as_float(a.y); v.pos[2] = __uint_as_float(a.z);
    v.nxy = a.w; v.nz_tw = b.x; v.tangentOct = b.y;
    v.uv[0] = __uint_as_float(b.z); v.uv[1] = __uint_as_float(b.w);
    return v;
}

FPT_D ShadingData load_shading_data(const DevScene& s, const HitRec& hit, float3 rayDir) {
    const DevInstance inst = s.instances[hit.instanceID];
    const uint32_t* ip = s.indices + inst.ibOffset + hit.primIndex * 3;
    const uint32_t i0 = __ldg(ip) + inst.vbOffset, i1 = __ldg(ip + 1) + inst.vbOffset, i2 = __ldg(ip + 2) + inst.vbOffset;
    const PackedVertex pv0 = load_vertex(s.vertices, i0), pv1 = load_vertex(s.vertices, i1), pv2 = load_vertex(s.vertices, i2);
    float3 p0, p1, p2, n0, n1, n2;
    unpack_vertex(pv0, p0, n0);
    unpack_vertex(pv1, p1, n1);
    unpack_vertex(pv2, p2, n2);
    // Tangent: decodeNormal2x16 + sign of the fp16 tangent w.
    const float3 t0 = decode_normal2x16(pv0.tangentOct), t1 = decode_normal2x16(pv1.tangentOct), t2 = decode_normal2x16(pv2.tangentOct);
    const float w0 = sgn(f16(pv0.nz_tw >> 16)), w1 = sgn(f16(pv1.nz_tw >> 16)), w2 = sgn(f16(pv2.nz_tw >> 16));
    const float bx = hit.baryX, by = hit.baryY;
    const float b0 = 1.f - bx - by, b1 = bx, b2 = by;
    float3 posW = p0 * b0;
    posW += p1 * b1;
    posW += p2 * b2;
    float3 normalW = n0 * b0;
    normalW += n1 * b1;
    normalW += n2 * b2;
    float3 tanW = t0 * b0;
    tanW += t1 * b1;
    tanW += t2 * b2;
    float tw = w0 * b0;
    tw += w1 * b1;
    tw += w2 * b2;
    tw = sgn(tw);
    float3 faceN = normalize(cross(p1 - p0, p2 - p0));
    if (inst.flags & FPT_INSTANCE_FRONT_FACE_CW) faceN = -faceN;
    normalW = normalize(normalW);
    faceN = normalize(faceN);
    tanW = normalize(tanW);

    ShadingData sd;
    sd.posW = posW;
    sd.V = -rayDir;
    sd.N = normalize(normalW);
    const float NdotT = dot(tanW, sd.N);
    const bool nonParallel = fabsf(NdotT) < 0.9999f;
    const bool nonZero = dot(tanW, tanW) > 0.f;
    const bool valid = fabsf(tw) == 1.f && nonZero && nonParallel;
    if (valid) {
        sd.T = normalize(tanW - sd.N * NdotT);
        sd.B = cross(sd.N, sd.T) * tw;
    } else {
        sd.T = perp_stark(sd.N);
        sd.B = cross(sd.N, sd.T);
    }
    sd.faceN = faceN;
    sd.frontFacing = dot(sd.V, sd.faceN) >= 0.f;
    sd.materialID = inst.materialID;
    return sd;
}

FPT_D float3 sd_ray_origin(const ShadingData& sd, bool viewside = true) {
    return compute_ray_origin(sd.posW, (sd.frontFacing == viewside) ? sd.faceN : -sd.faceN);
}
FPT_D float3 sd_oriented_face_n(const ShadingData& sd) { return sd.frontFacing ? sd.faceN : -sd.faceN; }

template <bool HAS_TRANSMISSION>
struct MaterialInstance {
    float3 T, B, N;
    BSDFData data;
    float3 emission;
    bool thin, lambert;
    uint32_t activeLobes;

    FPT_D float3 toLocal(float3 v) const { return make_float3(dot(v, T), dot(v, B), dot(v, N)); }
    FPT_D float3 fromLocal(float3 v) const { return T * v.x + B * v.y + N * v.z; }
    FPT_D uint32_t lobeTypes() const { return bsdf_lobe_types(data); }
    FPT_D float propRoughness() const { return data.roughness * data.roughness < kMinGGXAlpha ? 0.f : data.roughness; }

    // isValidHemisphereReflectionOrTransmission (Scene/Material/ShadingUtils.slang:216-245).
    FPT_D bool valid_hemisphere(const ShadingData& sd, float3 wiL, float3 woL, float3 wo) const {
        const bool isT = wiL.z * woL.z < 0.f;
        if (hmin(wiL.z, fabsf(woL.z)) < kMinCosTheta) return false;
        const bool wiTop = sd.frontFacing, woTop = dot(wo, sd.faceN) >= 0.f;
        if (isT) { if (wiTop == woTop) return false; }
        else { if (wiTop != woTop) return false; }
        const bool shadingTop = dot(N, sd.faceN) >= 0.f;
        if (wiTop != shadingTop) return false;
        return true;
    }
    FPT_D StandardBSDF<HAS_TRANSMISSION> bsdf(float3 wiL) const {
        StandardBSDF<HAS_TRANSMISSION> b;
        b.init(wiL, data, thin, activeLobes, lambert);
        return b;
    }
    FPT_D float3 eval(const ShadingData& sd, float3 wo) const {
        const float3 wiL = toLocal(sd.V), woL = toLocal(wo);
        if (!valid_hemisphere(sd, wiL, woL, wo)) return f3(0.f);
        return bsdf(wiL).eval(wiL, woL);
    }
    FPT_D float evalPdf(const ShadingData& sd, float3 wo, bool useIS) const {
        const float3 wiL = toLocal(sd.V), woL = toLocal(wo);
        if (!valid_hemisphere(sd, wiL, woL, wo)) return 0.f;
        if (!useIS) {
            if (lobeTypes() & L_TRANSMISSION) {
                if (hmin(fabsf(wiL.z), fabsf(woL.z)) < kMinCosTheta) return 0.f;
                return 0.5f * woL.z * kInvPi;
            }
            if (hmin(wiL.z, woL.z) < kMinCosTheta) return 0.f;
            return woL.z * kInvPi;
        }
        return bsdf(wiL).eval_pdf(wiL, woL);
    }
    template <class SG>
    FPT_D bool sample(const ShadingData& sd, SG& sg, float3& wo, float3& weight, float& pdf, uint32_t& lobe, bool useIS) const {
        const float3 wiL = toLocal(sd.V);
        float3 woL = f3(0.f);
        if (!useIS) {
            // sampleReference (StandardMaterialInstance.slang:202-230).
            weight = f3(0.f);
            lobe = 0;
            const bool isTransmissive = (lobeTypes() & L_TRANSMISSION) != 0;
            woL = sample_cosine_hemisphere_concentric(next2D(sg), pdf);
            if (isTransmissive) {
                if (next1D(sg) < 0.5f) woL.z = -woL.z;
                pdf *= 0.5f;
                if (hmin(fabsf(wiL.z), fabsf(woL.z)) < kMinCosTheta || pdf == 0.f) return false;
            } else {
                if (hmin(wiL.z, woL.z) < kMinCosTheta || pdf == 0.f) return false;
            }
            weight = bsdf(wiL).eval(wiL, woL) / pdf;
            lobe = woL.z > 0.f ? L_DIFF_R : L_DIFF_T;
        } else {
            const StandardBSDF<HAS_TRANSMISSION> b = bsdf(wiL);
            if (!b.sample(wiL, woL, pdf, weight, lobe, sg)) return false;
        }
        wo = fromLocal(woL);
        if (!valid_hemisphere(sd, wiL, woL, wo)) return false;
        return true;
    }
};

template <bool HAS_TRANSMISSION>
FPT_D MaterialInstance<HAS_TRANSMISSION> material_instance(const DevScene& s, const ShadingData& sd, bool lambert) {
    const uint4* mp = reinterpret_cast<const uint4*>(s.materials + sd.materialID);
    const uint4 m0 = __ldg(mp), m1 = __ldg(mp + 1), m2 = __ldg(mp + 2);
    MaterialInstance<HAS_TRANSMISSION> mi;
    mi.lambert = lambert;
    const uint32_t flags = m2.w & 0xffffu;
    mi.thin = (flags & 2u) != 0;
    mi.activeLobes = m2.w >> 16;
    BSDFData& d = mi.data;
    const float IoR = f16(m2.x & 0xffffu);
    d.eta = sd.frontFacing ? (1.f / IoR) : (IoR / 1.f);
    d.specTrans = f16(m2.x >> 16);
    d.diffTrans = f16(m2.y & 0xffffu);
    d.transmission = f3(1.f);
    if (d.diffTrans > 0.f || d.specTrans > 0.f) d.transmission = make_float3(f16(m2.y >> 16), f16(m2.z & 0xffffu), f16(m2.z >> 16));
    const float f = (IoR - 1.f) / (IoR + 1.f);
    const float F0 = f * f;
    const float3 baseColor = make_float3(f16(m0.x & 0xffffu), f16(m0.x >> 16), f16(m0.y & 0xffffu));
    const float specG = f16(m0.z >> 16), specB = f16(m0.w & 0xffffu);
    d.diffuse = lerp(baseColor, f3(0.f), specB);
    d.specular = lerp(f3(F0), baseColor, specB);
    d.roughness = specG;
    d.metallic = specB;
    mi.T = sd.T; mi.B = sd.B; mi.N = sd.N;
    if (!sd.frontFacing && (flags & 1u)) mi.N = -mi.N;  // flipShadingNormal
    mi.emission = f3(0.f);
    if (sd.frontFacing) {
        const float fac = __uint_as_float(m1.w);
        mi.emission = make_float3(__uint_as_float(m1.x), __uint_as_float(m1.y), __uint_as_float(m1.z)) * fac;
    }
    return mi;
}

// ---------------------------------------------------------------------------
// Environment map (Scene/Lights/EnvMap.slang:58-68) with software bilinear
// filtering (wrap in u, clamp in v), and EnvMapSampler (EnvMapSampler.slang:75-164).
// ---------------------------------------------------------------------------
FPT_D float3 env_texel(const DevScene& s, int x, int y) {
    const float4 t = __ldg(s.env + size_t(y) * s.envW + x);
    return make_float3(t.x, t.y, t.z);
}
FPT_D float3 env_eval(const DevScene& s, float3 dir) {
    const float2 uv = world_to_latlong_map(dir);
    const float fx = uv.x * float(s.envW) - 0.5f, fy = uv.y * float(s.envH) - 0.5f;
    const float x0f = floorf(fx), y0f = floorf(fy);
    const float ax = fx - x0f, ay = fy - y0f;
    const int x0 = int(x0f), y0 = int(y0f);
    const int W = int(s.envW), H = int(s.envH);
    const int xa = ((x0 % W) + W) % W, xb = (((x0 + 1) % W) + W) % W;
    const int ya = min(max(y0, 0), H - 1), yb = min(max(y0 + 1, 0), H - 1);
    const float3 c = env_texel(s, xa, ya) * ((1.f - ax) * (1.f - ay)) + env_texel(s, xb, ya) * (ax * (1.f - ay)) +
                     env_texel(s, xa, yb) * ((1.f - ax) * ay) + env_texel(s, xb, yb) * (ax * ay);
    return c * make_float3(s.envScale[0], s.envScale[1], s.envScale[2]);
}
FPT_D float imp_load(const DevScene& s, uint32_t mip, uint32_t x, uint32_t y) {
    return __ldg(s.impMips + s.impMipOffset[mip] + size_t(y) * (s.impDim >> mip) + x);
}
FPT_D bool env_sample(const DevScene& s, float2 p, float3& dir, float& pdf, float3& Le) {
    uint32_t px = 0, py = 0;
    for (int mip = int(s.impBaseMip) - 1; mip >= 0; mip--) {
        px *= 2; py *= 2;
        const float w0 = imp_load(s, mip, px, py), w1 = imp_load(s, mip, px + 1, py);
        const float w2 = imp_load(s, mip, px, py + 1), w3 = imp_load(s, mip, px + 1, py + 1);
        const float q0 = w0 + w2, q1 = w1 + w3;
        uint32_t ox, oy;
        const float dd = q0 / (q0 + q1);
        if (p.x < dd) { ox = 0; p.x = p.x / dd; }
        else { ox = 1; p.x = (p.x - dd) / (1.f - dd); }
        const float e = ox == 0 ? (w0 / q0) : (w1 / q1);
        if (p.y < e) { oy = 0; p.y = p.y / e; }
        else { oy = 1; p.y = (p.y - e) / (1.f - e); }
        px += ox; py += oy;
    }
    const float inv = 1.f / float(s.impDim);
    const float2 uv = make_float2((float(px) + p.x) * inv, (float(py) + p.y) * inv);
    dir = oct_to_ndir_equal_area_unorm(uv);
    const float avg = imp_load(s, s.impBaseMip, 0, 0);
    const float pr = imp_load(s, 0, px, py) / avg;
    pdf = pr * kInv4Pi;
    Le = env_eval(s, dir);
    return true;
}
FPT_D float env_eval_pdf(const DevScene& s, float3 dir) {
    const float2 uv = ndir_to_oct_equal_area_unorm(dir);
    const float avg = imp_load(s, s.impBaseMip, 0, 0);
    int x = int(floorf(uv.x * float(s.impDim))), y = int(floorf(uv.y * float(s.impDim)));
    x = min(max(x, 0), int(s.impDim) - 1);
    y = min(max(y, 0), int(s.impDim) - 1);
    const float pr = imp_load(s, 0, uint32_t(x), uint32_t(y)) / avg;
    return pr * (1.f / k4Pi);
}

// ---------------------------------------------------------------------------
// Emissive triangle lights (EmissiveLightSamplerHelpers.slang:54-124,
// EmissiveUniformSampler.slang:55-110, EmissivePowerSampler.slang:61-124).
// ---------------------------------------------------------------------------
struct TriLightSample {
    float3 posW, normalW, dir, Le;
    float distance, pdf;
};

FPT_D bool sample_triangle_light(const DevScene& s, float3 posW, uint32_t tri, float2 u, TriLightSample& ls) {
    const uint4* tp = reinterpret_cast<const uint4*>(s.emissive + tri);
    const uint4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2), e = __ldg(tp + 3);
    const float3 P0 = make_float3(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z));
    const float3 P1 = make_float3(__uint_as_float(b.x), __uint_as_float(b.y), __uint_as_float(b.z));
    const float3 P2 = make_float3(__uint_as_float(c.x), __uint_as_float(c.y), __uint_as_float(c.z));
    const float3 bc = sample_triangle_bary(u);
    ls.posW = P0 * bc.x + P1 * bc.y + P2 * bc.z;
    const float3 toLight = ls.posW - posW;
    const float distSqr = hmax(kFltMin, dot(toLight, toLight));
    ls.distance = sqrtf(distSqr);
    ls.dir = toLight / ls.distance;
    ls.normalW = decode_normal2x16(e.x);
    const float cosTheta = dot(ls.normalW, -ls.dir);
    if (cosTheta <= 0.f) return false;
    const DevMaterial* m = s.materials + e.z;
    const float4 em = __ldg(reinterpret_cast<const float4*>(m) + 1);
    ls.Le = make_float3(em.x, em.y, em.z) * em.w;
    const float denom = hmax(kFltMin, cosTheta * __uint_as_float(e.y));
    ls.pdf = distSqr / denom;
    return true;
}
FPT_D float eval_triangle_pdf(const DevScene& s, float3 posW, uint32_t tri, float3 hitPos, float3 hitN) {
    const float3 toLight = hitPos - posW;
    const float distSqr = dot(toLight, toLight);
    if (distSqr <= kFltMin) return 0.f;
    const float3 L = toLight / sqrtf(distSqr);
    const float cosTheta = dot(hitN, -L);
    if (cosTheta <= 0.f) return 0.f;
    const float area = __ldg(&s.emissive[tri].area);
    const float denom = hmax(kFltMin, cosTheta * area);
    return distSqr / denom;
}
template <class SG>
FPT_D bool emissive_sample(const DevScene& s, uint32_t samplerType, float3 posW, SG& sg, TriLightSample& ls) {
    if (samplerType == 0) {
        if (s.activeCount == 0) return false;
        const float uLight = next1D(sg);
        const uint32_t n = s.activeCount;
        const uint32_t idx = min(uint32_t(uLight * float(n)), n - 1);
        const uint32_t tri = __ldg(s.activeTris + idx);
        const float selPdf = 1.f / float(n);
        const float2 u = next2D(sg);
        if (!sample_triangle_light(s, posW, tri, u, ls)) return false;
        ls.pdf *= selPdf;
        return true;
    }
    if (s.emissiveCount == 0) return false;
    const float uLight = next1D(sg);
    const uint32_t n = s.emissiveCount;
    uint32_t tri = min(uint32_t(uLight * float(n)), n - 1);
    const uint2 e = __ldg(s.alias + tri);
    const float threshold = f16(e.x >> 16);
    const uint32_t above = ((e.x & 0xFFFFu) << 8) | ((e.y >> 24) & 0xFFu);
    const uint32_t below = e.y & 0xFFFFFFu;
    tri = (next1D(sg) >= threshold) ? above : below;
    const float selPdf = __ldg(s.flux + tri) * s.invWeightSum;
    const float2 u = next2D(sg);
    if (!sample_triangle_light(s, posW, tri, u, ls)) return false;
    ls.pdf *= selPdf;
    return true;
}
FPT_D float emissive_eval_pdf(const DevScene& s, uint32_t samplerType, float3 posW, uint32_t tri, float3 hitPos, float3 hitN) {
    if (tri == 0xffffffffu) return 0.f;
    float sel;
    if (samplerType == 0) sel = s.activeCount > 0 ? 1.f / float(s.activeCount) : 0.f;
    else sel = __ldg(s.flux + tri) * s.invWeightSum;
    return sel * eval_triangle_pdf(s, posW, tri, hitPos, hitN);
}

}  // namespace dev
}  // namespace fpt
