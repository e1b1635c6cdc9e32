// war_common.cuh -- WARDiffPathTracer device pieces shared by the
// megakernel (wardiff.cu) and the wavefront scheduler (war_wavefront.cu):
// launch parameters, the AttachToRay intersection, loadShadingData, evalMIS,
// material parameters and the local Jacobians of evalAD.
#pragma once

#include "diff_bsdf.cuh"
#include "kernels.cuh"
#include "path_logic.cuh"

#include "war_wavefront.h"

namespace fpt {
namespace {

using namespace dev;

constexpr int kMaxWarVertices = 16;   // maxBounces <= 14 in the adjoint
constexpr uint32_t kMatParams = 20;   // DiffMaterialData::kMaterialParamCount



// Intersection recomputed from the hit triangle (DiffSceneQuery.slang:148-219).
struct WarIsect {
    uint32_t inst, prim;
    float b[3];
    float3 posW;
    float3 normalW, tangentW;    // interpolated, unnormalised
    float tw;                    // sign of the interpolated tangent w
    uint32_t local[3];           // vertex indices within the mesh
    uint32_t vbOffset;           // first vertex of the mesh in the scene's vertex buffer
};

// Mesh-position gradient target: one mesh (InverseOptimizationParams.meshID),
// or every mesh with scene-global vertex indices when meshID is kAllMeshes.
constexpr uint32_t kAllMeshes = 0xffffffffu;
FPT_D bool war_pos_target(uint32_t meshID, const WarIsect& is) { return meshID == kAllMeshes || is.inst == meshID; }
FPT_D uint32_t war_pos_index(uint32_t meshID, const WarIsect& is, int v) {
    return (meshID == kAllMeshes ? is.vbOffset + is.local[v] : is.local[v]) * 3u;
}

FPT_D float war_ray_distance(float3 v0, float3 v1, float3 v2, float3 o, float3 d) {
    const float3 e1 = v1 - v0, e2 = v2 - v0;
    const float3 pvec = cross(d, e2);
    const float det = dot(e1, pvec);
    const float3 tvec = o - v0;
    const float3 qvec = cross(tvec, e1);
    return dot(e2, qvec) / det;
}

// Completes a WarIsect from the hit triangle and its barycentrics; these come
// from the ray (AttachToRay) or from a stored path vertex.
FPT_D WarIsect war_isect_bary(const DevScene& s, uint32_t instID, uint32_t prim, float b0, float b1, float b2);

FPT_D WarIsect war_intersect(const DevScene& s, const HitRec& h, float3 o, float3 d) {
    const DevInstance inst = s.instances[h.instanceID];
    const uint32_t* ip = s.indices + inst.ibOffset + h.primIndex * 3;
    float3 v0, v1, v2, n0, n1, n2;
    unpack_vertex(load_vertex(s.vertices, __ldg(ip) + inst.vbOffset), v0, n0);
    unpack_vertex(load_vertex(s.vertices, __ldg(ip + 1) + inst.vbOffset), v1, n1);
    unpack_vertex(load_vertex(s.vertices, __ldg(ip + 2) + inst.vbOffset), v2, n2);
    // computeBarycentrics of the ray/triangle-plane point (GeometryHelpers.slang:442-482).
    const float t = war_ray_distance(v0, v1, v2, o, d);
    const float3 p = o + d * t;
    const float3 e0 = v0 - p, e1 = v1 - p, e2 = v2 - p;
    const float a0 = length(cross(e1, e2));
    const float a1 = length(cross(e2, e0));
    const float a2 = length(cross(e0, e1));
    const float area = a0 + a1 + a2;
    return war_isect_bary(s, h.instanceID, h.primIndex, a0 / area, a1 / area, a2 / area);
}

FPT_D WarIsect war_isect_bary(const DevScene& s, uint32_t instID, uint32_t prim, float b0, float b1, float b2) {
    WarIsect is;
    is.inst = instID;
    is.prim = prim;
    const DevInstance inst = s.instances[instID];
    const uint32_t* ip = s.indices + inst.ibOffset + prim * 3;
    is.local[0] = __ldg(ip);
    is.local[1] = __ldg(ip + 1);
    is.local[2] = __ldg(ip + 2);
    is.vbOffset = inst.vbOffset;
    const PackedVertex pv0 = load_vertex(s.vertices, is.local[0] + inst.vbOffset);
    const PackedVertex pv1 = load_vertex(s.vertices, is.local[1] + inst.vbOffset);
    const PackedVertex pv2 = load_vertex(s.vertices, is.local[2] + inst.vbOffset);
    float3 v0, v1, v2, n0, n1, n2;
    unpack_vertex(pv0, v0, n0);
    unpack_vertex(pv1, v1, n1);
    unpack_vertex(pv2, v2, n2);
    is.b[0] = b0;
    is.b[1] = b1;
    is.b[2] = b2;
    is.posW = v0 * is.b[0] + v1 * is.b[1] + v2 * is.b[2];
    // loadVertexNormalsW / loadVertexTangentsW (DiffSceneIO.slang:145-258), identity world matrices.
    n0 = normalize(n0); n1 = normalize(n1); n2 = normalize(n2);
    const float3 t0 = normalize(decode_normal2x16(pv0.tangentOct)), t1 = normalize(decode_normal2x16(pv1.tangentOct)),
                 t2 = normalize(decode_normal2x16(pv2.tangentOct));
    is.normalW = n0 * is.b[0] + n1 * is.b[1] + n2 * is.b[2];
    is.tangentW = t0 * is.b[0] + t1 * is.b[1] + t2 * is.b[2];
    // VertexData.tangentW.w with the TriangleHit barycentric weights (Scene.slang:452-455).
    const float w0 = sgn(f16(pv0.nz_tw >> 16)), w1 = sgn(f16(pv1.nz_tw >> 16)), w2 = sgn(f16(pv2.nz_tw >> 16));
    const float bx = is.b[1], by = is.b[2];
    float tw = w0 * (1.f - bx - by);
    tw += w1 * bx;
    tw += w2 * by;
    is.tw = sgn(tw);
    return is;
}

// loadShadingData (PTUtils.slang:97-123): the vertex data of the hit with
// sd.frame = ShadingFrame::createSafe(isect.normalW, float4(isect.tangentW, v.tangentW.w)).
FPT_D ShadingData war_shading_data(const DevScene& s, const WarIsect& is, float3 rayDir) {
    HitRec th;
    th.instanceID = is.inst;
    th.primIndex = is.prim;
    th.globalTri = 0;
    th.baryX = is.b[1];
    th.baryY = is.b[2];
    th.t = 0.f;
    th.valid = true;
    ShadingData sd = load_shading_data(s, th, rayDir);
    sd.N = normalize(is.normalW);
    const float3 tg = is.tangentW;
    const float NdotT = dot(tg, sd.N);
    const bool valid = fabsf(is.tw) == 1.f && dot(tg, tg) > 0.f && fabsf(NdotT) < 0.9999f;
    if (valid) {
        sd.T = normalize(tg - sd.N * NdotT);
        sd.B = cross(sd.N, sd.T) * is.tw;
    } else {
        sd.T = perp_stark(sd.N);
        sd.B = cross(sd.N, sd.T);
    }
    return sd;
}

// evalMIS, power-two heuristic (PTUtils.slang:87-93).
FPT_D float war_mis(float n0, float p0, float n1, float p1) {
    const float q0 = (n0 * p0) * (n0 * p0);
    const float q1 = (n1 * p1) * (n1 * p1);
    return q0 / (q0 + q1);
}

// Raw material parameters (StandardMaterialParamLayout order) of a material.
struct MatParams {
    float3 baseColor, transmission;
    float metallic, roughness, ior, diffTrans, specTrans;
};
// A textured material's base colour is its texture's value at uv.
FPT_D MatParams load_mat_params(const DevScene& s, uint32_t id, float2 uv) {
    const uint4* mp = reinterpret_cast<const uint4*>(s.materials + id);
    const uint4 m0 = __ldg(mp), m2 = __ldg(mp + 2);
    MatParams m;
    m.baseColor = make_float3(f16(m0.x & 0xffffu), f16(m0.x >> 16), f16(m0.y & 0xffffu));
    if (m2.w & kMatFlagBaseColorTexture) m.baseColor = tex_sample(s, __ldg(reinterpret_cast<const uint32_t*>(mp + 3)), uv);
    m.roughness = f16(m0.z >> 16);
    m.metallic = f16(m0.w & 0xffffu);
    m.ior = f16(m2.x & 0xffffu);
    m.specTrans = f16(m2.x >> 16);
    m.diffTrans = f16(m2.y & 0xffffu);
    m.transmission = make_float3(f16(m2.y >> 16), f16(m2.z & 0xffffu), f16(m2.z >> 16));
    return m;
}

// Jacobian of one evalAD with respect to the 11 material parameters (slots
// 0-10), for N >= 14 the local outgoing direction (slots 11-13) and, for
// N = 17, the local incident direction (slots 14-16).
template <int N, bool HAS_T>
FPT_D DV3<N> eval_jacobian(const MaterialInstance<HAS_T>& mi, const MatParams& mp, bool frontFacing, float3 wiL, float3 woL) {
    const StandardBSDF<HAS_T> b = mi.bsdf(wiL);
    const DBSDFData<N> d = diff_bsdf_data<N>(mp.baseColor, mp.metallic, mp.roughness, mp.ior, mp.transmission, mp.diffTrans,
                                             mp.specTrans, frontFacing);
    const DV3<N> wi = N >= 17 ? dv3(dvar<N>(wiL.x, 14), dvar<N>(wiL.y, 15), dvar<N>(wiL.z, 16)) : dv3c<N>(wiL);
    const DV3<N> wo = dv3(dvar<N>(woL.x, 11), dvar<N>(woL.y, 12), dvar<N>(woL.z, 13));
    return diff_bsdf_eval<N>(d, wi, wo, mi.thin, mi.activeLobes, mi.lambert, b.pDR, HAS_T ? b.pDT : 0.f, b.pSR,
                             HAS_T ? b.pST : 0.f);
}

FPT_D uint32_t war_hash(uint32_t pixelID, uint32_t hashSize) { return jenkins_hash(pixelID) % hashSize; }

// Debug gradient image (ForwardDiffDebug / BackwardDiffDebug): one scene
// variable -- the floats one material read returns (GradientIOWrapper.slang:87-94)
// or the translation of one mesh (DiffSceneIO.slang:85-93, 122-131) -- whose
// derivative d(color.r)/d(variable) goes to dbgColor[pixel].x.  DiffVariableType
// values (DiffRendering/SharedTypes.slang:90-96).
constexpr uint32_t kDbgNone = 0, kDbgMaterial = 1, kDbgTranslation = 2;

// The adjoint of a pixel's radiance: dLdI, or (1, 0, 0) for the debug image.
FPT_D float3 war_dLdI(const WarParams& p, uint32_t pid) {
    if (!p.dLdI) return make_float3(1.f, 0.f, 0.f);
    return make_float3(p.dLdI[3 * size_t(pid)], p.dLdI[3 * size_t(pid) + 1], p.dLdI[3 * size_t(pid) + 2]);
}
// Whether vertex-position derivatives are wanted (gradients or the translation image).
FPT_D bool war_wants_pos(const WarParams& p) { return p.gradPos != nullptr || (p.dbgColor && p.dbgType == kDbgTranslation); }

// Tangent of material parameter `slot` under the debug variable: the floats of
// the getFloat read at dbgOffset (3 for the colours at 0, 6 and 11, else 1).
FPT_D float war_dbg_tangent(const WarParams& p, uint32_t slot) {
    const uint32_t o = p.dbgOffset;
    const uint32_t width = (o == 0 || o == 6 || o == 11) ? 3u : 1u;
    if (slot < o || slot - o >= width) return 0.f;
    const uint32_t i = slot - o;
    return i == 0 ? p.dbgGrad.x : (i == 1 ? p.dbgGrad.y : p.dbgGrad.z);
}

// Warp-aggregated gradient atomics (SceneGradients::atomicAddGrad,
// DiffRendering/SceneGradients.slang:50-57, InterlockedAddF32): the lanes of a
// warp that add to the same N-float row find one another with match.any, sum
// their values with shuffles, and the lowest lane of each group issues one
// atomic per non-zero float.  Lanes adding to distinct rows pay one match, one
// max-reduction and one shuffle per value.
template <int N>
FPT_D void atomic_add_row(float* row, const float (&v)[N]) {
    const uint32_t active = __activemask();
    const uint32_t peers = __match_any_sync(active, reinterpret_cast<unsigned long long>(row));
    uint32_t lane;
    asm("mov.u32 %0, %%laneid;" : "=r"(lane));
    const uint32_t rounds = __reduce_max_sync(active, uint32_t(__popc(peers)));
    float sum[N];
#pragma unroll
    for (int i = 0; i < N; i++) sum[i] = 0.f;
    uint32_t rem = peers;
    for (uint32_t k = 0; k < rounds; k++) {
        const int src = rem ? __ffs(rem) - 1 : int(lane);
#pragma unroll
        for (int i = 0; i < N; i++) {
            const float x = __shfl_sync(active, v[i], src);
            if (rem) sum[i] += x;
        }
        if (rem) rem &= rem - 1u;
    }
    if (int(lane) == __ffs(peers) - 1) {
#pragma unroll
        for (int i = 0; i < N; i++)
            if (sum[i] != 0.f) atomicAdd(row + i, sum[i]);
    }
}

// Gradient of a textured base colour.  The reference samples textures no_diff
// (StandardMaterial.slang:164); here dL/d(texel rgb) += w_k dL/d(baseColor)
// for the four texels k of the bilinear lookup at uv, into a flat buffer of 3
// floats per texel of every texture (DevTexture::texelBase order).
FPT_D void add_texture_grad(const DevScene& s, const WarParams& p, uint32_t tex, float2 uv, float g0, float g1, float g2) {
    if (!p.gradTex || (g0 == 0.f && g1 == 0.f && g2 == 0.f)) return;
    const DevTexture t = load_texture(s, tex);
    const fpt_tex::Bilinear b = fpt_tex::bilinear(uv.x, uv.y, t.width, t.height);
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const uint32_t x = (k & 1) ? b.x1 : b.x0, y = (k & 2) ? b.y1 : b.y0;
        const uint64_t idx = (uint64_t(t.texelBase) + uint64_t(y) * t.width + x) * 3u;
        if (idx + 3u > p.texDim) continue;
        const float row[3] = {g0 * b.w[k], g1 * b.w[k], g2 * b.w[k]};
        atomic_add_row<3>(p.gradTex + idx, row);
    }
}

// Material-parameter gradients G[0..10] of material matID from pixel pid; the
// base-colour entries of a textured material go to its texture at uv.
FPT_D void add_material_grad_values(const DevScene& s, const WarParams& p, uint32_t pid, uint32_t hash, uint32_t matID, float2 uv,
                                    const float (&G0)[11]) {
    float G[11];
#pragma unroll
    for (int i = 0; i < 11; i++) G[i] = G0[i];
    const uint32_t tex = material_base_texture(s, matID);
    if (tex != ~0u) {
        add_texture_grad(s, p, tex, uv, G[0], G[1], G[2]);
        G[0] = G[1] = G[2] = 0.f;
    }
    if (p.dbgColor && p.dbgType == kDbgMaterial) {
        if (matID != p.dbgId) return;
        float acc = 0.f;
#pragma unroll
        for (int i = 0; i < 11; i++) acc += G[i] * war_dbg_tangent(p, uint32_t(i));
        if (acc != 0.f) atomicAdd(&p.dbgColor[pid].x, acc);
        return;
    }
    if (!p.gradMat) return;
    const uint32_t base = matID * kMatParams;
    if (base + 11 > p.matDim) return;
    atomic_add_row<11>(p.gradMat + size_t(hash) * p.matDim + base, G);
}

// Adds sum_c G_c * J_c[i] for the 11 material parameters.
template <int N>
FPT_D void add_material_grads(const DevScene& s, const WarParams& p, uint32_t pid, uint32_t hash, uint32_t matID, float2 uv,
                              const DV3<N>& J, float3 G) {
    float v[11];
#pragma unroll
    for (int i = 0; i < 11; i++) v[i] = G.x * J.x.d[i] + G.y * J.y.d[i] + G.z * J.z.d[i];
    add_material_grad_values(s, p, pid, hash, matID, uv, v);
}

// Position gradient g of a point sum_v b_v x_v of a target mesh's triangle whose
// vertices sit at gradient offsets off[v] (the caller checks the target mesh).
FPT_D void add_position_grad(const WarParams& p, uint32_t pid, const uint32_t (&off)[3], const float (&b)[3], float3 g) {
    if (p.dbgColor && p.dbgType == kDbgTranslation) {
        // sum_v dot(velocity, dPos_v) (DiffSceneIO.slang:127-129).
        const float v = dot(make_float3(p.dbgGrad.x, p.dbgGrad.y, p.dbgGrad.z), g) * (b[0] + b[1] + b[2]);
        if (v != 0.f) atomicAdd(&p.dbgColor[pid].x, v);
        return;
    }
    if (!p.gradPos) return;
    float* gp = p.gradPos + size_t(war_hash(pid, p.posHash)) * p.posDim;
#pragma unroll
    for (int v = 0; v < 3; v++) {
        const uint32_t o = off[v];
        if (o + 3 > p.posDim) continue;
        const float row[3] = {b[v] * g.x, b[v] * g.y, b[v] * g.z};
        atomic_add_row<3>(gp + o, row);
    }
}
FPT_D void add_position_grad(const WarParams& p, uint32_t pid, const WarIsect& is, float3 g) {
    const uint32_t off[3] = {war_pos_index(p.meshID, is, 0), war_pos_index(p.meshID, is, 1), war_pos_index(p.meshID, is, 2)};
    add_position_grad(p, pid, off, is.b, g);
}

// Whether vertex normal / tangent gradients are wanted.
FPT_D bool war_wants_frame(const WarParams& p) { return p.gradNrm != nullptr || p.gradTan != nullptr; }

// Adjoint of the interpolated (unnormalised) vertex normal and tangent of a
// path vertex from the adjoints gwiL, gwoL of one evalAD's local directions
// wiL = frame(V), woL = frame(wo).  The frame is loadShadingData's
// ShadingFrame::createSafe(normalW, float4(tangentW, w)) (ShadingFrame.slang:76-153)
// with flipShadingNormal (ShadingUtils.slang:111-117); perp_stark is no_diff.
FPT_D void war_frame_adjoint(const WarIsect& is, bool flip, float3 V, float3 wo, float3 gwiL, float3 gwoL, float3& gn, float3& gt) {
    const float ln = length(is.normalW);
    const float3 N0 = is.normalW / ln;
    const float3 t = is.tangentW;
    const float tn = dot(t, N0);
    const bool valid = fabsf(is.tw) == 1.f && dot(t, t) > 0.f && fabsf(tn) < 0.9999f;
    float3 u = f3(0.f), T;
    float lu = 1.f, sw = 1.f;
    if (valid) {
        u = t - N0 * tn;
        lu = length(u);
        T = u / lu;
        sw = is.tw;
    } else {
        T = perp_stark(N0);
    }
    float3 gT = V * gwiL.x + wo * gwoL.x;
    const float3 gB = V * gwiL.y + wo * gwoL.y;
    float3 gN0 = (V * gwiL.z + wo * gwoL.z) * (flip ? -1.f : 1.f);
    // B = cross(N0, T) * w.
    gN0 += cross(T, gB) * sw;
    gT += cross(gB, N0) * sw;
    gt = f3(0.f);
    if (valid) {
        // T = normalize(t - N0 (t . N0)).
        const float3 gu = (gT - T * dot(T, gT)) / lu;
        gt = gu - N0 * dot(N0, gu);
        gN0 -= gu * tn + t * dot(N0, gu);
    }
    // N0 = normalize(normalW).
    gn = (gN0 - N0 * dot(N0, gN0)) / ln;
}

// Normal / tangent gradients gn, gt of the interpolation sum_v b_v n_v of a
// target mesh's triangle (vertex gradient offsets off[v]).
FPT_D void add_frame_grad(const WarParams& p, uint32_t pid, const uint32_t (&off)[3], const float (&b)[3], float3 gn, float3 gt) {
    float* an = p.gradNrm ? p.gradNrm + size_t(war_hash(pid, p.nrmHash)) * p.nrmDim : nullptr;
    float* at = p.gradTan ? p.gradTan + size_t(war_hash(pid, p.tanHash)) * p.tanDim : nullptr;
#pragma unroll
    for (int v = 0; v < 3; v++) {
        const uint32_t o = off[v];
        if (an && o + 3 <= p.nrmDim) {
            const float row[3] = {b[v] * gn.x, b[v] * gn.y, b[v] * gn.z};
            atomic_add_row<3>(an + o, row);
        }
        if (at && o + 3 <= p.tanDim && (gt.x != 0.f || gt.y != 0.f || gt.z != 0.f)) {
            const float row[3] = {b[v] * gt.x, b[v] * gt.y, b[v] * gt.z};
            atomic_add_row<3>(at + o, row);
        }
    }
}

}  // namespace
}  // namespace fpt
