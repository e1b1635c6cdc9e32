// wardiff.cu -- WARDiffPathTracer on sm_100a: the primal render and the
// reverse-mode gradients of material parameters and mesh vertex positions
// (bwd_diff(tracePaths), RenderPasses/WARDiffPathTracer/WARDiffPathTracer.rt.slang:167-180),
// plus SceneGradients (DiffRendering/SceneGradients.cpp:42-206).
//
// One thread traces one path per pixel (WARDiffPathTracer.rt.slang:146-212).
// The adjoint kernel re-traces the same path (same sample generator state), so
// the primal does not have to be stored between the passes.  While tracing it
//  * accumulates the NEE term's gradients at once -- the adjoint of a radiance
//    increment is dL/dI itself -- and
//  * records, per path vertex, what the scatter term needs (local directions,
//    throughput, pdf, BSDF weight, radiance increments), then sweeps the
//    vertices backwards carrying the adjoint of the throughput:
//        A_k = dLdI * e_k + A_{k+1} * w_k,
//        dS/df_k(ws) = A_{k+1} * thp_k / pdf_k,
//    which is exactly the reverse-mode derivative of the loop, with no
//    division by the path throughput.
// Local Jacobians of StandardBSDF.eval come from diff_bsdf.cuh.  Which
// quantities are differentiable follows the Slang sources:
//  * sampling, light selection, MIS weights and emission are not
//    (PTUtils.slang:177-207, StandardMaterialInstance.slang:92-160);
//  * the AttachToRay hit position is sum(v_i * b_i) with the barycentrics of
//    computeBarycentrics detached (GeometryHelpers.slang:465-482,
//    DiffSceneQuery.slang:195-219), so positions enter only through the NEE
//    direction and the area-to-solid-angle ratio x / detach(x)
//    (PTUtils.slang:211-249);
//  * warped-area reparameterisation leaves every value unchanged
//    (WarpedAreaReparam.slang:226-263); its boundary gradients are not
//    produced by this adjoint (useWAR is accepted and reported).
#include <cstring>
#include <string>

#include "diff_bsdf.cuh"
#include "kernels.cuh"
#include "path_logic.cuh"
#include "passes.h"
#include "scene_device.h"
#include "wardiff.h"

namespace fpt {

using namespace dev;

namespace {

constexpr int kWarBlock = 128;
constexpr int kMaxWarVertices = 16;   // maxBounces <= 14 in the adjoint
constexpr uint32_t kMatParams = 20;   // DiffMaterialData::kMaterialParamCount

struct WarParams {
    uint32_t width, height, maxBounces;
    uint32_t useBSDFSampling, useNEE, useMIS, useAntithetic;
    uint32_t frameSeed, lambert, meshID;
    float4* color;               // primal output
    const float* dLdI;           // float3 per pixel (adjoint)
    float* gradMat;              // [hash][matDim]
    uint32_t matDim, matHash;
    float* gradPos;              // [hash][posDim]
    uint32_t posDim, posHash;
    unsigned long long* counters;  // [0] paths, [1] rays
};

// Intersection recomputed from the hit triangle (DiffSceneQuery.slang:148-219).
struct WarIsect {
    uint32_t inst, prim;
    float b[3];
    float3 posW;
    float3 normalW, tangentW;    // interpolated, unnormalised
    float tw;                    // sign of the interpolated tangent w
    uint32_t local[3];           // vertex indices within the mesh
};

FPT_D float war_ray_distance(float3 v0, float3 v1, float3 v2, float3 o, float3 d) {
    const float3 e1 = v1 - v0, e2 = v2 - v0;
    const float3 pvec = cross(d, e2);
    const float det = dot(e1, pvec);
    const float3 tvec = o - v0;
    const float3 qvec = cross(tvec, e1);
    return dot(e2, qvec) / det;
}

FPT_D WarIsect war_intersect(const DevScene& s, const HitRec& h, float3 o, float3 d) {
    WarIsect is;
    is.inst = h.instanceID;
    is.prim = h.primIndex;
    const DevInstance inst = s.instances[h.instanceID];
    const uint32_t* ip = s.indices + inst.ibOffset + h.primIndex * 3;
    is.local[0] = __ldg(ip);
    is.local[1] = __ldg(ip + 1);
    is.local[2] = __ldg(ip + 2);
    const PackedVertex pv0 = load_vertex(s.vertices, is.local[0] + inst.vbOffset);
    const PackedVertex pv1 = load_vertex(s.vertices, is.local[1] + inst.vbOffset);
    const PackedVertex pv2 = load_vertex(s.vertices, is.local[2] + inst.vbOffset);
    float3 v0, v1, v2, n0, n1, n2;
    unpack_vertex(pv0, v0, n0);
    unpack_vertex(pv1, v1, n1);
    unpack_vertex(pv2, v2, n2);
    // computeBarycentrics of the ray/triangle-plane point (GeometryHelpers.slang:442-482).
    const float t = war_ray_distance(v0, v1, v2, o, d);
    const float3 p = o + d * t;
    const float3 e0 = v0 - p, e1 = v1 - p, e2 = v2 - p;
    const float a0 = length(cross(e1, e2));
    const float a1 = length(cross(e2, e0));
    const float a2 = length(cross(e0, e1));
    const float area = a0 + a1 + a2;
    is.b[0] = a0 / area;
    is.b[1] = a1 / area;
    is.b[2] = a2 / area;
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
FPT_D MatParams load_mat_params(const DevScene& s, uint32_t id) {
    const uint4* mp = reinterpret_cast<const uint4*>(s.materials + id);
    const uint4 m0 = __ldg(mp), m2 = __ldg(mp + 2);
    MatParams m;
    m.baseColor = make_float3(f16(m0.x & 0xffffu), f16(m0.x >> 16), f16(m0.y & 0xffffu));
    m.roughness = f16(m0.z >> 16);
    m.metallic = f16(m0.w & 0xffffu);
    m.ior = f16(m2.x & 0xffffu);
    m.specTrans = f16(m2.x >> 16);
    m.diffTrans = f16(m2.y & 0xffffu);
    m.transmission = make_float3(f16(m2.y >> 16), f16(m2.z & 0xffffu), f16(m2.z >> 16));
    return m;
}

// Jacobian of one evalAD with respect to the 11 material parameters (slots
// 0-10) and, for N = 14, the local outgoing direction (slots 11-13).
template <int N, bool HAS_T>
FPT_D DV3<N> eval_jacobian(const MaterialInstance<HAS_T>& mi, const MatParams& mp, bool frontFacing, float3 wiL, float3 woL) {
    const StandardBSDF<HAS_T> b = mi.bsdf(wiL);
    const DBSDFData<N> d = diff_bsdf_data<N>(mp.baseColor, mp.metallic, mp.roughness, mp.ior, mp.transmission, mp.diffTrans,
                                             mp.specTrans, frontFacing);
    const DV3<N> wi = dv3c<N>(wiL);
    const DV3<N> wo = dv3(dvar<N>(woL.x, 11), dvar<N>(woL.y, 12), dvar<N>(woL.z, 13));
    return diff_bsdf_eval<N>(d, wi, wo, mi.thin, mi.activeLobes, mi.lambert, b.pDR, HAS_T ? b.pDT : 0.f, b.pSR,
                             HAS_T ? b.pST : 0.f);
}

FPT_D uint32_t war_hash(uint32_t pixelID, uint32_t hashSize) { return jenkins_hash(pixelID) % hashSize; }

// Adds sum_c G_c * J_c[i] for the 11 material parameters.
template <int N>
FPT_D void add_material_grads(const WarParams& p, uint32_t hash, uint32_t matID, const DV3<N>& J, float3 G) {
    if (!p.gradMat) return;
    const uint32_t base = matID * kMatParams;
    if (base + 11 > p.matDim) return;
    float* g = p.gradMat + size_t(hash) * p.matDim + base;
#pragma unroll
    for (int i = 0; i < 11; i++) {
        const float v = G.x * J.x.d[i] + G.y * J.y.d[i] + G.z * J.z.d[i];
        if (v != 0.f) atomicAdd(g + i, v);
    }
}

struct WarVertex {
    float3 wiL, wsL, thp, bw, e;
    float pdf;
    uint32_t matID;
    uint32_t flags;  // 1 front facing, 2 scattered with a valid evaluation
};

template <bool HAS_T, bool BWD>
__global__ void __launch_bounds__(kWarBlock) war_kernel(DevScene s, WarParams p) {
    __shared__ uint2 stackMem[kStackSize * kWarBlock];
    uint2* stack = stackMem + threadIdx.x;
    Counters cnt;
    const uint32_t pixels = p.width * p.height;
    const bool useEmissive = s.hasEmissive != 0 && s.activeCount > 0;
    for (uint32_t pid = blockIdx.x * blockDim.x + threadIdx.x; pid < pixels; pid += gridDim.x * blockDim.x) {
        const uint32_t x = pid % p.width, y = pid / p.width;
        // tracePaths (WARDiffPathTracer.rt.slang:115-143).
        UniformSG sg;
        sg.init(x, y, p.frameSeed / 2);
        next2D(sg);
        next2D(sg);
        next2D(sg);
        const float2 u = next2D(sg);
        const float r = sqrtf(-2.f * logf(u.x));
        const float ang = 6.28318530717958647692f * u.y;
        float jx = (r * cosf(ang)) * 0.5f, jy = (r * sinf(ang)) * 0.5f;
        if (p.useAntithetic && p.frameSeed % 2 == 0) { jx = -jx; jy = -jy; }
        const float px = (float(x) + 0.5f) + jx, py = (float(y) + 0.5f) + jy;
        // computeCameraRayDirection (DiffSceneQuery.slang:314-323).
        const float qx = px / float(p.width), qy = py / float(p.height);
        const float ndcx = 2.f * qx + -1.f, ndcy = -2.f * qy + 1.f;
        const float3 dirU = load3(s.camera.cameraU) * ndcx + load3(s.camera.cameraV) * ndcy + load3(s.camera.cameraW);
        const float len = length(dirU);
        float3 rayDir = len > 0.f ? dirU / len : f3(0.f);
        float3 rayOrigin = load3(s.camera.posW);

        float3 radiance = f3(0.f), thp = f3(1.f);
        float pathPdf = 0.f;
        uint32_t pathLen = 0;
        float3 g = f3(0.f);
        uint32_t hash = 0, hashPos = 0;
        if (BWD) {
            g = make_float3(p.dLdI[3 * size_t(pid)], p.dLdI[3 * size_t(pid) + 1], p.dLdI[3 * size_t(pid) + 2]);
            hash = war_hash(pid, p.matHash ? p.matHash : 1);
            hashPos = war_hash(pid, p.posHash ? p.posHash : 1);
        }
        WarVertex rec[BWD ? kMaxWarVertices : 1];
        int nv = 0;

        cnt.v[0]++;
        cnt.v[1]++;
        cnt.v[2]++;
        HitRec h;
        trace_bvh<false>(s, rayOrigin, rayDir, 0.f, 3.402823466e+38f, h, stack, kWarBlock);
        if (h.valid) {
            WarIsect is = war_intersect(s, h, rayOrigin, rayDir);
            for (;;) {
                // handleHit (PTUtils.slang:253-341).
                cnt.v[6]++;
                const ShadingData sd = war_shading_data(s, is, rayDir);
                const MaterialInstance<HAS_T> mi = material_instance<HAS_T>(s, sd, p.lambert != 0);
                float3 e = f3(0.f);
                const bool isPrimaryHit = pathLen == 0;
                const bool computeEmissive = isPrimaryHit || (useEmissive && (!p.useNEE || p.useMIS));
                if (computeEmissive && any_pos(mi.emission)) {
                    float misWeight = 1.f;
                    if (!isPrimaryHit && useEmissive && p.useNEE && p.useMIS) {
                        const uint32_t off = __ldg(s.instEmissiveOffset + is.inst);
                        const uint32_t tri = off == 0xffffffffu ? 0xffffffffu : off + is.prim;
                        const float lightPdf = emissive_eval_pdf(s, 0, rayOrigin, tri, sd.posW, sd_oriented_face_n(sd));
                        misWeight = war_mis(1.f, pathPdf, 1.f, lightPdf);
                    }
                    radiance += (thp * mi.emission) * misWeight;
                    if (BWD) e += mi.emission * misWeight;
                }
                WarVertex* vr = BWD ? &rec[nv] : nullptr;
                if (BWD) {
                    vr->thp = thp;
                    vr->wiL = vr->wsL = vr->bw = vr->e = f3(0.f);
                    vr->pdf = 1.f;
                    vr->flags = sd.frontFacing ? 1u : 0u;
                    vr->matID = sd.materialID;
                    nv++;
                }
                if (pathLen >= p.maxBounces + 1) {
                    if (BWD) vr->e = e;
                    break;
                }
                if (p.useNEE && useEmissive) {
                    // generateEmissiveSample (PTUtils.slang:177-207) with the uniform sampler.
                    TriLightSample tls;
                    cnt.v[7]++;
                    if (emissive_sample(s, 0, is.posW, sg, tls)) {
                        const float3 Li = tls.pdf > 0.f ? tls.Le / tls.pdf : f3(0.f);
                        const float3 lightPos = compute_ray_origin(tls.posW, tls.normalW);
                        const float3 origin = compute_ray_origin(is.posW, is.normalW);
                        const float3 toLight = lightPos - origin;
                        const float distance = length(toLight);
                        const float3 ldir = normalize(toLight);
                        if (any_pos(Li)) {
                            HitRec sh;
                            cnt.v[1]++;
                            cnt.v[3]++;
                            trace_bvh<true>(s, origin, ldir, 0.f, distance, sh, stack, kWarBlock);
                            if (!sh.valid) {
                                // computeNEE (PTUtils.slang:211-249).
                                float3 wo = tls.posW - is.posW;
                                const float dist = length(wo);
                                wo /= dist;
                                const float a2s = (dist * dist) / dot(tls.normalW, -wo);
                                const float3 bsdfValue = mi.eval(sd, wo);
                                float3 weight = ((Li * bsdfValue) * a2s) / a2s;
                                float mis = 1.f;
                                if (p.useMIS) {
                                    const float scatterPdf = mi.evalPdf(sd, ldir, p.useBSDFSampling != 0);
                                    mis = war_mis(1.f, tls.pdf, 1.f, scatterPdf);
                                    weight *= mis;
                                }
                                radiance += thp * weight;
                                if (BWD) {
                                    e += weight;
                                    const float3 wiL = mi.toLocal(sd.V), woL = mi.toLocal(wo);
                                    if (mi.valid_hemisphere(sd, wiL, woL, wo)) {
                                        const MatParams mp = load_mat_params(s, sd.materialID);
                                        const DV3<14> J = eval_jacobian<14, HAS_T>(mi, mp, sd.frontFacing, wiL, woL);
                                        const float3 Gf = ((g * thp) * Li) * mis;
                                        add_material_grads<14>(p, hash, sd.materialID, J, Gf);
                                        if (p.gradPos && is.inst == p.meshID) {
                                            // Through wo = (L - P) / |L - P| and the ratio a2s / detach(a2s).
                                            const float3 gL = make_float3(Gf.x * J.x.d[11] + Gf.y * J.y.d[11] + Gf.z * J.z.d[11],
                                                                          Gf.x * J.x.d[12] + Gf.y * J.y.d[12] + Gf.z * J.z.d[12],
                                                                          Gf.x * J.x.d[13] + Gf.y * J.y.d[13] + Gf.z * J.z.d[13]);
                                            const float3 gwo = mi.T * gL.x + mi.B * gL.y + mi.N * gL.z;
                                            const float gRatio = dot(Gf, make_float3(J.x.v, J.y.v, J.z.v));
                                            const float nlwo = dot(tls.normalW, wo);
                                            float3 dP = (gwo - wo * dot(wo, gwo)) * (-1.f / dist);
                                            dP += (wo * (-3.f / dist) + tls.normalW * (1.f / (dist * nlwo))) * gRatio;
                                            float* gp = p.gradPos + size_t(hashPos) * p.posDim;
#pragma unroll
                                            for (int i = 0; i < 3; i++) {
                                                const uint32_t o = is.local[i] * 3;
                                                if (o + 3 > p.posDim) continue;
                                                atomicAdd(gp + o, is.b[i] * dP.x);
                                                atomicAdd(gp + o + 1, is.b[i] * dP.y);
                                                atomicAdd(gp + o + 2, is.b[i] * dP.z);
                                            }
                                        }
                                    }
                                }
                            }
                        }
                    }
                }
                if (BWD) vr->e = e;
                // generateScatterRay (PTUtils.slang:136-172).
                float3 wo, w;
                float pdf;
                uint32_t lobe;
                if (!(mi.sample(sd, sg, wo, w, pdf, lobe, p.useBSDFSampling != 0) && pdf > 0.f)) break;
                rayDir = wo;
                rayOrigin = compute_ray_origin(is.posW, sd.frontFacing ? sd.faceN : -sd.faceN);
                const float3 bsdfWeight = mi.eval(sd, wo) / pdf;
                if (BWD) {
                    vr->wiL = mi.toLocal(sd.V);
                    vr->wsL = mi.toLocal(wo);
                    vr->pdf = pdf;
                    vr->bw = bsdfWeight;
                    if (mi.valid_hemisphere(sd, vr->wiL, vr->wsL, wo)) vr->flags |= 2u;
                }
                thp *= bsdfWeight;
                pathPdf = pdf;
                if (!any_pos(thp)) break;
                pathLen++;
                if (BWD && nv >= kMaxWarVertices) break;  // guarded by the host (maxBounces <= 14)
                cnt.v[1]++;
                cnt.v[2]++;
                trace_bvh<false>(s, rayOrigin, rayDir, 0.f, 3.402823466e+38f, h, stack, kWarBlock);
                if (!h.valid) break;
                is = war_intersect(s, h, rayOrigin, rayDir);
            }
        }
        if (!BWD) {
            if (p.color) p.color[pid] = make_float4(radiance.x, radiance.y, radiance.z, 1.f);
        } else {
            // Reverse sweep over the scatter terms: A = adjoint of thp_{k+1}.
            float3 A = f3(0.f);
            for (int k = nv - 1; k >= 0; k--) {
                const WarVertex& v = rec[k];
                if ((v.flags & 2u) && (A.x != 0.f || A.y != 0.f || A.z != 0.f)) {
                    const MatParams mp = load_mat_params(s, v.matID);
                    ShadingData sd;
                    sd.frontFacing = (v.flags & 1u) != 0;
                    sd.materialID = v.matID;
                    const MaterialInstance<HAS_T> mi = material_instance<HAS_T>(s, sd, p.lambert != 0);
                    const DV3<11> J = eval_jacobian<11, HAS_T>(mi, mp, sd.frontFacing, v.wiL, v.wsL);
                    const float3 Gs = (A * v.thp) / v.pdf;
                    add_material_grads<11>(p, hash, v.matID, J, Gs);
                }
                A = A * v.bw + g * v.e;
            }
        }
    }
    flush_counters(p.counters, cnt);
}

__global__ void war_aggregate(const float* tmp, float* out, uint32_t dim, uint32_t hash) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += gridDim.x * blockDim.x) {
        float v = 0.f;
        for (uint32_t h = 0; h < hash; h++) v += tmp[size_t(h) * dim + i];
        out[i] += v;
    }
}

int war_blocks(const void* k) {
    int perSM = 0, dev = 0, sms = 148;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k, kWarBlock, 0);
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, perSM) * sms;
}

template <bool HAS_T, bool BWD>
cudaError_t launch_war(const DevScene& s, const WarParams& p, cudaStream_t st) {
    static int blocks = 0;
    if (!blocks) blocks = war_blocks(reinterpret_cast<const void*>(war_kernel<HAS_T, BWD>));
    const int need = int((p.width * p.height + kWarBlock - 1) / kWarBlock);
    war_kernel<HAS_T, BWD><<<std::min(blocks, std::max(need, 1)), kWarBlock, 0, st>>>(s, p);
    return cudaGetLastError();
}

}  // namespace

}  // namespace fpt

// ---------------------------------------------------------------------------
// SceneGradients.
// ---------------------------------------------------------------------------
using fpt::set_error;

extern "C" {

FPT_API fpt_status fpt_scene_gradients_create(const fpt_grad_config* configs, uint32_t count, fpt_scene_gradients** out) {
    if (!out || (count && !configs)) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_gradients_create: null argument");
    auto g = new fpt_scene_gradients();
    for (uint32_t i = 0; i < count; i++) {
        const fpt_grad_config& c = configs[i];
        if (c.grad_type >= FPT_GRAD_TYPE_COUNT || c.dim == 0 || c.hash_size == 0) {
            delete g;
            return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_gradients_create: invalid gradient config " + std::to_string(i));
        }
        auto& e = g->e[c.grad_type];
        if (e.active) {
            delete g;
            return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_gradients_create: gradient type given twice");
        }
        e.active = true;
        e.dim = c.dim;
        e.hash = c.hash_size;
        if (cudaMalloc(&e.grads, size_t(c.dim) * 4) != cudaSuccess ||
            cudaMalloc(&e.tmp, size_t(c.dim) * c.hash_size * 4) != cudaSuccess) {
            delete g;
            return set_error(FPT_ERR_OOM, "fpt_scene_gradients_create: out of device memory");
        }
        cudaMemset(e.grads, 0, size_t(c.dim) * 4);
        cudaMemset(e.tmp, 0, size_t(c.dim) * c.hash_size * 4);
    }
    *out = g;
    return FPT_OK;
}

FPT_API void fpt_scene_gradients_destroy(fpt_scene_gradients* g) { delete g; }

FPT_API fpt_status fpt_scene_gradients_clear(fpt_scene_gradients* g, uint32_t type, void* stream) {
    if (!g || type >= FPT_GRAD_TYPE_COUNT) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_gradients_clear: invalid argument");
    auto& e = g->e[type];
    if (!e.active) return FPT_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(e.tmp, 0, size_t(e.dim) * e.hash * 4, st) != cudaSuccess ||
        cudaMemsetAsync(e.grads, 0, size_t(e.dim) * 4, st) != cudaSuccess)
        return set_error(FPT_ERR_CUDA, "fpt_scene_gradients_clear: memset failed");
    return FPT_OK;
}

FPT_API fpt_status fpt_scene_gradients_aggregate(fpt_scene_gradients* g, uint32_t type, void* stream) {
    if (!g || type >= FPT_GRAD_TYPE_COUNT) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_gradients_aggregate: invalid argument");
    auto& e = g->e[type];
    if (!e.active) return FPT_OK;
    const int blocks = int(std::min<uint32_t>((e.dim + 255) / 256, 4096));
    fpt::war_aggregate<<<std::max(blocks, 1), 256, 0, static_cast<cudaStream_t>(stream)>>>(e.tmp, e.grads, e.dim, e.hash);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return set_error(FPT_ERR_CUDA, std::string("fpt_scene_gradients_aggregate: ") + cudaGetErrorString(err));
    return FPT_OK;
}

FPT_API fpt_status fpt_scene_gradients_get(const fpt_scene_gradients* g, uint32_t type, float** grads, uint32_t* dim,
                                           uint32_t* hash_size) {
    if (!g || type >= FPT_GRAD_TYPE_COUNT) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_gradients_get: invalid argument");
    const auto& e = g->e[type];
    if (grads) *grads = e.active ? e.grads : nullptr;
    if (dim) *dim = e.active ? e.dim : 0;
    if (hash_size) *hash_size = e.active ? e.hash : 0;
    return FPT_OK;
}

}  // extern "C"

fpt_scene_gradients::~fpt_scene_gradients() {
    for (auto& x : e) {
        if (x.grads) cudaFree(x.grads);
        if (x.tmp) cudaFree(x.tmp);
    }
}

namespace fpt {

// WARDiffPathTracer::execute (WARDiffPathTracer.cpp:218-244, 519-606).
fpt_status wardiff_execute(fpt_pass& pass, const fpt_frame_io* io, const float* dLdI, const fpt_grad_buffers* grads,
                           cudaStream_t st) {
    fpt_scene* scene = pass.scene;
    if (!scene) return set_error(FPT_ERR_NO_SCENE, "WARDiffPathTracer: no scene set");
    if (scene->dev.hasEnv) log_warning("WARDiffPathTracer: This render pass does not support environment lights.");
    const std::string diffMode = pass.str("diffMode");
    const int mode = diffMode == "BackwardDiff" ? 1 : (diffMode == "ForwardDiffDebug" ? 2 : (diffMode == "BackwardDiffDebug" ? 3 : 0));
    const bool direct = dLdI != nullptr;  // fpt_pass_backward: caller-owned flat buffers
    const bool backward = direct || (mode == 1 && pass.num("runBackward") != 0);
    WarParams p{};
    p.width = io->width;
    p.height = io->height;
    p.maxBounces = uint32_t(std::max(0.0, pass.num("maxBounces")));
    p.useBSDFSampling = pass.num("useBSDFSampling") != 0;
    p.useNEE = pass.num("useNEE") != 0;
    p.useMIS = pass.num("useMIS") != 0;
    p.useAntithetic = pass.num("useAntitheticSampling") != 0;
    p.lambert = pass.str("diffuseBrdf") == "Lambert";
    p.meshID = uint32_t(pass.num("meshToOptimize"));
    p.frameSeed = pass.useFixedSeed ? uint32_t(pass.num("fixedSeed")) : pass.frameCount;
    p.counters = static_cast<unsigned long long*>(pass.scratch);
    if (p.width == 0 || p.height == 0) return set_error(FPT_ERR_INVALID_ARG, "WARDiffPathTracer: empty frame");
    if (p.width > 4096 || p.height > 4096)
        return set_error(FPT_ERR_INVALID_ARG, "WARDiffPathTracer: frame dimension exceeds kMaxFrameDimension (4096)");
    cudaError_t e = cudaMemsetAsync(pass.scratch, 0, kNumCounters * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, "WARDiffPathTracer: counter reset failed");
    const bool hasT = scene->dev.hasTransmission != 0;
    if (!backward) {
        if (!io->color) return set_error(FPT_ERR_INVALID_ARG, "WARDiffPathTracer: 'color' is required");
        p.color = reinterpret_cast<float4*>(io->color);
        if (io->d_color) cudaMemsetAsync(io->d_color, 0, size_t(p.width) * p.height * 16, st);
        e = hasT ? launch_war<true, false>(scene->dev, p, st) : launch_war<false, false>(scene->dev, p, st);
    } else {
        if (p.maxBounces + 2 > uint32_t(kMaxWarVertices))
            return set_error(FPT_ERR_UNSUPPORTED, "WARDiffPathTracer: the adjoint supports maxBounces <= 14");
        if (direct) {
            p.dLdI = dLdI;
            p.gradMat = grads->material;
            p.matDim = grads->material ? grads->material_dim : 0;
            p.matHash = 1;
            p.gradPos = grads->mesh_position;
            p.posDim = grads->mesh_position ? grads->position_dim : 0;
            p.posHash = 1;
        } else {
            if (!pass.dLdI) return set_error(FPT_ERR_INVALID_ARG, "WARDiffPathTracer: dL_dI is not set (fpt_pass_set_dLdI)");
            if (!pass.sceneGradients)
                return set_error(FPT_ERR_INVALID_ARG, "WARDiffPathTracer: scene_gradients is not set (fpt_pass_set_scene_gradients)");
            p.dLdI = pass.dLdI;
            const auto& gm = pass.sceneGradients->e[FPT_GRAD_MATERIAL];
            const auto& gp = pass.sceneGradients->e[FPT_GRAD_MESH_POSITION];
            if (gm.active) { p.gradMat = gm.tmp; p.matDim = gm.dim; p.matHash = gm.hash; }
            if (gp.active) { p.gradPos = gp.tmp; p.posDim = gp.dim; p.posHash = gp.hash; }
        }
        e = hasT ? launch_war<true, true>(scene->dev, p, st) : launch_war<false, true>(scene->dev, p, st);
    }
    pass.launches = 1;
    pass.frameCount++;
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, std::string("WARDiffPathTracer: kernel launch failed: ") + cudaGetErrorString(e));
    return FPT_OK;
}

}  // namespace fpt
