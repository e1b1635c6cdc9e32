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
//    (WarpedAreaReparam.slang:226-332) and only adds position derivatives;
//    with useWAR and position gradients, the NEE warp's gradient is formed at
//    the NEE sample and the scatter and screen warps' in the sweep
//    (war_reparam.cuh).
#include <cmath>
#include <cstring>
#include <string>

#include "diff_bsdf.cuh"
#include "kernels.cuh"
#include "path_logic.cuh"
#include "passes.h"
#include "scene_device.h"
#include "wardiff.h"
#include "war_common.cuh"
#include "war_reparam.cuh"

namespace fpt {

using namespace dev;

namespace {

constexpr int kWarBlock = 128;

template <bool HAS_T, bool BWD, bool WAR>
__global__ void __launch_bounds__(kWarBlock) war_kernel(DevScene s, WarParams p) {
    constexpr int NJ = WAR ? 17 : 14;
    __shared__ uint2 stackMem[kStackSize * kWarBlock];
    uint2* stack = stackMem + threadIdx.x;
    Counters cnt;
    const uint32_t pixels = p.width * p.height;
    const bool useEmissive = s.hasEmissive != 0 && s.activeCount > 0;
    for (uint32_t pid = blockIdx.x * blockDim.x + threadIdx.x; pid < pixels; pid += gridDim.x * blockDim.x) {
        const uint32_t x = pid % p.width, y = pid / p.width;
        // tracePaths (WARDiffPathTracer.rt.slang:115-143).
        UniformSG sg;
        const float2 pix = war_camera_sample(p, x, y, sg);
        const float px = pix.x, py = pix.y;
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
        uint32_t hash = 0;
        if (BWD) {
            g = war_dLdI(p, pid);
            hash = war_hash(pid, p.matHash ? p.matHash : 1);
        }
        WarSweepVertex rec[BWD ? kMaxWarVertices : 1];
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
                WarSweepVertex* vr = BWD ? &rec[nv] : nullptr;
                if (BWD) {
                    vr->thp = thp;
                    vr->wiL = vr->wsL = vr->bw = vr->e = f3(0.f);
                    vr->pdf = 1.f;
                    vr->flags = sd.frontFacing ? 1u : 0u;
                    vr->matID = sd.materialID;
                    vr->uv = sd.uv;
                    if (WAR) {
                        vr->inDir = rayDir;
                        vr->outDir = vr->gV = f3(0.f);
                        vr->inst = is.inst;
                        vr->prim = is.prim;
                        vr->b[0] = is.b[0];
                        vr->b[1] = is.b[1];
                        vr->b[2] = is.b[2];
                    }
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
                                        const MatParams mp = load_mat_params(s, sd.materialID, sd.uv);
                                        const DV3<NJ> J = eval_jacobian<NJ, HAS_T>(mi, mp, sd.frontFacing, wiL, woL);
                                        const float3 Gf = ((g * thp) * Li) * mis;
                                        add_material_grads<NJ>(s, p, pid, hash, sd.materialID, sd.uv, J, Gf);
                                        if (war_wants_pos(p) || (WAR && war_wants_frame(p))) {
                                            // Through wo = (L - P) / |L - P| and the ratio a2s / detach(a2s).
                                            const float3 gL = make_float3(Gf.x * J.x.d[11] + Gf.y * J.y.d[11] + Gf.z * J.z.d[11],
                                                                          Gf.x * J.x.d[12] + Gf.y * J.y.d[12] + Gf.z * J.z.d[12],
                                                                          Gf.x * J.x.d[13] + Gf.y * J.y.d[13] + Gf.z * J.z.d[13]);
                                            const float3 gwo = mi.T * gL.x + mi.B * gL.y + mi.N * gL.z;
                                            const float gRatio = dot(Gf, make_float3(J.x.v, J.y.v, J.z.v));
                                            const float nlwo = dot(tls.normalW, wo);
                                            float3 dP = (gwo - wo * dot(wo, gwo)) * (-1.f / dist);
                                            dP += (wo * (-3.f / dist) + tls.normalW * (1.f / (dist * nlwo))) * gRatio;
                                            if (WAR) {
                                                // computeNEE's reparameterizeRay, adjoint dLdI: the warped
                                                // direction feeds evalAD and the area-to-solid-angle ratio.
                                                constexpr int q0 = NJ - 3;
                                                const float3 gI = make_float3(Gf.x * J.x.d[q0] + Gf.y * J.y.d[q0] + Gf.z * J.z.d[q0],
                                                                              Gf.x * J.x.d[q0 + 1] + Gf.y * J.y.d[q0 + 1] + Gf.z * J.z.d[q0 + 1],
                                                                              Gf.x * J.x.d[q0 + 2] + Gf.y * J.y.d[q0 + 2] + Gf.z * J.z.d[q0 + 2]);
                                                vr->gV += mi.T * gI.x + mi.B * gI.y + mi.N * gI.z;
                                                if (war_wants_frame(p) && war_pos_target(p.meshID, is)) {
                                                    float3 gn, gt;
                                                    war_frame_adjoint(is, dot(mi.N, sd.N) < 0.f, sd.V, wo, gI, gL, gn, gt);
                                                    const uint32_t off[3] = {war_pos_index(p.meshID, is, 0), war_pos_index(p.meshID, is, 1),
                                                                             war_pos_index(p.meshID, is, 2)};
                                                    add_frame_grad(p, pid, off, is.b, gn, gt);
                                                }
                                                const float3 gdN = gRatio != 0.f ? gwo - tls.normalW * (gRatio / nlwo) : gwo;
                                                if (p.useWAR && war_wants_pos(p) && (gdN.x != 0.f || gdN.y != 0.f || gdN.z != 0.f || gRatio != 0.f)) {
                                                    const float3 no = compute_ray_origin(is.posW, sd.frontFacing ? sd.faceN : -sd.faceN);
                                                    float3 gO = f3(0.f), gD = f3(0.f);
                                                    war_ray_grad(s, p, pid, no, wo, true, sg, gdN, gRatio, stack, kWarBlock, gO, gD);
                                                    dP += gO - (gD - wo * dot(wo, gD)) * (1.f / dist);
                                                }
                                            }
                                            if (war_wants_pos(p) && war_pos_target(p.meshID, is)) add_position_grad(p, pid, is, dP);
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
                    if (WAR) {
                        vr->outDir = wo;
                        vr->sg = make_uint4(sg.s0, sg.s1, sg.s2, sg.s3);
                    }
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
            float3 A = f3(0.f), gV = f3(0.f);
            for (int k = nv - 1; k >= 0; k--) war_sweep_vertex<HAS_T, WAR>(s, p, pid, hash, rec[k], g, A, gV, stack, kWarBlock);
            if (WAR && p.useWAR && war_wants_pos(p) && nv > 0) war_sweep_screen(s, p, pid, A, gV, stack, kWarBlock);
        }
    }
    flush_counters(p.counters, cnt);
}

__global__ void war_debug_finalize(float4* dColor, uint32_t n, float maxValue) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float d = dColor[i].x;
        dColor[i] = (d >= -maxValue && d <= maxValue) ? make_float4(d, 0.f, 0.f, 1.f) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

__global__ void war_aggregate(const float* tmp, float* out, uint32_t dim, uint32_t hash) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < dim; i += gridDim.x * blockDim.x) {
        float v = 0.f;
        for (uint32_t h = 0; h < hash; h++) v += tmp[size_t(h) * dim + i];
        out[i] += v;
    }
}

// SceneGradients::atomicAddGrad over arrays of contributions: value i goes to
// scratch row hashIndex[i], element gradIndex[i] (ignored beyond the dimension).
__global__ void war_atomic_add_grads(float* tmp, uint32_t dim, uint32_t hash, uint32_t n, const uint32_t* gradIndex,
                                     const uint32_t* hashIndex, const float* values) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t g = gradIndex[i], h = hashIndex[i];
        if (g >= dim || h >= hash) continue;
        const float v[1] = {values[i]};
        atomic_add_row<1>(tmp + size_t(h) * dim + g, v);
    }
}

int war_blocks(const void* k) {
    int perSM = 0, dev = 0, sms = 148;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, k, kWarBlock, 0);
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, perSM) * sms;
}

template <bool HAS_T, bool BWD, bool WAR>
cudaError_t launch_war(const DevScene& s, const WarParams& p, cudaStream_t st) {
    static int blocks = 0;
    if (!blocks) blocks = war_blocks(reinterpret_cast<const void*>(war_kernel<HAS_T, BWD, WAR>));
    const int need = int((p.width * p.height + kWarBlock - 1) / kWarBlock);
    war_kernel<HAS_T, BWD, WAR><<<std::min(blocks, std::max(need, 1)), kWarBlock, 0, st>>>(s, p);
    return cudaGetLastError();
}

template <bool BWD>
cudaError_t launch_war_any(const DevScene& s, const WarParams& p, cudaStream_t st) {
    // Extended records: the warps (position derivatives only) and normal / tangent gradients.
    const bool war = BWD && ((p.useWAR && (p.gradPos || (p.dbgColor && p.dbgType == kDbgTranslation))) || p.gradNrm || p.gradTan);
    if (s.hasTransmission) return war ? launch_war<true, BWD, BWD>(s, p, st) : launch_war<true, BWD, false>(s, p, st);
    return war ? launch_war<false, BWD, BWD>(s, p, st) : launch_war<false, BWD, false>(s, p, st);
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

FPT_API fpt_status fpt_scene_gradients_atomic_add(fpt_scene_gradients* g, uint32_t type, uint32_t count,
                                                  const uint32_t* grad_index, const uint32_t* hash_index, const float* values,
                                                  void* stream) {
    if (!g || type >= FPT_GRAD_TYPE_COUNT) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_gradients_atomic_add: invalid argument");
    auto& e = g->e[type];
    if (!e.active || count == 0) return FPT_OK;
    if (!grad_index || !hash_index || !values) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_gradients_atomic_add: null array");
    const int blocks = int(std::min<uint32_t>((count + 255) / 256, 148u * 8u));
    fpt::war_atomic_add_grads<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(e.tmp, e.dim, e.hash, count, grad_index,
                                                                                       hash_index, values);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) return set_error(FPT_ERR_CUDA, std::string("fpt_scene_gradients_atomic_add: ") + cudaGetErrorString(err));
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
    const double mesh = pass.num("meshToOptimize");
    p.meshID = mesh < 0 ? 0xffffffffu : uint32_t(mesh);  // -1: every mesh, scene-global vertex indices
    p.frameSeed = pass.useFixedSeed ? uint32_t(pass.num("fixedSeed")) : pass.frameCount;
    p.useWAR = pass.num("useWAR") != 0;
    p.auxCount = uint32_t(std::max(0.0, pass.num("auxSampleCount")));
    // kappa = pow(10, Log10vMFConcentration) (WarpedAreaReparam.slang:241, 318).
    p.kappa = std::pow(10.f, float(pass.num("Log10vMFConcentration")));
    p.kappaScreen = std::pow(10.f, float(pass.num("Log10vMFConcentrationScreen")));
    p.counters = static_cast<unsigned long long*>(pass.scratch);
    if (p.width == 0 || p.height == 0) return set_error(FPT_ERR_INVALID_ARG, "WARDiffPathTracer: empty frame");
    if (p.width > 4096 || p.height > 4096)
        return set_error(FPT_ERR_INVALID_ARG, "WARDiffPathTracer: frame dimension exceeds kMaxFrameDimension (4096)");
    cudaError_t e = cudaMemsetAsync(pass.scratch, 0, kNumCounters * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, "WARDiffPathTracer: counter reset failed");
    const bool wavefront = pass.str("scheduler") != "Megakernel";
    if (backward || wavefront) {
        if (p.maxBounces + 2 > uint32_t(kMaxWarVertices))
            return set_error(FPT_ERR_UNSUPPORTED, "WARDiffPathTracer: the adjoint supports maxBounces <= 14");
    }
    const bool debug = !backward && (mode == 2 || mode == 3) && io->d_color != nullptr;
    if (!backward) {
        if (!io->color) return set_error(FPT_ERR_INVALID_ARG, "WARDiffPathTracer: 'color' is required");
        p.color = reinterpret_cast<float4*>(io->color);
        // Outputs are cleared every frame except in BackwardDiff with runBackward
        // (WARDiffPathTracer.cpp:518-529).
        if (io->d_color) cudaMemsetAsync(io->d_color, 0, size_t(p.width) * p.height * 16, st);
        if (mode == 3) cudaMemsetAsync(io->color, 0, size_t(p.width) * p.height * 16, st);
    }
    auto adjointScratch = [&](bool war) -> fpt_status {
        const size_t need = war_adjoint_bytes(pass.wavefront.capacity, p.maxBounces, war);
        if (pass.adjointScratchBytes < need) {
            if (pass.adjointScratch) cudaFree(pass.adjointScratch);
            pass.adjointScratch = nullptr;
            pass.adjointScratchBytes = 0;
            if (cudaMalloc(&pass.adjointScratch, need) != cudaSuccess)
                return set_error(FPT_ERR_OOM, "WARDiffPathTracer: adjoint scratch allocation failed");
            pass.adjointScratchBytes = need;
        }
        return FPT_OK;
    };
    auto checkWar = [&](const WarParams& q) -> fpt_status {
        const bool pos = q.gradPos || (q.dbgColor && q.dbgType == kDbgTranslation);
        if (!q.useWAR || !pos) return FPT_OK;
        if (q.auxCount == 0 || q.auxCount > uint32_t(kMaxAux))
            return set_error(FPT_ERR_UNSUPPORTED, "WARDiffPathTracer: auxSampleCount must be in [1, 32]");
        if (q.useAntithetic && (q.auxCount & 1u))
            return set_error(FPT_ERR_UNSUPPORTED, "WARDiffPathTracer: antithetic sampling needs an even auxSampleCount");
        if (!(q.kappa > 0.f) || !(q.kappaScreen > 0.f) || std::isinf(q.kappa) || std::isinf(q.kappaScreen))
            return set_error(FPT_ERR_INVALID_ARG, "WARDiffPathTracer: vMF concentrations must be finite");
        return FPT_OK;
    };
    if (wavefront) {
        const uint32_t pixels = p.width * p.height;
        const uint32_t cap = std::min<uint32_t>(pixels, uint32_t(std::max(1.0, pass.num("wavefrontCapacity"))));
        e = pass.wavefront.ensure(cap);
        if (e != cudaSuccess) return set_error(FPT_ERR_OOM, std::string("WARDiffPathTracer: wavefront buffers: ") + cudaGetErrorString(e));
        if (backward || debug) {
            // The extended record layout (warps, normal / tangent gradients) covers every adjoint.
            const fpt_status s = adjointScratch(true);
            if (s != FPT_OK) return s;
        }
    }
    // Checkpointed vertices belong to one frame: seed, size and the settings and
    // scene state that decide the paths.
    const bool checkpointMode = wavefront && pass.str("adjointMode") == "Checkpoint";
    const uint64_t key[8] = {p.frameSeed, (uint64_t(p.width) << 32) | p.height, p.maxBounces,
                             (uint64_t(p.useBSDFSampling) << 3) | (p.useNEE << 2) | (p.useMIS << 1) | p.useAntithetic,
                             p.lambert, reinterpret_cast<uint64_t>(scene), scene->version, 0};
    pass.lastAdjointCheckpointed = false;
    if (!backward) {
        if (mode != 3) {
            WarCheckpoint ck{};
            bool record = false;
            if (checkpointMode && wavefront) {
                // Where memory allows: at most half of the free device memory.
                const uint32_t pixels = p.width * p.height;
                const size_t need = war_checkpoint_bytes(pixels, p.maxBounces);
                if (pass.checkpointBytes < need) {
                    if (pass.checkpoint) cudaFree(pass.checkpoint);
                    pass.checkpoint = nullptr;
                    pass.checkpointBytes = 0;
                    size_t freeB = 0, totalB = 0;
                    if (cudaMemGetInfo(&freeB, &totalB) == cudaSuccess && need <= freeB / 2 &&
                        cudaMalloc(&pass.checkpoint, need) == cudaSuccess)
                        pass.checkpointBytes = need;
                    else
                        log_warning("WARDiffPathTracer: not enough device memory for checkpointed vertices; the adjoint replays");
                }
                if (pass.checkpoint) {
                    ck.hits = static_cast<uint4*>(pass.checkpoint);
                    ck.visible = reinterpret_cast<uint32_t*>(ck.hits + size_t(p.maxBounces + 2) * pixels);
                    ck.pixels = pixels;
                    ck.mode = 1;
                    record = cudaMemsetAsync(ck.visible, 0, size_t(pixels) * 4, st) == cudaSuccess;
                }
            }
            pass.checkpointValid = false;
            if (wavefront) e = launch_war_wavefront(scene->dev, p, pass.wavefront, nullptr, false, st, pass.launches, record ? &ck : nullptr);
            else e = launch_war_any<false>(scene->dev, p, st);
            if (record && e == cudaSuccess) {
                std::memcpy(pass.checkpointKey, key, sizeof(key));
                pass.checkpointValid = true;
            }
        }
        if (debug && e == cudaSuccess) {
            // ForwardDiffDebug / BackwardDiffDebug (WARDiffPathTracer.rt.slang:182-210): the
            // reverse sweep with adjoint (1, 0, 0) per pixel gives d(color.r)/d(variable)
            // pixel by pixel, each path belonging to one pixel.
            WarParams q = p;
            q.color = nullptr;
            q.dLdI = nullptr;
            q.dbgColor = reinterpret_cast<float4*>(io->d_color);
            uint32_t type = pass.diffDebugType, id = pass.diffDebugId[0], offset = pass.diffDebugOffset;
            float4 grad = make_float4(pass.diffDebugGrad[0], pass.diffDebugGrad[1], pass.diffDebugGrad[2], pass.diffDebugGrad[3]);
            if (!pass.diffDebugExplicit) {
                // The diffVarName presets of the WARDiffPathTracer constructor (WARDiffPathTracer.cpp:83-93).
                const std::string var = pass.str("diffVarName");
                type = kDbgNone;
                if (var == "CBOX_BUNNY_MATERIAL") { type = kDbgMaterial; id = 0; offset = 0; grad = make_float4(1.f, 1.f, 1.f, 0.f); }
                else if (var == "CBOX_BUNNY_TRANSLATION") { type = kDbgTranslation; id = 0; offset = 0; grad = make_float4(0.f, 1.f, 0.f, 0.f); }
            }
            // Reverse mode routes material derivatives to the scene gradients, not to
            // the image (GradientIOWrapper.slang:97-104 has no debug branch).
            if (mode == 3 && type == kDbgMaterial) type = kDbgNone;
            q.dbgType = type;
            q.dbgId = id;
            q.dbgOffset = offset;
            q.dbgGrad = grad;
            if (type == kDbgTranslation) q.meshID = id;
            if (mode == 3 && pass.sceneGradients && pass.sceneGradients->e[FPT_GRAD_MATERIAL].active) {
                const auto& gm = pass.sceneGradients->e[FPT_GRAD_MATERIAL];
                q.gradMat = gm.tmp;
                q.matDim = gm.dim;
                q.matHash = gm.hash;
            }
            q.matHash = std::max(q.matHash, 1u);
            q.posHash = std::max(q.posHash, 1u);
            const fpt_status cs = checkWar(q);
            if (cs != FPT_OK) return cs;
            uint32_t launches = 0;
            if (wavefront) e = launch_war_wavefront(scene->dev, q, pass.wavefront, pass.adjointScratch, true, st, launches);
            else e = launch_war_any<true>(scene->dev, q, st);
            pass.launches += launches;
            if (e == cudaSuccess && mode == 2) {
                // gOutputDColor = (d.r, 0, 0, 1) when |d| <= assertThreshold (Params.slang:61), else cleared.
                const uint32_t n = p.width * p.height;
                war_debug_finalize<<<(n + 255) / 256, 256, 0, st>>>(q.dbgColor, n, 1e9f);
                e = cudaGetLastError();
            }
        }
    } else {
        if (direct) {
            p.dLdI = dLdI;
            p.gradMat = grads->material;
            p.matDim = grads->material ? grads->material_dim : 0;
            p.matHash = 1;
            p.gradPos = grads->mesh_position;
            p.posDim = grads->mesh_position ? grads->position_dim : 0;
            p.posHash = 1;
            p.gradNrm = grads->mesh_normal;
            p.nrmDim = grads->mesh_normal ? grads->normal_dim : 0;
            p.gradTan = grads->mesh_tangent;
            p.tanDim = grads->mesh_tangent ? grads->tangent_dim : 0;
            p.gradTex = grads->base_color_texture;
            p.texDim = grads->base_color_texture ? grads->texture_dim : 0;
        } else {
            if (!pass.dLdI) return set_error(FPT_ERR_INVALID_ARG, "WARDiffPathTracer: dL_dI is not set (fpt_pass_set_dLdI)");
            if (!pass.sceneGradients)
                return set_error(FPT_ERR_INVALID_ARG, "WARDiffPathTracer: scene_gradients is not set (fpt_pass_set_scene_gradients)");
            p.dLdI = pass.dLdI;
            const auto& gm = pass.sceneGradients->e[FPT_GRAD_MATERIAL];
            const auto& gp = pass.sceneGradients->e[FPT_GRAD_MESH_POSITION];
            if (gm.active) { p.gradMat = gm.tmp; p.matDim = gm.dim; p.matHash = gm.hash; }
            if (gp.active) { p.gradPos = gp.tmp; p.posDim = gp.dim; p.posHash = gp.hash; }
            const auto& gn = pass.sceneGradients->e[FPT_GRAD_MESH_NORMAL];
            const auto& gt = pass.sceneGradients->e[FPT_GRAD_MESH_TANGENT];
            if (gn.active) { p.gradNrm = gn.tmp; p.nrmDim = gn.dim; p.nrmHash = gn.hash; }
            if (gt.active) { p.gradTan = gt.tmp; p.tanDim = gt.dim; p.tanHash = gt.hash; }
        }
        p.matHash = std::max(p.matHash, 1u);
        p.posHash = std::max(p.posHash, 1u);
        p.nrmHash = std::max(p.nrmHash, 1u);
        p.tanHash = std::max(p.tanHash, 1u);
        const fpt_status cs = checkWar(p);
        if (cs != FPT_OK) return cs;
        WarCheckpoint ck{};
        if (checkpointMode && pass.checkpointValid && std::memcmp(pass.checkpointKey, key, sizeof(key)) == 0) {
            const uint32_t pixels = p.width * p.height;
            ck.hits = static_cast<uint4*>(pass.checkpoint);
            ck.visible = reinterpret_cast<uint32_t*>(ck.hits + size_t(p.maxBounces + 2) * pixels);
            ck.pixels = pixels;
            ck.mode = 2;
            pass.lastAdjointCheckpointed = true;
        }
        if (wavefront)
            e = launch_war_wavefront(scene->dev, p, pass.wavefront, pass.adjointScratch, true, st, pass.launches, ck.mode ? &ck : nullptr);
        else e = launch_war_any<true>(scene->dev, p, st);
    }
    if (!wavefront) pass.launches = 1;
    pass.frameCount++;
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, std::string("WARDiffPathTracer: kernel launch failed: ") + cudaGetErrorString(e));
    return FPT_OK;
}

}  // namespace fpt
