// war_wavefront.cu -- wavefront scheduler of the WARDiffPathTracer primal
// and adjoint (the default; the per-pixel megakernel in wardiff.cu is the
// "Megakernel" scheduler).
//
// The frame's paths (one per pixel, WARDiffPathTracer.rt.slang:115-143) run in
// waves whose state lives in the structure-of-arrays buffers of the PathTracer
// wavefront.  Per bounce:
//   extend    closest-hit traversal with dynamic ray fetch (shared with the PathTracer)
//   shade     handleHit (PTUtils.slang:253-341): emission, the uniform light
//             sample, the scatter sample; pushes the visibility ray and the
//             continuing path
//   shadow    any-hit traversal; adds thp * weight when unoccluded
//   nee_grad  (adjoint) applies the NEE gradients of the visible samples
// The adjoint re-traces the frame from its seeds (path replay: the primal
// stores nothing).  The shade kernel writes, per path vertex, the record the
// scatter term needs (local directions, throughput, pdf, BSDF weight and the
// vertex's radiance increments); after the last bounce a sweep kernel walks
// each path's records backwards with the throughput adjoint
//     A_k = dLdI * e_k + A_{k+1} * w_k,   dS/df_k(ws) = A_{k+1} * thp_k / pdf_k.
// The NEE term's adjoint is dLdI itself, so its gradients are formed in the
// shade kernel and applied when the visibility ray finds the light unoccluded.
//
// With the warped-area reparameterisation (WAR) and position gradients, the
// records also keep what the reparameterised rays need -- the sample
// generator state at each reparameterisation, the unwarped directions and the
// hit -- and the adjoints of the warped directions and weights are formed
// where they become known: the NEE warp in the nee_grad kernel (its adjoint is
// dLdI), the scatter warps in the sweep (the adjoint of the next vertex's
// incident direction and throughput is known once that vertex has been swept)
// and the screen warp after the sweep.  Each one traces its auxiliary rays
// there (war_reparam.cuh); the primal never traces them, since the warps leave
// every value unchanged.
#include <algorithm>

#include "passes.h"
#include "scene_device.h"
#include "war_common.cuh"
#include "war_reparam.cuh"
#include "war_wavefront.h"
#include "wavefront_common.cuh"

namespace fpt {

namespace {

// Adjoint scratch layout (float4 arrays of `capacity` entries): the pending
// NEE gradients (kNeeArrays, kNeeArraysWar with WAR) and, per path vertex, the
// record (kRecArrays, kRecArraysWar with WAR).
//   nee  0-2 material gradients, material ID   rec 0 wiL, pdf
//        3   dP, position-gradient flag            1 wsL, material ID
//        4-5 barycentrics, vertex offsets          2 thp, flags
//        6   NEE weight                            3 BSDF weight
//   WAR: 7   NEE ray origin, distance              4 emission + NEE weight
//        8   unwarped direction, gRatio      WAR: 5 incident direction, instance
//        9   adjoint of the warped direction      6 scatter direction, primitive
//        10  sample generator                     7 sample generator after the BSDF sample
//        11  adjoint of V (incident direction)    8 NEE adjoint of V, b0
//        12  normal adjoint, flag                 9 b1, b2
//        13  tangent adjoint
// ("WAR" = the extended layout, used for the warps and for normal / tangent gradients.)
constexpr int kNeeArrays = 7, kNeeArraysWar = 14;
constexpr int kRecArrays = 5, kRecArraysWar = 10;

struct WarWave {
    uint32_t waveFirstPixel, wavePixels, capacity;
    float4* nee;        // neeArrays x capacity
    float4* rec;        // maxVertices x recArrays x capacity
    uint32_t* nv;       // records per path
    uint32_t maxVertices, recArrays;
    // Reparameterisation requests of the reverse sweep (WAR), served by
    // ww_war_requests: scatter rays (kReqArrays x maxVertices * capacity
    // entries) and screen samples (kScreenReqArrays x capacity), with their
    // counters in reqCount[0] / reqCount[1].
    float4* req;
    float4* sreq;
    uint32_t* reqCount;
    uint32_t reqCapacity;
};
// Scatter request: origin + gJ, direction + pixel, gDir + b1, sample generator,
// gradient offsets + b0, b2.  Screen request: sample + gPix, sample generator,
// gJ + pixel.
constexpr int kReqArrays = 6, kScreenReqArrays = 3;

FPT_D float4& nee_at(const WarWave& ww, int j, uint32_t i) { return ww.nee[size_t(j) * ww.capacity + i]; }
FPT_D float4& rec_at(const WarWave& ww, uint32_t k, int j, uint32_t i) {
    return ww.rec[(size_t(k) * ww.recArrays + j) * ww.capacity + i];
}
FPT_D float4& req_at(const WarWave& ww, int j, uint32_t k) { return ww.req[size_t(j) * ww.reqCapacity + k]; }
FPT_D float4& sreq_at(const WarWave& ww, int j, uint32_t k) { return ww.sreq[size_t(j) * ww.capacity + k]; }
FPT_D uint4& as_u4(float4& v) { return reinterpret_cast<uint4&>(v); }
FPT_D float3 xyz(const float4& v) { return make_float3(v.x, v.y, v.z); }
FPT_D bool nonzero(float3 v) { return v.x != 0.f || v.y != 0.f || v.z != 0.f; }

// Seeds the wave: camera ray of pixel waveFirstPixel + i (tracePaths,
// WARDiffPathTracer.rt.slang:115-143 and tracePath :75-112).
// Resident blocks per SM of the adjoint's shading kernels (registers are
// capped accordingly).  Uncapped they took up to 255 registers (2 blocks per
// SM); on the displaced-sphere adjoint 4 blocks measured best: replay adjoint
// 168.5 -> 176 Mpaths/s, with the boundary term 16.8 -> 19.1, checkpointed
// forward + adjoint 142.8 -> 149.
#ifndef FPT_WW_MIN_BLOCKS
#define FPT_WW_MIN_BLOCKS 4
#endif
template <bool BWD>
__global__ void __launch_bounds__(kShadeBlock) ww_generate(DevScene s, WarParams p, WaveParams wp, SoA w, WarWave ww) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < wp.wavePixels; i += gridDim.x * blockDim.x) {
        const uint32_t pid = wp.waveFirstPixel + i;
        const uint32_t x = pid % p.width, y = pid / p.width;
        UniformSG sg;
        const float2 pix = war_camera_sample(p, x, y, sg);
        const float px = pix.x, py = pix.y;
        const float qx = px / float(p.width), qy = py / float(p.height);
        const float ndcx = 2.f * qx + -1.f, ndcy = -2.f * qy + 1.f;
        const float3 dirU = load3(s.camera.cameraU) * ndcx + load3(s.camera.cameraV) * ndcy + load3(s.camera.cameraW);
        const float len = length(dirU);
        const float3 d = len > 0.f ? dirU / len : f3(0.f);
        const float3 o = load3(s.camera.posW);
        w.originPdf[i] = make_float4(o.x, o.y, o.z, 0.f);
        w.dirV[i] = make_float4(d.x, d.y, d.z, __uint_as_float(PF_ACTIVE));
        w.thpB[i] = make_float4(1.f, 1.f, 1.f, __uint_as_float(0u));
        w.L[i] = make_float4(0.f, 0.f, 0.f, 0.f);
        store_sg(w.sg[i], sg);
        wp.extQueue[i] = i;
        if (BWD) ww.nv[i] = 0;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        wp.counts[1] = wp.wavePixels;
        if (p.counters) {
            atomicAdd(p.counters + 0, (unsigned long long)wp.wavePixels);
        }
    }
}

// handleHit for every path of the shade queue whose extension ray hit.
template <bool HAS_T, bool BWD, bool WAR>
__global__ void __launch_bounds__(kShadeBlock, FPT_WW_MIN_BLOCKS) ww_shade(DevScene s, WarParams p, WaveParams wp, SoA w, WarWave ww) {
    constexpr int NJ = WAR ? 17 : 14;  // NEE Jacobian: material, wo and (WAR) wi slots
    Counters cnt;
    const bool useEmissive = s.hasEmissive != 0 && s.activeCount > 0;
    const uint32_t n = wp.counts[0];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t i = wp.shadeQueue[k];
        const float4 od = w.originPdf[i], dv = w.dirV[i];
        const uint32_t fv = __float_as_uint(dv.w);
        if (!(fv & 0x2u)) continue;  // the extension ray missed: the path is done (no environment light)
        const uint32_t pid = wp.waveFirstPixel + i;
        float3 rayOrigin = make_float3(od.x, od.y, od.z), rayDir = make_float3(dv.x, dv.y, dv.z);
        const float pathPdf = od.w;
        const float4 tb = w.thpB[i];
        float3 thp = make_float3(tb.x, tb.y, tb.z);
        uint32_t pathLen = __float_as_uint(tb.w);
        float4 Lr = w.L[i];
        float3 radiance = make_float3(Lr.x, Lr.y, Lr.z);
        UniformSG sg;
        load_sg(w.sg[i], sg);
        const uint4 hr = w.hit[i];
        HitRec h;
        h.instanceID = hr.x;
        h.primIndex = hr.y;
        h.baryX = __uint_as_float(hr.z);
        h.baryY = __uint_as_float(hr.w);
        h.valid = true;
        cnt.v[6]++;
        const WarIsect is = war_intersect(s, h, rayOrigin, rayDir);
        const ShadingData sd = war_shading_data(s, is, rayDir);
        const MaterialInstance<HAS_T> mi = material_instance<HAS_T>(s, sd, p.lambert != 0);
        float3 g = f3(0.f), e = f3(0.f);
        uint32_t vk = 0;
        if (BWD) {
            g = war_dLdI(p, pid);
            vk = ww.nv[i];
            ww.nv[i] = vk + 1;
            rec_at(ww, vk, 0, i) = make_float4(0.f, 0.f, 0.f, 1.f);  // wiL, pdf
            rec_at(ww, vk, 1, i) = make_float4(0.f, 0.f, 0.f, __uint_as_float(sd.materialID));
            rec_at(ww, vk, 2, i) = make_float4(thp.x, thp.y, thp.z, __uint_as_float(sd.frontFacing ? 1u : 0u));
            rec_at(ww, vk, 3, i) = make_float4(0.f, 0.f, 0.f, sd.uv.x);  // bw, texture coordinate x
            if (WAR) {
                rec_at(ww, vk, 5, i) = make_float4(rayDir.x, rayDir.y, rayDir.z, __uint_as_float(is.inst));
                rec_at(ww, vk, 6, i) = make_float4(0.f, 0.f, 0.f, __uint_as_float(is.prim));
                rec_at(ww, vk, 8, i) = make_float4(0.f, 0.f, 0.f, is.b[0]);
                rec_at(ww, vk, 9, i) = make_float4(is.b[1], is.b[2], 0.f, 0.f);
            }
        }
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
        bool cont = false, shadowRay = false;
        if (pathLen < p.maxBounces + 1) {
            if (p.useNEE && useEmissive) {
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
                        // computeNEE (PTUtils.slang:211-249); applied if the light is visible.
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
                        const float3 contrib = thp * weight;
                        w.sOrigin[i] = make_float4(origin.x, origin.y, origin.z, distance);
                        w.sDir[i] = make_float4(ldir.x, ldir.y, ldir.z, 0.f);
                        w.sLr[i] = make_float4(contrib.x, contrib.y, contrib.z, 0.f);
                        shadowRay = true;
                        if (BWD) {
                            float G[11];
#pragma unroll
                            for (int q = 0; q < 11; q++) G[q] = 0.f;
                            float3 dP = f3(0.f), gwo = f3(0.f), gwi = f3(0.f), gn = f3(0.f), gt = f3(0.f);
                            float gRatio = 0.f;
                            bool frameGrad = false;
                            const float3 wiL = mi.toLocal(sd.V), woL = mi.toLocal(wo);
                            if (mi.valid_hemisphere(sd, wiL, woL, wo)) {
                                const MatParams mp = load_mat_params(s, sd.materialID, sd.uv);
                                const DV3<NJ> J = eval_jacobian<NJ, HAS_T>(mi, mp, sd.frontFacing, wiL, woL);
                                const float3 Gf = ((g * thp) * Li) * mis;
#pragma unroll
                                for (int q = 0; q < 11; q++) G[q] = Gf.x * J.x.d[q] + Gf.y * J.y.d[q] + Gf.z * J.z.d[q];
                                if (war_wants_pos(p) || (WAR && war_wants_frame(p))) {
                                    const float3 gL = make_float3(Gf.x * J.x.d[11] + Gf.y * J.y.d[11] + Gf.z * J.z.d[11],
                                                                  Gf.x * J.x.d[12] + Gf.y * J.y.d[12] + Gf.z * J.z.d[12],
                                                                  Gf.x * J.x.d[13] + Gf.y * J.y.d[13] + Gf.z * J.z.d[13]);
                                    gwo = mi.T * gL.x + mi.B * gL.y + mi.N * gL.z;
                                    gRatio = dot(Gf, make_float3(J.x.v, J.y.v, J.z.v));
                                    if (WAR) {
                                        const int q0 = NJ - 3;  // wi slots
                                        const float3 gI = make_float3(Gf.x * J.x.d[q0] + Gf.y * J.y.d[q0] + Gf.z * J.z.d[q0],
                                                                      Gf.x * J.x.d[q0 + 1] + Gf.y * J.y.d[q0 + 1] + Gf.z * J.z.d[q0 + 1],
                                                                      Gf.x * J.x.d[q0 + 2] + Gf.y * J.y.d[q0 + 2] + Gf.z * J.z.d[q0 + 2]);
                                        gwi = mi.T * gI.x + mi.B * gI.y + mi.N * gI.z;
                                        if (war_wants_frame(p) && war_pos_target(p.meshID, is)) {
                                            frameGrad = true;
                                            war_frame_adjoint(is, dot(mi.N, sd.N) < 0.f, sd.V, wo, gI, gL, gn, gt);
                                        }
                                    }
                                    if (war_wants_pos(p) && war_pos_target(p.meshID, is)) {
                                        const float nlwo = dot(tls.normalW, wo);
                                        dP = (gwo - wo * dot(wo, gwo)) * (-1.f / dist);
                                        dP += (wo * (-3.f / dist) + tls.normalW * (1.f / (dist * nlwo))) * gRatio;
                                    }
                                }
                            }
                            const bool posGrad = war_wants_pos(p) && war_pos_target(p.meshID, is);
                            nee_at(ww, 0, i) = make_float4(G[0], G[1], G[2], G[3]);
                            nee_at(ww, 1, i) = make_float4(G[4], G[5], G[6], G[7]);
                            nee_at(ww, 2, i) = make_float4(G[8], G[9], G[10], __uint_as_float(sd.materialID));
                            nee_at(ww, 3, i) = make_float4(dP.x, dP.y, dP.z, __uint_as_float(posGrad ? 1u : 0u));
                            nee_at(ww, 4, i) = make_float4(is.b[0], is.b[1], is.b[2], __uint_as_float(war_pos_index(p.meshID, is, 0)));
                            nee_at(ww, 5, i) = make_float4(__uint_as_float(war_pos_index(p.meshID, is, 1)),
                                                           __uint_as_float(war_pos_index(p.meshID, is, 2)), sd.uv.x, sd.uv.y);
                            nee_at(ww, 6, i) = make_float4(weight.x, weight.y, weight.z, 0.f);
                            if (WAR) {
                                // computeNEE's reparameterizeRay: origin computeRayOrigin(posW, +-faceN),
                                // direction wo, sample generator after the light sample.
                                const float3 no = compute_ray_origin(is.posW, sd.frontFacing ? sd.faceN : -sd.faceN);
                                // Adjoint of the warped direction: evalAD's wo and the
                                // area-to-solid-angle ratio, d ln(a2s)/d dir = -nl / (nl . dir).
                                const float3 gdN = gRatio != 0.f ? gwo - tls.normalW * (gRatio / dot(tls.normalW, wo)) : gwo;
                                nee_at(ww, 7, i) = make_float4(no.x, no.y, no.z, dist);
                                nee_at(ww, 8, i) = make_float4(wo.x, wo.y, wo.z, gRatio);
                                nee_at(ww, 9, i) = make_float4(gdN.x, gdN.y, gdN.z, 0.f);
                                store_sg(as_u4(nee_at(ww, 10, i)), sg);
                                nee_at(ww, 11, i) = make_float4(gwi.x, gwi.y, gwi.z, 0.f);
                                nee_at(ww, 12, i) = make_float4(gn.x, gn.y, gn.z, __uint_as_float(frameGrad ? 1u : 0u));
                                nee_at(ww, 13, i) = make_float4(gt.x, gt.y, gt.z, 0.f);
                            }
                        }
                    }
                }
            }
            // generateScatterRay (PTUtils.slang:136-172).
            float3 wo, wgt;
            float pdf;
            uint32_t lobe;
            if (mi.sample(sd, sg, wo, wgt, pdf, lobe, p.useBSDFSampling != 0) && pdf > 0.f) {
                rayDir = wo;
                rayOrigin = compute_ray_origin(is.posW, sd.frontFacing ? sd.faceN : -sd.faceN);
                const float3 bsdfWeight = mi.eval(sd, wo) / pdf;
                if (BWD) {
                    const float3 wiL = mi.toLocal(sd.V), wsL = mi.toLocal(wo);
                    const bool valid = mi.valid_hemisphere(sd, wiL, wsL, wo);
                    rec_at(ww, vk, 0, i) = make_float4(wiL.x, wiL.y, wiL.z, pdf);
                    rec_at(ww, vk, 1, i) = make_float4(wsL.x, wsL.y, wsL.z, __uint_as_float(sd.materialID));
                    rec_at(ww, vk, 2, i) = make_float4(thp.x, thp.y, thp.z,
                                                       __uint_as_float((sd.frontFacing ? 1u : 0u) | (valid ? 2u : 0u)));
                    rec_at(ww, vk, 3, i) = make_float4(bsdfWeight.x, bsdfWeight.y, bsdfWeight.z, sd.uv.x);
                    if (WAR) {
                        rec_at(ww, vk, 6, i) = make_float4(wo.x, wo.y, wo.z, __uint_as_float(is.prim));
                        store_sg(as_u4(rec_at(ww, vk, 7, i)), sg);
                    }
                }
                thp *= bsdfWeight;
                if (any_pos(thp)) {
                    pathLen++;
                    cont = true;
                }
                w.originPdf[i] = make_float4(rayOrigin.x, rayOrigin.y, rayOrigin.z, pdf);
                w.dirV[i] = make_float4(rayDir.x, rayDir.y, rayDir.z, __uint_as_float(fv & ~0x2u));
            }
        }
        push(shadowRay, i, wp.shadowQueue, wp.counts + 2);
        if (BWD) rec_at(ww, vk, 4, i) = make_float4(e.x, e.y, e.z, sd.uv.y);  // radiance increment, texture coordinate y
        if (BWD && vk + 1 >= ww.maxVertices) cont = false;  // guarded by the host
        w.thpB[i] = make_float4(thp.x, thp.y, thp.z, __uint_as_float(pathLen));
        w.L[i] = make_float4(radiance.x, radiance.y, radiance.z, 0.f);
        store_sg(w.sg[i], sg);
        push(cont, i, wp.extQueue, wp.counts + 1);
    }
    flush_counters(p.counters, cnt);
}

// Applies the NEE gradients of the samples whose visibility ray found the
// light unoccluded (sLr.w set by the shadow kernel) and adds the NEE weight to
// the vertex's radiance increment.  With WAR it also forms the gradient of the
// NEE ray's reparameterisation and hands the adjoint of the incident
// direction to the vertex record.
template <bool WAR>
__global__ void __launch_bounds__(kShadeBlock, FPT_WW_MIN_BLOCKS) ww_nee_grad(DevScene s, WarParams p, WaveParams wp, SoA w, WarWave ww) {
    __shared__ uint2 stackMem[WAR ? kStackSize * kShadeBlock : 1];
    uint2* stack = stackMem + threadIdx.x;
    const uint32_t n = wp.counts[2];
    // Warp-uniform trip count: with WAR the reparameterisations of the warp's
    // samples are served together (war_coop), which needs converged warps.
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t k0 = blockIdx.x * blockDim.x + threadIdx.x - lane; k0 < n; k0 += gridDim.x * blockDim.x) {
        const uint32_t k = k0 + lane;
        uint32_t i = 0, pid = 0;
        bool live = false;
        if (k < n) {
            i = wp.shadowQueue[k];
            live = w.sLr[i].w == 1.f;
            pid = wp.waveFirstPixel + i;
        }
        WarCoopReq rq;
        rq.active = false;
        float3 dP = f3(0.f), wo = f3(0.f);
        float invDist = 0.f;
        bool posGrad = false;
        uint32_t loc[3] = {0, 0, 0};
        float bw[3] = {0.f, 0.f, 0.f};
        if (live) {
            const float4 a = nee_at(ww, 0, i), b = nee_at(ww, 1, i), c = nee_at(ww, 2, i);
            const float G[11] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w, c.x, c.y, c.z};
            const uint32_t matID = __float_as_uint(c.w);
            const float4 bb = nee_at(ww, 4, i), ll = nee_at(ww, 5, i);
            add_material_grad_values(s, p, pid, war_hash(pid, p.matHash), matID, make_float2(ll.z, ll.w), G);
            const float4 d = nee_at(ww, 3, i);
            dP = xyz(d);
            posGrad = __float_as_uint(d.w) != 0;
            const uint32_t vk = ww.nv[i] - 1;
            bw[0] = bb.x; bw[1] = bb.y; bw[2] = bb.z;
            loc[0] = __float_as_uint(bb.w); loc[1] = __float_as_uint(ll.x); loc[2] = __float_as_uint(ll.y);  // gradient offsets
            if (WAR) {
                const float4 o7 = nee_at(ww, 7, i), o8 = nee_at(ww, 8, i), o9 = nee_at(ww, 9, i);
                const float3 gdN = xyz(o9);
                const float gRatio = o8.w;  // also the adjoint of the reparameterisation weight
                const float4 fn = nee_at(ww, 12, i);
                if (__float_as_uint(fn.w)) add_frame_grad(p, pid, loc, bw, xyz(fn), xyz(nee_at(ww, 13, i)));
                if (p.useWAR && war_wants_pos(p) && (nonzero(gdN) || gRatio != 0.f)) {
                    wo = xyz(o8);
                    invDist = 1.f / o7.w;
                    rq.active = true;
                    rq.origin = xyz(o7);
                    rq.dir = wo;
                    rq.sg = as_u4(nee_at(ww, 10, i));
                    rq.gDir = gdN;
                    rq.gJ = gRatio;
                    rq.needD = true;
                }
                const float4 gv = nee_at(ww, 11, i);
                float4& r8 = rec_at(ww, vk, 8, i);
                r8.x += gv.x;
                r8.y += gv.y;
                r8.z += gv.z;
            }
            const float4 wt = nee_at(ww, 6, i);
            float4& e = rec_at(ww, vk, 4, i);
            e.x += wt.x;
            e.y += wt.y;
            e.z += wt.z;
        }
        if (WAR) {
            float3 gO = f3(0.f), gD = f3(0.f);
            war_coop<3>(s, p, pid, rq, stack, kShadeBlock, gO, gD);
            // The origin follows posW (computeRayOrigin passes its derivative
            // through); the unwarped direction is (P_light - posW) / dist.
            if (rq.active) dP += gO - (gD - wo * dot(wo, gD)) * invDist;
        }
        if (live && posGrad) add_position_grad(p, pid, loc, bw, dP);
    }
}

// Reverse sweep over each path's records (war_sweep_vertex), then the
// screen-sample reparameterisation (WAR).
// Claims one slot of a request queue per lane with want set (warp-aggregated);
// ~0u when not wanted or when the queue is full (recorded in the error word).
FPT_D uint32_t claim_slot(const DevScene& s, bool want, uint32_t* count, uint32_t capacity) {
    const uint32_t group = __activemask();
    const uint32_t mask = __ballot_sync(group, want);
    if (mask == 0) return ~0u;
    const uint32_t lane = threadIdx.x & 31u;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (int(lane) == leader) base = atomicAdd(count, uint32_t(__popc(mask)));
    base = __shfl_sync(group, base, leader);
    if (!want) return ~0u;
    const uint32_t pos = base + uint32_t(__popc(mask & ((1u << lane) - 1u)));
    if (pos >= capacity) {
        atomicOr(s.errorWord, FPT_DEVERR_QUEUE);
        return ~0u;
    }
    return pos;
}

// Reverse sweep over each path's records (war_sweep_vertex).  With WAR the
// scatter and screen reparameterisations are not evaluated here: they are
// queued for ww_war_requests, which traces their auxiliary rays with the lanes
// of a warp cooperating -- a separate, smaller kernel, as the sweep with the
// cooperative pass inline was bound by instruction fetch.
template <bool HAS_T, bool WAR>
__global__ void __launch_bounds__(kShadeBlock, FPT_WW_MIN_BLOCKS) ww_sweep(DevScene s, WarParams p, WaveParams wp, WarWave ww) {
    __shared__ uint2 stackMem[1];
    uint2* stack = stackMem;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < wp.wavePixels; i += gridDim.x * blockDim.x) {
        const uint32_t pid = wp.waveFirstPixel + i;
        const float3 g = war_dLdI(p, pid);
        const uint32_t hash = war_hash(pid, p.matHash);
        float3 A = f3(0.f), gV = f3(0.f);
        const int nv = int(ww.nv[i]);
        for (int k = nv - 1; k >= 0; k--) {
            const float4 r0 = rec_at(ww, k, 0, i), r1 = rec_at(ww, k, 1, i), r2 = rec_at(ww, k, 2, i);
            WarSweepVertex v;
            v.wiL = xyz(r0);
            v.pdf = r0.w;
            v.wsL = xyz(r1);
            v.matID = __float_as_uint(r1.w);
            v.thp = xyz(r2);
            v.flags = __float_as_uint(r2.w);
            const float4 r3 = rec_at(ww, k, 3, i), r4 = rec_at(ww, k, 4, i);
            v.bw = xyz(r3);
            v.e = xyz(r4);
            v.uv = make_float2(r3.w, r4.w);
            WarCoopReq rq;
            rq.active = false;
            uint32_t off[3] = {0, 0, 0};
            float bwt[3] = {0.f, 0.f, 0.f};
            bool posT = false;
            if (WAR) {
                const float4 r5 = rec_at(ww, k, 5, i), r6 = rec_at(ww, k, 6, i), r8 = rec_at(ww, k, 8, i), r9 = rec_at(ww, k, 9, i);
                v.inDir = xyz(r5);
                v.inst = __float_as_uint(r5.w);
                v.outDir = xyz(r6);
                v.prim = __float_as_uint(r6.w);
                v.sg = as_u4(rec_at(ww, k, 7, i));
                v.gV = xyz(r8);
                v.b[0] = r8.w;
                v.b[1] = r9.x;
                v.b[2] = r9.y;
            }
            war_sweep_vertex<HAS_T, WAR>(s, p, pid, hash, v, g, A, gV, stack, kShadeBlock, WAR ? &rq : nullptr, &off, &bwt, &posT);
            if (WAR) {
                // Queued whenever the warp is wanted: the auxiliary hits can be on
                // the optimised mesh although this vertex is not (posT).
                const uint32_t slot = claim_slot(s, rq.active, ww.reqCount, ww.reqCapacity);
                if (slot != ~0u) {
                    req_at(ww, 0, slot) = make_float4(rq.origin.x, rq.origin.y, rq.origin.z, rq.gJ);
                    req_at(ww, 1, slot) = make_float4(rq.dir.x, rq.dir.y, rq.dir.z, __uint_as_float(pid));
                    req_at(ww, 2, slot) = make_float4(rq.gDir.x, rq.gDir.y, rq.gDir.z, bwt[1]);
                    as_u4(req_at(ww, 3, slot)) = rq.sg;
                    req_at(ww, 4, slot) = make_float4(__uint_as_float(off[0]), __uint_as_float(off[1]), __uint_as_float(off[2]), bwt[0]);
                    req_at(ww, 5, slot) = make_float4(bwt[2], __uint_as_float(posT ? 1u : 0u), 0.f, 0.f);
                }
            }
        }
        if (WAR && p.useWAR && war_wants_pos(p) && nv > 0) {
            WarCoopReq rq;
            rq.active = false;
            war_sweep_screen(s, p, pid, A, gV, stack, kShadeBlock, &rq);
            const uint32_t slot = claim_slot(s, rq.active, ww.reqCount + 1, ww.capacity);
            if (slot != ~0u) {
                sreq_at(ww, 0, slot) = make_float4(rq.posS.x, rq.posS.y, rq.gPix.x, rq.gPix.y);
                as_u4(sreq_at(ww, 1, slot)) = rq.sg;
                sreq_at(ww, 2, slot) = make_float4(rq.gJ, __uint_as_float(pid), 0.f, 0.f);
            }
        }
    }
}

// Serves the queued reparameterisations (J = 3 scatter rays, J = 2 screen
// samples): each lane loads one request and the warp traces their auxiliary
// rays together (war_coop); the origin's adjoint of a scatter ray goes to its
// vertex's position gradient.
// FPT_WAR_REQ_ROUND 1: a warp takes only the requests that war_coop serves in
// one round (32 / G for G lanes per request), so that a launch with few
// requests spreads them over all resident warps instead of giving a few warps
// many sequential rounds; 0: one request per lane.
#ifndef FPT_WAR_REQ_ROUND
#define FPT_WAR_REQ_ROUND 1
#endif
template <int J>
__global__ void __launch_bounds__(kShadeBlock, FPT_WW_MIN_BLOCKS) ww_war_requests(DevScene s, WarParams p, WarWave ww) {
    __shared__ uint2 stackMem[kStackSize * kShadeBlock];
    uint2* stack = stackMem + threadIdx.x;
    const uint32_t n = min(ww.reqCount[J == 3 ? 0 : 1], J == 3 ? ww.reqCapacity : ww.capacity);
    const uint32_t lane = threadIdx.x & 31u;
    uint32_t G = 1;
    while (G < p.auxCount) G <<= 1;
    const uint32_t perWarp = FPT_WAR_REQ_ROUND ? 32u / G : 32u;  // G <= 32 (auxCount <= kMaxAux)
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t warps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t k0 = warp * perWarp; k0 < n; k0 += warps * perWarp) {
        const uint32_t k = k0 + lane;
        WarCoopReq rq;
        rq.active = lane < perWarp && k < n;
        rq.needD = false;
        uint32_t pid = 0;
        uint32_t off[3] = {0, 0, 0};
        float bw[3] = {0.f, 0.f, 0.f};
        bool posT = false;
        if (rq.active) {
            if (J == 3) {
                const float4 a = req_at(ww, 0, k), b = req_at(ww, 1, k), c = req_at(ww, 2, k), d = req_at(ww, 4, k);
                rq.origin = xyz(a);
                rq.gJ = a.w;
                rq.dir = xyz(b);
                pid = __float_as_uint(b.w);
                rq.gDir = xyz(c);
                bw[1] = c.w;
                rq.sg = as_u4(req_at(ww, 3, k));
                off[0] = __float_as_uint(d.x);
                off[1] = __float_as_uint(d.y);
                off[2] = __float_as_uint(d.z);
                bw[0] = d.w;
                const float4 e = req_at(ww, 5, k);
                bw[2] = e.x;
                posT = __float_as_uint(e.y) != 0u;
            } else {
                const float4 a = sreq_at(ww, 0, k);
                rq.posS = make_float2(a.x, a.y);
                rq.gPix = make_float2(a.z, a.w);
                rq.sg = as_u4(sreq_at(ww, 1, k));
                const float4 c = sreq_at(ww, 2, k);
                rq.gJ = c.x;
                pid = __float_as_uint(c.y);
            }
        }
        float3 gO = f3(0.f), gD = f3(0.f);
        war_coop<J>(s, p, pid, rq, stack, kShadeBlock, gO, gD);
        if (J == 3 && rq.active && posT) add_position_grad(p, pid, off, bw, gO);
    }
}

// Checkpoint record (forward): the hits of the extension rays just traced.
__global__ void ww_ck_record_hits(WaveParams wp, SoA w, WarCheckpoint ck, uint32_t it) {
    const uint32_t n = wp.counts[1];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t i = wp.extQueue[k];
        const uint32_t f = __float_as_uint(w.dirV[i].w);
        ck.hits[size_t(it) * ck.pixels + wp.waveFirstPixel + i] = (f & 0x2u) ? w.hit[i] : make_uint4(kCkMiss, 0, 0, 0);
    }
}
// Checkpoint record (forward): the visibility rays that found the light.
__global__ void ww_ck_record_visible(WaveParams wp, SoA w, WarCheckpoint ck, uint32_t it) {
    const uint32_t n = wp.counts[2];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t i = wp.shadowQueue[k];
        if (w.sLr[i].w == 1.f) ck.visible[wp.waveFirstPixel + i] |= 1u << it;
    }
}
// Checkpoint read (adjoint): the extension kernel's effect on the path state
// (trace_queue, closest hit) from the stored hit.
__global__ void ww_ck_extend(WaveParams wp, SoA w, WarCheckpoint ck, uint32_t it) {
    const uint32_t n = wp.counts[1];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t i = wp.extQueue[k];
        const uint4 h = ck.hits[size_t(it) * ck.pixels + wp.waveFirstPixel + i];
        float4 d = w.dirV[i];
        uint32_t f = __float_as_uint(d.w) + (1u << 16);  // vertexIndex++
        if (h.x != kCkMiss) {
            f |= 0x2u;
            w.hit[i] = h;
        } else {
            f &= ~0x2u;
        }
        d.w = __uint_as_float(f);
        w.dirV[i] = d;
    }
}
// Checkpoint read (adjoint): the visibility kernel's effect (trace_queue, any hit).
__global__ void ww_ck_shadow(WaveParams wp, SoA w, WarCheckpoint ck, uint32_t it) {
    const uint32_t n = wp.counts[2];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t i = wp.shadowQueue[k];
        if (!((ck.visible[wp.waveFirstPixel + i] >> it) & 1u)) continue;
        const float4 lr = w.sLr[i];
        float4 L = w.L[i];
        L.x += lr.x;
        L.y += lr.y;
        L.z += lr.z;
        w.L[i] = L;
        w.sLr[i].w = 1.f;
    }
}

__global__ void ww_resolve(WarParams p, WaveParams wp, SoA w) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < wp.wavePixels; i += gridDim.x * blockDim.x) {
        const float4 L = w.L[i];
        p.color[wp.waveFirstPixel + i] = make_float4(L.x, L.y, L.z, 1.f);
    }
}

__global__ void ww_advance(WaveParams wp) {
    wp.counts[0] = wp.counts[1];
    wp.counts[1] = 0;
    wp.counts[2] = 0;
    wp.counts[kFetchExtend] = 0;
    wp.counts[kFetchShadow] = 0;
}

__global__ void __launch_bounds__(kTraceBlock, FPT_TRACE_MIN_BLOCKS) ww_extend(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    __shared__ uint2 stackMem[kStackSize * kTraceBlock];
    trace_queue<false>(s, p, wp, w, stackMem + threadIdx.x);
}
template <bool MARK>
__global__ void __launch_bounds__(kTraceBlock, FPT_TRACE_MIN_BLOCKS) ww_shadow(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    __shared__ uint2 stackMem[kStackSize * kTraceBlock];
    trace_queue<true, MARK>(s, p, wp, w, stackMem + threadIdx.x);
}

template <bool HAS_T, bool BWD, bool WAR>
cudaError_t run_war_wavefront(const DevScene& s, const WarParams& p, WavefrontBuffers& b, void* adj, cudaStream_t st,
                              uint32_t& launches, const WarCheckpoint* ck) {
    const int ckMode = ck ? ck->mode : 0;
    SoA w;
    w.originPdf = b.f4(0); w.dirV = b.f4(1); w.thpB = b.f4(2); w.L = b.f4(3);
    w.sg = reinterpret_cast<uint4*>(b.f4(4)); w.hit = reinterpret_cast<uint4*>(b.f4(5));
    w.sOrigin = b.f4(6); w.sDir = b.f4(7); w.sLr = b.f4(8);
    w.nrm = nullptr;
    w.sampleL = b.sampleL;
    WarWave ww{};
    ww.capacity = b.capacity;
    ww.maxVertices = p.maxBounces + 2;
    ww.recArrays = WAR ? kRecArraysWar : kRecArrays;
    if (BWD) {
        char* q = static_cast<char*>(adj);
        ww.nee = reinterpret_cast<float4*>(q);
        q += size_t(WAR ? kNeeArraysWar : kNeeArrays) * b.capacity * sizeof(float4);
        ww.rec = reinterpret_cast<float4*>(q);
        q += size_t(ww.maxVertices) * ww.recArrays * b.capacity * sizeof(float4);
        ww.nv = reinterpret_cast<uint32_t*>(q);
        q += size_t(b.capacity) * sizeof(uint32_t);
        ww.req = ww.sreq = nullptr;
        ww.reqCount = nullptr;
        ww.reqCapacity = 0;
        if (WAR) {
            q = reinterpret_cast<char*>((reinterpret_cast<uintptr_t>(q) + 255) & ~uintptr_t(255));
            ww.reqCapacity = ww.maxVertices * b.capacity;
            ww.req = reinterpret_cast<float4*>(q);
            q += size_t(kReqArrays) * ww.reqCapacity * sizeof(float4);
            ww.sreq = reinterpret_cast<float4*>(q);
            q += size_t(kScreenReqArrays) * b.capacity * sizeof(float4);
            ww.reqCount = reinterpret_cast<uint32_t*>(q);
        }
    }
    // Trace kernels read the ray counters through FrameParams.
    FrameParams fp{};
    fp.counters = p.counters;
    static int gShade = 0, gTrace = 0, gSweep = 0, gNee = 0, gReq3 = 0, gReq2 = 0;
    if (!gShade) {
        gShade = blocks_for(reinterpret_cast<const void*>(ww_shade<HAS_T, BWD, WAR>), kShadeBlock);
        gTrace = blocks_for(reinterpret_cast<const void*>(ww_extend), kTraceBlock);
        gSweep = BWD ? blocks_for(reinterpret_cast<const void*>(ww_sweep<HAS_T, WAR>), kShadeBlock) : 1;
        gNee = BWD ? blocks_for(reinterpret_cast<const void*>(ww_nee_grad<WAR>), kShadeBlock) : 1;
        gReq3 = WAR ? blocks_for(reinterpret_cast<const void*>(ww_war_requests<3>), kShadeBlock) : 1;
        gReq2 = WAR ? blocks_for(reinterpret_cast<const void*>(ww_war_requests<2>), kShadeBlock) : 1;
    }
    const uint32_t pixels = p.width * p.height;
    const uint32_t maxIter = p.maxBounces + 2;
    launches = 0;
    for (uint32_t first = 0; first < pixels; first += b.capacity) {
        WaveParams wp{};  // every field not set below stays null / zero (no sort, split, binning)
        wp.waveFirstPixel = first;
        wp.wavePixels = std::min(b.capacity, pixels - first);
        wp.wavePaths = wp.wavePixels;
        wp.counts = b.counts;
        cudaError_t e = cudaMemsetAsync(b.counts, 0, kNumWaveCounts * sizeof(uint32_t), st);
        if (e != cudaSuccess) return e;
        uint32_t* qa = b.queueA;
        uint32_t* qb = b.queueB;
        wp.shadeQueue = qa;
        wp.extQueue = qb;
        wp.shadowQueue = b.shadowQueue;
        const int genBlocks = std::min<int>(gShade, int((wp.wavePixels + kShadeBlock - 1) / kShadeBlock));
        ww_generate<BWD><<<genBlocks, kShadeBlock, 0, st>>>(s, p, wp, w, ww);
        launches++;
        const int ckBlocks = std::min<int>(gShade, int((wp.wavePixels + kShadeBlock - 1) / kShadeBlock));
        for (uint32_t it = 0; it < maxIter; it++) {
            if (ckMode == 2) {
                ww_ck_extend<<<ckBlocks, kShadeBlock, 0, st>>>(wp, w, *ck, it);
            } else {
                ww_extend<<<gTrace, kTraceBlock, 0, st>>>(s, fp, wp, w);
                if (ckMode == 1) {
                    ww_ck_record_hits<<<ckBlocks, kShadeBlock, 0, st>>>(wp, w, *ck, it);
                    launches++;
                }
            }
            ww_advance<<<1, 1, 0, st>>>(wp);
            std::swap(qa, qb);
            wp.shadeQueue = qa;
            wp.extQueue = qb;
            ww_shade<HAS_T, BWD, WAR><<<gShade, kShadeBlock, 0, st>>>(s, p, wp, w, ww);
            if (ckMode == 2) {
                ww_ck_shadow<<<ckBlocks, kShadeBlock, 0, st>>>(wp, w, *ck, it);
            } else if (ckMode == 1) {
                ww_shadow<true><<<gTrace, kTraceBlock, 0, st>>>(s, fp, wp, w);
                ww_ck_record_visible<<<ckBlocks, kShadeBlock, 0, st>>>(wp, w, *ck, it);
                launches++;
            } else {
                ww_shadow<BWD><<<gTrace, kTraceBlock, 0, st>>>(s, fp, wp, w);
            }
            launches += 4;
            if (BWD) {
                ww_nee_grad<WAR><<<gNee, kShadeBlock, 0, st>>>(s, p, wp, w, ww);
                launches++;
            }
        }
        if (BWD) {
            if (WAR) {
                e = cudaMemsetAsync(ww.reqCount, 0, 2 * sizeof(uint32_t), st);
                if (e != cudaSuccess) return e;
            }
            ww_sweep<HAS_T, WAR><<<std::min<int>(gSweep, int((wp.wavePixels + kShadeBlock - 1) / kShadeBlock)), kShadeBlock, 0, st>>>(
                s, p, wp, ww);
            if (WAR) {
                ww_war_requests<3><<<gReq3, kShadeBlock, 0, st>>>(s, p, ww);
                ww_war_requests<2><<<gReq2, kShadeBlock, 0, st>>>(s, p, ww);
                launches += 2;
            }
        } else {
            ww_resolve<<<(wp.wavePixels + 255) / 256, 256, 0, st>>>(p, wp, w);
        }
        launches++;
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

size_t war_checkpoint_bytes(uint32_t pixels, uint32_t maxBounces) {
    return (size_t(maxBounces) + 2) * pixels * sizeof(uint4) + size_t(pixels) * sizeof(uint32_t);
}

size_t war_adjoint_bytes(uint32_t capacity, uint32_t maxBounces, bool war) {
    const size_t maxVertices = size_t(maxBounces) + 2;
    const size_t nee = war ? kNeeArraysWar : kNeeArrays, rec = war ? kRecArraysWar : kRecArrays;
    size_t bytes = (nee + maxVertices * rec) * capacity * sizeof(float4) + size_t(capacity) * sizeof(uint32_t);
    if (war)  // alignment, scatter and screen requests, two counters
        bytes += 256 + (size_t(kReqArrays) * maxVertices + kScreenReqArrays) * capacity * sizeof(float4) + 2 * sizeof(uint32_t);
    return bytes;
}

cudaError_t launch_war_wavefront(const DevScene& s, const WarParams& p, WavefrontBuffers& b, void* adjointScratch, bool backward,
                                 cudaStream_t st, uint32_t& launches, const WarCheckpoint* ck) {
    // Extended records: the warps (position derivatives only) and normal / tangent gradients.
    const bool war = backward && ((p.useWAR && (p.gradPos || (p.dbgColor && p.dbgType == kDbgTranslation))) ||
                                  p.gradNrm || p.gradTan);
    if (s.hasTransmission) {
        if (!backward) return run_war_wavefront<true, false, false>(s, p, b, adjointScratch, st, launches, ck);
        return war ? run_war_wavefront<true, true, true>(s, p, b, adjointScratch, st, launches, ck)
                   : run_war_wavefront<true, true, false>(s, p, b, adjointScratch, st, launches, ck);
    }
    if (!backward) return run_war_wavefront<false, false, false>(s, p, b, adjointScratch, st, launches, ck);
    return war ? run_war_wavefront<false, true, true>(s, p, b, adjointScratch, st, launches, ck)
               : run_war_wavefront<false, true, false>(s, p, b, adjointScratch, st, launches, ck);
}

}  // namespace fpt
