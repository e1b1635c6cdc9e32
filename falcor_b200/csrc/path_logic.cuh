// path_logic.cuh -- per-vertex PathTracer logic shared by the megakernel and
// the wavefront kernels: handleHit / handleMiss of PathTracer.slang with
// NEE + MIS over the env map and emissive triangles, and the event counters.
#pragma once

#include "kernels.cuh"

namespace fpt {
namespace dev {

// Per-thread event counts, reduced per warp and added to the pass's device
// counters once per thread: [0] paths, [1] rays, [2] closest-hit rays,
// [3] visibility rays, [4] BVH node visits, [5] triangle tests, [6] shaded
// hits, [7] emissive light samples, [8] env-map importance samples,
// [9] env-map evaluations, [10] env-map pdf evaluations, [11] node visits and
// [12] triangle tests of visibility rays (included in [4] and [5]).
struct Counters {
    uint32_t v[kNumCounters] = {0};
    FPT_D void trace(bool shadow, const TraceStats& ts) {
        v[1]++;
        v[shadow ? 3 : 2]++;
        v[4] += ts.nodes;
        v[5] += ts.tris;
        if (shadow) {
            v[11] += ts.nodes;
            v[12] += ts.tris;
        }
    }
};

FPT_D void flush_counters(unsigned long long* out, const Counters& c) {
    if (!out) return;
#pragma unroll
    for (int i = 0; i < kNumCounters; i++) {
        unsigned long long x = c.v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if ((threadIdx.x & 31) == 0 && x) atomicAdd(out + i, x);
    }
}

// ---------------------------------------------------------------------------
// PathTracer.
// ---------------------------------------------------------------------------
constexpr uint32_t PF_ACTIVE = 0x1, PF_TRANSMISSION = 0x4, PF_SPECULAR = 0x8, PF_DELTA = 0x10;
constexpr uint32_t PF_LIGHT_UPPER = 0x40, PF_LIGHT_LOWER = 0x80;

FPT_D float eval_mis(const FrameParams& p, float p0, float p1) {
    if (p.misHeuristic == 0) { const float q0 = p0, q1 = p1; return q0 / (q0 + q1); }
    if (p.misHeuristic == 1) { const float q0 = p0 * p0, q1 = p1 * p1; return q0 / (q0 + q1); }
    const float q0 = fm::pow(p0, p.misPowerExponent), q1 = fm::pow(p1, p.misPowerExponent);
    return q0 / (q0 + q1);
}

template <class SG>
struct PathState {
    uint32_t flags, bounces, vertexIndex;
    float3 origin, dir, normal, thp, L;
    float pdf;
    HitRec hit;
    SG sg;
    // Pending visibility ray of the last NEE sample and its contribution.
    bool shadowPending;
    float3 sOrigin, sDir, sLr;
    float sDist;
    FPT_D bool has(uint32_t f) const { return (flags & f) != 0; }
    FPT_D void set(uint32_t f, bool v) { flags = v ? (flags | f) : (flags & ~f); }
    FPT_D uint32_t getBounces(int t) const { return (bounces >> (t * 8)) & 0xffu; }
    FPT_D bool isLightSampled() const { return (flags & (PF_LIGHT_UPPER | PF_LIGHT_LOWER)) != 0; }
    FPT_D bool isLightSamplable() const { return !has(PF_DELTA); }
};

// Optional record of the hit of path vertex `vertexIndex` (1 = the primary
// hit) of one sample: (instanceID + 1, primitiveIndex, bary.x, bary.y bits), or
// zeros for a miss.  `perSample` entries per sample, `spp` samples per pixel
// (fpt_frame_io::hit_trace).
FPT_D void record_vertex(const FrameParams& p, uint32_t spp, uint32_t perSample, uint32_t pix, uint32_t sample,
                         uint32_t vertexIndex, bool valid, const HitRec& h) {
    if (vertexIndex == 0 || vertexIndex > perSample) return;
    const uint4 v = valid ? make_uint4(h.instanceID + 1u, h.primIndex, __float_as_uint(h.baryX), __float_as_uint(h.baryY))
                          : make_uint4(0u, 0u, 0u, 0u);
    p.hitTrace[(size_t(pix) * spp + sample) * perSample + (vertexIndex - 1)] = v;
}

FPT_D bool finished_surface_bounces(const FrameParams& p, uint32_t bounces) {
    const uint32_t d = bounces & 0xffu, sp = (bounces >> 8) & 0xffu, tr = (bounces >> 16) & 0xffu;
    return (d + sp + tr > p.maxSurfaceBounces) || (d > p.maxDiffuseBounces) || (sp > p.maxSpecularBounces) ||
           (tr > p.maxTransmissionBounces);
}

// generateLightSample (PathTracer.slang:705-738) for env + emissive lights.
template <class SG>
FPT_D bool generate_light_sample(const DevScene& s, const FrameParams& p, const ShadingData& sd, bool upper, bool lower,
                                 SG& sg, float3& Li, float& lpdf, float3& lorigin, float3& ldir, float& ldist, Counters& cnt) {
    const bool useEnv = s.hasEnv != 0, useEm = s.hasEmissive != 0;
    float pr0 = useEnv ? 1.f : 0.f, pr1 = useEm ? 1.f : 0.f;
    const float sum = pr0 + pr1;
    if (sum != 0.f) { const float inv = 1.f / sum; pr0 *= inv; pr1 *= inv; }
    float u = next1D(sg);
    uint32_t lightType;
    float selPdf;
    if (u < pr0) { lightType = 0; selPdf = pr0; }
    else {
        u -= pr0;
        if (u < pr1) { lightType = 1; selPdf = pr1; }
        else return false;
    }
    bool valid = false;
    if (useEnv && lightType == 0) {
        float3 dir, Le;
        float epdf;
        env_sample(s, next2D(sg), dir, epdf, Le);
        cnt.v[8]++;
        Li = epdf > 0.f ? Le / epdf : f3(0.f);
        lpdf = epdf;
        lorigin = compute_ray_origin(sd.posW, dot(sd.faceN, dir) >= 0.f ? sd.faceN : -sd.faceN);
        ldist = 1e30f;
        ldir = dir;
        valid = any_pos(Li);
    }
    if (useEm && lightType == 1) {
        TriLightSample tls;
        cnt.v[7]++;
        // generateEmissiveSample: upperHemisphere = upper && !lower (PathTracer.slang:705-720).
        if (emissive_sample(s, p.emissiveSampler, sd.posW, sg, tls, sd_oriented_face_n(sd), upper && !lower)) {
            Li = tls.pdf > 0.f ? tls.Le / tls.pdf : f3(0.f);
            lpdf = tls.pdf;
            const float3 lightPos = compute_ray_origin(tls.posW, tls.normalW);
            const float3 toL0 = lightPos - sd.posW;
            lorigin = compute_ray_origin(sd.posW, dot(sd.faceN, toL0) >= 0.f ? sd.faceN : -sd.faceN);
            const float3 toLight = lightPos - lorigin;
            ldist = length(toLight);
            ldir = normalize(toLight);
            valid = any_pos(Li);
        }
    }
    if (!valid) return false;
    const float NdotL = dot(sd_oriented_face_n(sd), ldir);
    if ((!upper && NdotL >= -kMinCosTheta) || (!lower && NdotL <= kMinCosTheta)) return false;
    lpdf *= selPdf;
    Li = Li / selPdf;
    return true;
}

// PathTracer::handleHit (PathTracer.slang:821-1066).
template <class SG, bool HAS_T, bool TEX = true>
FPT_D void pt_handle_hit(const DevScene& s, const FrameParams& p, PathState<SG>& path, Counters& cnt) {
    const bool isPrimaryHit = path.vertexIndex == 1;
    const bool useEnv = s.hasEnv != 0, useEm = s.hasEmissive != 0;
    const ShadingData sd = load_shading_data(s, path.hit, path.dir);
    cnt.v[6]++;
    const MaterialInstance<HAS_T> mi = material_instance<HAS_T, TEX>(s, sd, p.lambert != 0);
    const float roughness = mi.propRoughness();
    const bool isLightSamplable = path.isLightSamplable();
    const bool computeEmissive =
        isPrimaryHit || (useEm && (!p.useNEE || p.useMIS || !path.isLightSampled() || !isLightSamplable));
    if (computeEmissive && any_pos(mi.emission)) {
        float misWeight = 1.f;
        if (useEm && p.useNEE && p.useMIS && !isPrimaryHit && path.isLightSampled() && isLightSamplable) {
            const uint32_t off = __ldg(s.instEmissiveOffset + path.hit.instanceID);
            const uint32_t triIdx = off == 0xffffffffu ? 0xffffffffu : off + path.hit.primIndex;
            const float emissiveSel = (useEnv && useEm) ? 0.5f : 1.f;
            // upperHemisphere = isLightSampledUpper && !isLightSampledLower (PathTracer.slang:909).
            const bool upperOnly = path.has(PF_LIGHT_UPPER) && !path.has(PF_LIGHT_LOWER);
            const float lightPdf = emissiveSel * emissive_eval_pdf(s, p.emissiveSampler, path.origin, triIdx, sd.posW,
                                                                   sd_oriented_face_n(sd), path.normal, upperOnly);
            misWeight = eval_mis(p, path.pdf, lightPdf);
        }
        path.L += path.thp * (misWeight * mi.emission);
    }
    if (finished_surface_bounces(p, path.bounces)) { path.set(PF_ACTIVE, false); return; }
    path.origin = sd_ray_origin(sd);
    const uint32_t lobeTypes = mi.lobeTypes();
    const bool applyNEE = p.useNEE && (lobeTypes & L_NON_DELTA) != 0;
    path.set(PF_LIGHT_UPPER | PF_LIGHT_LOWER, false);
    // One BSDF set-up for the light sample's evaluation and the scatter sample.
    const float3 wiL = mi.toLocal(sd.V);
    const StandardBSDF<HAS_T> bs = mi.bsdf(wiL);
    if (applyNEE) {
        const bool upper = (lobeTypes & L_NON_DELTA_R) != 0, lower = (lobeTypes & L_NON_DELTA_T) != 0;
        float3 Li, lorigin, ldir;
        float lpdf, ldist;
        const bool validSample = generate_light_sample(s, p, sd, upper, lower, path.sg, Li, lpdf, lorigin, ldir, ldist, cnt);
        path.set(PF_LIGHT_UPPER, upper);
        path.set(PF_LIGHT_LOWER, lower);
        if (validSample) {
            float3 f;
            float scatterPdf;
            mi.eval_with_pdf(sd, bs, wiL, ldir, p.useBSDFSampling != 0, f, scatterPdf);
            if (p.useMIS) Li *= eval_mis(p, lpdf, scatterPdf);
            const float3 Lr = f * Li;
            if (any_pos(Lr)) {
                // The visibility ray is traced by the caller's single traversal
                // site before the next extension ray; its contribution thp * Lr
                // uses the throughput before scattering, as in the reference.
                path.shadowPending = true;
                path.sOrigin = lorigin;
                path.sDir = ldir;
                path.sDist = ldist;
                path.sLr = path.thp * Lr;
            }
        }
    }
    // generateScatterRay (PathTracer.slang:385-513).
    float3 wo, w;
    float bpdf;
    uint32_t lobe;
    bool valid = mi.sample_with(sd, bs, wiL, path.sg, wo, w, bpdf, lobe, p.useBSDFSampling != 0);
    if (valid) {
        path.dir = wo;
        path.thp *= w;
        path.pdf = bpdf;
        path.set(PF_TRANSMISSION | PF_SPECULAR | PF_DELTA, false);
        if (lobe & L_REFLECTION) {
            const bool isDiffuse = (lobe & L_DIFF_R) || roughness > p.specularRoughnessThreshold;
            if (isDiffuse) path.bounces += 1u;
            else { path.bounces += 1u << 8; path.set(PF_SPECULAR, true); }
        }
        if (lobe & L_DELTA) path.set(PF_DELTA, true);
        if (lobe & L_TRANSMISSION) {
            path.bounces += 1u << 16;
            path.set(PF_TRANSMISSION, true);
            path.origin = sd_ray_origin(sd, false);
        }
        path.normal = sd_oriented_face_n(sd);
        valid = any_pos(path.thp);
    }
    if (p.useNEE && !p.useMIS && finished_surface_bounces(p, path.bounces) && path.isLightSamplable()) valid = false;
    if (!valid) path.set(PF_ACTIVE, false);
}

// PathTracer::handleMiss (PathTracer.slang:1071-1157).
template <class SG>
FPT_D void pt_handle_miss(const DevScene& s, const FrameParams& p, PathState<SG>& path, Counters& cnt) {
    const bool useEnv = s.hasEnv != 0, useEm = s.hasEmissive != 0;
    const bool isLightSamplable = path.isLightSamplable();
    const bool computeEnv = useEnv && (!p.useNEE || p.useMIS || !path.isLightSampled() || !isLightSamplable);
    if (computeEnv) {
        float misWeight = 1.f;
        if (p.useNEE && p.useMIS && path.isLightSampled() && isLightSamplable) {
            const float envSel = (useEnv && useEm) ? 0.5f : 1.f;
            const float lightPdf = envSel * env_eval_pdf(s, path.dir);
            cnt.v[10]++;
            misWeight = eval_mis(p, path.pdf, lightPdf);
        }
        path.L += path.thp * (misWeight * env_eval(s, path.dir));
        cnt.v[9]++;
    }
    path.set(PF_ACTIVE, false);
}

}  // namespace dev
}  // namespace fpt
