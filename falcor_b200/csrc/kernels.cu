// kernels.cu -- render-pass kernels for sm_100a:
//   vbuffer_kernel      VBufferRT primary hits (VBufferRT.rt.slang:47-86)
//   minimal_pt_kernel   MinimalPathTracer (MinimalPathTracer.rt.slang:297-468)
//   path_tracer_kernel  PathTracer with NEE + MIS (PathTracer.slang:241-1202,
//                       TracePass.rt.slang:385-507, GeneratePaths.cs.slang,
//                       ResolvePass.cs.slang)
//
// Each thread traces whole paths; BVH traversal stacks live in shared memory
// (kStackSize entries per thread, interleaved across the block so that the
// threads of a warp hit distinct banks).  The path tracer runs persistent
// warps that fetch 32 pixels at a time from a global work counter, and each
// lane loops over the pixel's samples, so lanes of a warp stay in the same
// trace/shade loop while their paths have different lengths.
#include "kernels.cuh"

namespace fpt {

using namespace dev;

namespace {

constexpr int kVBufferBlock = 128;
constexpr int kMinimalBlock = 128;
constexpr int kPathBlock = 128;

// Per-thread event counts, reduced per warp and added to the pass's device
// counters once per thread: [0] paths, [1] rays, [2] closest-hit rays,
// [3] visibility rays, [4] BVH node visits, [5] triangle tests, [6] shaded
// hits, [7] emissive light samples, [8] env-map importance samples,
// [9] env-map evaluations, [10] env-map pdf evaluations.
struct Counters {
    uint32_t v[kNumCounters] = {0};
    FPT_D void trace(bool shadow, const TraceStats& ts) {
        v[1]++;
        v[shadow ? 3 : 2]++;
        v[4] += ts.nodes;
        v[5] += ts.tris;
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
// VBufferRT.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(kVBufferBlock) vbuffer_kernel(DevScene s, FrameParams p) {
    __shared__ uint2 stackMem[kStackSize * kVBufferBlock];
    uint2* stack = stackMem + threadIdx.x;
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= p.width * p.height) return;
    const uint32_t x = idx % p.width, y = idx / p.width;
    float tMin, tMax;
    const float3 dir = camera_ray_dir(s.camera, x, y, p.width, p.height, tMin, tMax);
    HitRec h;
    trace_bvh<false>(s, load3(s.camera.posW), dir, tMin, tMax, h, stack, kVBufferBlock);
    p.vbufferOut[idx] = pack_hit(s.bits, h);
}

// ---------------------------------------------------------------------------
// MinimalPathTracer: one path per pixel, BSDF sampling only.
// ---------------------------------------------------------------------------
template <bool HAS_T>
__global__ void __launch_bounds__(kMinimalBlock) minimal_pt_kernel(DevScene s, FrameParams p) {
    __shared__ uint2 stackMem[kStackSize * kMinimalBlock];
    uint2* stack = stackMem + threadIdx.x;
    const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
    Counters cnt;
    if (idx < p.width * p.height) {
        const uint32_t x = idx % p.width, y = idx / p.width;
        float tMin, tMax;
        const float3 primaryDir = camera_ray_dir(s.camera, x, y, p.width, p.height, tMin, tMax);
        HitRec hit;
        float3 outColor = f3(0.f);
        uint32_t rays = 0;
        const bool useEmissive = s.hasEmissive != 0, useEnv = s.hasEnv != 0;
        const bool lambert = p.lambert != 0, useIS = p.useImportanceSampling != 0;
        if (unpack_hit(s.bits, __ldg(p.vbuffer + idx), hit)) {
            ShadingData sd = load_shading_data(s, hit, primaryDir);
            MaterialInstance<HAS_T> mi = material_instance<HAS_T>(s, sd, lambert);
            UniformSG sg;
            sg.init(x, y, p.frameIndex);
            for (uint32_t i = 0; i < p.prngDimension; i++) next1D(sg);
            if (p.computeDirect) outColor += mi.emission;
            float3 radiance = f3(0.f), thp = f3(1.f), origin = f3(0.f), direction = f3(0.f);
            bool terminated = false;
            uint32_t pathLength = 0;
            // generateScatterRay at the primary hit (.rt.slang:297-314).
            {
                float3 wo, w;
                float pdf;
                uint32_t lobe;
                const float3 ro = sd_ray_origin(sd);
                if (mi.sample(sd, sg, wo, w, pdf, lobe, useIS)) {
                    origin = (lobe & L_TRANSMISSION) ? sd_ray_origin(sd, false) : ro;
                    direction = wo;
                    thp *= w;
                    if (!any_pos(thp)) terminated = true;
                } else {
                    terminated = true;
                }
            }
            for (uint32_t depth = 0; depth <= p.maxBounces && !terminated; depth++) {
                rays++;
                HitRec h;
                TraceStats ts;
                trace_bvh<false>(s, origin, direction, 0.f, 3.402823466e+38f, h, stack, kMinimalBlock, &ts);
                cnt.trace(false, ts);
                if (!h.valid) {
                    terminated = true;
                    if (useEnv && (p.computeDirect || pathLength > 0)) radiance += thp * env_eval(s, direction);
                    continue;
                }
                ShadingData hsd = load_shading_data(s, h, direction);
                MaterialInstance<HAS_T> hmi = material_instance<HAS_T>(s, hsd, lambert);
                if (useEmissive && (p.computeDirect || pathLength > 0)) radiance += thp * hmi.emission;
                if (pathLength >= p.maxBounces) { terminated = true; continue; }
                const float3 ro = sd_ray_origin(hsd);
                float3 wo, w;
                float pdf;
                uint32_t lobe;
                if (hmi.sample(hsd, sg, wo, w, pdf, lobe, useIS)) {
                    origin = (lobe & L_TRANSMISSION) ? sd_ray_origin(hsd, false) : ro;
                    direction = wo;
                    thp *= w;
                    if (!any_pos(thp)) { terminated = true; continue; }
                } else {
                    terminated = true;
                    continue;
                }
                pathLength++;
            }
            outColor += radiance;
        } else {
            outColor = useEnv ? env_eval(s, primaryDir) : f3(0.f);
        }
        p.color[idx] = make_float4(outColor.x, outColor.y, outColor.z, 1.f);
        if (p.rayCount) p.rayCount[idx] = rays;
        cnt.v[0] = 1;
    }
    flush_counters(p.counters, cnt);
}

// ---------------------------------------------------------------------------
// PathTracer.
// ---------------------------------------------------------------------------
constexpr uint32_t PF_ACTIVE = 0x1, PF_TRANSMISSION = 0x4, PF_SPECULAR = 0x8, PF_DELTA = 0x10;
constexpr uint32_t PF_LIGHT_UPPER = 0x40, PF_LIGHT_LOWER = 0x80;

FPT_D float eval_mis(const FrameParams& p, float p0, float p1) {
    if (p.misHeuristic == 0) { const float q0 = p0, q1 = p1; return q0 / (q0 + q1); }
    if (p.misHeuristic == 1) { const float q0 = p0 * p0, q1 = p1 * p1; return q0 / (q0 + q1); }
    const float q0 = powf(p0, p.misPowerExponent), q1 = powf(p1, p.misPowerExponent);
    return q0 / (q0 + q1);
}

template <class SG>
struct PathState {
    uint32_t flags, bounces, vertexIndex;
    float3 origin, dir, normal, thp, L;
    float pdf;
    HitRec hit;
    SG sg;
    FPT_D bool has(uint32_t f) const { return (flags & f) != 0; }
    FPT_D void set(uint32_t f, bool v) { flags = v ? (flags | f) : (flags & ~f); }
    FPT_D uint32_t getBounces(int t) const { return (bounces >> (t * 8)) & 0xffu; }
    FPT_D bool isLightSampled() const { return (flags & (PF_LIGHT_UPPER | PF_LIGHT_LOWER)) != 0; }
    FPT_D bool isLightSamplable() const { return !has(PF_DELTA); }
};

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
        if (emissive_sample(s, p.emissiveSampler, sd.posW, sg, tls)) {
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
template <class SG, bool HAS_T>
FPT_D void pt_handle_hit(const DevScene& s, const FrameParams& p, PathState<SG>& path, uint2* stack, Counters& cnt) {
    const bool isPrimaryHit = path.vertexIndex == 1;
    const bool useEnv = s.hasEnv != 0, useEm = s.hasEmissive != 0;
    const ShadingData sd = load_shading_data(s, path.hit, path.dir);
    cnt.v[6]++;
    const MaterialInstance<HAS_T> mi = material_instance<HAS_T>(s, sd, p.lambert != 0);
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
            const float lightPdf = emissiveSel * emissive_eval_pdf(s, p.emissiveSampler, path.origin, triIdx, sd.posW, sd_oriented_face_n(sd));
            misWeight = eval_mis(p, path.pdf, lightPdf);
        }
        path.L += path.thp * (misWeight * mi.emission);
    }
    if (finished_surface_bounces(p, path.bounces)) { path.set(PF_ACTIVE, false); return; }
    path.origin = sd_ray_origin(sd);
    const uint32_t lobeTypes = mi.lobeTypes();
    const bool applyNEE = p.useNEE && (lobeTypes & L_NON_DELTA) != 0;
    path.set(PF_LIGHT_UPPER | PF_LIGHT_LOWER, false);
    if (applyNEE) {
        const bool upper = (lobeTypes & L_NON_DELTA_R) != 0, lower = (lobeTypes & L_NON_DELTA_T) != 0;
        float3 Li, lorigin, ldir;
        float lpdf, ldist;
        const bool validSample = generate_light_sample(s, p, sd, upper, lower, path.sg, Li, lpdf, lorigin, ldir, ldist, cnt);
        path.set(PF_LIGHT_UPPER, upper);
        path.set(PF_LIGHT_LOWER, lower);
        if (validSample) {
            if (p.useMIS) {
                const float scatterPdf = mi.evalPdf(sd, ldir, p.useBSDFSampling != 0);
                Li *= eval_mis(p, lpdf, scatterPdf);
            }
            const float3 Lr = mi.eval(sd, ldir) * Li;
            if (any_pos(Lr)) {
                HitRec sh;
                TraceStats ts;
                trace_bvh<true>(s, lorigin, ldir, 0.f, ldist, sh, stack, kPathBlock, &ts);
                cnt.trace(true, ts);
                if (!sh.valid) path.L += path.thp * Lr;
            }
        }
    }
    // generateScatterRay (PathTracer.slang:385-513).
    float3 wo, w;
    float bpdf;
    uint32_t lobe;
    bool valid = mi.sample(sd, path.sg, wo, w, bpdf, lobe, p.useBSDFSampling != 0);
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

template <class SG, bool HAS_T>
FPT_D float3 pt_trace_path(const DevScene& s, const FrameParams& p, uint32_t x, uint32_t y, uint32_t sampleIdx,
                           const HitRec& primary, float3 primaryDir, uint2* stack, Counters& cnt, uint32_t& rays) {
    PathState<SG> path;
    path.sg.init(x, y, p.seed * p.spp + sampleIdx);
    path.flags = PF_ACTIVE;
    path.bounces = 0;
    path.thp = f3(1.f);
    path.L = f3(0.f);
    path.pdf = 0.f;
    path.normal = f3(0.f);
    path.origin = load3(s.camera.posW);
    path.dir = primaryDir;
    path.hit = primary;
    path.vertexIndex = 1;
    pt_handle_hit<SG, HAS_T>(s, p, path, stack, cnt);
    while (path.has(PF_ACTIVE)) {
        path.vertexIndex++;
        rays++;
        HitRec h;
        TraceStats ts;
        trace_bvh<false>(s, path.origin, path.dir, 0.f, 1e30f, h, stack, kPathBlock, &ts);
        cnt.trace(false, ts);
        if (h.valid) {
            path.hit = h;
            pt_handle_hit<SG, HAS_T>(s, p, path, stack, cnt);
        } else {
            pt_handle_miss<SG>(s, p, path, cnt);
        }
    }
    cnt.v[0]++;
    return path.L;
}

template <class SG, bool HAS_T>
__global__ void __launch_bounds__(kPathBlock) path_tracer_kernel(DevScene s, FrameParams p) {
    __shared__ uint2 stackMem[kStackSize * kPathBlock];
    uint2* stack = stackMem + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    Counters cnt;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(p.workCounter, 32u);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= p.workItems) break;
        const uint32_t idx = base + lane;
        if (idx < p.workItems) {
            const uint32_t x = idx % p.width, y = idx / p.width;
            float tMin, tMax;
            const float3 primaryDir = camera_ray_dir(s.camera, x, y, p.width, p.height, tMin, tMax);
            HitRec hit;
            const bool isHit = unpack_hit(s.bits, __ldg(p.vbuffer + idx), hit);
            const uint32_t spp = p.spp;
            float3 color = f3(0.f);
            uint32_t rays = 0;
            if (!isHit) {
                // GeneratePaths::writeBackground (GeneratePaths.cs.slang:208-245).
                const float3 bg = s.hasEnv ? env_eval(s, primaryDir) : f3(0.f);
                if (s.hasEnv) cnt.v[9]++;
                for (uint32_t i = 0; i < spp; i++) {
                    if (p.sampleColor) {
                        float* o = p.sampleColor + (size_t(idx) * spp + i) * 3;
                        o[0] = bg.x; o[1] = bg.y; o[2] = bg.z;
                    }
                    color += (spp != 1 && p.colorFormat == 1) ? decode_logluv_hdr(encode_logluv_hdr(bg)) : bg;
                }
            } else {
                for (uint32_t i = 0; i < spp; i++) {
                    const float3 L = (p.sampleGenerator == 0)
                                         ? pt_trace_path<TinyUniformSG, HAS_T>(s, p, x, y, i, hit, primaryDir, stack, cnt, rays)
                                         : pt_trace_path<UniformSG, HAS_T>(s, p, x, y, i, hit, primaryDir, stack, cnt, rays);
                    if (p.sampleColor) {
                        float* o = p.sampleColor + (size_t(idx) * spp + i) * 3;
                        o[0] = L.x; o[1] = L.y; o[2] = L.z;
                    }
                    color += (spp != 1 && p.colorFormat == 1) ? decode_logluv_hdr(encode_logluv_hdr(L)) : L;
                }
            }
            // ResolvePass (ResolvePass.cs.slang:80-101); 1 spp writes the colour directly.
            const float3 out = spp == 1 ? color : color * (1.f / float(spp));
            if (!isfinite(out.x) || !isfinite(out.y) || !isfinite(out.z)) atomicOr(s.errorWord, FPT_DEVERR_NAN);
            p.color[idx] = make_float4(out.x, out.y, out.z, 1.f);
            if (p.rayCount) p.rayCount[idx] = rays;
        }
    }
    flush_counters(p.counters, cnt);
}

int g_numSMs = 0;
int num_sms() {
    if (g_numSMs == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&g_numSMs, cudaDevAttrMultiProcessorCount, dev);
        if (g_numSMs <= 0) g_numSMs = 148;
    }
    return g_numSMs;
}

}  // namespace

cudaError_t launch_vbuffer(const DevScene& s, const FrameParams& p, cudaStream_t st) {
    const uint32_t n = p.width * p.height;
    vbuffer_kernel<<<(n + kVBufferBlock - 1) / kVBufferBlock, kVBufferBlock, 0, st>>>(s, p);
    return cudaGetLastError();
}

cudaError_t launch_minimal_pt(const DevScene& s, const FrameParams& p, cudaStream_t st) {
    const uint32_t n = p.width * p.height;
    const uint32_t blocks = (n + kMinimalBlock - 1) / kMinimalBlock;
    if (s.hasTransmission) minimal_pt_kernel<true><<<blocks, kMinimalBlock, 0, st>>>(s, p);
    else minimal_pt_kernel<false><<<blocks, kMinimalBlock, 0, st>>>(s, p);
    return cudaGetLastError();
}

int path_tracer_grid_blocks(int) {
    int perSM = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, path_tracer_kernel<TinyUniformSG, false>, kPathBlock, 0);
    if (perSM <= 0) perSM = 1;
    return perSM * num_sms();
}

cudaError_t launch_path_tracer(const DevScene& s, const FrameParams& p, cudaStream_t st, int) {
    cudaError_t e = cudaMemsetAsync(p.workCounter, 0, sizeof(uint32_t), st);
    if (e != cudaSuccess) return e;
    const int blocks = path_tracer_grid_blocks(kPathBlock);
    if (s.hasTransmission) path_tracer_kernel<TinyUniformSG, true><<<blocks, kPathBlock, 0, st>>>(s, p);
    else path_tracer_kernel<TinyUniformSG, false><<<blocks, kPathBlock, 0, st>>>(s, p);
    return cudaGetLastError();
}

}  // namespace fpt
