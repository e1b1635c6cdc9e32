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
#include "path_logic.cuh"

namespace fpt {

using namespace dev;

namespace {

constexpr int kVBufferBlock = 128;
constexpr int kMinimalBlock = 128;
constexpr int kPathBlock = 128;

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
    if (p.viewWOut) p.viewWOut[idx] = make_float4(-dir.x, -dir.y, -dir.z, 0.f);  // writeAux
    if (!p.depthOut && !p.mvecOut && !p.maskOut) return;
    float depth = 1.f, mask = 0.f;
    float2 mvec = make_float2(0.f, 0.f);
    if (h.valid) {
        // writeHit: NDC depth of the perspective projection without jitter
        // (right-handed, depth 0 at nearZ and 1 at farZ), and the motion vector
        // from the previous camera's projection of the hit (static geometry),
        // with the jitter added back.
        const DevInstance inst = s.instances[h.instanceID];
        const uint32_t* ip = s.indices + inst.ibOffset + h.primIndex * 3;
        float3 p0, p1, p2, n;
        unpack_vertex(load_vertex(s.vertices, __ldg(ip) + inst.vbOffset), p0, n);
        unpack_vertex(load_vertex(s.vertices, __ldg(ip + 1) + inst.vbOffset), p1, n);
        unpack_vertex(load_vertex(s.vertices, __ldg(ip + 2) + inst.vbOffset), p2, n);
        float3 posW = p0 * (1.f - h.baryX - h.baryY);
        posW += p1 * h.baryX;
        posW += p2 * h.baryY;
        const fpt_camera_data& c = s.camera;
        const float d = dot(posW - load3(c.posW), normalize(load3(c.cameraW)));
        depth = (c.farZ * (d - c.nearZ)) / (d * (c.farZ - c.nearZ));
        const fpt_camera_data& q = p.prevCamera;
        const float3 r = posW - load3(q.posW), U = load3(q.cameraU), V = load3(q.cameraV), Wq = load3(q.cameraW);
        const float t = dot(r, Wq) / dot(Wq, Wq);
        const float nx = dot(r, U) / (dot(U, U) * t), ny = dot(r, V) / (dot(V, V) * t);
        const float2 prevCrd = make_float2(nx * 0.5f + 0.5f, ny * -0.5f + 0.5f);
        mvec = make_float2(prevCrd.x - (float(x) + 0.5f) / float(p.width) + c.jitterX,
                           prevCrd.y - (float(y) + 0.5f) / float(p.height) - c.jitterY);
        mask = 1.f;
    }
    if (p.depthOut) p.depthOut[idx] = depth;
    if (p.mvecOut) p.mvecOut[idx] = mvec;
    if (p.maskOut) p.maskOut[idx] = mask;
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
        const uint32_t traceLen = p.maxBounces + 2;
        if (unpack_hit(s.bits, __ldg(p.vbuffer + idx), hit)) {
            if (p.hitTrace) record_vertex(p, 1, traceLen, idx, 0, 1, true, hit);
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
                if (p.hitTrace) record_vertex(p, 1, traceLen, idx, 0, depth + 2, h.valid, h);
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

// Per-lane state of the path-tracer state machine.
enum LaneState : uint32_t { LS_FETCH = 0, LS_SHADE = 1, LS_TRACE = 2, LS_MISS = 3, LS_DONE = 4 };

// Persistent path tracer.  Each lane owns one pixel at a time and runs its
// spp samples one after the other (TracePass.rt.slang:490-506); a lane that
// finishes its pixel fetches the next one with a warp-aggregated atomic, so
// lanes regenerate work independently.  Every loop iteration has one
// traversal call site (a visibility ray pending from NEE, else the extension
// ray) followed by one shading call site (handleHit or handleMiss), which
// keeps the warp converged in both phases and the kernel small.
template <class SG, bool HAS_T>
__global__ void __launch_bounds__(kPathBlock) path_tracer_kernel(DevScene s, FrameParams p) {
    __shared__ uint2 stackMem[kStackSize * kPathBlock];
    uint2* stack = stackMem + threadIdx.x;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t laneMaskLt = (1u << lane) - 1u;
    const uint32_t spp = p.spp;
    Counters cnt;
    uint32_t state = LS_FETCH;
    uint32_t idx = 0, x = 0, y = 0, sampleIdx = 0, rays = 0;
    float3 primaryDir = f3(0.f), color = f3(0.f);
    HitRec primary;
    primary.valid = false;
    PathState<SG> path;
    path.flags = 0;
    path.shadowPending = false;
    for (;;) {
        // (1) Work fetch for lanes without a pixel.  Background pixels are
        // written right away (GeneratePaths::writeBackground).
        for (;;) {
            const bool need = state == LS_FETCH;
            const uint32_t mask = __ballot_sync(0xffffffffu, need);
            if (mask == 0) break;
            const int leader = __ffs(mask) - 1;
            uint32_t base = 0;
            if (int(lane) == leader) base = atomicAdd(p.workCounter, uint32_t(__popc(mask)));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (!need) continue;
            idx = base + uint32_t(__popc(mask & laneMaskLt));
            if (idx >= p.workItems) { state = LS_DONE; continue; }
            x = idx % p.width;
            y = idx / p.width;
            float tMin, tMax;
            primaryDir = camera_ray_dir(s.camera, x, y, p.width, p.height, tMin, tMax);
            color = f3(0.f);
            rays = 0;
            sampleIdx = 0;
            if (unpack_hit(s.bits, __ldg(p.vbuffer + idx), primary)) {
                state = LS_SHADE;  // primary hit of sample 0
                path.sg.init(x, y, p.seed * spp);
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
                path.shadowPending = false;
            } else {
                const float3 bg = s.hasEnv ? env_eval(s, primaryDir) : f3(0.f);
                if (s.hasEnv) cnt.v[9]++;
                float3 c = f3(0.f);
                for (uint32_t i = 0; i < spp; i++) {
                    if (p.sampleColor) {
                        float* o = p.sampleColor + (size_t(idx) * spp + i) * 3;
                        o[0] = bg.x; o[1] = bg.y; o[2] = bg.z;
                    }
                    c += (spp != 1 && p.colorFormat == 1) ? decode_logluv_hdr(encode_logluv_hdr(bg)) : bg;
                }
                const float3 out = spp == 1 ? c : c * (1.f / float(spp));
                p.color[idx] = make_float4(out.x, out.y, out.z, 1.f);
                if (p.rayCount) p.rayCount[idx] = 0;
                // stays LS_FETCH
            }
        }
        if (__all_sync(0xffffffffu, state == LS_DONE)) break;

        // (2) Traversal: the pending visibility ray, else the extension ray.
        if (state == LS_TRACE) {
            const bool shadow = path.shadowPending;
            HitRec h;
            TraceStats ts;
            if (shadow) trace_bvh<true>(s, path.sOrigin, path.sDir, 0.f, path.sDist, h, stack, kPathBlock, &ts);
            else trace_bvh<false>(s, path.origin, path.dir, 0.f, 1e30f, h, stack, kPathBlock, &ts);
            cnt.trace(shadow, ts);
            rays++;
            if (shadow) {
                path.shadowPending = false;
                if (!h.valid) path.L += path.sLr;
                // The extension ray is traced on the next iteration (if the path continues).
            } else {
                path.vertexIndex++;
                if (h.valid) { path.hit = h; state = LS_SHADE; }
                else state = LS_MISS;
            }
        }

        // (3) Shading: handleHit / handleMiss.
        if (p.hitTrace && (state == LS_SHADE || state == LS_MISS))
            record_vertex(p, spp, p.maxSurfaceBounces + 2, idx, sampleIdx, path.vertexIndex, state == LS_SHADE, path.hit);
        if (state == LS_SHADE) pt_handle_hit<SG, HAS_T>(s, p, path, cnt);
        else if (state == LS_MISS) pt_handle_miss<SG>(s, p, path, cnt);
        if (state == LS_SHADE || state == LS_MISS || state == LS_TRACE) {
            if (path.has(PF_ACTIVE) || path.shadowPending) {
                state = LS_TRACE;
            } else {
                // Sample finished (writeOutput + ResolvePass accumulation).
                cnt.v[0]++;
                const float3 L = path.L;
                if (p.sampleColor) {
                    float* o = p.sampleColor + (size_t(idx) * spp + sampleIdx) * 3;
                    o[0] = L.x; o[1] = L.y; o[2] = L.z;
                }
                color += (spp != 1 && p.colorFormat == 1) ? decode_logluv_hdr(encode_logluv_hdr(L)) : L;
                sampleIdx++;
                if (sampleIdx < spp) {
                    path.sg.init(x, y, p.seed * spp + sampleIdx);
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
                    path.shadowPending = false;
                    state = LS_SHADE;
                    // The primary hit of the next sample is shaded on the next iteration.
                    continue;
                }
                // ResolvePass (ResolvePass.cs.slang:80-101); 1 spp writes the colour directly.
                const float3 out = spp == 1 ? color : color * (1.f / float(spp));
                if (!isfinite(out.x) || !isfinite(out.y) || !isfinite(out.z)) atomicOr(s.errorWord, FPT_DEVERR_NAN);
                p.color[idx] = make_float4(out.x, out.y, out.z, 1.f);
                if (p.rayCount) p.rayCount[idx] = rays;
                state = LS_FETCH;
            }
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
    const bool uniform = p.sampleGenerator == 1;
    if (s.hasTransmission) {
        if (uniform) path_tracer_kernel<UniformSG, true><<<blocks, kPathBlock, 0, st>>>(s, p);
        else path_tracer_kernel<TinyUniformSG, true><<<blocks, kPathBlock, 0, st>>>(s, p);
    } else {
        if (uniform) path_tracer_kernel<UniformSG, false><<<blocks, kPathBlock, 0, st>>>(s, p);
        else path_tracer_kernel<TinyUniformSG, false><<<blocks, kPathBlock, 0, st>>>(s, p);
    }
    return cudaGetLastError();
}

}  // namespace fpt
