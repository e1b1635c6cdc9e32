// wavefront.cu -- wavefront PathTracer for sm_100a.
//
// The frame's (pixel, sample) paths are processed in waves of up to
// `capacity` paths whose state lives in structure-of-arrays buffers.  Each
// bounce runs three small kernels over compacted queues of path indices:
//   shade   handleHit / handleMiss (PathTracer.slang:821-1157): emission with
//           MIS, NEE light sample, BSDF sample; pushes the visibility ray to
//           the shadow queue and the continuing path to the extension queue
//   shadow  any-hit traversal of the NEE rays; adds thp * Lr when visible
//   extend  closest-hit traversal of the continuing paths
// Queue pushes are warp-aggregated (ballot + one atomic per warp), so every
// kernel runs on dense, converged warps.  A resolve kernel sums the samples
// of each pixel in sample order with the per-sample colour format
// (ResolvePass.cs.slang:80-101), and a generate kernel seeds the wave
// (PathTracer.slang:273-301, GeneratePaths.cs.slang:93-256).
#include <algorithm>

#include "kernels.cuh"
#include "path_logic.cuh"
#include "wavefront.h"

namespace fpt {

using namespace dev;

namespace {

constexpr int kTraceBlock = 128;
constexpr int kShadeBlock = 128;

// Counts: [0] shade queue, [1] extension queue, [2] shadow queue, [4] and [5]
// the fetch counters of the extension and visibility ray kernels.
constexpr int kFetchExtend = 4, kFetchShadow = 5, kNumWaveCounts = 8;
struct WaveParams {
    uint32_t waveFirstPixel;   // first pixel of the wave
    uint32_t wavePixels;       // pixels in the wave
    uint32_t wavePaths;        // wavePixels * spp
    uint32_t* counts;
    const uint32_t* shadeQueue;
    uint32_t* extQueue;
    uint32_t* shadowQueue;
};

struct SoA {
    float4* originPdf;    // origin.xyz, pdf
    float4* dirV;         // dir.xyz, flags | vertexIndex << 16 (bits)
    float4* thpB;         // thp.xyz, bounce counters (bits)
    float4* L;            // L.xyz, -
    uint4* sg;            // sample generator state
    uint4* hit;           // instanceID, primIndex, baryX, baryY
    float4* sOrigin;      // shadow origin, distance
    float4* sDir;         // shadow direction, -
    float4* sLr;          // shadow contribution thp * Lr
    float* sampleL;       // per-path radiance (3 floats), wave slot order
};

template <class SG> FPT_D void store_sg(uint4& o, const SG& g);
template <class SG> FPT_D void load_sg(const uint4& i, SG& g);
template <> FPT_D void store_sg<TinyUniformSG>(uint4& o, const TinyUniformSG& g) { o = make_uint4(g.state, 0, 0, 0); }
template <> FPT_D void load_sg<TinyUniformSG>(const uint4& i, TinyUniformSG& g) { g.state = i.x; }
template <> FPT_D void store_sg<UniformSG>(uint4& o, const UniformSG& g) { o = make_uint4(g.s0, g.s1, g.s2, g.s3); }
template <> FPT_D void load_sg<UniformSG>(const uint4& i, UniformSG& g) { g.s0 = i.x; g.s1 = i.y; g.s2 = i.z; g.s3 = i.w; }

template <class SG>
FPT_D void load_path(const SoA& w, uint32_t i, PathState<SG>& path) {
    const float4 a = w.originPdf[i], b = w.dirV[i], c = w.thpB[i], d = w.L[i];
    path.origin = make_float3(a.x, a.y, a.z);
    path.pdf = a.w;
    path.dir = make_float3(b.x, b.y, b.z);
    const uint32_t fv = __float_as_uint(b.w);
    path.flags = fv & 0xffffu;
    path.vertexIndex = fv >> 16;
    path.thp = make_float3(c.x, c.y, c.z);
    path.bounces = __float_as_uint(c.w);
    path.L = make_float3(d.x, d.y, d.z);
    load_sg(w.sg[i], path.sg);
    const uint4 h = w.hit[i];
    path.hit.instanceID = h.x;
    path.hit.primIndex = h.y;
    path.hit.baryX = __uint_as_float(h.z);
    path.hit.baryY = __uint_as_float(h.w);
    path.hit.valid = true;
    path.normal = f3(0.f);
    path.shadowPending = false;
}

template <class SG>
FPT_D void store_path(const SoA& w, uint32_t i, const PathState<SG>& path) {
    w.originPdf[i] = make_float4(path.origin.x, path.origin.y, path.origin.z, path.pdf);
    w.dirV[i] = make_float4(path.dir.x, path.dir.y, path.dir.z, __uint_as_float((path.flags & 0xffffu) | (path.vertexIndex << 16)));
    w.thpB[i] = make_float4(path.thp.x, path.thp.y, path.thp.z, __uint_as_float(path.bounces));
    w.L[i] = make_float4(path.L.x, path.L.y, path.L.z, 0.f);
    store_sg(w.sg[i], path.sg);
}

// Warp-aggregated push of `item` onto queue q (count at *cnt).
FPT_D void push(bool pred, uint32_t item, uint32_t* q, uint32_t* cnt) {
    const uint32_t mask = __ballot_sync(__activemask(), pred);
    if (mask == 0) return;
    const uint32_t lane = threadIdx.x & 31u;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (int(lane) == leader) base = atomicAdd(cnt, uint32_t(__popc(mask)));
    base = __shfl_sync(__activemask(), base, leader);
    if (pred) q[base + uint32_t(__popc(mask & ((1u << lane) - 1u)))] = item;
}

// Seeds a wave: slot i <-> (pixel waveFirstPixel + i % wavePixels, sample i / wavePixels).
// Background pixels write their samples directly; hit pixels enter the shade queue.
template <class SG>
__global__ void __launch_bounds__(kShadeBlock) wf_generate(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    Counters cnt;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i - threadIdx.x < wp.wavePaths; i += gridDim.x * blockDim.x) {
        bool enqueue = false;
        if (i < wp.wavePaths) {
            const uint32_t pixIn = i % wp.wavePixels, sample = i / wp.wavePixels;
            const uint32_t pix = wp.waveFirstPixel + pixIn;
            const uint32_t x = pix % p.width, y = pix / p.width;
            float tMin, tMax;
            const float3 dir = camera_ray_dir(s.camera, x, y, p.width, p.height, tMin, tMax);
            HitRec hit;
            if (unpack_hit(s.bits, __ldg(p.vbuffer + pix), hit)) {
                PathState<SG> path;
                path.sg.init(x, y, p.seed * p.spp + sample);
                path.flags = PF_ACTIVE | 0x2u;  // active, hit (primary hit from the V-buffer)
                path.vertexIndex = 1;
                path.bounces = 0;
                path.thp = f3(1.f);
                path.L = f3(0.f);
                path.pdf = 0.f;
                path.origin = load3(s.camera.posW);
                path.dir = dir;
                store_path(w, i, path);
                w.hit[i] = make_uint4(hit.instanceID, hit.primIndex, __float_as_uint(hit.baryX), __float_as_uint(hit.baryY));
                enqueue = true;
            } else {
                const float3 bg = s.hasEnv ? env_eval(s, dir) : f3(0.f);
                if (s.hasEnv) cnt.v[9]++;
                float* o = w.sampleL + size_t(i) * 3;
                o[0] = bg.x; o[1] = bg.y; o[2] = bg.z;
            }
        }
        push(enqueue, i, const_cast<uint32_t*>(wp.shadeQueue), wp.counts + 0);
    }
    flush_counters(p.counters, cnt);
}

// handleHit / handleMiss for every path of the shade queue.  The hit flag of
// a path is PF_HIT (0x2) in its flags.
template <class SG, bool HAS_T>
__global__ void __launch_bounds__(kShadeBlock) wf_shade(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    Counters cnt;
    const uint32_t n = wp.counts[0];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k - threadIdx.x < n; k += gridDim.x * blockDim.x) {
        bool ext = false, shadow = false;
        uint32_t i = 0;
        if (k < n) {
            i = wp.shadeQueue[k];
            PathState<SG> path;
            load_path(w, i, path);
            if (path.flags & 0x2u) pt_handle_hit<SG, HAS_T>(s, p, path, cnt);
            else pt_handle_miss<SG>(s, p, path, cnt);
            shadow = path.shadowPending;
            if (shadow) {
                w.sOrigin[i] = make_float4(path.sOrigin.x, path.sOrigin.y, path.sOrigin.z, path.sDist);
                w.sDir[i] = make_float4(path.sDir.x, path.sDir.y, path.sDir.z, 0.f);
                w.sLr[i] = make_float4(path.sLr.x, path.sLr.y, path.sLr.z, 0.f);
            }
            ext = path.has(PF_ACTIVE);
            store_path(w, i, path);
            if (!ext) cnt.v[0]++;
        }
        push(shadow, i, wp.shadowQueue, wp.counts + 2);
        push(ext, i, wp.extQueue, wp.counts + 1);
    }
    flush_counters(p.counters, cnt);
}

// Visibility rays: L += thp * Lr when unoccluded.
// Ray tracing kernels (visibility and extension rays) with per-lane dynamic
// ray fetch: each warp takes chunks of kFetchChunk queue entries with one
// atomic and hands them to its idle lanes, and a lane whose ray has finished
// takes the next one as soon as fewer than kRefillBelow lanes of its warp are
// still tracing.  The traversal itself advances one node visit per step, so
// rays of very different lengths share a warp without leaving most of its
// lanes idle until the longest ray is done.
#ifndef FPT_REFILL_BELOW
#define FPT_REFILL_BELOW 24
#endif
#ifndef FPT_TRACE_MIN_BLOCKS
#define FPT_TRACE_MIN_BLOCKS 6
#endif
constexpr uint32_t kFetchChunk = 128;
constexpr int kRefillBelow = FPT_REFILL_BELOW;

template <bool SHADOW>
FPT_D void trace_queue(const DevScene& s, const FrameParams& p, const WaveParams& wp, const SoA& w, uint2* stack) {
    const uint32_t lane = threadIdx.x & 31u;
    Counters cnt;
    const uint32_t n = wp.counts[SHADOW ? 2 : 1];
    uint32_t* fetch = wp.counts + (SHADOW ? kFetchShadow : kFetchExtend);
    const uint32_t* queue = SHADOW ? wp.shadowQueue : wp.extQueue;
    const int postponeLimit = kStackSize - int(s.bvhDepth);
    uint32_t chunkNext = 0, chunkEnd = 0;  // warp-uniform
    bool drained = n == 0 || s.nodeCount == 0;
    bool active = false;
    uint32_t path = 0, fv = 0;
    TraceRay r;
    TraceState t;
    for (;;) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !active);
        if (idle && !drained) {
            if (chunkNext >= chunkEnd) {
                uint32_t base = 0;
                if (lane == 0) base = atomicAdd(fetch, kFetchChunk);
                base = __shfl_sync(0xffffffffu, base, 0);
                if (base >= n) drained = true;
                else { chunkNext = base; chunkEnd = min(base + kFetchChunk, n); }
            }
            if (!drained) {
                const uint32_t avail = chunkEnd - chunkNext;
                const uint32_t rank = __popc(idle & ((1u << lane) - 1u));
                if (!active && rank < avail) {
                    path = queue[chunkNext + rank];
                    float4 o, d;
                    if (SHADOW) { o = w.sOrigin[path]; d = w.sDir[path]; }
                    else { o = w.originPdf[path]; d = w.dirV[path]; }
                    fv = __float_as_uint(d.w);
                    r = make_trace_ray(make_float3(o.x, o.y, o.z), make_float3(d.x, d.y, d.z), 0.f);
                    trace_init(r, SHADOW ? o.w : 1e30f, t);
                    active = true;
                }
                chunkNext += min(avail, uint32_t(__popc(idle)));
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0) break;
        for (;;) {
            if (active) {
                trace_step<SHADOW>(s, r, t, stack, kTraceBlock, postponeLimit);
                if (t.status != kTraceRunning) {
                    active = false;
                    cnt.v[1]++;
                    cnt.v[SHADOW ? 3 : 2]++;
                    cnt.v[4] += t.visits;
                    cnt.v[5] += t.triTests;
                    if (SHADOW) { cnt.v[11] += t.visits; cnt.v[12] += t.triTests; }
                    HitRec h;
                    trace_result(t, h);
                    if (SHADOW) {
                        if (!h.valid && t.status != kTraceError) {
                            const float4 lr = w.sLr[path];
                            float4 L = w.L[path];
                            L.x += lr.x; L.y += lr.y; L.z += lr.z;
                            w.L[path] = L;
                        }
                    } else {
                        uint32_t f = fv + (1u << 16);  // vertexIndex++
                        if (h.valid) {
                            f |= 0x2u;
                            w.hit[path] = make_uint4(h.instanceID, h.primIndex, __float_as_uint(h.baryX), __float_as_uint(h.baryY));
                        } else {
                            f &= ~0x2u;
                        }
                        float4 d = w.dirV[path];
                        d.w = __uint_as_float(f);
                        w.dirV[path] = d;
                    }
                }
            }
            const uint32_t a = __ballot_sync(0xffffffffu, active);
            if (a == 0) break;
            if (!drained && __popc(a) < kRefillBelow) break;
        }
    }
    flush_counters(p.counters, cnt);
}

// Visibility rays of the NEE samples: any hit; adds thp * Lr when unoccluded.
__global__ void __launch_bounds__(kTraceBlock, FPT_TRACE_MIN_BLOCKS) wf_shadow(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    __shared__ uint2 stackMem[kStackSize * kTraceBlock];
    trace_queue<true>(s, p, wp, w, stackMem + threadIdx.x);
}

// Extension rays: closest hit; the path re-enters the shade queue.
__global__ void __launch_bounds__(kTraceBlock, FPT_TRACE_MIN_BLOCKS) wf_extend(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    __shared__ uint2 stackMem[kStackSize * kTraceBlock];
    trace_queue<false>(s, p, wp, w, stackMem + threadIdx.x);
}

// Finished paths keep their radiance in L; copy it into the per-sample buffer.
__global__ void wf_collect(FrameParams p, WaveParams wp, SoA w, const uint32_t* hitPixelFlags) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < wp.wavePaths; i += gridDim.x * blockDim.x) {
        const uint32_t pix = wp.waveFirstPixel + i % wp.wavePixels;
        if (!(__ldg(p.vbuffer + pix).x)) continue;  // background: written by wf_generate
        const float4 L = w.L[i];
        float* o = w.sampleL + size_t(i) * 3;
        o[0] = L.x; o[1] = L.y; o[2] = L.z;
    }
}

// ResolvePass: per-pixel average of the per-sample colours in sample order.
__global__ void wf_resolve(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < wp.wavePixels; j += gridDim.x * blockDim.x) {
        const uint32_t pix = wp.waveFirstPixel + j;
        float3 c = f3(0.f);
        for (uint32_t smp = 0; smp < p.spp; smp++) {
            const float* q = w.sampleL + (size_t(smp) * wp.wavePixels + j) * 3;
            const float3 L = make_float3(q[0], q[1], q[2]);
            if (p.sampleColor) {
                float* o = p.sampleColor + (size_t(pix) * p.spp + smp) * 3;
                o[0] = L.x; o[1] = L.y; o[2] = L.z;
            }
            c += (p.spp != 1 && p.colorFormat == 1) ? decode_logluv_hdr(encode_logluv_hdr(L)) : L;
        }
        const float3 out = p.spp == 1 ? c : c * (1.f / float(p.spp));
        if (!isfinite(out.x) || !isfinite(out.y) || !isfinite(out.z)) atomicOr(s.errorWord, FPT_DEVERR_NAN);
        p.color[pix] = make_float4(out.x, out.y, out.z, 1.f);
    }
}

// Moves the extension queue into the shade queue for the next bounce.
__global__ void wf_advance(WaveParams wp) {
    wp.counts[0] = wp.counts[1];
    wp.counts[1] = 0;
    wp.counts[2] = 0;
    wp.counts[kFetchExtend] = 0;
    wp.counts[kFetchShadow] = 0;
}

int blocks_for(const void* kernel, int block) {
    int perSM = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, block, 0);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, perSM) * sms;
}

template <class SG, bool HAS_T>
cudaError_t run_wavefront(const DevScene& s, const FrameParams& p, WavefrontBuffers& b, cudaStream_t st, KernelTimer* kt) {
    auto T0 = [&](int cat) { if (kt && kt->enabled) kt->begin(cat, st); };
    auto T1 = [&]() { if (kt && kt->enabled) kt->end(st); };
    SoA w;
    w.originPdf = b.f4(0); w.dirV = b.f4(1); w.thpB = b.f4(2); w.L = b.f4(3);
    w.sg = reinterpret_cast<uint4*>(b.f4(4)); w.hit = reinterpret_cast<uint4*>(b.f4(5));
    w.sOrigin = b.f4(6); w.sDir = b.f4(7); w.sLr = b.f4(8);
    w.sampleL = b.sampleL;
    const uint32_t pixels = p.width * p.height;
    const uint32_t wavePixels = std::max<uint32_t>(1, std::min<uint32_t>(pixels, b.capacity / p.spp));
    static int gShade = 0, gTrace = 0, gGen = 0;
    if (!gShade) {
        gShade = blocks_for(reinterpret_cast<const void*>(wf_shade<SG, HAS_T>), kShadeBlock);
        gTrace = blocks_for(reinterpret_cast<const void*>(wf_extend), kTraceBlock);
        gGen = blocks_for(reinterpret_cast<const void*>(wf_generate<SG>), kShadeBlock);
    }
    const uint32_t maxIter = p.maxSurfaceBounces + 2;
    for (uint32_t first = 0; first < pixels; first += wavePixels) {
        WaveParams wp;
        wp.waveFirstPixel = first;
        wp.wavePixels = std::min(wavePixels, pixels - first);
        wp.wavePaths = wp.wavePixels * p.spp;
        wp.counts = b.counts;
        cudaError_t e = cudaMemsetAsync(b.counts, 0, kNumWaveCounts * sizeof(uint32_t), st);
        if (e != cudaSuccess) return e;
        uint32_t* qa = b.queueA;
        uint32_t* qb = b.queueB;
        wp.shadeQueue = qa;
        wp.extQueue = qb;
        wp.shadowQueue = b.shadowQueue;
        const int genBlocks = std::min<int>(gGen, int((wp.wavePaths + kShadeBlock - 1) / kShadeBlock));
        T0(KC_GENERATE);
        wf_generate<SG><<<genBlocks, kShadeBlock, 0, st>>>(s, p, wp, w);
        T1();
        for (uint32_t it = 0; it < maxIter; it++) {
            T0(KC_SHADE);
            wf_shade<SG, HAS_T><<<gShade, kShadeBlock, 0, st>>>(s, p, wp, w);
            T1();
            T0(KC_SHADOW);
            wf_shadow<<<gTrace, kTraceBlock, 0, st>>>(s, p, wp, w);
            T1();
            T0(KC_EXTEND);
            wf_extend<<<gTrace, kTraceBlock, 0, st>>>(s, p, wp, w);
            T1();
            wf_advance<<<1, 1, 0, st>>>(wp);
            std::swap(qa, qb);
            wp.shadeQueue = qa;
            wp.extQueue = qb;
        }
        T0(KC_RESOLVE);
        wf_collect<<<gGen, 256, 0, st>>>(p, wp, w, nullptr);
        wf_resolve<<<(wp.wavePixels + 255) / 256, 256, 0, st>>>(s, p, wp, w);
        T1();
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

cudaError_t WavefrontBuffers::ensure(uint32_t cap) {
    if (capacity >= cap && base) return cudaSuccess;
    release();
    const size_t f4Bytes = size_t(cap) * sizeof(float4);
    const size_t bytes = kFloat4Arrays * f4Bytes + size_t(cap) * 3 * sizeof(float) + 3 * size_t(cap) * sizeof(uint32_t) + 256;
    cudaError_t e = cudaMalloc(&base, bytes);
    if (e != cudaSuccess) { base = nullptr; return e; }
    capacity = cap;
    char* q = static_cast<char*>(base);
    arrays = reinterpret_cast<float4*>(q);
    q += kFloat4Arrays * f4Bytes;
    sampleL = reinterpret_cast<float*>(q);
    q += size_t(cap) * 3 * sizeof(float);
    queueA = reinterpret_cast<uint32_t*>(q);
    q += size_t(cap) * sizeof(uint32_t);
    queueB = reinterpret_cast<uint32_t*>(q);
    q += size_t(cap) * sizeof(uint32_t);
    shadowQueue = reinterpret_cast<uint32_t*>(q);
    q += size_t(cap) * sizeof(uint32_t);
    counts = reinterpret_cast<uint32_t*>(q);
    bytesAllocated = bytes;
    return cudaSuccess;
}

void WavefrontBuffers::release() {
    if (base) cudaFree(base);
    base = nullptr;
    capacity = 0;
}

size_t WavefrontBuffers::bytes_for(uint32_t cap) {
    return kFloat4Arrays * size_t(cap) * sizeof(float4) + size_t(cap) * 3 * sizeof(float) + 3 * size_t(cap) * sizeof(uint32_t) + 256;
}

void WavefrontBuffers::view(void* mem, uint32_t cap) {
    // Same layout as ensure(), over memory that the caller owns.
    owning = false;
    base = mem;
    capacity = cap;
    char* q = static_cast<char*>(mem);
    arrays = reinterpret_cast<float4*>(q);
    q += kFloat4Arrays * size_t(cap) * sizeof(float4);
    sampleL = reinterpret_cast<float*>(q);
    q += size_t(cap) * 3 * sizeof(float);
    queueA = reinterpret_cast<uint32_t*>(q);
    q += size_t(cap) * sizeof(uint32_t);
    queueB = reinterpret_cast<uint32_t*>(q);
    q += size_t(cap) * sizeof(uint32_t);
    shadowQueue = reinterpret_cast<uint32_t*>(q);
    q += size_t(cap) * sizeof(uint32_t);
    counts = reinterpret_cast<uint32_t*>(q);
    bytesAllocated = bytes_for(cap);
}

cudaError_t launch_path_tracer_wavefront(const DevScene& s, const FrameParams& p, WavefrontBuffers& b, cudaStream_t st,
                                         KernelTimer* kt) {
    const bool uniform = p.sampleGenerator == 1;
    if (s.hasTransmission)
        return uniform ? run_wavefront<UniformSG, true>(s, p, b, st, kt) : run_wavefront<TinyUniformSG, true>(s, p, b, st, kt);
    return uniform ? run_wavefront<UniformSG, false>(s, p, b, st, kt) : run_wavefront<TinyUniformSG, false>(s, p, b, st, kt);
}

void KernelTimer::begin(int cat, cudaStream_t st) {
    if (used + 2 > events.size()) {
        const size_t grow = std::max<size_t>(64, events.size());
        for (size_t i = 0; i < grow; i++) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) { enabled = false; return; }
            events.push_back(e);
        }
    }
    pendingCat.push_back(cat);
    cudaEventRecord(events[used], st);
}

void KernelTimer::end(cudaStream_t st) {
    if (!enabled || pendingCat.empty() || used + 1 >= events.size()) return;
    cudaEventRecord(events[used + 1], st);
    used += 2;
}

cudaError_t KernelTimer::collect() {
    const size_t pairs = std::min(used / 2, pendingCat.size());
    for (size_t k = 0; k < pairs; k++) {
        cudaError_t e = cudaEventSynchronize(events[k * 2 + 1]);
        if (e != cudaSuccess) return e;
        float t = 0.f;
        e = cudaEventElapsedTime(&t, events[k * 2], events[k * 2 + 1]);
        if (e != cudaSuccess) return e;
        ms[pendingCat[k]] += t;
        launches[pendingCat[k]] += 1;
    }
    used = 0;
    pendingCat.clear();
    return cudaSuccess;
}

void KernelTimer::reset() {
    used = 0;
    pendingCat.clear();
    for (int i = 0; i < KC_COUNT; i++) { ms[i] = 0; launches[i] = 0; }
}

KernelTimer::~KernelTimer() {
    for (cudaEvent_t e : events) cudaEventDestroy(e);
}

}  // namespace fpt
