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
#include <cstring>

#include "kernels.cuh"
#include "path_logic.cuh"
#include "wavefront.h"
// The PathTracer's generate and shade kernels run 1024-thread blocks, one per
// SM (the adjoint's kernels keep the 128 of wavefront_common.cuh).  Every
// queue push of a launch is an atomic on the same counter word, which the L2
// serialises; one push per block per grid-stride iteration makes bigger blocks
// cheaper.  Measured on the 1080p heightfield frame (shading ms per 16-spp
// frame): 15.97 with 64-thread blocks, 15.07 with 128, 14.62 with 256, 13.43
// with 512, 12.69 with 1024 (generate 0.72 -> 0.79 ms from 512 to 1024).
#ifndef FPT_SHADE_BLOCK
#define FPT_SHADE_BLOCK 1024
#endif
#include "wavefront_common.cuh"

namespace fpt {

using namespace dev;

namespace {

// Seeds one slot: (pixel pix, sample) of a frame.  Background pixels write
// their samples directly; returns true for hit pixels (shade queue).
template <class SG>
FPT_D bool generate_slot(const DevScene& s, const FrameParams& p, const SoA& w, uint32_t i, uint32_t pix, uint32_t sample,
                         Counters& cnt) {
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
        return true;
    }
    const float3 bg = s.hasEnv ? env_eval(s, dir) : f3(0.f);
    if (s.hasEnv) cnt.v[9]++;
    float* o = w.sampleL + size_t(i) * 3;
    o[0] = bg.x; o[1] = bg.y; o[2] = bg.z;
    return false;
}

// Tile of slot (or resolved pixel) `x` of a batched wave: the last tile whose
// offset is <= x (tiles are in slot order).
template <bool PIXELS>
FPT_D uint32_t find_tile(const WaveParams& wp, uint32_t x) {
    uint32_t lo = 0, hi = wp.tileCount;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t off = PIXELS ? wp.tiles[mid].pixelOffset : wp.tiles[mid].slotOffset;
        if (off <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Seeds a wave.  Single frame: slot i <-> (pixel waveFirstPixel + i % wavePixels,
// sample i / wavePixels).  Batched (MULTI): slot i of tile t <-> (pixel
// firstPixel + j % numPixels, sample j / numPixels), j = i - slotOffset.
// FPT_BLOCK_PUSH: 1 = the generate kernel pushes the shade queue with one
// atomic per block, 2 = the shade kernel its two queues too; 0 = one atomic
// per warp everywhere.  On the 1080p heightfield frame 2 measured 940.6
// Mpaths/s against 906.6 with 0 (shading 15.55 -> 15.05 ms per frame).
#ifndef FPT_BLOCK_PUSH
#define FPT_BLOCK_PUSH 2
#endif
template <class SG, bool MULTI>
__global__ void __launch_bounds__(kShadeBlock) wf_generate(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    Counters cnt;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i - threadIdx.x < wp.wavePaths; i += gridDim.x * blockDim.x) {
        bool enqueue = false;
        if (i < wp.wavePaths) {
            if (MULTI) {
                const uint32_t t = find_tile<false>(wp, i);
                wp.slotTile[i] = t;
                const BatchTile tile = wp.tiles[t];
                const uint32_t j = i - tile.slotOffset;
                enqueue = generate_slot<SG>(wp.scenes[tile.req], wp.frames[tile.req], w, i, tile.firstPixel + j % tile.numPixels,
                                            j / tile.numPixels, cnt);
            } else {
                enqueue = generate_slot<SG>(s, p, w, i, wp.waveFirstPixel + i % wp.wavePixels, i / wp.wavePixels, cnt);
            }
        }
#if FPT_BLOCK_PUSH
        __shared__ uint32_t pushWords[2 * (kShadeBlock / 32 + 1)];
        uint32_t pa, pb;
        block_push2<kShadeBlock / 32>(enqueue, i, const_cast<uint32_t*>(wp.shadeQueue), wp.counts + 0, false, 0u, nullptr, nullptr,
                                      pushWords, pa, pb);
#else
        push(enqueue, i, const_cast<uint32_t*>(wp.shadeQueue), wp.counts + 0);
#endif
    }
    flush_counters(p.counters, cnt);
}

template <class SG, bool HAS_T, bool TEX = true>
FPT_D void shade_slot(const DevScene& s, const FrameParams& p, const SoA& w, uint32_t i, bool& ext, bool& shadow, Counters& cnt,
                      const WaveParams* wp = nullptr, uint32_t* binKey = nullptr, uint32_t* shadowKey = nullptr) {
    PathState<SG> path;
    load_path(w, i, path);
    if (wp && p.hitTrace)
        record_vertex(p, p.spp, p.maxSurfaceBounces + 2, wp->waveFirstPixel + i % wp->wavePixels, i / wp->wavePixels, path.vertexIndex,
                      (path.flags & 0x2u) != 0, path.hit);
    if (path.flags & 0x2u) pt_handle_hit<SG, HAS_T, TEX>(s, p, path, cnt);
    else pt_handle_miss<SG>(s, p, path, cnt);
    shadow = path.shadowPending;
    if (shadow) {
        if (shadowKey) *shadowKey = ray_bin_key(s, path.sOrigin, path.sDir);
        w.sOrigin[i] = make_float4(path.sOrigin.x, path.sOrigin.y, path.sOrigin.z, path.sDist);
        w.sDir[i] = make_float4(path.sDir.x, path.sDir.y, path.sDir.z, 0.f);
        w.sLr[i] = make_float4(path.sLr.x, path.sLr.y, path.sLr.z, 0.f);
    }
    ext = path.has(PF_ACTIVE);
    if (binKey && ext) *binKey = ray_bin_key(s, path.origin, path.dir);
    // A finished path is read again only for its radiance (its visibility ray
    // and the collect kernel), so only L is written back.
    if (ext) store_path(w, i, path);
    else w.L[i] = make_float4(path.L.x, path.L.y, path.L.z, 0.f);
    if (!ext) cnt.v[0]++;
}

// handleHit / handleMiss for every path of the shade queue.  The hit flag of
// a path is PF_HIT (0x2) in its flags.
#ifndef FPT_SHADE_MIN_BLOCKS
// 1024 resident threads per SM (64 registers, spills to L1) measured best on
// the 1080p heightfield frame with the sampler-specialised kernel, as 128-thread
// blocks: shading 18.77 ms per frame at 6 blocks (80 registers), 17.88 at 7,
// 17.68 at 8, 19.51 at 5; after later shading changes 14.94 at 7, 15.05 at 8.
#define FPT_SHADE_MIN_BLOCKS (1024 / FPT_SHADE_BLOCK)
#endif
// ES >= 0: the emissive sampler (0 Uniform, 1 LightBVH, 2 Power) fixed at
// compile time, so that the code of the other two samplers is not in the
// kernel (a smaller kernel stalls less on instruction fetch); -1: read from
// the frame parameters.
#ifndef FPT_SPECIALIZE_SAMPLER
#define FPT_SPECIALIZE_SAMPLER 1
#endif
template <class SG, bool HAS_T, bool MULTI, int ES = -1, bool TEX = true>
__global__ void __launch_bounds__(kShadeBlock, FPT_SHADE_MIN_BLOCKS) wf_shade(DevScene s, FrameParams pk, WaveParams wp, SoA w) {
    FrameParams p = pk;
    if (ES >= 0) p.emissiveSampler = uint32_t(ES);
    Counters cnt;
    const uint32_t n = wp.counts[0];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k - threadIdx.x < n; k += gridDim.x * blockDim.x) {
        bool ext = false, shadow = false;
        uint32_t i = 0, key = 0, skey = 0;
        if (k < n) {
            i = wp.shadeQueue[k];
            if (MULTI) {
                const uint32_t r = slot_request(wp, i);
                shade_slot<SG, HAS_T>(wp.scenes[r], wp.frames[r], w, i, ext, shadow, cnt);
            } else {
                shade_slot<SG, HAS_T, TEX>(s, p, w, i, ext, shadow, cnt, &wp, wp.extKeys ? &key : nullptr,
                                           wp.shadowKeys ? &skey : nullptr);
            }
        }
#if FPT_BLOCK_PUSH >= 2
        __shared__ uint32_t pushWords[2 * (kShadeBlock / 32 + 1)];
        uint32_t spos, pos;
        block_push2<kShadeBlock / 32>(shadow, i, wp.shadowQueue, wp.counts + 2, ext, i, wp.extQueue, wp.counts + 1, pushWords, spos, pos);
#else
        const uint32_t spos = push(shadow, i, wp.shadowQueue, wp.counts + 2);
        const uint32_t pos = push(ext, i, wp.extQueue, wp.counts + 1);
#endif
        if (!MULTI && wp.shadowKeys && spos != 0xffffffffu) wp.shadowKeys[spos] = skey;
        if (!MULTI && wp.extKeys && pos != 0xffffffffu) wp.extKeys[pos] = key;
    }
    flush_counters(p.counters, cnt);
}

// Visibility rays of the NEE samples: any hit; adds thp * Lr when unoccluded.
// Scenes whose tree is at most kShortStack levels deep trace with a stack of
// that many entries (half the shared memory per block).
#ifndef FPT_TRACE_MIN_BLOCKS_SHORT
#define FPT_TRACE_MIN_BLOCKS_SHORT 6
#endif
constexpr int kShortStack = 16;
// FPT_TOP_NODES: the trace kernels stage the BVH's top levels in shared memory
// (stage_top_nodes) and read them from there.
#ifndef FPT_TOP_NODES
#define FPT_TOP_NODES 0
#endif
template <int STACK>
__global__ void __launch_bounds__(kTraceBlock, STACK <= kShortStack ? FPT_TRACE_MIN_BLOCKS_SHORT : FPT_TRACE_MIN_BLOCKS)
    wf_shadow(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    __shared__ uint2 stackMem[STACK * kTraceBlock];
    __shared__ __align__(16) uint4 topMem[FPT_TOP_NODES ? kTopNodes * 5 : 1];
    __shared__ __align__(8) unsigned long long topBar;
    const uint32_t topCount = FPT_TOP_NODES ? stage_top_nodes(s, topMem, &topBar) : 0u;
    trace_queue<true, false, false, STACK>(s, p, wp, w, stackMem + threadIdx.x, topMem, topCount);
}

// Extension rays: closest hit; the path re-enters the shade queue.
template <int STACK>
__global__ void __launch_bounds__(kTraceBlock, STACK <= kShortStack ? FPT_TRACE_MIN_BLOCKS_SHORT : FPT_TRACE_MIN_BLOCKS)
    wf_extend(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    __shared__ uint2 stackMem[STACK * kTraceBlock];
    __shared__ __align__(16) uint4 topMem[FPT_TOP_NODES ? kTopNodes * 5 : 1];
    __shared__ __align__(8) unsigned long long topBar;
    const uint32_t topCount = FPT_TOP_NODES ? stage_top_nodes(s, topMem, &topBar) : 0u;
    trace_queue<false, false, false, STACK>(s, p, wp, w, stackMem + threadIdx.x, topMem, topCount);
}

// Batched waves: each ray traced in its own request's scene.
__global__ void __launch_bounds__(kTraceBlock, FPT_TRACE_MIN_BLOCKS) wf_shadow_batch(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    __shared__ uint2 stackMem[kStackSize * kTraceBlock];
    trace_queue<true, false, true>(s, p, wp, w, stackMem + threadIdx.x);
}
__global__ void __launch_bounds__(kTraceBlock, FPT_TRACE_MIN_BLOCKS) wf_extend_batch(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    __shared__ uint2 stackMem[kStackSize * kTraceBlock];
    trace_queue<false, false, true>(s, p, wp, w, stackMem + threadIdx.x);
}

// Finished paths keep their radiance in L; copy it into the per-sample buffer.
template <bool MULTI>
__global__ void wf_collect(FrameParams p, WaveParams wp, SoA w) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < wp.wavePaths; i += gridDim.x * blockDim.x) {
        if (MULTI) {
            const BatchTile tile = wp.tiles[wp.slotTile[i]];
            const uint32_t pix = tile.firstPixel + (i - tile.slotOffset) % tile.numPixels;
            if (!(__ldg(wp.frames[tile.req].vbuffer + pix).x)) continue;
        } else {
            const uint32_t pix = wp.waveFirstPixel + i % wp.wavePixels;
            if (!(__ldg(p.vbuffer + pix).x)) continue;  // background: written by wf_generate
        }
        const float4 L = w.L[i];
        float* o = w.sampleL + size_t(i) * 3;
        o[0] = L.x; o[1] = L.y; o[2] = L.z;
    }
}

// ResolvePass: per-pixel average of the per-sample colours in sample order.
FPT_D void resolve_pixel(const DevScene& s, const FrameParams& p, const SoA& w, uint32_t pix, uint32_t slot0, uint32_t stride) {
    float3 c = f3(0.f);
    for (uint32_t smp = 0; smp < p.spp; smp++) {
        const float* q = w.sampleL + (size_t(smp) * stride + slot0) * 3;
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

template <bool MULTI>
__global__ void wf_resolve(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < wp.wavePixels; j += gridDim.x * blockDim.x) {
        if (MULTI) {
            const BatchTile tile = wp.tiles[find_tile<true>(wp, j)];
            const uint32_t jt = j - tile.pixelOffset;
            // Slot of (pixel jt, sample smp) = slotOffset + smp * numPixels + jt.
            resolve_pixel(wp.scenes[tile.req], wp.frames[tile.req], w, tile.firstPixel + jt,
                          tile.slotOffset + jt - 0u, tile.numPixels);
        } else {
            resolve_pixel(s, p, w, wp.waveFirstPixel + j, j, wp.wavePixels);
        }
    }
}

// Counting sort of the shade queue by material (misses in the last bin), so
// that the warps of the shade kernel see one material -- and hits apart from
// misses -- instead of a random mix.  The keys were written by the extension
// kernel at the queue positions; sorting moves 12 B per path.
__global__ void wf_sort_count(WaveParams wp, uint32_t* bins) {
    __shared__ uint32_t h[WavefrontBuffers::kMaxSortBins];
    for (uint32_t b = threadIdx.x; b < wp.sortBins; b += blockDim.x) h[b] = 0;
    __syncthreads();
    const uint32_t n = wp.counts[0];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        atomicAdd(&h[min(wp.sortKeys[k], wp.sortBins - 1u)], 1u);
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < wp.sortBins; b += blockDim.x)
        if (h[b]) atomicAdd(&bins[b], h[b]);
}

// Exclusive prefix sum of the bin counts into the cursors (one block of
// kMaxSortBins threads).
__global__ void wf_sort_scan(WaveParams wp, uint32_t* bins) {
    __shared__ uint32_t v[WavefrontBuffers::kMaxSortBins];
    const uint32_t t = threadIdx.x;
    const uint32_t own = t < wp.sortBins ? bins[t] : 0u;
    v[t] = own;
    __syncthreads();
    for (uint32_t off = 1; off < blockDim.x; off <<= 1) {
        const uint32_t add = t >= off ? v[t - off] : 0u;
        __syncthreads();
        v[t] += add;
        __syncthreads();
    }
    if (t < wp.sortBins) bins[WavefrontBuffers::kMaxSortBins + t] = v[t] - own;
}

// Scatters queue entries to their bins (warp-aggregated per key).
__global__ void wf_sort_scatter(WaveParams wp, uint32_t* bins, uint32_t* out) {
    const uint32_t n = wp.counts[0];
    uint32_t* cursor = bins + WavefrontBuffers::kMaxSortBins;
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k - lane < n; k += gridDim.x * blockDim.x) {
        const bool valid = k < n;
        const uint32_t key = valid ? min(wp.sortKeys[k], wp.sortBins - 1u) : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        if (!valid) continue;
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (int(lane) == leader) base = atomicAdd(&cursor[key], uint32_t(__popc(peers)));
        base = __shfl_sync(peers, base, leader);
        out[base + uint32_t(__popc(peers & ((1u << lane) - 1u)))] = wp.shadeQueue[k];
    }
}

// Counting sort of the extension queue by ray bin (coherence of the next
// traversal): histogram, scan (wf_sort_scan over nBins), scatter.
__global__ void wf_bin_count(const uint32_t* keys, const uint32_t* count, uint32_t nBins, uint32_t* bins) {
    __shared__ uint32_t h[WavefrontBuffers::kMaxSortBins];
    for (uint32_t b = threadIdx.x; b < nBins; b += blockDim.x) h[b] = 0;
    __syncthreads();
    const uint32_t n = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x)
        atomicAdd(&h[min(keys[k], nBins - 1u)], 1u);
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < nBins; b += blockDim.x)
        if (h[b]) atomicAdd(&bins[b], h[b]);
}
__global__ void wf_bin_scatter(const uint32_t* keys, const uint32_t* in, const uint32_t* count, uint32_t nBins, uint32_t* bins,
                               uint32_t* out) {
    const uint32_t n = *count;
    uint32_t* cursor = bins + WavefrontBuffers::kMaxSortBins;
    const uint32_t lane = threadIdx.x & 31u;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k - lane < n; k += gridDim.x * blockDim.x) {
        const bool valid = k < n;
        const uint32_t key = valid ? min(keys[k], nBins - 1u) : 0xffffffffu;
        const uint32_t peers = __match_any_sync(0xffffffffu, key);
        if (!valid) continue;
        const int leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (int(lane) == leader) base = atomicAdd(&cursor[key], uint32_t(__popc(peers)));
        base = __shfl_sync(peers, base, leader);
        out[base + uint32_t(__popc(peers & ((1u << lane) - 1u)))] = in[k];
    }
}

// handleMiss for the paths of the miss queue (hit/miss split): the short
// environment-light branch of the shade stage, run apart so that the shade
// kernel's warps hold hits only.
template <class SG>
__global__ void __launch_bounds__(kShadeBlock) wf_miss(DevScene s, FrameParams p, WaveParams wp, SoA w) {
    Counters cnt;
    const uint32_t n = wp.counts[kMissCount];
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t i = wp.missQueue[k];
        PathState<SG> path;
        load_path(w, i, path);
        pt_handle_miss<SG>(s, p, path, cnt);
        w.L[i] = make_float4(path.L.x, path.L.y, path.L.z, 0.f);  // a miss ends the path: only L is read again
        if (!path.has(PF_ACTIVE)) cnt.v[0]++;
    }
    flush_counters(p.counters, cnt);
}

// Moves the extension queue (or, with the hit/miss split, the next-bounce hit
// and miss queues) into the shade (and miss) queue for the next bounce.
__global__ void wf_advance(WaveParams wp) {
    if (wp.nextHitQueue) {
        wp.counts[0] = wp.counts[kNextHitCount];
        wp.counts[kMissCount] = wp.counts[kNextMissCount];
        wp.counts[kNextHitCount] = 0;
        wp.counts[kNextMissCount] = 0;
    } else {
        wp.counts[0] = wp.counts[1];
    }
    wp.counts[1] = 0;
    wp.counts[2] = 0;
    wp.counts[kFetchExtend] = 0;
    wp.counts[kFetchShadow] = 0;
}

// The shade stage: the kernel specialised for the emissive sampler and for
// whether the scene has textures.
template <class SG, bool HAS_T, bool TEX>
void launch_shade(const DevScene& s, const FrameParams& p, const WaveParams& wp, const SoA& w, int grid, cudaStream_t st) {
    if (FPT_SPECIALIZE_SAMPLER && p.emissiveSampler == 2) wf_shade<SG, HAS_T, false, 2, TEX><<<grid, kShadeBlock, 0, st>>>(s, p, wp, w);
    else if (FPT_SPECIALIZE_SAMPLER && p.emissiveSampler == 1) wf_shade<SG, HAS_T, false, 1, TEX><<<grid, kShadeBlock, 0, st>>>(s, p, wp, w);
    else if (FPT_SPECIALIZE_SAMPLER && p.emissiveSampler == 0) wf_shade<SG, HAS_T, false, 0, TEX><<<grid, kShadeBlock, 0, st>>>(s, p, wp, w);
    else wf_shade<SG, HAS_T, false, -1, TEX><<<grid, kShadeBlock, 0, st>>>(s, p, wp, w);
}

// overlapTraces launch order: 0 enqueues the visibility kernel (second
// stream) before the extension kernel, 1 after it.  FPT_OVERLAP_AUX_PRIORITY 1
// gives the visibility stream the device's highest priority.
#ifndef FPT_OVERLAP_EXTEND_FIRST
#define FPT_OVERLAP_EXTEND_FIRST 0
#endif
#ifndef FPT_OVERLAP_AUX_PRIORITY
#define FPT_OVERLAP_AUX_PRIORITY 0
#endif

template <class SG, bool HAS_T>
cudaError_t run_wavefront(const DevScene& s, const FrameParams& p, WavefrontBuffers& b, cudaStream_t st, KernelTimer* kt) {
    int openPairs[4] = {-1, -1, -1, -1};  // pairs begun by T0 and not yet ended (T0 / T1 nest)
    int depth = 0;
    auto T0 = [&](int cat) { const int q = kt && kt->enabled ? kt->begin(cat, st) : -1; if (depth < 4) openPairs[depth] = q; depth++; };
    auto T1 = [&]() { if (depth > 0 && --depth < 4 && kt) kt->end(openPairs[depth], st); };
    SoA w;
    w.originPdf = b.f4(0); w.dirV = b.f4(1); w.thpB = b.f4(2); w.L = b.f4(3);
    w.sg = reinterpret_cast<uint4*>(b.f4(4)); w.hit = reinterpret_cast<uint4*>(b.f4(5));
    w.sOrigin = b.f4(6); w.sDir = b.f4(7); w.sLr = b.f4(8);
    w.nrm = p.emissiveSampler == 1 ? b.f4(9) : nullptr;  // the LightBVH pdf needs the previous vertex's normal
    w.sampleL = b.sampleL;
    const uint32_t pixels = p.width * p.height;
    const uint32_t wavePixels = std::max<uint32_t>(1, std::min<uint32_t>(pixels, b.capacity / p.spp));
    static int gShade = 0, gTrace = 0, gTraceShort = 0, gGen = 0;
    if (!gShade) {
        gShade = blocks_for(reinterpret_cast<const void*>(wf_shade<SG, HAS_T, false>), kShadeBlock);
        // The specialised variants have the same launch bounds.
        gTrace = blocks_for(reinterpret_cast<const void*>(wf_extend<kStackSize>), kTraceBlock);
        gTraceShort = blocks_for(reinterpret_cast<const void*>(wf_extend<kShortStack>), kTraceBlock);
        gGen = blocks_for(reinterpret_cast<const void*>(wf_generate<SG, false>), kShadeBlock);
    }
    const bool shortStack = s.bvhDepth <= uint32_t(kShortStack);
    // Material sort of the secondary shade queues (primary hits come in pixel
    // order, already coherent).
    // Extension-ray binning (sortExtensionRays) shares the sort buffers and
    // takes precedence over the material sort.
    const bool binRays = p.sortRays && !p.splitMisses && b.owning && b.ensure_sort() == cudaSuccess;
    const bool binShadow = p.sortShadowRays && b.owning && b.ensure_sort() == cudaSuccess;
    const bool sortQueue = !binRays && p.sortMaterials && b.owning && b.ensure_sort() == cudaSuccess;
    const uint32_t sortBins = std::min<uint32_t>(std::max<uint32_t>(s.materialCount, 1u), WavefrontBuffers::kMaxSortBins - 1u) + 1u;
    // Hit/miss split of the shade stage.
    const bool split = p.splitMisses && b.owning && b.ensure_split() == cudaSuccess;
    // Visibility rays beside the extension rays: after shading they only add
    // to L, which the extension kernel neither reads nor writes, and the
    // extension kernel writes only the hit record and the flags word.
    const bool overlap = p.overlapTraces && b.owning && b.ensure_aux() == cudaSuccess;
    const cudaStream_t ss = overlap ? b.aux : st;
    const uint32_t maxIter = p.maxSurfaceBounces + 2;
    for (uint32_t first = 0; first < pixels; first += wavePixels) {
        WaveParams wp{};
        wp.waveFirstPixel = first;
        wp.wavePixels = std::min(wavePixels, pixels - first);
        wp.wavePaths = wp.wavePixels * p.spp;
        wp.counts = b.counts;
        cudaError_t e = cudaMemsetAsync(b.counts, 0, kNumWaveCounts * sizeof(uint32_t), st);
        if (e != cudaSuccess) return e;
        uint32_t* qa = b.queueA;
        uint32_t* qb = b.queueB;
        uint32_t* spare = b.sortQueue;  // binning: scatter target (three distinct buffers rotate within a wave)
        wp.shadeQueue = qa;
        wp.extQueue = qb;
        wp.shadowQueue = b.shadowQueue;
        wp.sortKeys = sortQueue ? b.sortKeys : nullptr;
        wp.sortBins = sortBins;
        wp.extKeys = binRays ? b.sortKeys : nullptr;
        wp.shadowKeys = binShadow ? b.shadowKeys : nullptr;
        uint32_t* qHit = qa;
        uint32_t* qMiss = b.missQueue;
        uint32_t* qNextHit = b.nextHitQueue;
        uint32_t* qNextMiss = b.nextMissQueue;
        wp.missQueue = split ? qMiss : nullptr;
        wp.nextHitQueue = split ? qNextHit : nullptr;
        wp.nextMissQueue = split ? qNextMiss : nullptr;
        const int genBlocks = std::min<int>(gGen, int((wp.wavePaths + kShadeBlock - 1) / kShadeBlock));
        T0(KC_GENERATE);
        wf_generate<SG, false><<<genBlocks, kShadeBlock, 0, st>>>(s, p, wp, w);
        T1();
        for (uint32_t it = 0; it < maxIter; it++) {
            if (sortQueue && it > 0) {
                T0(KC_SORT);
                e = cudaMemsetAsync(b.sortBins, 0, WavefrontBuffers::kMaxSortBins * sizeof(uint32_t), st);
                if (e != cudaSuccess) return e;
                wf_sort_count<<<gGen, kShadeBlock, 0, st>>>(wp, b.sortBins);
                wf_sort_scan<<<1, WavefrontBuffers::kMaxSortBins, 0, st>>>(wp, b.sortBins);
                wf_sort_scatter<<<gGen, kShadeBlock, 0, st>>>(wp, b.sortBins, b.sortQueue);
                T1();
                wp.shadeQueue = b.sortQueue;
            }
            T0(KC_SHADE);
            if (s.textureCount) launch_shade<SG, HAS_T, true>(s, p, wp, w, gShade, st);
            else launch_shade<SG, HAS_T, false>(s, p, wp, w, gShade, st);
            if (split && it > 0) wf_miss<SG><<<gGen, kShadeBlock, 0, st>>>(s, p, wp, w);
            T1();
            WaveParams ws = wp;  // the visibility kernel's view (binned queue)
            if (binShadow) {
                T0(KC_SORT);
                constexpr uint32_t kRayBins = 512;
                e = cudaMemsetAsync(b.sortBins, 0, WavefrontBuffers::kMaxSortBins * sizeof(uint32_t), st);
                if (e != cudaSuccess) return e;
                wf_bin_count<<<gGen, kShadeBlock, 0, st>>>(b.shadowKeys, wp.counts + 2, kRayBins, b.sortBins);
                WaveParams sp = wp;
                sp.sortBins = kRayBins;
                wf_sort_scan<<<1, WavefrontBuffers::kMaxSortBins, 0, st>>>(sp, b.sortBins);
                wf_bin_scatter<<<gGen, kShadeBlock, 0, st>>>(b.shadowKeys, wp.shadowQueue, wp.counts + 2, kRayBins, b.sortBins,
                                                             b.shadowSorted);
                T1();
                ws.shadowQueue = b.shadowSorted;
            }
            if (overlap) {
                T0(KC_TRACE);  // ended on the caller's stream after the join
                if ((e = cudaEventRecord(b.forkEv, st)) != cudaSuccess) return e;
                if ((e = cudaStreamWaitEvent(b.aux, b.forkEv, 0)) != cudaSuccess) return e;
            }
            auto shadowStage = [&]() -> cudaError_t {
                const int shadowPair = kt && kt->enabled ? kt->begin(KC_SHADOW, ss) : -1;
                if (shortStack) wf_shadow<kShortStack><<<gTraceShort, kTraceBlock, 0, ss>>>(s, p, ws, w);
                else wf_shadow<kStackSize><<<gTrace, kTraceBlock, 0, ss>>>(s, p, ws, w);
                if (kt) kt->end(shadowPair, ss);
                return overlap ? cudaEventRecord(b.joinEv, b.aux) : cudaSuccess;
            };
            const bool extendFirst = overlap && FPT_OVERLAP_EXTEND_FIRST;
            if (!extendFirst && (e = shadowStage()) != cudaSuccess) return e;
            if (binRays) {
                T0(KC_SORT);
                constexpr uint32_t kRayBins = 512;
                e = cudaMemsetAsync(b.sortBins, 0, WavefrontBuffers::kMaxSortBins * sizeof(uint32_t), st);
                if (e != cudaSuccess) return e;
                wf_bin_count<<<gGen, kShadeBlock, 0, st>>>(b.sortKeys, wp.counts + 1, kRayBins, b.sortBins);
                WaveParams sp = wp;
                sp.sortBins = kRayBins;
                wf_sort_scan<<<1, WavefrontBuffers::kMaxSortBins, 0, st>>>(sp, b.sortBins);
                wf_bin_scatter<<<gGen, kShadeBlock, 0, st>>>(b.sortKeys, wp.extQueue, wp.counts + 1, kRayBins, b.sortBins, spare);
                T1();
                // The sorted order becomes the extension queue (and the next shade
                // queue); the unsorted buffer is the next bounce's scatter target.
                uint32_t* sorted = spare;
                spare = qb;
                qb = sorted;
                wp.extQueue = sorted;
            }
            T0(KC_EXTEND);
            if (shortStack) wf_extend<kShortStack><<<gTraceShort, kTraceBlock, 0, st>>>(s, p, wp, w);
            else wf_extend<kStackSize><<<gTrace, kTraceBlock, 0, st>>>(s, p, wp, w);
            T1();
            if (extendFirst && (e = shadowStage()) != cudaSuccess) return e;
            // Both traversals of the bounce end before the queues advance.
            if (overlap) {
                if ((e = cudaStreamWaitEvent(st, b.joinEv, 0)) != cudaSuccess) return e;
                T1();
            }
            wf_advance<<<1, 1, 0, st>>>(wp);
            if (split) {
                // Hits of this bounce are the next shade queue; the extension
                // queue buffer is reused as is.
                std::swap(qHit, qNextHit);
                std::swap(qMiss, qNextMiss);
                wp.shadeQueue = qHit;
                wp.missQueue = qMiss;
                wp.nextHitQueue = qNextHit;
                wp.nextMissQueue = qNextMiss;
            } else {
                std::swap(qa, qb);
                wp.shadeQueue = qa;
                wp.extQueue = qb;
            }
        }
        T0(KC_RESOLVE);
        wf_collect<false><<<gGen, 256, 0, st>>>(p, wp, w);
        wf_resolve<false><<<(wp.wavePixels + 255) / 256, 256, 0, st>>>(s, p, wp, w);
        T1();
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// All waves of a batch (one stream-ordered sequence; the caller captures it
// in a CUDA graph).
template <class SG, bool HAS_T>
cudaError_t run_batch(const BatchDevice& bd, const std::vector<BatchWave>& waves, WavefrontBuffers& b, int shadeScale,
                      cudaStream_t st, uint32_t& launches) {
    SoA w;
    w.originPdf = b.f4(0); w.dirV = b.f4(1); w.thpB = b.f4(2); w.L = b.f4(3);
    w.sg = reinterpret_cast<uint4*>(b.f4(4)); w.hit = reinterpret_cast<uint4*>(b.f4(5));
    w.sOrigin = b.f4(6); w.sDir = b.f4(7); w.sLr = b.f4(8);
    w.nrm = nullptr;  // batched requests use the Power sampler
    w.sampleL = b.sampleL;
    DevScene none;
    std::memset(&none, 0, sizeof(none));
    FrameParams fp;
    std::memset(&fp, 0, sizeof(fp));
    fp.counters = bd.counters;
    static int gShade = 0, gTrace = 0, gGen = 0;
    if (!gShade) {
        gShade = blocks_for(reinterpret_cast<const void*>(wf_shade<SG, HAS_T, true>), kShadeBlock);
        gTrace = blocks_for(reinterpret_cast<const void*>(wf_extend_batch), kTraceBlock);
        gGen = blocks_for(reinterpret_cast<const void*>(wf_generate<SG, true>), kShadeBlock);
    }
    const int shadeBlocks = gShade * std::max(1, shadeScale);
    // overlapTraces: the caller created the second stream before any capture
    // (ensure_aux); in a captured graph the two traversals become parallel
    // branches between the shade and advance nodes.
    const bool overlap = b.owning && b.aux && b.forkEv && b.joinEv;
    launches = 0;
    for (const BatchWave& wv : waves) {
        WaveParams wp{};
        wp.fetchChunk = bd.fetchChunk;
        wp.waveFirstPixel = 0;
        wp.wavePixels = wv.pixels;
        wp.wavePaths = wv.paths;
        wp.counts = b.counts;
        wp.scenes = bd.scenes;
        wp.frames = bd.frames;
        wp.tiles = bd.tiles + wv.firstTile;
        wp.tileCount = wv.tileCount;
        wp.slotTile = bd.slotTile;
        cudaError_t e = cudaMemsetAsync(b.counts, 0, kNumWaveCounts * sizeof(uint32_t), st);
        if (e != cudaSuccess) return e;
        uint32_t* qa = b.queueA;
        uint32_t* qb = b.queueB;
        wp.shadeQueue = qa;
        wp.extQueue = qb;
        wp.shadowQueue = b.shadowQueue;
        const int genBlocks = std::min<int>(gGen, int((wp.wavePaths + kShadeBlock - 1) / kShadeBlock));
        wf_generate<SG, true><<<genBlocks, kShadeBlock, 0, st>>>(none, fp, wp, w);
        launches++;
        for (uint32_t it = 0; it < wv.maxIter; it++) {
            wf_shade<SG, HAS_T, true><<<shadeBlocks, kShadeBlock, 0, st>>>(none, fp, wp, w);
            if (overlap) {
                if ((e = cudaEventRecord(b.forkEv, st)) != cudaSuccess) return e;
                if ((e = cudaStreamWaitEvent(b.aux, b.forkEv, 0)) != cudaSuccess) return e;
            }
            wf_shadow_batch<<<gTrace, kTraceBlock, 0, overlap ? b.aux : st>>>(none, fp, wp, w);
            if (overlap && (e = cudaEventRecord(b.joinEv, b.aux)) != cudaSuccess) return e;
            wf_extend_batch<<<gTrace, kTraceBlock, 0, st>>>(none, fp, wp, w);
            if (overlap && (e = cudaStreamWaitEvent(st, b.joinEv, 0)) != cudaSuccess) return e;
            wf_advance<<<1, 1, 0, st>>>(wp);
            launches += 4;
            std::swap(qa, qb);
            wp.shadeQueue = qa;
            wp.extQueue = qb;
        }
        wf_collect<true><<<gGen, 256, 0, st>>>(fp, wp, w);
        wf_resolve<true><<<(wp.wavePixels + 255) / 256, 256, 0, st>>>(none, fp, wp, w);
        launches += 2;
        e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace

cudaError_t launch_batch_wavefront(const BatchDevice& bd, const std::vector<BatchWave>& waves, bool uniformSG, bool hasT,
                                   WavefrontBuffers& b, int shadeScale, cudaStream_t st, uint32_t& launches) {
    if (uniformSG)
        return hasT ? run_batch<UniformSG, true>(bd, waves, b, shadeScale, st, launches)
                    : run_batch<UniformSG, false>(bd, waves, b, shadeScale, st, launches);
    return hasT ? run_batch<TinyUniformSG, true>(bd, waves, b, shadeScale, st, launches)
                : run_batch<TinyUniformSG, false>(bd, waves, b, shadeScale, st, launches);
}

cudaError_t WavefrontBuffers::ensure(uint32_t cap) {
    if (capacity >= cap && base) return cudaSuccess;
    release();
    const size_t f4Bytes = size_t(cap) * sizeof(float4);
    const size_t bytes = bytes_for(cap);
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
    if (base && owning) cudaFree(base);
    if (sortBase) cudaFree(sortBase);
    if (splitBase) cudaFree(splitBase);
    base = nullptr;
    capacity = 0;
    sortBase = nullptr;
    sortCapacity = 0;
    sortKeys = sortQueue = sortBins = nullptr;
    splitBase = nullptr;
    splitCapacity = 0;
    missQueue = nextHitQueue = nextMissQueue = nullptr;
}

cudaError_t WavefrontBuffers::ensure_aux() {
    if (!owning) return cudaErrorNotSupported;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (aux && auxDevice == dev) return cudaSuccess;
    release_aux();
    int least = 0, greatest = 0;
    if (FPT_OVERLAP_AUX_PRIORITY && cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) greatest = 0;
    if ((e = cudaStreamCreateWithPriority(&aux, cudaStreamNonBlocking, FPT_OVERLAP_AUX_PRIORITY ? greatest : 0)) != cudaSuccess) {
        aux = nullptr;
        return e;
    }
    if ((e = cudaEventCreateWithFlags(&forkEv, cudaEventDisableTiming)) != cudaSuccess) { forkEv = nullptr; release_aux(); return e; }
    if ((e = cudaEventCreateWithFlags(&joinEv, cudaEventDisableTiming)) != cudaSuccess) { joinEv = nullptr; release_aux(); return e; }
    auxDevice = dev;
    return cudaSuccess;
}

void WavefrontBuffers::release_aux() {
    if (joinEv) cudaEventDestroy(joinEv);
    if (forkEv) cudaEventDestroy(forkEv);
    if (aux) cudaStreamDestroy(aux);
    aux = nullptr;
    forkEv = joinEv = nullptr;
    auxDevice = -1;
}

cudaError_t WavefrontBuffers::ensure_split() {
    if (!owning) return cudaErrorNotSupported;
    if (splitBase && splitCapacity >= capacity) return cudaSuccess;
    if (splitBase) cudaFree(splitBase);
    splitBase = nullptr;
    splitCapacity = 0;
    cudaError_t e = cudaMalloc(&splitBase, 3 * size_t(capacity) * sizeof(uint32_t));
    if (e != cudaSuccess) { splitBase = nullptr; return e; }
    splitCapacity = capacity;
    missQueue = static_cast<uint32_t*>(splitBase);
    nextHitQueue = missQueue + capacity;
    nextMissQueue = nextHitQueue + capacity;
    return cudaSuccess;
}

cudaError_t WavefrontBuffers::ensure_sort() {
    if (!owning) return cudaErrorNotSupported;
    if (sortBase && sortCapacity >= capacity) return cudaSuccess;
    if (sortBase) cudaFree(sortBase);
    sortBase = nullptr;
    sortCapacity = 0;
    const size_t bytes = 4 * size_t(capacity) * sizeof(uint32_t) + 2 * kMaxSortBins * sizeof(uint32_t);
    cudaError_t e = cudaMalloc(&sortBase, bytes);
    if (e != cudaSuccess) { sortBase = nullptr; return e; }
    sortCapacity = capacity;
    sortKeys = static_cast<uint32_t*>(sortBase);
    sortQueue = sortKeys + capacity;
    shadowKeys = sortQueue + capacity;
    shadowSorted = shadowKeys + capacity;
    sortBins = shadowSorted + capacity;
    return cudaSuccess;
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

int KernelTimer::begin(int cat, cudaStream_t st) {
    if (!enabled) return -1;
    if (used + 2 > events.size()) {
        const size_t grow = std::max<size_t>(64, events.size());
        for (size_t i = 0; i < grow; i++) {
            cudaEvent_t e;
            if (cudaEventCreate(&e) != cudaSuccess) { enabled = false; return -1; }
            events.push_back(e);
        }
    }
    const int pair = int(used / 2);
    pendingCat.push_back(cat);
    ended.push_back(0);
    cudaEventRecord(events[used], st);
    used += 2;
    return pair;
}

void KernelTimer::end(int pair, cudaStream_t st) {
    if (pair < 0 || size_t(pair) >= ended.size()) return;
    cudaEventRecord(events[size_t(pair) * 2 + 1], st);
    ended[size_t(pair)] = 1;
}

cudaError_t KernelTimer::collect() {
    const size_t pairs = std::min(used / 2, pendingCat.size());
    for (size_t k = 0; k < pairs; k++) {
        if (!ended[k]) continue;  // a launch sequence that returned early
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
    ended.clear();
    return cudaSuccess;
}

void KernelTimer::reset() {
    used = 0;
    pendingCat.clear();
    ended.clear();
    for (int i = 0; i < KC_COUNT; i++) { ms[i] = 0; launches[i] = 0; }
}

KernelTimer::~KernelTimer() {
    for (cudaEvent_t e : events) cudaEventDestroy(e);
}

}  // namespace fpt
