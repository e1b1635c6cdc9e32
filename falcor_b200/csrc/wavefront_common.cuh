// wavefront_common.cuh -- structure-of-arrays path state, warp-aggregated
// queues and the dynamic-fetch ray tracing loop shared by the wavefront
// PathTracer (wavefront.cu) and the wavefront WARDiffPathTracer
// (war_wavefront.cu).  Everything here has internal linkage per translation
// unit.
#pragma once

#include "kernels.cuh"
#include "path_logic.cuh"

namespace fpt {
namespace {

using namespace dev;

constexpr int kTraceBlock = 128;
// Threads per block of the generate and shade kernels (each grid-stride
// iteration of the shade kernel ends in a block-wide queue push).
#ifndef FPT_SHADE_BLOCK
#define FPT_SHADE_BLOCK 128
#endif
constexpr int kShadeBlock = FPT_SHADE_BLOCK;

// Counts: [0] shade queue, [1] extension queue, [2] shadow queue, [4] and [5]
// the fetch counters of the extension and visibility ray kernels.
// Wave counters: [0] shade (hit) queue, [1] extension, [2] shadow, [3] miss
// queue, [4]/[5] fetch cursors, [6]/[7] next-bounce hit / miss queues.
constexpr int kFetchExtend = 4, kFetchShadow = 5, kNumWaveCounts = 8;
constexpr int kMissCount = 3, kNextHitCount = 6, kNextMissCount = 7;
struct WaveParams {
    uint32_t waveFirstPixel;   // first pixel of the wave
    uint32_t wavePixels;       // pixels in the wave
    uint32_t wavePaths;        // wavePixels * spp
    uint32_t* counts;
    const uint32_t* shadeQueue;
    uint32_t* extQueue;
    uint32_t* shadowQueue;
    // Material sort of the next shade queue: the extension kernel writes the
    // sort key of queue position k to sortKeys[k] (null: no sort).
    uint32_t* sortKeys;
    uint32_t sortBins;         // material bins + 1 miss bin
    // Hit/miss split (null: the extension queue itself becomes the next
    // shade queue, hits and misses mixed).
    const uint32_t* missQueue;
    uint32_t* nextHitQueue;
    uint32_t* nextMissQueue;
    // Batched waves only: per-request scenes/frames, this wave's tiles, slot -> tile.
    const DevScene* scenes;
    const FrameParams* frames;
    const BatchTile* tiles;
    uint32_t tileCount;
    uint32_t* slotTile;
    // Queue entries a warp of the trace kernels claims per atomic (0: kFetchChunk).
    uint32_t fetchChunk;
    // Extension-ray binning: the shade kernel writes the bin key (ray_bin_key)
    // of extension queue position k to extKeys[k] (null: no binning).
    uint32_t* extKeys;
    uint32_t* shadowKeys;  // visibility-ray binning keys at shadow queue positions (null: none)
};

// Request of wave slot i in a batched wave.
FPT_D uint32_t slot_request(const WaveParams& wp, uint32_t i) { return wp.tiles[wp.slotTile[i]].req; }

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
    float4* nrm;          // oriented face normal of the last scatter vertex (LightBVH MIS), or null
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
    if (w.nrm) {
        const float4 n = w.nrm[i];
        path.normal = make_float3(n.x, n.y, n.z);
    }
    path.shadowPending = false;
}

template <class SG>
FPT_D void store_path(const SoA& w, uint32_t i, const PathState<SG>& path) {
    w.originPdf[i] = make_float4(path.origin.x, path.origin.y, path.origin.z, path.pdf);
    w.dirV[i] = make_float4(path.dir.x, path.dir.y, path.dir.z, __uint_as_float((path.flags & 0xffffu) | (path.vertexIndex << 16)));
    w.thpB[i] = make_float4(path.thp.x, path.thp.y, path.thp.z, __uint_as_float(path.bounces));
    w.L[i] = make_float4(path.L.x, path.L.y, path.L.z, 0.f);
    store_sg(w.sg[i], path.sg);
    if (w.nrm) w.nrm[i] = make_float4(path.normal.x, path.normal.y, path.normal.z, 0.f);
}

// Warp-aggregated push of `item` onto queue q (count at *cnt).
// Returns the queue position of the pushed item (or 0xffffffff).  The lanes
// taking part are those converged at the call, read once: the ballot and the
// shuffle run over the same set even where the caller's control flow has
// split the warp.
FPT_D uint32_t push(bool pred, uint32_t item, uint32_t* q, uint32_t* cnt) {
    const uint32_t group = __activemask();
    const uint32_t mask = __ballot_sync(group, pred);
    if (mask == 0) return 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if (int(lane) == leader) base = atomicAdd(cnt, uint32_t(__popc(mask)));
    base = __shfl_sync(group, base, leader);
    if (!pred) return 0xffffffffu;
    const uint32_t pos = base + uint32_t(__popc(mask & ((1u << lane) - 1u)));
    q[pos] = item;
    return pos;
}

// Block-aggregated push onto two queues at once: one atomic per queue per
// block instead of one per warp (every push of a launch goes to the same
// counter word, whose atomics the L2 serialises).  Every thread of the block
// must reach the call (block-uniform loops only).  `sh` is 2 * (NW + 1) words
// of shared memory; positions are returned in posA / posB (0xffffffff: none).
template <int NW>
FPT_D void block_push2(bool predA, uint32_t itemA, uint32_t* qA, uint32_t* cntA, bool predB, uint32_t itemB, uint32_t* qB,
                       uint32_t* cntB, uint32_t* sh, uint32_t& posA, uint32_t& posB) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t mA = __ballot_sync(0xffffffffu, predA), mB = __ballot_sync(0xffffffffu, predB);
    if (lane == 0) {
        sh[warp] = __popc(mA);
        sh[NW + 1 + warp] = __popc(mB);
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        uint32_t* s = sh + threadIdx.x * (NW + 1);
        uint32_t tot = 0;
        for (int w = 0; w < NW; w++) {
            const uint32_t c = s[w];
            s[w] = tot;
            tot += c;
        }
        s[NW] = tot ? atomicAdd(threadIdx.x ? cntB : cntA, tot) : 0u;
    }
    __syncthreads();
    const uint32_t below = (1u << lane) - 1u;
    posA = predA ? sh[NW] + sh[warp] + uint32_t(__popc(mA & below)) : 0xffffffffu;
    posB = predB ? sh[2 * NW + 1] + sh[NW + 1 + warp] + uint32_t(__popc(mB & below)) : 0xffffffffu;
    __syncthreads();  // the words are reused by the next call
    if (predA) qA[posA] = itemA;
    if (predB) qB[posB] = itemB;
}

// Ray tracing kernels (visibility and extension rays) with per-lane dynamic
// ray fetch: each warp takes chunks of kFetchChunk queue entries with one
// atomic and hands them to its idle lanes, and a lane whose ray has finished
// takes the next one as soon as fewer than kRefillBelow lanes of its warp are
// still tracing.  The traversal itself advances one node visit per step, so
// rays of very different lengths share a warp without leaving most of its
// lanes idle until the longest ray is done.
#ifndef FPT_REFILL_BELOW
#define FPT_REFILL_BELOW 28
#endif
#ifndef FPT_TRACE_MIN_BLOCKS
#define FPT_TRACE_MIN_BLOCKS 6
#endif
// Triangle tests per traversal step of the queue kernels (measured on the
// 1080p heightfield frame: extension rays 8 % faster with 1, visibility rays
// 6 % faster with 2, than testing a whole leaf list per step).
#ifndef FPT_EXTEND_TRIS_PER_STEP
#define FPT_EXTEND_TRIS_PER_STEP 1
#endif
#ifndef FPT_SHADOW_TRIS_PER_STEP
#define FPT_SHADOW_TRIS_PER_STEP 2
#endif
// Queue entries a warp claims per atomic: one per lane.  On the 1080p
// heightfield frame 32 beat 64, 128 and 256 (739.8, 730.3, 700.5, 645.6
// Mpaths/s): smaller claims spread the long rays of a bounce over more warps.
#ifndef FPT_FETCH_CHUNK
#define FPT_FETCH_CHUNK 32
#endif
constexpr uint32_t kFetchChunk = FPT_FETCH_CHUNK;
constexpr int kRefillBelow = FPT_REFILL_BELOW;

// MULTI: rays of a batched wave, each traced in its own request's scene.
// STACK: traversal-stack entries per thread (>= the tree depth).
template <bool SHADOW, bool MARK_VISIBLE = false, bool MULTI = false, int STACK = kStackSize>
FPT_D void trace_queue(const DevScene& s, const FrameParams& p, const WaveParams& wp, const SoA& w, uint2* stack,
                       const uint4* top = nullptr, uint32_t topCount = 0) {
    const uint32_t lane = threadIdx.x & 31u;
    Counters cnt;
    const uint32_t n = wp.counts[SHADOW ? 2 : 1];
    uint32_t* fetch = wp.counts + (SHADOW ? kFetchShadow : kFetchExtend);
    const uint32_t* queue = SHADOW ? wp.shadowQueue : wp.extQueue;
    const int postponeLimit = MULTI ? 0 : STACK - int(s.bvhDepth);
    uint32_t chunkNext = 0, chunkEnd = 0;  // warp-uniform
    bool drained = n == 0 || (!MULTI && s.nodeCount == 0);
    bool active = false;
    uint32_t path = 0, fv = 0, qpos = 0;
    const DevScene* S = nullptr;  // MULTI: this lane's scene
    TraceRay r;
    TraceState t;
    for (;;) {
        const uint32_t idle = __ballot_sync(0xffffffffu, !active);
        if (idle && !drained) {
            if (chunkNext >= chunkEnd) {
                uint32_t base = 0;
                const uint32_t chunk = wp.fetchChunk ? wp.fetchChunk : kFetchChunk;
                if (lane == 0) base = atomicAdd(fetch, chunk);
                base = __shfl_sync(0xffffffffu, base, 0);
                if (base >= n) drained = true;
                else { chunkNext = base; chunkEnd = min(base + chunk, n); }
            }
            if (!drained) {
                const uint32_t avail = chunkEnd - chunkNext;
                const uint32_t rank = __popc(idle & ((1u << lane) - 1u));
                if (!active && rank < avail) {
                    qpos = chunkNext + rank;
                    path = queue[qpos];
                    float4 o, d;
                    if (SHADOW) { o = w.sOrigin[path]; d = w.sDir[path]; }
                    else { o = w.originPdf[path]; d = w.dirV[path]; }
                    fv = __float_as_uint(d.w);
                    r = make_trace_ray(make_float3(o.x, o.y, o.z), make_float3(d.x, d.y, d.z), 0.f);
                    trace_init(r, SHADOW ? o.w : 1e30f, t);
                    if (MULTI) {
                        S = wp.scenes + slot_request(wp, path);
                        if (S->nodeCount == 0) t.status = kTraceDone;  // empty scene: a miss
                    }
                    active = true;
                }
                chunkNext += min(avail, uint32_t(__popc(idle)));
            }
        }
        if (__ballot_sync(0xffffffffu, active) == 0) break;
        for (;;) {
            if (active) {
                if (MULTI) {
                    if (t.status == kTraceRunning)
                        trace_step<SHADOW, STACK, SHADOW ? FPT_SHADOW_TRIS_PER_STEP : FPT_EXTEND_TRIS_PER_STEP>(*S, r, t, stack, kTraceBlock, 0);
                } else {
                    trace_step<SHADOW, STACK, SHADOW ? FPT_SHADOW_TRIS_PER_STEP : FPT_EXTEND_TRIS_PER_STEP>(s, r, t, stack, kTraceBlock,
                                                                                                         postponeLimit, top, topCount);
                }
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
                            if (MARK_VISIBLE) w.sLr[path].w = 1.f;  // read by the adjoint's NEE-gradient kernel
                        }
                    } else {
                        uint32_t f = fv + (1u << 16);  // vertexIndex++
                        if (h.valid) {
                            f |= 0x2u;
                            w.hit[path] = make_uint4(h.instanceID, h.primIndex, __float_as_uint(h.baryX), __float_as_uint(h.baryY));
                        } else {
                            f &= ~0x2u;
                        }
                        if (!MULTI) {
                            // Material bin of the hit (misses in the last bin).
                            const uint32_t last = wp.sortBins - 1u;
                            const uint32_t key = h.valid ? min(__ldg(&s.instances[h.instanceID].materialID), last - 1u) : last;
                            if (wp.nextHitQueue) {
                                const uint32_t pos = push(h.valid, path, wp.nextHitQueue, wp.counts + kNextHitCount);
                                push(!h.valid, path, wp.nextMissQueue, wp.counts + kNextMissCount);
                                if (wp.sortKeys && h.valid) wp.sortKeys[pos] = key;
                            } else if (wp.sortKeys) {
                                wp.sortKeys[qpos] = key;
                            }
                        }
                        // Only the flags word changes: a 4-byte store, no re-read of the direction.
                        reinterpret_cast<uint32_t*>(w.dirV + path)[3] = f;
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

inline int blocks_for(const void* kernel, int block) {
    int perSM = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, kernel, block, 0);
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return std::max(1, perSM) * sms;
}

}  // namespace
}  // namespace fpt
