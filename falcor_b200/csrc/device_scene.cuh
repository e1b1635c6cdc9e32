// device_scene.cuh -- device view of a scene and the per-hit operations of the
// hot path: compressed 8-wide BVH traversal with a shared-memory stack, the
// watertight ray/triangle test, shading-data load, StandardMaterial set-up,
// emissive and environment light sampling.
#pragma once

#include "device_math.cuh"
#include "texture.h"

namespace fpt {

// Kernel-parameter view of a device scene (all pointers are device memory).
struct DevScene {
    const uint4* nodes;               // BVH8Node, 5 x uint4 each
    const float4* tris;               // TriRecord, 3 x float4 each
    const PackedVertex* vertices;
    const uint32_t* indices;
    const DevInstance* instances;
    const DevMaterial* materials;
    const DevEmissiveTri* emissive;
    const float* flux;
    const uint2* alias;
    const uint32_t* instEmissiveOffset;
    const uint32_t* activeTris;
    const uint4* lbvhNodes;           // light BVH: PackedNode, 2 x uint4 each
    const uint32_t* lbvhTriIndices;   // emissive triangle indices of the leaves
    const uint2* lbvhBitmasks;        // per emissive triangle: bit path to its leaf (lo, hi)
    uint32_t lbvhNodeCount;
    const float4* env;                // envW x envH texels (rgb, 0)
    const float* impMips;             // importance mips, concatenated
    uint32_t emissiveCount, activeCount;
    float invWeightSum;
    uint32_t envW, envH;
    float envScale[3];
    uint32_t impDim, impBaseMip;
    uint32_t impMipOffset[16];
    fpt_camera_data camera;
    fpt_hitinfo_bits bits;
    uint32_t hasEnv, hasEmissive, hasTransmission;
    uint32_t nodeCount, triCount;
    uint32_t bvhDepth;                // levels of the 8-wide tree (root = 1)
    uint32_t materialCount;
    uint32_t* errorWord;              // device error word (FPT_DEVERR_*)
    const uint8_t* texData;           // texels of all material textures
    const DevTexture* textures;
    const float* srgbDecode;          // 256-entry sRGB decode table
    uint32_t textureCount;
    float sceneLo[3], sceneInvExtent[3]; // scene bounds at creation (ray binning keys)
};

// Bin of an extension ray for coherence sorting: the Morton code of its
// origin's cell in a 4 x 4 x 4 grid over the scene bounds, then its direction
// octant (512 bins).
FPT_D uint32_t ray_bin_key(const DevScene& s, float3 o, float3 d) {
    uint32_t c[3];
    const float p[3] = {o.x, o.y, o.z};
#pragma unroll
    for (int a = 0; a < 3; a++) {
        const float f = (p[a] - s.sceneLo[a]) * s.sceneInvExtent[a] * 4.f;
        c[a] = f >= 3.f ? 3u : (f > 0.f ? uint32_t(f) : 0u);
    }
    uint32_t m = 0;
#pragma unroll
    for (int b = 1; b >= 0; b--) m = (m << 3) | (((c[0] >> b) & 1u) << 2) | (((c[1] >> b) & 1u) << 1) | ((c[2] >> b) & 1u);
    return (m << 3) | (d.x < 0.f ? 4u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 1u : 0u);
}

namespace dev {

constexpr int kStackSize = 32;  // entries per thread; the host checks BVH depth <= kStackSize

struct HitRec {
    uint32_t instanceID, primIndex, globalTri;
    float baryX, baryY, t;
    bool valid;
};

// Watertight ray/triangle test (Utils/Geometry/IntersectionHelpers.slang:118-189).
// kx/ky/kz and the shear constants depend on the ray only.
struct RayShear {
    int kx, ky, kz;
    float Sx, Sy, Sz;
};
FPT_D RayShear make_shear(float3 d) {
    RayShear s;
    const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
    int axis = 0;
    if (ay > ax && ay > az) axis = 1;
    if (az > ax && az > ay) axis = 2;
    s.kz = axis;
    s.kx = (s.kz + 1) % 3;
    s.ky = (s.kx + 1) % 3;
    if (comp(d, s.kz) < 0.f) { int t = s.kx; s.kx = s.ky; s.ky = t; }
    s.Sx = comp(d, s.kx) / comp(d, s.kz);
    s.Sy = comp(d, s.ky) / comp(d, s.kz);
    s.Sz = 1.f / comp(d, s.kz);
    return s;
}
FPT_D bool intersect_triangle(const RayShear& rs, float3 o, float3 v0, float3 v1, float3 v2, float& t, float& bu, float& bv) {
    const float3 A = v0 - o, B = v1 - o, C = v2 - o;
    const float Akx = comp(A, rs.kx), Aky = comp(A, rs.ky), Akz = comp(A, rs.kz);
    const float Bkx = comp(B, rs.kx), Bky = comp(B, rs.ky), Bkz = comp(B, rs.kz);
    const float Ckx = comp(C, rs.kx), Cky = comp(C, rs.ky), Ckz = comp(C, rs.kz);
    const float Ax = Akx - rs.Sx * Akz, Ay = Aky - rs.Sy * Akz;
    const float Bx = Bkx - rs.Sx * Bkz, By = Bky - rs.Sy * Bkz;
    const float Cx = Ckx - rs.Sx * Ckz, Cy = Cky - rs.Sy * Ckz;
    float U = Cx * By - Cy * Bx;
    float V = Ax * Cy - Ay * Cx;
    float W = Bx * Ay - By * Ax;
    if (U == 0.f || V == 0.f || W == 0.f) {
        double CxBy = double(Cx) * double(By), CyBx = double(Cy) * double(Bx);
        U = float(CxBy - CyBx);
        double AxCy = double(Ax) * double(Cy), AyCx = double(Ay) * double(Cx);
        V = float(AxCy - AyCx);
        double BxAy = double(Bx) * double(Ay), ByAx = double(By) * double(Ax);
        W = float(BxAy - ByAx);
    }
    if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
    float det = U + V + W;
    if (det == 0.f) return false;
    const float Az = rs.Sz * Akz, Bz = rs.Sz * Bkz, Cz = rs.Sz * Ckz;
    const float T = U * Az + V * Bz + W * Cz;
    const float rcpDet = 1.f / det;
    t = T * rcpDet;
    bu = V * rcpDet;
    bv = W * rcpDet;
    return true;
}

// ---------------------------------------------------------------------------
// Compressed 8-wide BVH traversal.
//
// Child boxes are stored as 8-bit offsets q from a per-node origin p with a
// power-of-two scale s per axis; the builder guarantees that
// fma(q, s, p) rounded to float encloses each child box.  The slab distance of
// a plane is evaluated as one FMA, t = q * (s * inv) + (p - o) * inv, where
// s * inv is exact (s is a power of two).  The rounding of p - o, of the
// products and of the FMA, the rounding of the decoded plane and of 1/d are
// each below 2^-24 of one of |p| * |inv|, |p - o| * |inv|, 255 s |inv| or |t|;
// the entry and exit distances of every axis are therefore moved outward by
// eps = 2^-18 (|p| + 2 |p - o| + 512 s) |inv| before the comparison, so no box
// that the ray touches is culled.  (Scene coordinates are limited to
// |x| <= 1e15 so that none of these terms overflows.)
// ---------------------------------------------------------------------------
struct TraceStats {
    uint32_t nodes = 0, tris = 0;
};

// Per-ray constants of the traversal.
struct TraceRay {
    float3 o, d;
    float ix, iy, iz;
    uint32_t octinv;  // bit a set when d[a] < 0
    float tMin;
    RayShear rs;
};

FPT_D TraceRay make_trace_ray(float3 o, float3 d, float tMin) {
    TraceRay r;
    r.o = o;
    r.d = d;
    r.ix = 1.f / (fabsf(d.x) > 1e-20f ? d.x : copysignf(1e-20f, d.x));
    r.iy = 1.f / (fabsf(d.y) > 1e-20f ? d.y : copysignf(1e-20f, d.y));
    r.iz = 1.f / (fabsf(d.z) > 1e-20f ? d.z : copysignf(1e-20f, d.z));
    r.octinv = (d.x < 0.f ? 1u : 0u) | (d.y < 0.f ? 2u : 0u) | (d.z < 0.f ? 4u : 0u);
    r.tMin = tMin;
    r.rs = make_shear(d);
    return r;
}

enum : uint32_t { kTraceRunning = 0, kTraceDone = 1, kTraceAnyHit = 2, kTraceError = 3 };
constexpr uint32_t kTriGroupFlag = 0x80000000u;  // stack entry holds a triangle group

// Resumable traversal state.  The current node group (gBase, gHits, gImask)
// holds the not yet visited children of the last visited node, as bits in
// octant order (bit i is child slot i ^ octinv); the triangle group
// (tBase, tHits) holds the leaf triangles still to be tested.
struct TraceState {
    float tBest;
    uint32_t bestTri, bestInst, bestPrim;
    float bestU, bestV;
    uint32_t gBase, gHits, gImask;
    uint32_t tBase, tHits;
    int sp;
    uint32_t visits, triTests;
    uint32_t status;
};

FPT_D void trace_init(const TraceRay& r, float tMax, TraceState& t) {
    t.tBest = tMax;
    t.bestTri = 0xffffffffu;
    t.bestInst = t.bestPrim = 0;
    t.bestU = t.bestV = 0.f;
    // Pseudo group whose only member is the root (node 0 in slot 0).
    t.gBase = 0;
    t.gHits = 1u << r.octinv;
    t.gImask = 1u;
    t.tBase = t.tHits = 0;
    t.sp = 0;
    t.visits = t.triTests = 0;
    t.status = kTraceRunning;
}

// Byte k (0..3) of w as an exact float: 0x4B0000qq is 2^23 + qq.
FPT_D float quant_to_float(uint32_t w, uint32_t k) {
    return __uint_as_float(__byte_perm(w, 0x4B000000u, 0x7440u | k)) - 8388608.f;
}

// Moves bit k of an 8-bit mask to bit k ^ o.
FPT_D uint32_t octant_permute(uint32_t m, uint32_t o) {
    if (o & 1u) m = ((m & 0x55u) << 1) | ((m >> 1) & 0x55u);
    if (o & 2u) m = ((m & 0x33u) << 2) | ((m >> 2) & 0x33u);
    if (o & 4u) m = ((m & 0x0fu) << 4) | ((m >> 4) & 0x0fu);
    return m;
}

struct AxisPlanes {
    uint32_t n0, n1, f0, f1;  // near / far quantised planes of slots 0-3, 4-7
    float si, bn, bf;         // s * inv, (p - o) * inv - eps, (p - o) * inv + eps
};

FPT_D AxisPlanes axis_planes(float p, float s, float o, float inv, uint32_t lo0, uint32_t lo1, uint32_t hi0, uint32_t hi1,
                             bool flip) {
    AxisPlanes a;
    a.n0 = flip ? hi0 : lo0;
    a.n1 = flip ? hi1 : lo1;
    a.f0 = flip ? lo0 : hi0;
    a.f1 = flip ? lo1 : hi1;
    const float base = p - o;
    const float bi = base * inv;
    const float eps = (fabsf(p) + 2.f * fabsf(base) + 512.f * s) * fabsf(inv) * 3.8146973e-6f;  // 2^-18
    a.si = s * inv;
    a.bn = bi - eps;
    a.bf = bi + eps;
    return a;
}

// Visits one node: tests its 8 child boxes against [tMin, tBest].  Returns
// the hit internal children as a group (octant order) and the triangles of
// the hit leaf children as a bit mask relative to the node's triangle base.
// `top` (shared memory, may be null) holds the first `topCount` nodes of the
// tree (breadth-first order: its top levels), which are read from there.
FPT_D void visit_node(const DevScene& s, const TraceRay& r, float tBest, uint32_t nodeIdx, uint32_t& innerHits,
                      uint32_t& childBase, uint32_t& imask, uint32_t& triBase, uint32_t& triHits, const uint4* top = nullptr,
                      uint32_t topCount = 0) {
    uint4 w0, w1, w2, w3, w4;
    if (nodeIdx < topCount) {
        const uint4* np = top + size_t(nodeIdx) * 5;
        w0 = np[0]; w1 = np[1]; w2 = np[2]; w3 = np[3]; w4 = np[4];
    } else {
        const uint4* np = s.nodes + size_t(nodeIdx) * 5;
        w0 = __ldg(np + 0); w1 = __ldg(np + 1); w2 = __ldg(np + 2); w3 = __ldg(np + 3); w4 = __ldg(np + 4);
    }
    const uint32_t ew = w0.w;
    const float sx = __uint_as_float((ew & 0xffu) << 23);
    const float sy = __uint_as_float(((ew >> 8) & 0xffu) << 23);
    const float sz = __uint_as_float(((ew >> 16) & 0xffu) << 23);
    imask = ew >> 24;
    childBase = w1.x;
    triBase = w1.y;
    // Quantised planes: lo x = w2.xy, lo y = w2.zw, lo z = w3.xy, hi x = w3.zw,
    // hi y = w4.xy, hi z = w4.zw (slots 0-3 in the first word, 4-7 in the second).
    const AxisPlanes X = axis_planes(__uint_as_float(w0.x), sx, r.o.x, r.ix, w2.x, w2.y, w3.z, w3.w, (r.octinv & 1u) != 0);
    const AxisPlanes Y = axis_planes(__uint_as_float(w0.y), sy, r.o.y, r.iy, w2.z, w2.w, w4.x, w4.y, (r.octinv & 2u) != 0);
    const AxisPlanes Z = axis_planes(__uint_as_float(w0.z), sz, r.o.z, r.iz, w3.x, w3.y, w4.z, w4.w, (r.octinv & 4u) != 0);
    uint32_t hits = 0;
#pragma unroll
    for (uint32_t k = 0; k < 8; k++) {
        const uint32_t b = k & 3u;
        const float tnx = fmaf(quant_to_float(k < 4 ? X.n0 : X.n1, b), X.si, X.bn);
        const float tfx = fmaf(quant_to_float(k < 4 ? X.f0 : X.f1, b), X.si, X.bf);
        const float tny = fmaf(quant_to_float(k < 4 ? Y.n0 : Y.n1, b), Y.si, Y.bn);
        const float tfy = fmaf(quant_to_float(k < 4 ? Y.f0 : Y.f1, b), Y.si, Y.bf);
        const float tnz = fmaf(quant_to_float(k < 4 ? Z.n0 : Z.n1, b), Z.si, Z.bn);
        const float tfz = fmaf(quant_to_float(k < 4 ? Z.f0 : Z.f1, b), Z.si, Z.bf);
        const float tn = fmaxf(fmaxf(tnx, tny), fmaxf(tnz, r.tMin));
        const float tf = fminf(fminf(tfx, tfy), fminf(tfz, tBest));
        hits |= (tn <= tf) ? (1u << k) : 0u;
    }
    // Empty slots hold the inverted box [p + 255 s, p], which no ray enters
    // (and whose meta byte is 0, so a hit would add nothing).
    innerHits = octant_permute(hits & imask, r.octinv);
    uint32_t leaves = hits & ~imask;
    triHits = 0;
    while (leaves) {
        const uint32_t k = uint32_t(__ffs(leaves) - 1);
        leaves &= leaves - 1u;
        const uint32_t m = __byte_perm(w1.z, w1.w, k) & 0xffu;  // (count << 5) | offset
        triHits |= ((1u << (m >> 5)) - 1u) << (m & 31u);
    }
}

// One traversal iteration: visit the next node of the current group (if
// any), then test the pending leaf triangles, then pop the stack when the
// group is exhausted.  `postponeLimit` > 0 lets a lane push its triangle
// group onto the stack and keep visiting nodes when fewer than
// kPostponeLanes lanes of its warp have triangles to test; it is the stack
// depth below which this is allowed (stack size minus tree depth, so that
// node groups always fit).  Postponing is off by default: on the 2.3 M
// triangle heightfield workload it cost 3 % (8 lanes) with dynamic ray fetch.
#ifndef FPT_POSTPONE_LANES
#define FPT_POSTPONE_LANES 0
#endif
constexpr int kPostponeLanes = FPT_POSTPONE_LANES;
// TRIS: triangle tests per traversal step (0: all of the visited node's
// leaves in one step).  A bounded count keeps the lanes of a warp in step when
// one lane has a long leaf list; the next node is visited only once the list
// is empty, so the visiting order -- and the result -- are unchanged.

// STACK: entries of this thread's stack (at least the tree depth).
template <bool ANY, int STACK = kStackSize, int TRIS = 0>
FPT_D void trace_step(const DevScene& s, const TraceRay& r, TraceState& t, uint2* stack, uint32_t stride, int postponeLimit,
                      const uint4* top = nullptr, uint32_t topCount = 0) {
    if (t.gHits && (TRIS == 0 || t.tHits == 0)) {
        const uint32_t i = uint32_t(__ffs(t.gHits) - 1);
        t.gHits &= t.gHits - 1u;
        const uint32_t slot = i ^ r.octinv;
        const uint32_t nodeIdx = t.gBase + __popc(t.gImask & ((1u << slot) - 1u));
        t.visits++;
        // A well-formed tree visits each node at most once per ray; guard
        // against corrupted input so that the loop always terminates.
        if (nodeIdx >= s.nodeCount || t.visits > s.nodeCount) {
            atomicOr(s.errorWord, FPT_DEVERR_BAD_INDEX);
            t.status = kTraceError;
            return;
        }
        uint32_t innerHits, childBase, imask, triBase, triHits;
        visit_node(s, r, t.tBest, nodeIdx, innerHits, childBase, imask, triBase, triHits, top, topCount);
        if (t.gHits) {
            if (t.sp >= STACK) {
                atomicOr(s.errorWord, FPT_DEVERR_STACK_OVERFLOW);
                t.status = kTraceError;
                return;
            }
            stack[size_t(t.sp) * stride] = make_uint2(t.gBase, t.gHits | (t.gImask << 8));
            t.sp++;
        }
        t.gBase = childBase;
        t.gHits = innerHits;
        t.gImask = imask;
        t.tBase = triBase;
        t.tHits = triHits;
    }
    for (int tested = 0; t.tHits && (TRIS == 0 || tested < TRIS); tested++) {
        if (postponeLimit > 0 && t.gHits && t.sp < postponeLimit && __popc(__activemask()) < kPostponeLanes) {
            stack[size_t(t.sp) * stride] = make_uint2(t.tBase | kTriGroupFlag, t.tHits);
            t.sp++;
            t.tHits = 0;
            break;
        }
        const uint32_t b = uint32_t(__ffs(t.tHits) - 1);
        t.tHits &= t.tHits - 1u;
        const uint32_t ti = t.tBase + b;
        if (ti >= s.triCount) {
            atomicOr(s.errorWord, FPT_DEVERR_BAD_INDEX);
            continue;
        }
        const float4* tp = s.tris + size_t(ti) * 3;
        const float4 a = __ldg(tp), bb = __ldg(tp + 1), c = __ldg(tp + 2);
        t.triTests++;
        float th, u, v;
        if (!intersect_triangle(r.rs, r.o, make_float3(a.x, a.y, a.z), make_float3(bb.x, bb.y, bb.z), make_float3(c.x, c.y, c.z),
                                th, u, v))
            continue;
        if (!(th >= r.tMin && th <= t.tBest)) continue;
        const uint32_t g = __float_as_uint(a.w);
        if (th == t.tBest && g > t.bestTri) continue;
        if (ANY) {
            t.status = kTraceAnyHit;
            return;
        }
        t.tBest = th;
        t.bestTri = g;
        t.bestInst = __float_as_uint(bb.w);
        t.bestPrim = __float_as_uint(c.w);
        t.bestU = u;
        t.bestV = v;
    }
    if (t.gHits == 0 && t.tHits == 0) {
        if (t.sp == 0) {
            t.status = kTraceDone;
            return;
        }
        t.sp--;
        const uint2 e = stack[size_t(t.sp) * stride];
        if (e.x & kTriGroupFlag) {
            t.tBase = e.x & ~kTriGroupFlag;
            t.tHits = e.y;
        } else {
            t.gBase = e.x;
            t.gHits = e.y & 0xffu;
            t.gImask = e.y >> 8;
        }
    }
}

// Top levels of the BVH in shared memory.  One thread of the block copies the
// first kTopNodes nodes (5 KB; every ray visits them) with one bulk copy
// (cp.async.bulk from this GPU's global memory to this CTA's shared memory,
// no multicast) completing on an mbarrier; the block waits with a bounded
// number of polls.  Returns the number of staged nodes (0 after a timeout,
// recorded in the error word: the traversal then reads global memory).
constexpr uint32_t kTopNodes = 64;
FPT_D uint32_t stage_top_nodes(const DevScene& s, uint4* dst, unsigned long long* bar) {
    const uint32_t count = min(s.nodeCount, kTopNodes);
    if (count == 0) return 0;
    const uint32_t bytes = count * 80u;  // a multiple of 16; node array and dst are 16-byte aligned
    const uint32_t barAddr = uint32_t(__cvta_generic_to_shared(bar));
    const uint32_t dstAddr = uint32_t(__cvta_generic_to_shared(dst));
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared.b64 [%0], 1;" ::"r"(barAddr) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared.b64 _, [%0], %1;" ::"r"(barAddr), "r"(bytes) : "memory");
        asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];"
                     ::"r"(dstAddr), "l"(s.nodes), "r"(bytes), "r"(barAddr) : "memory");
    }
    uint32_t done = 0;
    for (uint32_t it = 0; it < (1u << 20) && !done; it++)
        asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
                     : "=r"(done) : "r"(barAddr) : "memory");
    if (!__syncthreads_and(int(done))) {
        if (threadIdx.x == 0) atomicOr(s.errorWord, FPT_DEVERR_TIMEOUT);
        return 0;
    }
    return count;
}

FPT_D void trace_result(const TraceState& t, HitRec& hit) {
    hit.valid = false;
    if (t.status == kTraceAnyHit) {
        hit.valid = true;
        return;
    }
    if (t.status == kTraceDone && t.bestTri != 0xffffffffu) {
        hit.valid = true;
        hit.globalTri = t.bestTri;
        hit.instanceID = t.bestInst;
        hit.primIndex = t.bestPrim;
        hit.baryX = t.bestU;
        hit.baryY = t.bestV;
        hit.t = t.tBest;
    }
}

// Traces one ray through the compressed 8-wide BVH.
//   ANY = false: closest hit in [tMin, tMax]; ties on t resolve to the
//                smaller global triangle index.
//   ANY = true : first hit in [tMin, tMax] (visibility rays).
// `stack` is this thread's slice of the block's shared-memory stack, strided
// by `stride` entries.  Returns false (and the ray counts as a miss) when the
// traversal stopped on an error, which is also recorded in the error word.
template <bool ANY>
FPT_D bool trace_bvh(const DevScene& s, float3 o, float3 d, float tMin, float tMax, HitRec& hit, uint2* stack,
                     uint32_t stride, TraceStats* ts = nullptr) {
    hit.valid = false;
    if (s.nodeCount == 0) return true;
    const TraceRay r = make_trace_ray(o, d, tMin);
    TraceState t;
    trace_init(r, tMax, t);
    while (t.status == kTraceRunning) trace_step<ANY>(s, r, t, stack, stride, 0);
    if (ts) {
        ts->nodes += t.visits;
        ts->tris += t.triTests;
    }
    trace_result(t, hit);
    return t.status != kTraceError;
}
// ---------------------------------------------------------------------------
// HitInfo packing (Scene/HitInfo.slang:457-487), uncompressed uint4.
// ---------------------------------------------------------------------------
FPT_D uint4 pack_hit(const fpt_hitinfo_bits& b, const HitRec& h) {
    if (!h.valid) return make_uint4(0, 0, 0, 0);
    const uint32_t header = b.type_bits + b.instance_id_bits + b.primitive_index_bits;
    const uint32_t typeOffset = 32u - b.type_bits;
    uint4 o;
    if (header <= 32) { o.x = (1u << typeOffset) | (h.instanceID << b.primitive_index_bits) | h.primIndex; o.y = 0; }
    else { o.x = (1u << typeOffset) | h.instanceID; o.y = h.primIndex; }
    o.z = __float_as_uint(h.baryX);
    o.w = __float_as_uint(h.baryY);
    return o;
}
FPT_D bool unpack_hit(const fpt_hitinfo_bits& b, uint4 in, HitRec& h) {
    h.valid = false;
    if ((in.x >> (32u - b.type_bits)) != 1u) return false;
    const uint32_t header = b.type_bits + b.instance_id_bits + b.primitive_index_bits;
    if (header <= 32) {
        h.instanceID = (in.x >> b.primitive_index_bits) & ((1u << b.instance_id_bits) - 1u);
        h.primIndex = in.x & ((1u << b.primitive_index_bits) - 1u);
    } else {
        h.instanceID = in.x & ((1u << b.instance_id_bits) - 1u);
        h.primIndex = in.y;
    }
    h.baryX = __uint_as_float(in.z);
    h.baryY = __uint_as_float(in.w);
    h.valid = true;
    return true;
}

// ---------------------------------------------------------------------------
// Camera (Scene/Camera/Camera.slang:46-78).
// ---------------------------------------------------------------------------
FPT_D float3 camera_ray_dir(const fpt_camera_data& c, uint32_t px, uint32_t py, uint32_t W, uint32_t H, float& tMin, float& tMax) {
    float2 p = make_float2((float(px) + 0.5f) / float(W), (float(py) + 0.5f) / float(H));
    p = make_float2(p.x + -c.jitterX, p.y + c.jitterY);
    const float ndcx = 2.f * p.x + -1.f, ndcy = -2.f * p.y + 1.f;
    const float3 U = load3(c.cameraU), V = load3(c.cameraV), Wv = load3(c.cameraW);
    const float3 dir = normalize(ndcx * U + ndcy * V + Wv);
    const float invCos = 1.f / dot(normalize(Wv), dir);
    tMin = c.nearZ * invCos;
    tMax = c.farZ * invCos;
    return dir;
}

// ---------------------------------------------------------------------------
// Shading data (Scene/Scene.slang:440-526, MaterialFactory.slang:78-106,
// ShadingFrame.slang:76-150) and StandardMaterial set-up
// (StandardMaterial.slang:50-133).
// ---------------------------------------------------------------------------
struct ShadingData {
    float3 posW, V, T, B, N, faceN;
    float2 uv;
    bool frontFacing;
    uint32_t materialID;
};

FPT_D void unpack_vertex(const PackedVertex& pv, float3& pos, float3& n) {
    pos = make_float3(pv.pos[0], pv.pos[1], pv.pos[2]);
    n = normalize(make_float3(f16(pv.nxy & 0xffffu), f16(pv.nxy >> 16), f16(pv.nz_tw & 0xffffu)));
}

// Reads one packed vertex as two 16-byte loads.
FPT_D PackedVertex load_vertex(const PackedVertex* vb, uint32_t i) {
    const uint4* p = reinterpret_cast<const uint4*>(vb + i);
    const uint4 a = __ldg(p), b = __ldg(p + 1);
    PackedVertex v;
    v.pos[0] = __uint_as_float(a.x); v.pos[1] = __uint_as_float(a.y); v.pos[2] = __uint_as_float(a.z);
    v.nxy = a.w; v.nz_tw = b.x; v.tangentOct = b.y;
    v.uv[0] = __uint_as_float(b.z); v.uv[1] = __uint_as_float(b.w);
    return v;
}

FPT_D ShadingData load_shading_data(const DevScene& s, const HitRec& hit, float3 rayDir) {
    const DevInstance inst = s.instances[hit.instanceID];
    const uint32_t* ip = s.indices + inst.ibOffset + hit.primIndex * 3;
    const uint32_t i0 = __ldg(ip) + inst.vbOffset, i1 = __ldg(ip + 1) + inst.vbOffset, i2 = __ldg(ip + 2) + inst.vbOffset;
    const PackedVertex pv0 = load_vertex(s.vertices, i0), pv1 = load_vertex(s.vertices, i1), pv2 = load_vertex(s.vertices, i2);
    float3 p0, p1, p2, n0, n1, n2;
    unpack_vertex(pv0, p0, n0);
    unpack_vertex(pv1, p1, n1);
    unpack_vertex(pv2, p2, n2);
    // Tangent: decodeNormal2x16 + sign of the fp16 tangent w.
    const float3 t0 = decode_normal2x16(pv0.tangentOct), t1 = decode_normal2x16(pv1.tangentOct), t2 = decode_normal2x16(pv2.tangentOct);
    const float w0 = sgn(f16(pv0.nz_tw >> 16)), w1 = sgn(f16(pv1.nz_tw >> 16)), w2 = sgn(f16(pv2.nz_tw >> 16));
    const float bx = hit.baryX, by = hit.baryY;
    const float b0 = 1.f - bx - by, b1 = bx, b2 = by;
    float3 posW = p0 * b0;
    posW += p1 * b1;
    posW += p2 * b2;
    float3 normalW = n0 * b0;
    normalW += n1 * b1;
    normalW += n2 * b2;
    float3 tanW = t0 * b0;
    tanW += t1 * b1;
    tanW += t2 * b2;
    float tw = w0 * b0;
    tw += w1 * b1;
    tw += w2 * b2;
    tw = sgn(tw);
    float2 uv = make_float2(pv0.uv[0] * b0, pv0.uv[1] * b0);
    uv.x += pv1.uv[0] * b1; uv.y += pv1.uv[1] * b1;
    uv.x += pv2.uv[0] * b2; uv.y += pv2.uv[1] * b2;
    float3 faceN = normalize(cross(p1 - p0, p2 - p0));
    if (inst.flags & FPT_INSTANCE_FRONT_FACE_CW) faceN = -faceN;
    normalW = normalize(normalW);
    faceN = normalize(faceN);
    tanW = normalize(tanW);

    ShadingData sd;
    sd.posW = posW;
    sd.V = -rayDir;
    sd.N = normalize(normalW);
    const float NdotT = dot(tanW, sd.N);
    const bool nonParallel = fabsf(NdotT) < 0.9999f;
    const bool nonZero = dot(tanW, tanW) > 0.f;
    const bool valid = fabsf(tw) == 1.f && nonZero && nonParallel;
    if (valid) {
        sd.T = normalize(tanW - sd.N * NdotT);
        sd.B = cross(sd.N, sd.T) * tw;
    } else {
        sd.T = perp_stark(sd.N);
        sd.B = cross(sd.N, sd.T);
    }
    sd.faceN = faceN;
    sd.uv = uv;
    sd.frontFacing = dot(sd.V, sd.faceN) >= 0.f;
    sd.materialID = inst.materialID;
    return sd;
}

// ---------------------------------------------------------------------------
// Base-colour textures: MaterialSystem::sampleTexture with
// ExplicitLodTextureSampler(0) (MaterialSystem.slang:308-320), bilinear at mip 0
// with wrap addressing (texture.h), texels decoded per format.
// ---------------------------------------------------------------------------
FPT_D float3 tex_texel(const DevScene& s, const DevTexture& t, uint32_t x, uint32_t y) {
    const size_t i = size_t(y) * t.width + x;
    if (t.format == fpt_tex::kRGBA32Float) {
        const float4 c = __ldg(reinterpret_cast<const float4*>(s.texData + t.offset) + i);
        return make_float3(c.x, c.y, c.z);
    }
    const uint32_t c = __ldg(reinterpret_cast<const uint32_t*>(s.texData + t.offset) + i);
    if (t.format == fpt_tex::kRGBA8Srgb)
        return make_float3(__ldg(s.srgbDecode + (c & 0xffu)), __ldg(s.srgbDecode + ((c >> 8) & 0xffu)),
                           __ldg(s.srgbDecode + ((c >> 16) & 0xffu)));
    return make_float3(fpt_tex::unorm8(c & 0xffu), fpt_tex::unorm8((c >> 8) & 0xffu), fpt_tex::unorm8((c >> 16) & 0xffu));
}
FPT_D DevTexture load_texture(const DevScene& s, uint32_t id) {
    const uint4* p = reinterpret_cast<const uint4*>(s.textures + id);
    const uint4 a = __ldg(p), b = __ldg(p + 1);
    DevTexture t;
    t.offset = uint64_t(a.x) | (uint64_t(a.y) << 32);
    t.width = a.z; t.height = a.w; t.format = b.x; t.texelBase = b.y;
    return t;
}
FPT_D float3 tex_sample(const DevScene& s, uint32_t id, float2 uv) {
    const DevTexture t = load_texture(s, id);
    const fpt_tex::Bilinear b = fpt_tex::bilinear(uv.x, uv.y, t.width, t.height);
    float3 c = tex_texel(s, t, b.x0, b.y0) * b.w[0];
    c += tex_texel(s, t, b.x1, b.y0) * b.w[1];
    c += tex_texel(s, t, b.x0, b.y1) * b.w[2];
    c += tex_texel(s, t, b.x1, b.y1) * b.w[3];
    return c;
}
// Texture index of material `id` if its base colour is textured, else ~0u.
FPT_D uint32_t material_base_texture(const DevScene& s, uint32_t id) {
    const uint4* mp = reinterpret_cast<const uint4*>(s.materials + id);
    const uint4 m2 = __ldg(mp + 2);
    if (!(m2.w & kMatFlagBaseColorTexture)) return ~0u;
    return __ldg(reinterpret_cast<const uint32_t*>(mp + 3));
}

FPT_D float3 sd_ray_origin(const ShadingData& sd, bool viewside = true) {
    return compute_ray_origin(sd.posW, (sd.frontFacing == viewside) ? sd.faceN : -sd.faceN);
}
FPT_D float3 sd_oriented_face_n(const ShadingData& sd) { return sd.frontFacing ? sd.faceN : -sd.faceN; }

template <bool HAS_TRANSMISSION>
struct MaterialInstance {
    float3 T, B, N;
    BSDFData data;
    float3 emission;
    bool thin, lambert;
    uint32_t activeLobes;

    FPT_D float3 toLocal(float3 v) const { return make_float3(dot(v, T), dot(v, B), dot(v, N)); }
    FPT_D float3 fromLocal(float3 v) const { return T * v.x + B * v.y + N * v.z; }
    FPT_D uint32_t lobeTypes() const { return bsdf_lobe_types(data); }
    FPT_D float propRoughness() const { return data.roughness * data.roughness < kMinGGXAlpha ? 0.f : data.roughness; }

    // isValidHemisphereReflectionOrTransmission (Scene/Material/ShadingUtils.slang:216-245).
    FPT_D bool valid_hemisphere(const ShadingData& sd, float3 wiL, float3 woL, float3 wo) const {
        const bool isT = wiL.z * woL.z < 0.f;
        if (hmin(wiL.z, fabsf(woL.z)) < kMinCosTheta) return false;
        const bool wiTop = sd.frontFacing, woTop = dot(wo, sd.faceN) >= 0.f;
        if (isT) { if (wiTop == woTop) return false; }
        else { if (wiTop != woTop) return false; }
        const bool shadingTop = dot(N, sd.faceN) >= 0.f;
        if (wiTop != shadingTop) return false;
        return true;
    }
    FPT_D StandardBSDF<HAS_TRANSMISSION> bsdf(float3 wiL) const {
        StandardBSDF<HAS_TRANSMISSION> b;
        b.init(wiL, data, thin, activeLobes, lambert);
        return b;
    }
    FPT_D float3 eval(const ShadingData& sd, float3 wo) const {
        const float3 wiL = toLocal(sd.V), woL = toLocal(wo);
        if (!valid_hemisphere(sd, wiL, woL, wo)) return f3(0.f);
        return bsdf(wiL).eval(wiL, woL);
    }
    FPT_D float evalPdf(const ShadingData& sd, float3 wo, bool useIS) const {
        const float3 wiL = toLocal(sd.V), woL = toLocal(wo);
        if (!valid_hemisphere(sd, wiL, woL, wo)) return 0.f;
        if (!useIS) {
            if (lobeTypes() & L_TRANSMISSION) {
                if (hmin(fabsf(wiL.z), fabsf(woL.z)) < kMinCosTheta) return 0.f;
                return 0.5f * woL.z * kInvPi;
            }
            if (hmin(wiL.z, woL.z) < kMinCosTheta) return 0.f;
            return woL.z * kInvPi;
        }
        return bsdf(wiL).eval_pdf(wiL, woL);
    }
    // eval and evalPdf of one direction, with the BSDF `b` set up for wiL =
    // toLocal(sd.V) by the caller (shared with sample_with).
    FPT_D void eval_with_pdf(const ShadingData& sd, const StandardBSDF<HAS_TRANSMISSION>& b, float3 wiL, float3 wo, bool useIS,
                             float3& f, float& pdf) const {
        f = f3(0.f);
        pdf = 0.f;
        const float3 woL = toLocal(wo);
        if (!valid_hemisphere(sd, wiL, woL, wo)) return;
        if (!useIS) {
            f = b.eval(wiL, woL);
            if (lobeTypes() & L_TRANSMISSION) {
                if (hmin(fabsf(wiL.z), fabsf(woL.z)) < kMinCosTheta) return;
                pdf = 0.5f * woL.z * kInvPi;
                return;
            }
            if (hmin(wiL.z, woL.z) < kMinCosTheta) return;
            pdf = woL.z * kInvPi;
            return;
        }
        b.eval_with_pdf(wiL, woL, f, pdf);
    }
    template <class SG>
    FPT_D bool sample(const ShadingData& sd, SG& sg, float3& wo, float3& weight, float& pdf, uint32_t& lobe, bool useIS) const {
        const float3 wiL = toLocal(sd.V);
        return sample_with(sd, bsdf(wiL), wiL, sg, wo, weight, pdf, lobe, useIS);
    }
    template <class SG>
    FPT_D bool sample_with(const ShadingData& sd, const StandardBSDF<HAS_TRANSMISSION>& b, float3 wiL, SG& sg, float3& wo,
                           float3& weight, float& pdf, uint32_t& lobe, bool useIS) const {
        float3 woL = f3(0.f);
        if (!useIS) {
            // sampleReference (StandardMaterialInstance.slang:202-230).
            weight = f3(0.f);
            lobe = 0;
            const bool isTransmissive = (lobeTypes() & L_TRANSMISSION) != 0;
            woL = sample_cosine_hemisphere_concentric(next2D(sg), pdf);
            if (isTransmissive) {
                if (next1D(sg) < 0.5f) woL.z = -woL.z;
                pdf *= 0.5f;
                if (hmin(fabsf(wiL.z), fabsf(woL.z)) < kMinCosTheta || pdf == 0.f) return false;
            } else {
                if (hmin(wiL.z, woL.z) < kMinCosTheta || pdf == 0.f) return false;
            }
            weight = b.eval(wiL, woL) / pdf;
            lobe = woL.z > 0.f ? L_DIFF_R : L_DIFF_T;
        } else {
            if (!b.sample(wiL, woL, pdf, weight, lobe, sg)) return false;
        }
        wo = fromLocal(woL);
        if (!valid_hemisphere(sd, wiL, woL, wo)) return false;
        return true;
    }
};

// TEX = false: the scene has no textures, and the texture lookup is compiled
// out (its code would sit in the instruction cache of the shading kernels).
template <bool HAS_TRANSMISSION, bool TEX = true>
FPT_D MaterialInstance<HAS_TRANSMISSION> material_instance(const DevScene& s, const ShadingData& sd, bool lambert) {
    const uint4* mp = reinterpret_cast<const uint4*>(s.materials + sd.materialID);
    const uint4 m0 = __ldg(mp), m1 = __ldg(mp + 1), m2 = __ldg(mp + 2);
    MaterialInstance<HAS_TRANSMISSION> mi;
    mi.lambert = lambert;
    const uint32_t flags = m2.w & 0xffffu;
    mi.thin = (flags & 2u) != 0;
    mi.activeLobes = m2.w >> 16;
    BSDFData& d = mi.data;
    const float IoR = f16(m2.x & 0xffffu);
    d.eta = sd.frontFacing ? (1.f / IoR) : (IoR / 1.f);
    d.specTrans = f16(m2.x >> 16);
    d.diffTrans = f16(m2.y & 0xffffu);
    d.transmission = f3(1.f);
    if (d.diffTrans > 0.f || d.specTrans > 0.f) d.transmission = make_float3(f16(m2.y >> 16), f16(m2.z & 0xffffu), f16(m2.z >> 16));
    const float f = (IoR - 1.f) / (IoR + 1.f);
    const float F0 = f * f;
    float3 baseColor = make_float3(f16(m0.x & 0xffffu), f16(m0.x >> 16), f16(m0.y & 0xffffu));
    if (TEX && (flags & kMatFlagBaseColorTexture)) baseColor = tex_sample(s, __ldg(reinterpret_cast<const uint32_t*>(mp + 3)), sd.uv);
    const float specG = f16(m0.z >> 16), specB = f16(m0.w & 0xffffu);
    d.diffuse = lerp(baseColor, f3(0.f), specB);
    d.specular = lerp(f3(F0), baseColor, specB);
    d.roughness = specG;
    d.metallic = specB;
    mi.T = sd.T; mi.B = sd.B; mi.N = sd.N;
    if (!sd.frontFacing && (flags & 1u)) mi.N = -mi.N;  // flipShadingNormal
    mi.emission = f3(0.f);
    if (sd.frontFacing) {
        const float fac = __uint_as_float(m1.w);
        mi.emission = make_float3(__uint_as_float(m1.x), __uint_as_float(m1.y), __uint_as_float(m1.z)) * fac;
    }
    return mi;
}

// ---------------------------------------------------------------------------
// Environment map (Scene/Lights/EnvMap.slang:58-68) with software bilinear
// filtering (wrap in u, clamp in v), and EnvMapSampler (EnvMapSampler.slang:75-164).
// ---------------------------------------------------------------------------
FPT_D float3 env_texel(const DevScene& s, int x, int y) {
    const float4 t = __ldg(s.env + size_t(y) * s.envW + x);
    return make_float3(t.x, t.y, t.z);
}
FPT_D float3 env_eval(const DevScene& s, float3 dir) {
    const float2 uv = world_to_latlong_map(dir);
    const float fx = uv.x * float(s.envW) - 0.5f, fy = uv.y * float(s.envH) - 0.5f;
    const float x0f = floorf(fx), y0f = floorf(fy);
    const float ax = fx - x0f, ay = fy - y0f;
    const int x0 = int(x0f), y0 = int(y0f);
    const int W = int(s.envW), H = int(s.envH);
    const int xa = ((x0 % W) + W) % W, xb = (((x0 + 1) % W) + W) % W;
    const int ya = min(max(y0, 0), H - 1), yb = min(max(y0 + 1, 0), H - 1);
    const float3 c = env_texel(s, xa, ya) * ((1.f - ax) * (1.f - ay)) + env_texel(s, xb, ya) * (ax * (1.f - ay)) +
                     env_texel(s, xa, yb) * ((1.f - ax) * ay) + env_texel(s, xb, yb) * (ax * ay);
    return c * make_float3(s.envScale[0], s.envScale[1], s.envScale[2]);
}
FPT_D float imp_load(const DevScene& s, uint32_t mip, uint32_t x, uint32_t y) {
    return __ldg(s.impMips + s.impMipOffset[mip] + size_t(y) * (s.impDim >> mip) + x);
}
FPT_D bool env_sample(const DevScene& s, float2 p, float3& dir, float& pdf, float3& Le) {
    uint32_t px = 0, py = 0;
    for (int mip = int(s.impBaseMip) - 1; mip >= 0; mip--) {
        px *= 2; py *= 2;
        const float w0 = imp_load(s, mip, px, py), w1 = imp_load(s, mip, px + 1, py);
        const float w2 = imp_load(s, mip, px, py + 1), w3 = imp_load(s, mip, px + 1, py + 1);
        const float q0 = w0 + w2, q1 = w1 + w3;
        uint32_t ox, oy;
        const float dd = q0 / (q0 + q1);
        if (p.x < dd) { ox = 0; p.x = p.x / dd; }
        else { ox = 1; p.x = (p.x - dd) / (1.f - dd); }
        const float e = ox == 0 ? (w0 / q0) : (w1 / q1);
        if (p.y < e) { oy = 0; p.y = p.y / e; }
        else { oy = 1; p.y = (p.y - e) / (1.f - e); }
        px += ox; py += oy;
    }
    const float inv = 1.f / float(s.impDim);
    const float2 uv = make_float2((float(px) + p.x) * inv, (float(py) + p.y) * inv);
    dir = oct_to_ndir_equal_area_unorm(uv);
    const float avg = imp_load(s, s.impBaseMip, 0, 0);
    const float pr = imp_load(s, 0, px, py) / avg;
    pdf = pr * kInv4Pi;
    Le = env_eval(s, dir);
    return true;
}
FPT_D float env_eval_pdf(const DevScene& s, float3 dir) {
    const float2 uv = ndir_to_oct_equal_area_unorm(dir);
    const float avg = imp_load(s, s.impBaseMip, 0, 0);
    int x = int(floorf(uv.x * float(s.impDim))), y = int(floorf(uv.y * float(s.impDim)));
    x = min(max(x, 0), int(s.impDim) - 1);
    y = min(max(y, 0), int(s.impDim) - 1);
    const float pr = imp_load(s, 0, uint32_t(x), uint32_t(y)) / avg;
    return pr * (1.f / k4Pi);
}

// ---------------------------------------------------------------------------
// Emissive triangle lights (EmissiveLightSamplerHelpers.slang:54-124,
// EmissiveUniformSampler.slang:55-110, EmissivePowerSampler.slang:61-124).
// ---------------------------------------------------------------------------
struct TriLightSample {
    float3 posW, normalW, dir, Le;
    float distance, pdf;
};

FPT_D bool sample_triangle_light(const DevScene& s, float3 posW, uint32_t tri, float2 u, TriLightSample& ls) {
    const uint4* tp = reinterpret_cast<const uint4*>(s.emissive + tri);
    const uint4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2), e = __ldg(tp + 3);
    const float3 P0 = make_float3(__uint_as_float(a.x), __uint_as_float(a.y), __uint_as_float(a.z));
    const float3 P1 = make_float3(__uint_as_float(b.x), __uint_as_float(b.y), __uint_as_float(b.z));
    const float3 P2 = make_float3(__uint_as_float(c.x), __uint_as_float(c.y), __uint_as_float(c.z));
    const float3 bc = sample_triangle_bary(u);
    ls.posW = P0 * bc.x + P1 * bc.y + P2 * bc.z;
    const float3 toLight = ls.posW - posW;
    const float distSqr = hmax(kFltMin, dot(toLight, toLight));
    ls.distance = sqrtf(distSqr);
    ls.dir = toLight / ls.distance;
    ls.normalW = decode_normal2x16(e.x);
    const float cosTheta = dot(ls.normalW, -ls.dir);
    if (cosTheta <= 0.f) return false;
    const DevMaterial* m = s.materials + e.z;
    const float4 em = __ldg(reinterpret_cast<const float4*>(m) + 1);
    ls.Le = make_float3(em.x, em.y, em.z) * em.w;
    const float denom = hmax(kFltMin, cosTheta * __uint_as_float(e.y));
    ls.pdf = distSqr / denom;
    return true;
}
FPT_D float eval_triangle_pdf(const DevScene& s, float3 posW, uint32_t tri, float3 hitPos, float3 hitN) {
    const float3 toLight = hitPos - posW;
    const float distSqr = dot(toLight, toLight);
    if (distSqr <= kFltMin) return 0.f;
    const float3 L = toLight / sqrtf(distSqr);
    const float cosTheta = dot(hitN, -L);
    if (cosTheta <= 0.f) return 0.f;
    const float area = __ldg(&s.emissive[tri].area);
    const float denom = hmax(kFltMin, cosTheta * area);
    return distSqr / denom;
}
// ---------------------------------------------------------------------------
// LightBVHSampler (Rendering/Lights/LightBVHSampler.slang:55-534) with its
// default options: bounding cone, lighting cone, node flux, uniform triangle
// selection in a leaf, SolidAngleBoundMethod::Sphere.
// ---------------------------------------------------------------------------
struct LbvhNode {
    uint32_t w0;  // leaf: 1 << 31 | count << 27 | offset; internal: right child
    float3 origin, extent, coneDir;
    float cosCone, flux;
};
FPT_D LbvhNode lbvh_node(const DevScene& s, uint32_t i) {
    const uint4 a = __ldg(s.lbvhNodes + 2 * i), b = __ldg(s.lbvhNodes + 2 * i + 1);
    LbvhNode n;
    n.w0 = a.x;
    n.origin = make_float3(__uint_as_float(a.y), __uint_as_float(a.z), __uint_as_float(a.w));
    n.extent = make_float3(f16(b.x & 0xffffu), f16(b.x >> 16), f16(b.y & 0xffffu));
    n.cosCone = float(b.y >> 16) * (1.f / 32767.f) - 1.f;
    n.coneDir = decode_normal2x16(b.z);
    n.flux = __uint_as_float(b.w);
    return n;
}
FPT_D bool lbvh_is_leaf(uint32_t w0) { return (w0 >> 31) != 0; }
FPT_D float cos_sub_clamped(float sinA, float cosA, float sinB, float cosB) {
    if (cosA > cosB) return 1.f;
    return cosA * cosB + sinA * sinB;
}
FPT_D float sin_sub_clamped(float sinA, float cosA, float sinB, float cosB) {
    if (cosA > cosB) return 0.f;
    return sinA * cosB - cosA * sinB;
}
// boundCosineTerm with boundSphereSubtendedConeAngle (GeometryHelpers.slang:222-240).
FPT_D float lbvh_bound_cosine(float3 posW, float3 normalW, float3 center, float3 extent, float& cosThetaCone) {
    const float sqrRadius = dot(extent, extent);
    const float3 c = center - posW;
    const float d2 = dot(c, c);
    float sinThetaCone;
    if (d2 < sqrRadius) {
        sinThetaCone = 0.f;
        cosThetaCone = -1.f;
    } else {
        const float sin2 = sqrRadius / d2;
        cosThetaCone = sqrtf(1.f - sin2);
        sinThetaCone = sqrtf(sin2);
    }
    const float3 L = normalize(center - posW);
    const float cosThetaL = fminf(fmaxf(dot(normalW, L), -1.f), 1.f);
    const float sinThetaL = sqrtf(1.f - cosThetaL * cosThetaL);
    return saturate(cos_sub_clamped(sinThetaL, cosThetaL, sinThetaCone, cosThetaCone));
}
// computeImportance (LightBVHSampler.slang:206-259).
FPT_D float lbvh_importance(const DevScene& s, float3 posW, float3 normalW, bool upper, uint32_t i) {
    const LbvhNode n = lbvh_node(s, i);
    float distance = length(n.origin - posW);
    float cosThetaBoundingCone = 0.f;
    float NdotL = lbvh_bound_cosine(posW, normalW, n.origin, n.extent, cosThetaBoundingCone);
    if (!upper) NdotL = 1.f;  // the NdotL bound only for the upper hemisphere
    float orientationWeight = 1.f;
    const float3 dirToAabb = (n.origin - posW) / distance;
    if (n.cosCone != -1.f && n.cosCone > 0.f) {
        const float sinConeAngle = sqrtf(fmaxf(0.f, 1.f - n.cosCone * n.cosCone));
        const float cosTheta = dot(n.coneDir, -dirToAabb);
        const float sinTheta = sqrtf(fmaxf(0.f, 1.f - cosTheta * cosTheta));
        const float sinThetaBoundingCone = sqrtf(fmaxf(0.f, 1.f - cosThetaBoundingCone * cosThetaBoundingCone));
        const float cosTheta0 = cos_sub_clamped(sinTheta, cosTheta, sinConeAngle, n.cosCone);
        const float sinTheta0 = sin_sub_clamped(sinTheta, cosTheta, sinConeAngle, n.cosCone);
        const float cosThetaPrime = cos_sub_clamped(sinTheta0, cosTheta0, sinThetaBoundingCone, cosThetaBoundingCone);
        orientationWeight = fmaxf(0.f, cosThetaPrime);
    }
    const float halfRadius = fmaxf(n.extent.x, fmaxf(n.extent.y, n.extent.z));
    distance = fmaxf(halfRadius, distance);
    return (n.flux * NdotL) * orientationWeight / (distance * distance);
}
// sampleLightViaBVH (traverseTree + pickTriangle, uniform in the leaf).
FPT_D bool lbvh_select(const DevScene& s, float3 posW, float3 normalW, bool upper, float u, float& pdf, uint32_t& tri) {
    pdf = 1.f;
    uint32_t node = 0;
    uint32_t w0 = __ldg(&s.lbvhNodes[0].x);
    for (int depth = 0; !lbvh_is_leaf(w0) && depth < 64; depth++) {
        const uint32_t left = node + 1, right = w0;
        const float il = lbvh_importance(s, posW, normalW, upper, left);
        const float ir = lbvh_importance(s, posW, normalW, upper, right);
        const float total = il + ir;
        if (total == 0.f) return false;
        const float pLeft = il / total;
        const float pRight = 1.f - pLeft;
        if (u < pLeft) {
            u = u / pLeft;
            pdf *= pLeft;
            node = left;
        } else {
            u = (u - pLeft) / pRight;
            pdf *= pRight;
            node = right;
        }
        w0 = __ldg(&s.lbvhNodes[2 * node].x);
    }
    if (!lbvh_is_leaf(w0)) return false;
    const uint32_t count = (w0 >> 27) & 15u, offset = w0 & ((1u << 27) - 1u);
    const uint32_t idx = min(uint32_t(u * float(count)), count - 1);
    tri = __ldg(s.lbvhTriIndices + offset + idx);
    pdf *= 1.f / float(count);
    return true;
}
// evalTriangleSelectionPdf (LightBVHSampler.slang:95-125): the traversal pdf along
// the triangle's bit path times the uniform leaf selection.
FPT_D float lbvh_selection_pdf(const DevScene& s, float3 posW, float3 normalW, bool upper, uint32_t tri) {
    const uint2 m = __ldg(s.lbvhBitmasks + tri);
    uint64_t bitmask = (uint64_t(m.y) << 32) | m.x;
    float pdf = 1.f;
    uint32_t node = 0;
    uint32_t w0 = __ldg(&s.lbvhNodes[0].x);
    for (int depth = 0; !lbvh_is_leaf(w0) && depth < 64; depth++) {
        const uint32_t left = node + 1, right = w0;
        const float il = lbvh_importance(s, posW, normalW, upper, left);
        const float ir = lbvh_importance(s, posW, normalW, upper, right);
        const float total = il + ir;
        if (total == 0.f) return 0.f;
        const float pLeft = il / total;
        const float pRight = 1.f - pLeft;
        if ((bitmask & 1ull) == 0) {
            pdf *= pLeft;
            node = left;
        } else {
            pdf *= pRight;
            node = right;
        }
        bitmask >>= 1;
        w0 = __ldg(&s.lbvhNodes[2 * node].x);
    }
    if (!lbvh_is_leaf(w0)) return 0.f;
    const uint32_t count = (w0 >> 27) & 15u;
    return pdf * (1.f / float(count));
}

template <class SG>
FPT_D bool emissive_sample(const DevScene& s, uint32_t samplerType, float3 posW, SG& sg, TriLightSample& ls,
                           float3 normalW = make_float3(0.f, 0.f, 0.f), bool upperHemisphere = false) {
    if (samplerType == 1) {
        // LightBVHSampler::sampleLight (LightBVHSampler.slang:70-90).
        if (s.emissiveCount == 0 || s.lbvhNodeCount == 0) return false;
        const float uLight = next1D(sg);
        float selPdf;
        uint32_t tri;
        if (!lbvh_select(s, posW, normalW, upperHemisphere, uLight, selPdf, tri)) return false;
        const float2 u = next2D(sg);
        if (!sample_triangle_light(s, posW, tri, u, ls)) return false;
        ls.pdf *= selPdf;
        return true;
    }
    if (samplerType == 0) {
        if (s.activeCount == 0) return false;
        const float uLight = next1D(sg);
        const uint32_t n = s.activeCount;
        const uint32_t idx = min(uint32_t(uLight * float(n)), n - 1);
        const uint32_t tri = __ldg(s.activeTris + idx);
        const float selPdf = 1.f / float(n);
        const float2 u = next2D(sg);
        if (!sample_triangle_light(s, posW, tri, u, ls)) return false;
        ls.pdf *= selPdf;
        return true;
    }
    if (s.emissiveCount == 0) return false;
    const float uLight = next1D(sg);
    const uint32_t n = s.emissiveCount;
    uint32_t tri = min(uint32_t(uLight * float(n)), n - 1);
    const uint2 e = __ldg(s.alias + tri);
    const float threshold = f16(e.x >> 16);
    const uint32_t above = ((e.x & 0xFFFFu) << 8) | ((e.y >> 24) & 0xFFu);
    const uint32_t below = e.y & 0xFFFFFFu;
    tri = (next1D(sg) >= threshold) ? above : below;
    const float selPdf = __ldg(s.flux + tri) * s.invWeightSum;
    const float2 u = next2D(sg);
    if (!sample_triangle_light(s, posW, tri, u, ls)) return false;
    ls.pdf *= selPdf;
    return true;
}
FPT_D float emissive_eval_pdf(const DevScene& s, uint32_t samplerType, float3 posW, uint32_t tri, float3 hitPos, float3 hitN,
                              float3 normalW = make_float3(0.f, 0.f, 0.f), bool upperHemisphere = false) {
    if (tri == 0xffffffffu) return 0.f;
    float sel;
    if (samplerType == 1) {
        if (s.lbvhNodeCount == 0) return 0.f;
        sel = lbvh_selection_pdf(s, posW, normalW, upperHemisphere, tri);
        if (sel == 0.f) return 0.f;
    } else if (samplerType == 0) sel = s.activeCount > 0 ? 1.f / float(s.activeCount) : 0.f;
    else sel = __ldg(s.flux + tri) * s.invWeightSum;
    return sel * eval_triangle_pdf(s, posW, tri, hitPos, hitN);
}

}  // namespace dev
}  // namespace fpt
