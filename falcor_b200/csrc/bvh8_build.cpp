// bvh8_build.cpp -- host builder of the compressed 8-wide BVH.
//
// The reference path has no software triangle BVH (DXR builds the
// acceleration structures in the driver, Scene::buildBlas Scene.cpp:3376), so
// this is new work: a binned-SAH binary BVH (leaves of at most 3 triangles),
// collapsed to 8-wide nodes by repeatedly opening the largest child, with the
// child slots ordered by direction octant so that traversal can visit them
// approximately front to back, and the child boxes quantised to 8 bits per
// plane relative to a per-node origin and power-of-two scale.  Quantisation is
// conservative with respect to the exact device decoding, fmaf(q, scale, p).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <future>
#include <limits>
#include <stdexcept>
#include <thread>

#include "common.h"

namespace fpt {

namespace {

struct AABB {
    float lo[3], hi[3];
    void reset() {
        for (int a = 0; a < 3; a++) { lo[a] = std::numeric_limits<float>::max(); hi[a] = -std::numeric_limits<float>::max(); }
    }
    void grow(const AABB& b) {
        for (int a = 0; a < 3; a++) { lo[a] = std::min(lo[a], b.lo[a]); hi[a] = std::max(hi[a], b.hi[a]); }
    }
    void grow(const float* p) {
        for (int a = 0; a < 3; a++) { lo[a] = std::min(lo[a], p[a]); hi[a] = std::max(hi[a], p[a]); }
    }
    float area() const {
        float d[3];
        for (int a = 0; a < 3; a++) d[a] = std::max(0.f, hi[a] - lo[a]);
        return 2.f * (d[0] * d[1] + d[1] * d[2] + d[2] * d[0]);
    }
};

struct Node2 {
    AABB box;
    uint32_t left = 0, right = 0;  // internal
    uint32_t first = 0, count = 0; // leaf (count > 0)
};

constexpr uint32_t kMaxLeaf = 3;
constexpr int kBins = 16;

struct Builder2 {
    std::vector<AABB> triBox;
    std::vector<float> cen;  // 3 per triangle
    std::vector<uint32_t> idx;
    std::vector<Node2> nodes;
    std::atomic<uint32_t> nextNode{0};

    uint32_t alloc() {
        uint32_t n = nextNode.fetch_add(1);
        if (n >= nodes.size()) throw std::runtime_error("BVH node pool exhausted");
        return n;
    }

    void build(uint32_t node, uint32_t first, uint32_t count, int depth) {
        Node2& nd = nodes[node];
        AABB box, cbox;
        box.reset();
        cbox.reset();
        for (uint32_t i = first; i < first + count; i++) {
            box.grow(triBox[idx[i]]);
            cbox.grow(&cen[size_t(idx[i]) * 3]);
        }
        nd.box = box;
        if (count <= 1) { nd.first = first; nd.count = count; return; }
        // Binned SAH over the three axes.
        float bestCost = std::numeric_limits<float>::max();
        int bestAxis = -1, bestSplit = -1;
        for (int a = 0; a < 3; a++) {
            float ext = cbox.hi[a] - cbox.lo[a];
            if (!(ext > 0.f)) continue;
            AABB bb[kBins];
            uint32_t bc[kBins] = {0};
            for (auto& b : bb) b.reset();
            const float k = float(kBins) * (1.f - 1e-6f) / ext;
            for (uint32_t i = first; i < first + count; i++) {
                int b = std::min(kBins - 1, int((cen[size_t(idx[i]) * 3 + a] - cbox.lo[a]) * k));
                bb[b].grow(triBox[idx[i]]);
                bc[b]++;
            }
            float rightArea[kBins];
            uint32_t rightCount[kBins];
            AABB acc;
            acc.reset();
            uint32_t n = 0;
            for (int b = kBins - 1; b > 0; b--) {
                acc.grow(bb[b]);
                n += bc[b];
                rightArea[b] = acc.area();
                rightCount[b] = n;
            }
            acc.reset();
            n = 0;
            for (int b = 0; b < kBins - 1; b++) {
                acc.grow(bb[b]);
                n += bc[b];
                if (n == 0 || rightCount[b + 1] == 0) continue;
                float cost = acc.area() * float(n) + rightArea[b + 1] * float(rightCount[b + 1]);
                if (cost < bestCost) { bestCost = cost; bestAxis = a; bestSplit = b; }
            }
        }
        const float leafCost = box.area() * float(count);
        const float travCost = box.area() * 0.5f;
        if (count <= kMaxLeaf && (bestAxis < 0 || leafCost <= bestCost + travCost)) {
            nd.first = first;
            nd.count = count;
            return;
        }
        uint32_t mid;
        if (bestAxis < 0) {
            mid = first + count / 2;  // all centroids equal: split by index
        } else {
            const float ext = cbox.hi[bestAxis] - cbox.lo[bestAxis];
            const float k = float(kBins) * (1.f - 1e-6f) / ext;
            auto it = std::partition(idx.begin() + first, idx.begin() + first + count, [&](uint32_t t) {
                int b = std::min(kBins - 1, int((cen[size_t(t) * 3 + bestAxis] - cbox.lo[bestAxis]) * k));
                return b <= bestSplit;
            });
            mid = uint32_t(it - idx.begin());
            if (mid == first || mid == first + count) mid = first + count / 2;
        }
        uint32_t l = alloc(), r = alloc();
        nd.left = l;
        nd.right = r;
        nd.count = 0;
        const uint32_t nl = mid - first, nr = first + count - mid;
        if (count > 200000 && depth < 6) {
            auto f = std::async(std::launch::async, [&, l, first, nl, depth] { build(l, first, nl, depth + 1); });
            build(r, mid, nr, depth + 1);
            f.get();
        } else {
            build(l, first, nl, depth + 1);
            build(r, mid, nr, depth + 1);
        }
    }
};

struct Collapse {
    const Builder2& b2;
    const std::vector<float>& triVerts;
    const std::vector<uint32_t>& triInstance;
    const std::vector<uint32_t>& triPrim;
    BVH8& out;
    uint32_t maxDepth = 0;

    static float pow2(int e) { return std::ldexp(1.f, e); }

    // Quantises child boxes of node `n` (slot-ordered) conservatively.
    void quantize(BVH8Node& n, const AABB* boxes, const bool* valid) {
        AABB u;
        u.reset();
        for (int s = 0; s < 8; s++)
            if (valid[s]) u.grow(boxes[s]);
        for (int a = 0; a < 3; a++) n.p[a] = u.lo[a];
        for (int a = 0; a < 3; a++) {
            float ext = u.hi[a] - u.lo[a];
            int e = -126;
            if (ext > 0.f) {
                e = int(std::ceil(std::log2(ext / 255.f)));
                e = std::max(e, -126);
            }
            for (;;) {
                const float scale = pow2(e);
                bool ok = true;
                uint8_t qlo[8], qhi[8];
                for (int s = 0; s < 8; s++) {
                    if (!valid[s]) { qlo[s] = 255; qhi[s] = 0; continue; }
                    const float lo = boxes[s].lo[a], hi = boxes[s].hi[a];
                    int ql = int(std::floor((lo - n.p[a]) / scale));
                    ql = std::min(std::max(ql, 0), 255);
                    while (ql > 0 && std::fma(float(ql), scale, n.p[a]) > lo) ql--;
                    if (std::fma(float(ql), scale, n.p[a]) > lo) { ok = false; break; }
                    int qh = int(std::ceil((hi - n.p[a]) / scale));
                    qh = std::min(std::max(qh, 0), 255);
                    while (qh < 255 && std::fma(float(qh), scale, n.p[a]) < hi) qh++;
                    if (std::fma(float(qh), scale, n.p[a]) < hi) { ok = false; break; }
                    qlo[s] = uint8_t(ql);
                    qhi[s] = uint8_t(qh);
                }
                if (!ok) { e++; if (e > 127) throw std::runtime_error("BVH quantisation failed"); continue; }
                n.e[a] = uint8_t(e + 127);
                uint8_t* L = a == 0 ? n.qlox : (a == 1 ? n.qloy : n.qloz);
                uint8_t* H = a == 0 ? n.qhix : (a == 1 ? n.qhiy : n.qhiz);
                std::memcpy(L, qlo, 8);
                std::memcpy(H, qhi, 8);
                break;
            }
        }
    }

    void emitTri(uint32_t t) {
        TriRecord r;
        std::memcpy(r.v0, &triVerts[size_t(t) * 9 + 0], 12);
        std::memcpy(r.v1, &triVerts[size_t(t) * 9 + 3], 12);
        std::memcpy(r.v2, &triVerts[size_t(t) * 9 + 6], 12);
        r.globalTri = t;
        r.instanceID = triInstance[t];
        r.primIndex = triPrim[t];
        out.tris.push_back(r);
    }

    // Fills BVH8 node `dst` from binary node `src` (breadth first).
    void run(uint32_t root2) {
        struct Job { uint32_t dst, src, depth; };
        std::vector<Job> queue;
        out.nodes.emplace_back();
        queue.push_back({0, root2, 1});
        for (size_t qi = 0; qi < queue.size(); qi++) {
            Job job = queue[qi];
            maxDepth = std::max(maxDepth, job.depth);
            // Gather up to 8 children by opening the largest internal child.
            std::vector<uint32_t> ch;
            const Node2& s = b2.nodes[job.src];
            if (s.count > 0) ch.push_back(job.src);
            else { ch.push_back(s.left); ch.push_back(s.right); }
            while (ch.size() < 8) {
                int best = -1;
                float bestA = -1.f;
                for (size_t i = 0; i < ch.size(); i++) {
                    const Node2& c = b2.nodes[ch[i]];
                    if (c.count == 0 && c.box.area() > bestA) { bestA = c.box.area(); best = int(i); }
                }
                if (best < 0) break;
                const Node2& c = b2.nodes[ch[size_t(best)]];
                ch[size_t(best)] = c.left;
                ch.push_back(c.right);
            }
            // Octant slot assignment: slot k faces corner (k&1 ? +x : -x, k&2 ? +y : -y, k&4 ? +z : -z).
            const Node2& sn = b2.nodes[job.src];
            float pc[3];
            for (int a = 0; a < 3; a++) pc[a] = 0.5f * (sn.box.lo[a] + sn.box.hi[a]);
            int slotOf[8];
            bool slotUsed[8] = {false};
            bool chUsed[8] = {false};
            for (size_t iter = 0; iter < ch.size(); iter++) {
                float best = -std::numeric_limits<float>::max();
                int bi = -1, bs = -1;
                for (size_t i = 0; i < ch.size(); i++) {
                    if (chUsed[i]) continue;
                    const AABB& cb = b2.nodes[ch[i]].box;
                    float d[3];
                    for (int a = 0; a < 3; a++) d[a] = 0.5f * (cb.lo[a] + cb.hi[a]) - pc[a];
                    for (int k = 0; k < 8; k++) {
                        if (slotUsed[k]) continue;
                        float v = (k & 1 ? d[0] : -d[0]) + (k & 2 ? d[1] : -d[1]) + (k & 4 ? d[2] : -d[2]);
                        if (v > best) { best = v; bi = int(i); bs = k; }
                    }
                }
                chUsed[bi] = true;
                slotUsed[bs] = true;
                slotOf[bi] = bs;
            }
            uint32_t slotChild[8];
            bool valid[8] = {false};
            AABB boxes[8];
            for (int k = 0; k < 8; k++) boxes[k].reset();
            for (size_t i = 0; i < ch.size(); i++) {
                slotChild[slotOf[i]] = ch[i];
                valid[slotOf[i]] = true;
                boxes[slotOf[i]] = b2.nodes[ch[i]].box;
            }
            BVH8Node n;
            std::memset(&n, 0, sizeof(n));
            n.imask = 0;
            n.childBase = uint32_t(out.nodes.size());
            n.triBase = uint32_t(out.tris.size());
            uint32_t triOffset = 0;
            for (int k = 0; k < 8; k++) {
                if (!valid[k]) continue;
                const Node2& c = b2.nodes[slotChild[k]];
                if (c.count > 0) {
                    if (c.count > kMaxLeaf) throw std::runtime_error("BVH leaf too large");
                    n.meta[k] = uint8_t((c.count << 5) | triOffset);
                    for (uint32_t t = 0; t < c.count; t++) emitTri(b2.idx[c.first + t]);
                    triOffset += c.count;
                } else {
                    n.imask |= uint8_t(1u << k);
                }
            }
            quantize(n, boxes, valid);
            // Internal children in slot order.
            for (int k = 0; k < 8; k++) {
                if (!(n.imask & (1u << k))) continue;
                uint32_t dst = uint32_t(out.nodes.size());
                out.nodes.emplace_back();
                queue.push_back({dst, slotChild[k], job.depth + 1});
            }
            out.nodes[job.dst] = n;
        }
    }
};

}  // namespace

void decode_child_box(const BVH8Node& n, int slot, float lo[3], float hi[3]) {
    const uint8_t* L[3] = {n.qlox, n.qloy, n.qloz};
    const uint8_t* H[3] = {n.qhix, n.qhiy, n.qhiz};
    for (int a = 0; a < 3; a++) {
        float scale = std::ldexp(1.f, int(n.e[a]) - 127);
        lo[a] = std::fma(float(L[a][slot]), scale, n.p[a]);
        hi[a] = std::fma(float(H[a][slot]), scale, n.p[a]);
    }
}

void build_bvh8(const std::vector<float>& triVerts, const std::vector<uint32_t>& triInstance,
                const std::vector<uint32_t>& triPrim, BVH8& out) {
    auto t0 = std::chrono::steady_clock::now();
    const uint32_t n = uint32_t(triInstance.size());
    out.nodes.clear();
    out.tris.clear();
    if (n == 0) {
        for (int a = 0; a < 3; a++) { out.lo[a] = 0.f; out.hi[a] = 0.f; }
        out.buildSeconds = 0;
        return;
    }
    Builder2 b;
    b.triBox.resize(n);
    b.cen.resize(size_t(n) * 3);
    b.idx.resize(n);
    for (uint32_t t = 0; t < n; t++) {
        AABB bx;
        bx.reset();
        for (int v = 0; v < 3; v++) bx.grow(&triVerts[size_t(t) * 9 + size_t(v) * 3]);
        b.triBox[t] = bx;
        for (int a = 0; a < 3; a++) b.cen[size_t(t) * 3 + a] = 0.5f * (bx.lo[a] + bx.hi[a]);
        b.idx[t] = t;
    }
    b.nodes.resize(size_t(n) * 2 + 1);
    uint32_t root = b.alloc();
    b.build(root, 0, n, 0);
    for (int a = 0; a < 3; a++) { out.lo[a] = b.nodes[root].box.lo[a]; out.hi[a] = b.nodes[root].box.hi[a]; }
    out.nodes.reserve(n / 3 + 16);
    out.tris.reserve(n);
    Collapse c{b, triVerts, triInstance, triPrim, out};
    c.run(root);
    out.maxDepth = c.maxDepth;
    out.buildSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace fpt

struct fpt_bvh {
    fpt::BVH8 bvh;
};

extern "C" {

FPT_API fpt_status fpt_bvh_build(const fpt_scene_desc* d, fpt_bvh** out) {
    using namespace fpt;
    if (!d || !out) return set_error(FPT_ERR_INVALID_ARG, "fpt_bvh_build: null argument");
    *out = nullptr;
    try {
        uint32_t total = 0;
        for (uint32_t i = 0; i < d->instance_count; i++) total += d->instances[i].triangle_count;
        std::vector<float> tv(size_t(total) * 9);
        std::vector<uint32_t> ti(total), tp(total);
        uint32_t g = 0;
        for (uint32_t i = 0; i < d->instance_count; i++) {
            const fpt_geometry_instance& in = d->instances[i];
            for (uint32_t t = 0; t < in.triangle_count; t++, g++) {
                for (int k = 0; k < 3; k++) {
                    const uint32_t vi = d->indices[in.ib_offset + t * 3 + k] + in.vb_offset;
                    if (vi >= d->vertex_count) return set_error(FPT_ERR_INVALID_ARG, "vertex index out of bounds");
                    std::memcpy(&tv[size_t(g) * 9 + size_t(k) * 3], d->vertices[vi].position, 12);
                }
                ti[g] = i;
                tp[g] = t;
            }
        }
        auto* b = new fpt_bvh();
        build_bvh8(tv, ti, tp, b->bvh);
        *out = b;
        return FPT_OK;
    } catch (const std::exception& e) {
        return set_error(FPT_ERR_INVALID_ARG, std::string("fpt_bvh_build: ") + e.what());
    }
}

FPT_API fpt_status fpt_bvh_get_view(const fpt_bvh* b, fpt_bvh_view* out, uint32_t* maxDepth, double* seconds) {
    if (!b || !out) return fpt::set_error(FPT_ERR_INVALID_ARG, "fpt_bvh_get_view: null argument");
    out->nodes = b->bvh.nodes.data();
    out->node_count = uint32_t(b->bvh.nodes.size());
    out->tris = b->bvh.tris.data();
    out->tri_count = uint32_t(b->bvh.tris.size());
    for (int a = 0; a < 3; a++) { out->scene_lo[a] = b->bvh.lo[a]; out->scene_hi[a] = b->bvh.hi[a]; }
    if (maxDepth) *maxDepth = b->bvh.maxDepth;
    if (seconds) *seconds = b->bvh.buildSeconds;
    return FPT_OK;
}

FPT_API void fpt_bvh_free(fpt_bvh* b) { delete b; }

}  // extern "C"
