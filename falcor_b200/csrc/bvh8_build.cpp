// bvh8_build.cpp -- host builder of the compressed 8-wide BVH.
//
// The reference path has no software triangle BVH (DXR builds the
// acceleration structures in the driver, Scene::buildBlas Scene.cpp:3376), so
// this is new work: a binned-SAH binary BVH with spatial splits (leaves of at
// most 3 triangle references), collapsed to 8-wide nodes by repeatedly opening the largest child, with the
// child slots ordered by direction octant so that traversal can visit them
// approximately front to back, and the child boxes quantised to 8 bits per
// plane relative to a per-node origin and power-of-two scale.  Quantisation is
// conservative with respect to the exact device decoding, fmaf(q, scale, p).
#include <algorithm>
#include <array>
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

// Leaf size limit (the node's leaf meta byte holds a 3-bit count and a 5-bit
// offset into a 32-triangle window, so 8 leaves of at most 4 triangles fit)
// and the SAH cost of a binary traversal step relative to one triangle test.
#ifndef FPT_BVH_MAX_LEAF
#define FPT_BVH_MAX_LEAF 3
#endif
#ifndef FPT_BVH_TRAV_COST
#define FPT_BVH_TRAV_COST 0.5f
#endif
constexpr uint32_t kMaxLeaf = FPT_BVH_MAX_LEAF;
static_assert(kMaxLeaf >= 1 && kMaxLeaf * 8 <= 32, "leaf triangles of a node must fit the 32-bit window");
#ifndef FPT_BVH_BINS
#define FPT_BVH_BINS 16
#endif
constexpr int kBins = FPT_BVH_BINS;

// Spatial splits (split BVH): a node may also split at a plane through its
// box, cutting the triangles that straddle the plane into two references
// whose boxes bound only the triangle's part on each side.  They are tried when
// the best object split's children overlap by more than kSplitAlpha of the
// root's area, within a budget of extra references (a fraction of the triangle
// count, handed down in proportion to the references of each subtree so that
// the tree does not depend on thread timing).  A triangle can then sit in
// several leaves; every copy is a full triangle record, so traversal results
// are unchanged (a repeated test finds the same t and triangle index).
#ifndef FPT_BVH_SPLIT_BUDGET
#define FPT_BVH_SPLIT_BUDGET 1.0
#endif
constexpr double kSplitBudget = FPT_BVH_SPLIT_BUDGET;
#ifndef FPT_BVH_SPLIT_ALPHA
#define FPT_BVH_SPLIT_ALPHA 1e-4f
#endif
constexpr float kSplitAlpha = FPT_BVH_SPLIT_ALPHA;
// Collapse of the binary tree into 8-wide nodes: 1 = SAH-optimal (dynamic
// programming, with kPrimCost the cost of a reference test relative to a node
// visit), 0 = repeatedly open the child of largest area.
#ifndef FPT_BVH_COLLAPSE_DP
#define FPT_BVH_COLLAPSE_DP 0
#endif
#ifndef FPT_BVH_PRIM_COST
#define FPT_BVH_PRIM_COST 0.3
#endif
#ifndef FPT_BVH_SPATIAL_BINS
#define FPT_BVH_SPATIAL_BINS 32
#endif
constexpr int kSpatialBins = FPT_BVH_SPATIAL_BINS;

struct Ref {
    AABB box;
    uint32_t tri;
};

// Rounds a double down / up to a float that bounds it.
inline float round_down(double v) {
    float f = float(v);
    if (double(f) > v) f = std::nextafter(f, -std::numeric_limits<float>::infinity());
    return f;
}
inline float round_up(double v) {
    float f = float(v);
    if (double(f) < v) f = std::nextafter(f, std::numeric_limits<float>::infinity());
    return f;
}

struct Builder2 {
    const std::vector<float>* verts = nullptr;  // 9 floats per triangle
    std::vector<Node2> nodes;
    std::vector<uint32_t> leafTris;  // triangle of each leaf reference
    std::atomic<uint32_t> nextNode{0};
    std::atomic<uint32_t> nextLeaf{0};
    float minOverlap = 0.f;

    uint32_t alloc() {
        uint32_t n = nextNode.fetch_add(1);
        if (n >= nodes.size()) throw std::runtime_error("BVH node pool exhausted");
        return n;
    }

    // Bounds of triangle t's part inside lo <= x[a] <= hi (double precision,
    // rounded outward), intersected with `within`.  Returns false when the
    // part is empty.
    bool clip(uint32_t t, int a, float lo, float hi, const AABB& within, AABB& out) const {
        const float* v = &(*verts)[size_t(t) * 9];
        double blo[3] = {INFINITY, INFINITY, INFINITY}, bhi[3] = {-INFINITY, -INFINITY, -INFINITY};
        auto grow = [&](const double* q) {
            for (int k = 0; k < 3; k++) { blo[k] = std::min(blo[k], q[k]); bhi[k] = std::max(bhi[k], q[k]); }
        };
        for (int e = 0; e < 3; e++) {
            const float* pf = v + e * 3;
            const float* qf = v + ((e + 1) % 3) * 3;
            const double P[3] = {pf[0], pf[1], pf[2]}, Q[3] = {qf[0], qf[1], qf[2]};
            if (P[a] >= lo && P[a] <= hi) grow(P);
            for (const double c : {double(lo), double(hi)}) {
                if ((P[a] < c && Q[a] > c) || (P[a] > c && Q[a] < c)) {
                    const double f = (c - P[a]) / (Q[a] - P[a]);
                    double X[3];
                    for (int k = 0; k < 3; k++) X[k] = P[k] + f * (Q[k] - P[k]);
                    X[a] = c;
                    grow(X);
                }
            }
        }
        if (!(blo[0] <= bhi[0])) return false;
        for (int k = 0; k < 3; k++) {
            out.lo[k] = std::max(round_down(blo[k]), within.lo[k]);
            out.hi[k] = std::min(round_up(bhi[k]), within.hi[k]);
        }
        out.lo[a] = std::max(out.lo[a], lo);
        out.hi[a] = std::min(out.hi[a], hi);
        for (int k = 0; k < 3; k++)
            if (out.lo[k] > out.hi[k]) return false;
        return true;
    }

    void make_leaf(Node2& nd, const std::vector<Ref>& refs) {
        const uint32_t first = nextLeaf.fetch_add(uint32_t(refs.size()));
        if (size_t(first) + refs.size() > leafTris.size()) throw std::runtime_error("BVH reference pool exhausted");
        for (size_t i = 0; i < refs.size(); i++) leafTris[first + i] = refs[i].tri;
        nd.first = first;
        nd.count = uint32_t(refs.size());
    }

    void build(uint32_t node, std::vector<Ref>& refs, int depth, int64_t budget) {
        Node2& nd = nodes[node];
        const uint32_t count = uint32_t(refs.size());
        AABB box, cbox;
        box.reset();
        cbox.reset();
        for (const Ref& r : refs) {
            box.grow(r.box);
            float c[3];
            for (int a = 0; a < 3; a++) c[a] = 0.5f * (r.box.lo[a] + r.box.hi[a]);
            cbox.grow(c);
        }
        nd.box = box;
        if (count <= 1) { make_leaf(nd, refs); return; }
        // Binned SAH object split over the three axes.
        float bestCost = std::numeric_limits<float>::max();
        int bestAxis = -1, bestSplit = -1;
        AABB bestL, bestR;
        for (int a = 0; a < 3; a++) {
            float ext = cbox.hi[a] - cbox.lo[a];
            if (!(ext > 0.f)) continue;
            AABB bb[kBins];
            uint32_t bc[kBins] = {0};
            for (auto& b : bb) b.reset();
            const float k = float(kBins) * (1.f - 1e-6f) / ext;
            for (const Ref& r : refs) {
                int b = std::min(kBins - 1, int((0.5f * (r.box.lo[a] + r.box.hi[a]) - cbox.lo[a]) * k));
                bb[b].grow(r.box);
                bc[b]++;
            }
            AABB rightBox[kBins];
            uint32_t rightCount[kBins];
            AABB acc;
            acc.reset();
            uint32_t n = 0;
            for (int b = kBins - 1; b > 0; b--) {
                acc.grow(bb[b]);
                n += bc[b];
                rightBox[b] = acc;
                rightCount[b] = n;
            }
            acc.reset();
            n = 0;
            for (int b = 0; b < kBins - 1; b++) {
                acc.grow(bb[b]);
                n += bc[b];
                if (n == 0 || rightCount[b + 1] == 0) continue;
                float cost = acc.area() * float(n) + rightBox[b + 1].area() * float(rightCount[b + 1]);
                if (cost < bestCost) { bestCost = cost; bestAxis = a; bestSplit = b; bestL = acc; bestR = rightBox[b + 1]; }
            }
        }
        // Spatial split, when the object split's children overlap.
        int spatialAxis = -1;
        float spatialPos = 0.f;
        if (budget > 0 && depth < 40) {
            float overlap = 0.f;
            if (bestAxis >= 0) {
                AABB o;
                for (int a = 0; a < 3; a++) { o.lo[a] = std::max(bestL.lo[a], bestR.lo[a]); o.hi[a] = std::min(bestL.hi[a], bestR.hi[a]); }
                overlap = (o.lo[0] <= o.hi[0] && o.lo[1] <= o.hi[1] && o.lo[2] <= o.hi[2]) ? o.area() : 0.f;
            }
            if (bestAxis < 0 || overlap > minOverlap) {
                for (int a = 0; a < 3; a++) {
                    const float ext = box.hi[a] - box.lo[a];
                    if (!(ext > 0.f)) continue;
                    float planes[kSpatialBins + 1];
                    for (int b = 0; b <= kSpatialBins; b++) planes[b] = box.lo[a] + ext * (float(b) / float(kSpatialBins));
                    planes[kSpatialBins] = box.hi[a];
                    const float k = float(kSpatialBins) / ext;
                    auto binOf = [&](float x) { return std::min(kSpatialBins - 1, std::max(0, int((x - box.lo[a]) * k))); };
                    AABB bb[kSpatialBins];
                    uint32_t enter[kSpatialBins] = {0}, exit[kSpatialBins] = {0};
                    for (auto& b : bb) b.reset();
                    for (const Ref& r : refs) {
                        const int b0 = binOf(r.box.lo[a]), b1 = binOf(r.box.hi[a]);
                        if (b0 == b1) {
                            bb[b0].grow(r.box);
                        } else {
                            for (int b = b0; b <= b1; b++) {
                                AABB c;
                                if (clip(r.tri, a, planes[b], planes[b + 1], r.box, c)) bb[b].grow(c);
                            }
                        }
                        enter[b0]++;
                        exit[b1]++;
                    }
                    AABB rightBox[kSpatialBins];
                    uint32_t rightCount[kSpatialBins];
                    AABB acc;
                    acc.reset();
                    uint32_t n = 0;
                    for (int b = kSpatialBins - 1; b > 0; b--) {
                        acc.grow(bb[b]);
                        n += exit[b];
                        rightBox[b] = acc;
                        rightCount[b] = n;
                    }
                    acc.reset();
                    n = 0;
                    for (int b = 0; b < kSpatialBins - 1; b++) {
                        acc.grow(bb[b]);
                        n += enter[b];
                        if (n == 0 || rightCount[b + 1] == 0) continue;
                        const float cost = acc.area() * float(n) + rightBox[b + 1].area() * float(rightCount[b + 1]);
                        if (cost < bestCost && int64_t(n) + int64_t(rightCount[b + 1]) - int64_t(count) <= budget) {
                            bestCost = cost;
                            spatialAxis = a;
                            spatialPos = planes[b + 1];
                        }
                    }
                }
            }
        }
        const float leafCost = box.area() * float(count);
        const float travCost = box.area() * float(FPT_BVH_TRAV_COST);
        if (count <= kMaxLeaf && ((bestAxis < 0 && spatialAxis < 0) || leafCost <= bestCost + travCost)) {
            make_leaf(nd, refs);
            return;
        }
        std::vector<Ref> left, right;
        if (spatialAxis >= 0) {
            const int a = spatialAxis;
            for (const Ref& r : refs) {
                if (r.box.hi[a] <= spatialPos) left.push_back(r);
                else if (r.box.lo[a] >= spatialPos) right.push_back(r);
                else {
                    Ref l{r.box, r.tri}, q{r.box, r.tri};
                    const bool hasL = clip(r.tri, a, -std::numeric_limits<float>::max(), spatialPos, r.box, l.box);
                    const bool hasR = clip(r.tri, a, spatialPos, std::numeric_limits<float>::max(), r.box, q.box);
                    if (hasL) left.push_back(l);
                    if (hasR) right.push_back(q);
                    if (!hasL && !hasR) left.push_back(r);  // cannot happen for a straddling box; keep the reference
                }
            }
            if (left.empty() || right.empty() || (left.size() == count && right.size() == count)) {
                left.clear();
                right.clear();
                spatialAxis = -1;
            }
        }
        if (spatialAxis < 0) {
            if (bestAxis < 0) {
                // All centroids equal: split by position in the list.
                left.assign(refs.begin(), refs.begin() + count / 2);
                right.assign(refs.begin() + count / 2, refs.end());
            } else {
                const float ext = cbox.hi[bestAxis] - cbox.lo[bestAxis];
                const float k = float(kBins) * (1.f - 1e-6f) / ext;
                for (const Ref& r : refs) {
                    int b = std::min(kBins - 1, int((0.5f * (r.box.lo[bestAxis] + r.box.hi[bestAxis]) - cbox.lo[bestAxis]) * k));
                    (b <= bestSplit ? left : right).push_back(r);
                }
                if (left.empty() || right.empty()) {
                    left.assign(refs.begin(), refs.begin() + count / 2);
                    right.assign(refs.begin() + count / 2, refs.end());
                }
            }
        }
        const int64_t extra = int64_t(left.size() + right.size()) - int64_t(count);
        const int64_t rest = std::max<int64_t>(0, budget - extra);
        const int64_t budgetL = int64_t(double(rest) * double(left.size()) / double(left.size() + right.size()));
        const int64_t budgetR = rest - budgetL;
        std::vector<Ref>().swap(refs);
        uint32_t l = alloc(), r = alloc();
        nd.left = l;
        nd.right = r;
        nd.count = 0;
        if (count > 200000 && depth < 6) {
            auto f = std::async(std::launch::async, [&, l, depth, budgetL] { build(l, left, depth + 1, budgetL); });
            build(r, right, depth + 1, budgetR);
            f.get();
        } else {
            build(l, left, depth + 1, budgetL);
            build(r, right, depth + 1, budgetR);
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

    // SAH-optimal collapse (dynamic programming over the binary tree): cost[n][j]
    // is the least expected cost of covering the subtree of binary node n with
    // at most j+1 roots, each root an 8-wide node (visit cost kNodeCost times its
    // area) or a leaf of at most kMaxLeaf references (kPrimCost per reference
    // times its area).  Children are allocated after their parent, so a reverse
    // sweep over the node indices sees both children of a node first.
    std::vector<std::array<float, 8>> cost;
    std::vector<std::array<uint8_t, 8>> how;  // j > 0: 0 = fewer roots, k = k roots on the left; j = 0: 1 leaf, 2 node
    std::vector<uint8_t> nodeSplit;           // 8-wide node: (roots on the left) | (all roots << 4)
    std::vector<uint32_t> refs;

    void optimise(uint32_t nodeCount) {
        const float kNodeCost = 1.f, kPrimCost = float(FPT_BVH_PRIM_COST);
        const float inf = std::numeric_limits<float>::infinity();
        cost.assign(nodeCount, {});
        how.assign(nodeCount, {});
        nodeSplit.assign(nodeCount, 0);
        refs.assign(nodeCount, 0);
        for (uint32_t n = nodeCount; n-- > 0;) {
            const Node2& nd = b2.nodes[n];
            const float A = nd.box.area();
            auto& C = cost[n];
            auto& H = how[n];
            if (nd.count > 0) {
                refs[n] = nd.count;
                C.fill(A * kPrimCost * float(nd.count));
                H.fill(0);
                H[0] = 1;
                continue;
            }
            refs[n] = refs[nd.left] + refs[nd.right];
            const auto& L = cost[nd.left];
            const auto& R = cost[nd.right];
            float dist[8];
            uint8_t distK[8];
            float best = inf;
            uint8_t bestJ = 0;
            for (int j = 1; j < 8; j++) {  // j + 1 roots
                dist[j] = inf;
                distK[j] = 0;
                for (int k = 1; k <= j; k++) {  // k roots on the left, j + 1 - k on the right
                    const float c = L[k - 1] + R[j - k];
                    if (c < dist[j]) { dist[j] = c; distK[j] = uint8_t(k); }
                }
                if (dist[j] < best) { best = dist[j]; bestJ = uint8_t(j); }
            }
            nodeSplit[n] = uint8_t(distK[bestJ] | ((bestJ + 1) << 4));
            const float nodeC = A * kNodeCost + best;
            const float leafC = refs[n] <= kMaxLeaf ? A * kPrimCost * float(refs[n]) : inf;
            C[0] = std::min(leafC, nodeC);
            H[0] = leafC <= nodeC ? 1 : 2;
            for (int j = 1; j < 8; j++) {
                if (C[j - 1] <= dist[j]) { C[j] = C[j - 1]; H[j] = 0; }
                else { C[j] = dist[j]; H[j] = distK[j]; }
            }
        }
    }

    struct Slot { uint32_t node; bool leaf; };
    void gather(uint32_t n, int roots, std::vector<Slot>& out2) const {
        const int j = roots - 1;
        if (j == 0) { out2.push_back({n, how[n][0] == 1}); return; }
        const uint8_t h = how[n][size_t(j)];
        if (h == 0) { gather(n, roots - 1, out2); return; }
        gather(b2.nodes[n].left, h, out2);
        gather(b2.nodes[n].right, roots - h, out2);
    }
    void leaf_refs(uint32_t n, std::vector<uint32_t>& out2) const {
        const Node2& nd = b2.nodes[n];
        if (nd.count > 0) {
            for (uint32_t t = 0; t < nd.count; t++) out2.push_back(b2.leafTris[nd.first + t]);
            return;
        }
        leaf_refs(nd.left, out2);
        leaf_refs(nd.right, out2);
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
            std::vector<uint32_t> ch;
            std::vector<bool> chLeaf;
            const Node2& s = b2.nodes[job.src];
            if (!cost.empty()) {
                // Children chosen by the SAH-optimal collapse.
                std::vector<Slot> slots;
                if (s.count > 0) slots.push_back({job.src, true});
                else {
                    const uint32_t k = nodeSplit[job.src] & 15u, all = nodeSplit[job.src] >> 4;
                    gather(s.left, int(k), slots);
                    gather(s.right, int(all - k), slots);
                }
                for (const Slot& sl : slots) { ch.push_back(sl.node); chLeaf.push_back(sl.leaf); }
            } else {
                // Gather up to 8 children by opening the largest internal child.
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
                for (uint32_t c : ch) chLeaf.push_back(b2.nodes[c].count > 0);
            }
            if (ch.size() > 8) throw std::runtime_error("BVH collapse produced more than 8 children");
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
            bool slotLeaf[8] = {false};
            bool valid[8] = {false};
            AABB boxes[8];
            for (int k = 0; k < 8; k++) boxes[k].reset();
            for (size_t i = 0; i < ch.size(); i++) {
                slotChild[slotOf[i]] = ch[i];
                slotLeaf[slotOf[i]] = chLeaf[i];
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
                if (slotLeaf[k]) {
                    std::vector<uint32_t> lr;
                    leaf_refs(slotChild[k], lr);
                    if (lr.empty() || lr.size() > kMaxLeaf) throw std::runtime_error("BVH leaf too large");
                    n.meta[k] = uint8_t((lr.size() << 5) | triOffset);
                    for (uint32_t t : lr) emitTri(t);
                    triOffset += uint32_t(lr.size());
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
    b.verts = &triVerts;
    std::vector<Ref> refs(n);
    for (uint32_t t = 0; t < n; t++) {
        refs[t].box.reset();
        for (int v = 0; v < 3; v++) refs[t].box.grow(&triVerts[size_t(t) * 9 + size_t(v) * 3]);
        refs[t].tri = t;
    }
    const int64_t budget = int64_t(double(n) * kSplitBudget);
    const size_t maxRefs = size_t(n) + size_t(budget);
    b.nodes.resize(maxRefs * 2 + 1);
    b.leafTris.resize(maxRefs);
    AABB rootBox;
    rootBox.reset();
    for (const Ref& r : refs) rootBox.grow(r.box);
    b.minOverlap = kSplitAlpha * rootBox.area();
    uint32_t root = b.alloc();
    b.build(root, refs, 0, budget);
    for (int a = 0; a < 3; a++) { out.lo[a] = b.nodes[root].box.lo[a]; out.hi[a] = b.nodes[root].box.hi[a]; }
    out.nodes.reserve(maxRefs / 3 + 16);
    out.tris.reserve(maxRefs);
    Collapse c{b, triVerts, triInstance, triPrim, out};
    if (FPT_BVH_COLLAPSE_DP) c.optimise(b.nextNode.load());
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
