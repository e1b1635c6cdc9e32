// light_bvh_build.cpp -- the light BVH over the emissive triangles
// (Rendering/Lights/LightBVHBuilder.cpp:228-882) with the options the
// LightBVHSampler uses by default (LightBVHBuilder.h:68-80): binned SAOH splits
// over 16 bins on all three axes, at most 10 triangles per leaf, leaves as soon
// as a range fits, the leaf-creation cost test, pre-integrated flux (triangles
// of zero flux are left out) and lighting cones; nodes in the compressed
// 32-byte format of PackedNode (LightBVHTypes.slang:102-200).
//
// The tree is stored depth first: an internal node's left child follows it,
// the right child's index is in the node.  Every light triangle also gets the
// bit path from the root to its leaf (bit d: right at depth d), used to
// evaluate the selection pdf of a triangle hit by a BSDF-sampled ray.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstring>
#include <limits>
#include <stdexcept>

#include "common.h"

namespace fpt {

namespace {

constexpr float kInvalidCos = -1.f;        // kInvalidCosConeAngle
constexpr uint32_t kMaxDepth = 64;         // bit path length
constexpr uint32_t kMaxLeafTris = 10;      // maxTriangleCountPerLeaf
constexpr uint32_t kBins = 16;             // binCount
constexpr float kPi = 3.14159265358979323846f;
constexpr float kInf = std::numeric_limits<float>::infinity();

struct Vec {
    float x = 0.f, y = 0.f, z = 0.f;
    float operator[](int a) const { return a == 0 ? x : (a == 1 ? y : z); }
};
Vec operator+(Vec a, Vec b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
Vec operator-(Vec a, Vec b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
Vec operator*(Vec a, float s) { return {a.x * s, a.y * s, a.z * s}; }
float dot(Vec a, Vec b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
float length(Vec a) { return std::sqrt(dot(a, a)); }
// normalize as v * rsqrt(dot(v, v)) (Utils/Math/VectorMath.h:1731-1734): a zero
// vector gives NaNs, which the cone code relies on to invalidate empty bins.
Vec normalize(Vec a) { return a * (1.f / std::sqrt(dot(a, a))); }
Vec vmin(Vec a, Vec b) { return {std::min(a.x, b.x), std::min(a.y, b.y), std::min(a.z, b.z)}; }
Vec vmax(Vec a, Vec b) { return {std::max(a.x, b.x), std::max(a.y, b.y), std::max(a.z, b.z)}; }

// AABB (Utils/Math/AABB.h): empty = (+inf, -inf).
struct Box {
    Vec lo{kInf, kInf, kInf};
    Vec hi{-kInf, -kInf, -kInf};
    void grow(const Box& b) {
        lo = vmin(lo, b.lo);
        hi = vmax(hi, b.hi);
    }
    void grow(Vec p) {
        lo = vmin(lo, p);
        hi = vmax(hi, p);
    }
    bool valid() const { return hi.x >= lo.x && hi.y >= lo.y && hi.z >= lo.z; }
    Vec center() const { return (lo + hi) * 0.5f; }
    Vec extent() const { return hi - lo; }
    float area() const {
        const Vec e = extent();
        return (e.x * e.y + e.x * e.z + e.y * e.z) * 2.f;
    }
};

struct LightTri {
    Box bounds;
    Vec coneDir;
    float cosCone = 1.f;
    float flux = 0.f;
    uint32_t index = 0;
};

struct Node {
    bool leaf = false;
    Box box;
    float flux = 0.f;
    Vec coneDir;
    float cosCone = kInvalidCos;
    uint32_t right = 0, triCount = 0, triOffset = 0;
};

float safe_acos(float v) { return std::acos(std::clamp(v, -1.f, 1.f)); }
float sin_from_cos(float c) { return std::sqrt(std::max(0.f, 1.f - c * c)); }

// computeCosConeAngle (LightBVHBuilder.cpp:66-89).
float cos_cone_angle(Vec coneDir, float cosTheta, Vec otherDir, float cosOther) {
    float r = kInvalidCos;
    if (cosTheta != kInvalidCos && cosOther != kInvalidCos) {
        const float cosDiff = dot(coneDir, otherDir);
        const float sinDiff = sin_from_cos(cosDiff);
        const float sinOther = sin_from_cos(cosOther);
        const float cosTotal = cosOther * cosDiff - sinOther * sinDiff;
        const float sinTotal = sinOther * cosDiff + cosOther * sinDiff;
        if (sinTotal > 0.f) r = std::min(cosTheta, cosTotal);
    }
    return r;
}

// coneUnionOld (LightBVHBuilder.cpp:94-109), the union used for internal nodes.
Vec cone_union(Vec a, float aCos, Vec b, float bCos, float& cosResult) {
    Vec dir = a + b;
    if (aCos == kInvalidCos || bCos == kInvalidCos || (dir.x == 0.f && dir.y == 0.f && dir.z == 0.f)) {
        cosResult = kInvalidCos;
        return Vec{};
    }
    dir = normalize(dir);
    const float aDiff = safe_acos(dot(dir, a));
    const float bDiff = safe_acos(dot(dir, b));
    cosResult = std::cos(std::max(aDiff + std::acos(aCos), bDiff + std::acos(bCos)));
    return dir;
}

// computeOrientationCost (LightBVHBuilder.cpp:659-665), flat diffuse emitters.
float orientation_cost(float thetaO) {
    const float thetaW = std::min(thetaO + kPi * 0.5f, kPi);
    const float s = std::sin(thetaO), c = std::cos(thetaO);
    return 2.f * kPi * (1.f - c) + kPi * 0.5f * (2.f * thetaW * s - std::cos(thetaO - 2.f * thetaW) - 2.f * thetaO * s + c);
}

// evalSAOH (LightBVHBuilder.cpp:671-680).
float eval_saoh(const Box& b, float flux, float cosTheta) {
    const float area = b.valid() ? b.area() : 0.f;
    const float theta = cosTheta != kInvalidCos ? safe_acos(cosTheta) : kPi;
    return flux * area * orientation_cost(theta);
}

struct Builder {
    std::vector<LightTri> tris;
    std::vector<Node> nodes;
    std::vector<uint32_t> triIndices;
    std::vector<uint64_t> bitmasks;
    float currentFlux = 0.f;

    // computeLightingCone (LightBVHBuilder.cpp:475-498).
    Vec lighting_cone(uint32_t b, uint32_t e, float& cosTheta) const {
        Vec dir{};
        cosTheta = kInvalidCos;
        Vec sum{};
        for (uint32_t i = b; i < e; i++) sum = sum + tris[i].coneDir;
        if (length(sum) >= FLT_MIN) {
            dir = normalize(sum);
            cosTheta = 1.f;
            for (uint32_t i = b; i < e; i++) cosTheta = cos_cone_angle(dir, cosTheta, tris[i].coneDir, tris[i].cosCone);
        }
        return dir;
    }

    struct Split {
        uint32_t axis = ~0u, index = ~0u;
        bool valid() const { return axis != ~0u && index != ~0u; }
    };

    // computeSplitWithEqual (LightBVHBuilder.cpp:500-513).
    static Split split_equal(uint32_t b, uint32_t e, const Box& nb) {
        const Vec d = nb.extent();
        Split s;
        s.axis = d.z >= d.x && d.z >= d.y ? 2u : (d.y >= d.x ? 1u : 0u);
        s.index = (b + e) / 2;
        return s;
    }

    struct Bin {
        Box bounds;
        uint32_t count = 0;
        float flux = 0.f;
        Vec coneDir{};
        float cosCone = 1.f;
        void add(const Bin& o) {
            bounds.grow(o.bounds);
            count += o.count;
            flux += o.flux;
            coneDir = coneDir + o.coneDir;
        }
    };

    // computeSplitWithBinnedSAOH (LightBVHBuilder.cpp:682-858).
    Split split_saoh(uint32_t b, uint32_t e, const Box& nb) const {
        float bestCost = std::numeric_limits<float>::infinity();
        Split best;
        const Vec dims = nb.extent();
        const uint32_t largest = dims.z >= dims.x && dims.z >= dims.y ? 2u : (dims.y >= dims.x && dims.y >= dims.z ? 1u : 0u);
        Bin bins[kBins];
        float costs[kBins - 1];
        for (uint32_t axis = 0; axis < 3; axis++) {
            const float bmin = nb.lo[int(axis)], bmax = nb.hi[int(axis)];
            const float w = bmax - bmin;
            const float scale = w > FLT_MIN ? float(kBins) / w : 0.f;
            auto binOf = [&](const LightTri& t) {
                const float p = t.bounds.center()[int(axis)];
                return std::min(uint32_t((p - bmin) * scale), kBins - 1);
            };
            for (Bin& bin : bins) bin = Bin();
            for (uint32_t i = b; i < e; i++) {
                Bin one;
                one.bounds = tris[i].bounds;
                one.count = 1;
                one.flux = tris[i].flux;
                one.coneDir = tris[i].coneDir;
                one.cosCone = tris[i].cosCone;
                bins[binOf(tris[i])].add(one);
            }
            for (Bin& bin : bins) {
                bin.cosCone = length(bin.coneDir) < FLT_MIN ? kInvalidCos : 1.f;
                bin.coneDir = normalize(bin.coneDir);
            }
            for (uint32_t i = b; i < e; i++) {
                Bin& bin = bins[binOf(tris[i])];
                bin.cosCone = cos_cone_angle(bin.coneDir, bin.cosCone, tris[i].coneDir, tris[i].cosCone);
            }
            // Left-to-right sweep: cost of bins 0..i.
            Bin total;
            for (uint32_t i = 0; i < kBins - 1; i++) {
                total.add(bins[i]);
                float cosTheta = kInvalidCos;
                if (length(total.coneDir) >= FLT_MIN) {
                    cosTheta = 1.f;
                    const Vec dir = normalize(total.coneDir);
                    for (uint32_t j = 0; j <= i; j++) cosTheta = cos_cone_angle(dir, cosTheta, bins[j].coneDir, bins[j].cosCone);
                }
                costs[i] = eval_saoh(total.bounds, total.flux, cosTheta);
            }
            // Right-to-left sweep: cost of bins i..n-1.
            total = Bin();
            for (uint32_t i = kBins - 1; i > 0; i--) {
                total.add(bins[i]);
                float cosTheta = kInvalidCos;
                if (length(total.coneDir) >= FLT_MIN) {
                    cosTheta = 1.f;
                    const Vec dir = normalize(total.coneDir);
                    for (uint32_t j = i; j <= kBins - 1; j++) cosTheta = cos_cone_angle(dir, cosTheta, bins[j].coneDir, bins[j].cosCone);
                }
                costs[i - 1] += eval_saoh(total.bounds, total.flux, cosTheta);
            }
            float axisCost = std::numeric_limits<float>::infinity();
            Split axisSplit;
            axisSplit.axis = axis;
            axisSplit.index = 0;
            for (uint32_t i = 0, idx = b; i < kBins - 1; i++) {
                idx += bins[i].count;
                if (costs[i] < axisCost) {
                    axisCost = costs[i];
                    axisSplit.index = idx;
                }
            }
            // Discourage long skinny nodes.
            axisCost *= dims[int(largest)] / dims[int(axis)];
            if (axisSplit.index == b || axisSplit.index == e) continue;
            if (axisCost < bestCost) {
                bestCost = axisCost;
                best = axisSplit;
            }
        }
        if (!best.valid()) {
            if (e - b <= kMaxLeafTris) return Split();
            return split_equal(b, e, nb);
        }
        if (e - b <= kMaxLeafTris) {
            float cosTheta = kInvalidCos;
            lighting_cone(b, e, cosTheta);
            const float leafCost = eval_saoh(nb, currentFlux, cosTheta);
            if (leafCost <= bestCost) return Split();
        }
        return best;
    }

    // buildInternal (LightBVHBuilder.cpp:352-438).
    uint32_t build(uint64_t bitmask, uint32_t depth, uint32_t b, uint32_t e) {
        float flux = 0.f;
        Box nb;
        for (uint32_t i = b; i < e; i++) {
            nb.grow(tris[i].bounds);
            flux += tris[i].flux;
        }
        currentFlux = flux;
        const bool trySplit = e - b > kMaxLeafTris;
        const Split s = trySplit ? split_saoh(b, e, nb) : Split();
        const uint32_t index = uint32_t(nodes.size());
        nodes.emplace_back();
        if (s.valid()) {
            const int axis = int(s.axis);
            std::nth_element(tris.begin() + b, tris.begin() + s.index, tris.begin() + e,
                             [axis](const LightTri& a, const LightTri& c) { return a.bounds.center()[axis] < c.bounds.center()[axis]; });
            if (depth >= kMaxDepth) throw std::runtime_error("light BVH deeper than 64 levels");
            Node n;
            n.box = nb;
            n.flux = flux;
            build(bitmask, depth + 1, b, s.index);
            n.right = build(bitmask | (1ull << depth), depth + 1, s.index, e);
            nodes[index] = n;
        } else {
            Node n;
            n.leaf = true;
            n.box = nb;
            n.flux = flux;
            n.coneDir = lighting_cone(b, e, n.cosCone);
            n.triCount = e - b;
            n.triOffset = uint32_t(triIndices.size());
            for (uint32_t i = b; i < e; i++) {
                triIndices.push_back(tris[i].index);
                bitmasks[tris[i].index] = bitmask;
            }
            nodes[index] = n;
        }
        return index;
    }

    // computeLightingConesInternal (LightBVHBuilder.cpp:440-473).
    Vec cones(uint32_t i, float& cosCone) {
        Node& n = nodes[i];
        if (n.leaf) {
            cosCone = n.cosCone;
            return n.coneDir;
        }
        float cl = kInvalidCos, cr = kInvalidCos;
        const Vec dl = cones(i + 1, cl);
        const Vec dr = cones(nodes[i].right, cr);
        Node& m = nodes[i];
        m.coneDir = cone_union(dl, cl, dr, cr, cosCone);
        m.cosCone = cosCone;
        return m.coneDir;
    }
};

}  // namespace

void build_light_bvh(const std::vector<float>& triVerts, const std::vector<float>& triNormals, const std::vector<float>& flux,
                     LightBVH& out) {
    out.nodes.clear();
    out.triIndices.clear();
    const size_t n = flux.size();
    out.bitmasks.assign(n, ~0ull);
    Builder bld;
    for (size_t i = 0; i < n; i++) {
        if (!(flux[i] > 0.f)) continue;  // pre-integration culls lights without flux
        LightTri t;
        for (int k = 0; k < 3; k++) t.bounds.grow(Vec{triVerts[9 * i + 3 * k], triVerts[9 * i + 3 * k + 1], triVerts[9 * i + 3 * k + 2]});
        t.coneDir = Vec{triNormals[3 * i], triNormals[3 * i + 1], triNormals[3 * i + 2]};
        t.cosCone = 1.f;
        t.flux = flux[i];
        t.index = uint32_t(i);
        bld.tris.push_back(t);
    }
    if (bld.tris.empty()) return;
    if (bld.tris.size() > (size_t(1) << 27) + 16) throw std::runtime_error("too many emissive triangles for the light BVH");
    bld.bitmasks.assign(n, ~0ull);
    bld.build(0ull, 0, 0, uint32_t(bld.tris.size()));
    float c = 0.f;
    bld.cones(0, c);
    out.bitmasks = bld.bitmasks;
    out.triIndices = bld.triIndices;
    out.nodes.resize(bld.nodes.size());
    for (size_t i = 0; i < bld.nodes.size(); i++) {
        const Node& s = bld.nodes[i];
        LightBVHNode& d = out.nodes[i];
        // PackedNode::setInternalNode / setLeafNode / setNodeAttributes (compressed).
        d.w[0] = s.leaf ? ((1u << 31) | (s.triCount << 27) | s.triOffset) : s.right;
        const Vec origin = (s.box.hi + s.box.lo) * 0.5f;
        const Vec extent = (s.box.hi - s.box.lo) * 0.5f;
        std::memcpy(&d.w[1], &origin.x, 4);
        std::memcpy(&d.w[2], &origin.y, 4);
        std::memcpy(&d.w[3], &origin.z, 4);
        const uint32_t packedAngle = uint32_t((s.cosCone + 1.f) * 32767.f);
        d.w[4] = uint32_t(f32_to_f16_host(extent.x)) | (uint32_t(f32_to_f16_host(extent.y)) << 16);
        d.w[5] = uint32_t(f32_to_f16_host(extent.z)) | (packedAngle << 16);
        const float cd[3] = {s.coneDir.x, s.coneDir.y, s.coneDir.z};
        d.w[6] = encode_normal_2x16_host(cd);
        std::memcpy(&d.w[7], &s.flux, 4);
    }
}

}  // namespace fpt
