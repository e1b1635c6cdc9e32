// oracle_lightbvh.h -- CPU restatement of the light BVH and its sampler:
// LightBVHBuilder::build (Rendering/Lights/LightBVHBuilder.cpp:228-309,
// buildInternal :352-438, binned SAOH :682-858, cones :66-109, :440-498) with
// the LightBVHSampler default options, the compressed PackedNode
// (LightBVHTypes.slang:102-200) and LightBVHSampler (LightBVHSampler.slang:70-534:
// traverseTree, computeImportance, pickTriangle with uniform leaf selection,
// evalTriangleSelectionPdf).
//
// TEST INFRASTRUCTURE ONLY (see oracle_math.h).
#pragma once

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <stdexcept>
#include <vector>

namespace orc {

struct LightBvhOracle {
    std::vector<uint32_t> nodes;        // 8 words per compressed node
    std::vector<uint32_t> triIndices;   // leaf order
    std::vector<uint64_t> bitmasks;     // per emissive triangle, ~0 if left out
};

namespace lbvh {

struct F3 {
    float v[3] = {0.f, 0.f, 0.f};
    float& operator[](int i) { return v[i]; }
    float operator[](int i) const { return v[i]; }
};
inline F3 f3(float x, float y, float z) { F3 r; r.v[0] = x; r.v[1] = y; r.v[2] = z; return r; }
inline F3 add(const F3& a, const F3& b) { return f3(a[0] + b[0], a[1] + b[1], a[2] + b[2]); }
inline F3 sub(const F3& a, const F3& b) { return f3(a[0] - b[0], a[1] - b[1], a[2] - b[2]); }
inline F3 mul(const F3& a, float s) { return f3(a[0] * s, a[1] * s, a[2] * s); }
inline float dot3(const F3& a, const F3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
inline float len3(const F3& a) { return std::sqrt(dot3(a, a)); }
inline F3 unit(const F3& a) { return mul(a, 1.f / std::sqrt(dot3(a, a))); }  // v * rsqrt(dot(v, v))

constexpr float kInvalid = -1.f;
constexpr float kPiF = 3.14159265358979323846f;

struct AABB {
    F3 mn = f3(std::numeric_limits<float>::infinity(), std::numeric_limits<float>::infinity(), std::numeric_limits<float>::infinity());
    F3 mx = f3(-std::numeric_limits<float>::infinity(), -std::numeric_limits<float>::infinity(), -std::numeric_limits<float>::infinity());
    void include(const AABB& b) {
        for (int a = 0; a < 3; a++) { mn[a] = std::min(mn[a], b.mn[a]); mx[a] = std::max(mx[a], b.mx[a]); }
    }
    void include(const F3& p) {
        for (int a = 0; a < 3; a++) { mn[a] = std::min(mn[a], p[a]); mx[a] = std::max(mx[a], p[a]); }
    }
    bool valid() const { return mx[0] >= mn[0] && mx[1] >= mn[1] && mx[2] >= mn[2]; }
    F3 center() const { return mul(add(mn, mx), 0.5f); }
    F3 extent() const { return sub(mx, mn); }
    float area() const { F3 e = extent(); return (e[0] * e[1] + e[0] * e[2] + e[1] * e[2]) * 2.f; }
};

struct SortTri { AABB bounds; F3 dir; float cosAngle; float flux; uint32_t index; };

inline float sacos(float v) { return std::acos(std::clamp(v, -1.f, 1.f)); }
inline float sin_of(float c) { return std::sqrt(std::max(0.f, 1.f - c * c)); }

inline float grow_cone(const F3& dir, float cosT, const F3& other, float cosO) {
    if (cosT == kInvalid || cosO == kInvalid) return kInvalid;
    const float cd = dot3(dir, other), sd = sin_of(cd), so = sin_of(cosO);
    const float ct = cosO * cd - so * sd, st = so * cd + cosO * sd;
    return st > 0.f ? std::min(cosT, ct) : kInvalid;
}
inline float orientation(float to) {
    const float tw = std::min(to + kPiF * 0.5f, kPiF);
    const float s = std::sin(to), c = std::cos(to);
    return 2.f * kPiF * (1.f - c) + kPiF * 0.5f * (2.f * tw * s - std::cos(to - 2.f * tw) - 2.f * to * s + c);
}
inline float saoh(const AABB& b, float flux, float cosT) {
    const float a = b.valid() ? b.area() : 0.f;
    const float t = cosT != kInvalid ? sacos(cosT) : kPiF;
    return flux * a * orientation(t);
}

struct Rec { bool leaf; AABB box; float flux; F3 dir; float cosAngle; uint32_t right, count, offset; };

struct Build {
    std::vector<SortTri> t;
    std::vector<Rec> recs;
    std::vector<uint32_t> leafTris;
    std::vector<uint64_t> masks;
    float nodeFlux = 0.f;

    F3 cone_of(uint32_t b, uint32_t e, float& c) const {
        F3 sum;
        for (uint32_t i = b; i < e; i++) sum = add(sum, t[i].dir);
        c = kInvalid;
        if (len3(sum) >= FLT_MIN) {
            F3 d = unit(sum);
            c = 1.f;
            for (uint32_t i = b; i < e; i++) c = grow_cone(d, c, t[i].dir, t[i].cosAngle);
            return d;
        }
        return F3();
    }

    // Returns {axis, index}; axis 3 = no split.
    void split(uint32_t b, uint32_t e, const AABB& nb, uint32_t& outAxis, uint32_t& outIdx) const {
        const uint32_t B = 16, maxLeaf = 10;
        const F3 d = nb.extent();
        const uint32_t big = d[2] >= d[0] && d[2] >= d[1] ? 2u : (d[1] >= d[0] && d[1] >= d[2] ? 1u : 0u);
        float best = std::numeric_limits<float>::infinity();
        uint32_t bestAxis = 3, bestIdx = 0;
        struct Bn { AABB box; uint32_t n = 0; float flux = 0.f; F3 dir; float c = 1.f; };
        for (uint32_t ax = 0; ax < 3; ax++) {
            std::vector<Bn> bins(B);
            const float lo = nb.mn[int(ax)], w = nb.mx[int(ax)] - lo;
            const float sc = w > FLT_MIN ? float(B) / w : 0.f;
            auto id = [&](const SortTri& s) { return std::min(uint32_t((s.bounds.center()[int(ax)] - lo) * sc), B - 1); };
            for (uint32_t i = b; i < e; i++) {
                Bn& bn = bins[id(t[i])];
                bn.box.include(t[i].bounds);
                bn.n++;
                bn.flux += t[i].flux;
                bn.dir = add(bn.dir, t[i].dir);
            }
            for (Bn& bn : bins) {
                bn.c = len3(bn.dir) < FLT_MIN ? kInvalid : 1.f;
                bn.dir = unit(bn.dir);
            }
            for (uint32_t i = b; i < e; i++) {
                Bn& bn = bins[id(t[i])];
                bn.c = grow_cone(bn.dir, bn.c, t[i].dir, t[i].cosAngle);
            }
            std::vector<float> cost(B - 1, 0.f);
            Bn acc;
            for (uint32_t i = 0; i + 1 < B; i++) {
                acc.box.include(bins[i].box); acc.n += bins[i].n; acc.flux += bins[i].flux; acc.dir = add(acc.dir, bins[i].dir);
                float c = kInvalid;
                if (len3(acc.dir) >= FLT_MIN) {
                    c = 1.f;
                    F3 u = unit(acc.dir);
                    for (uint32_t j = 0; j <= i; j++) c = grow_cone(u, c, bins[j].dir, bins[j].c);
                }
                cost[i] = saoh(acc.box, acc.flux, c);
            }
            acc = Bn();
            for (uint32_t i = B - 1; i > 0; i--) {
                acc.box.include(bins[i].box); acc.n += bins[i].n; acc.flux += bins[i].flux; acc.dir = add(acc.dir, bins[i].dir);
                float c = kInvalid;
                if (len3(acc.dir) >= FLT_MIN) {
                    c = 1.f;
                    F3 u = unit(acc.dir);
                    for (uint32_t j = i; j < B; j++) c = grow_cone(u, c, bins[j].dir, bins[j].c);
                }
                cost[i - 1] += saoh(acc.box, acc.flux, c);
            }
            float axCost = std::numeric_limits<float>::infinity();
            uint32_t axIdx = 0;
            uint32_t run = b;
            for (uint32_t i = 0; i + 1 < B; i++) {
                run += bins[i].n;
                if (cost[i] < axCost) { axCost = cost[i]; axIdx = run; }
            }
            axCost *= d[int(big)] / d[int(ax)];
            if (axIdx == b || axIdx == e) continue;
            if (axCost < best) { best = axCost; bestAxis = ax; bestIdx = axIdx; }
        }
        if (bestAxis == 3) {
            if (e - b <= maxLeaf) { outAxis = 3; return; }
            // computeSplitWithEqual
            outAxis = d[2] >= d[0] && d[2] >= d[1] ? 2u : (d[1] >= d[0] ? 1u : 0u);
            outIdx = (b + e) / 2;
            return;
        }
        if (e - b <= maxLeaf) {
            float c;
            cone_of(b, e, c);
            if (saoh(nb, nodeFlux, c) <= best) { outAxis = 3; return; }
        }
        outAxis = bestAxis;
        outIdx = bestIdx;
    }

    uint32_t node(uint64_t mask, uint32_t depth, uint32_t b, uint32_t e) {
        AABB nb;
        float flux = 0.f;
        for (uint32_t i = b; i < e; i++) { nb.include(t[i].bounds); flux += t[i].flux; }
        nodeFlux = flux;
        uint32_t ax = 3, at = 0;
        if (e - b > 10) split(b, e, nb, ax, at);
        const uint32_t me = uint32_t(recs.size());
        recs.push_back(Rec{});
        Rec r{};
        r.box = nb;
        r.flux = flux;
        r.cosAngle = kInvalid;
        if (ax != 3) {
            std::nth_element(t.begin() + b, t.begin() + at, t.begin() + e,
                             [ax](const SortTri& x, const SortTri& y) { return x.bounds.center()[int(ax)] < y.bounds.center()[int(ax)]; });
            if (depth >= 64) throw std::runtime_error("light BVH too deep");
            node(mask, depth + 1, b, at);
            r.leaf = false;
            r.right = node(mask | (1ull << depth), depth + 1, at, e);
        } else {
            r.leaf = true;
            r.dir = cone_of(b, e, r.cosAngle);
            r.count = e - b;
            r.offset = uint32_t(leafTris.size());
            for (uint32_t i = b; i < e; i++) { leafTris.push_back(t[i].index); masks[t[i].index] = mask; }
        }
        recs[me] = r;
        return me;
    }

    F3 cones(uint32_t i, float& c) {
        if (recs[i].leaf) { c = recs[i].cosAngle; return recs[i].dir; }
        float cl, cr;
        F3 dl = cones(i + 1, cl), dr = cones(recs[i].right, cr);
        // coneUnionOld
        F3 dir = add(dl, dr);
        if (cl == kInvalid || cr == kInvalid || (dir[0] == 0.f && dir[1] == 0.f && dir[2] == 0.f)) {
            c = kInvalid;
            dir = F3();
        } else {
            dir = unit(dir);
            c = std::cos(std::max(sacos(dot3(dir, dl)) + std::acos(cl), sacos(dot3(dir, dr)) + std::acos(cr)));
        }
        recs[i].dir = dir;
        recs[i].cosAngle = c;
        return dir;
    }
};

}  // namespace lbvh

// verts: 9 floats, normals: 3 floats (decoded), flux: 1 float per emissive triangle.
// f16 / encodeNormal2x16 come from the caller (the oracle's host conversions).
template <class F16, class EncN>
inline void build_light_bvh_oracle(const std::vector<float>& verts, const std::vector<float>& normals, const std::vector<float>& flux,
                                   F16 f16, EncN encn, LightBvhOracle& out) {
    using namespace lbvh;
    Build bd;
    const size_t n = flux.size();
    bd.masks.assign(n, ~0ull);
    for (size_t i = 0; i < n; i++) {
        if (!(flux[i] > 0.f)) continue;
        SortTri s;
        for (int k = 0; k < 3; k++) s.bounds.include(f3(verts[9 * i + 3 * k], verts[9 * i + 3 * k + 1], verts[9 * i + 3 * k + 2]));
        s.dir = f3(normals[3 * i], normals[3 * i + 1], normals[3 * i + 2]);
        s.cosAngle = 1.f;
        s.flux = flux[i];
        s.index = uint32_t(i);
        bd.t.push_back(s);
    }
    out.nodes.clear();
    out.triIndices.clear();
    out.bitmasks = bd.masks;
    if (bd.t.empty()) return;
    bd.node(0ull, 0, 0, uint32_t(bd.t.size()));
    float c;
    bd.cones(0, c);
    out.triIndices = bd.leafTris;
    out.bitmasks = bd.masks;
    out.nodes.assign(bd.recs.size() * 8, 0u);
    for (size_t i = 0; i < bd.recs.size(); i++) {
        const Rec& r = bd.recs[i];
        uint32_t* w = &out.nodes[8 * i];
        w[0] = r.leaf ? (0x80000000u | (r.count << 27) | r.offset) : r.right;
        const F3 o = mul(add(r.box.mx, r.box.mn), 0.5f), ext = mul(sub(r.box.mx, r.box.mn), 0.5f);
        std::memcpy(&w[1], &o.v[0], 4);
        std::memcpy(&w[2], &o.v[1], 4);
        std::memcpy(&w[3], &o.v[2], 4);
        w[4] = uint32_t(f16(ext[0])) | (uint32_t(f16(ext[1])) << 16);
        w[5] = uint32_t(f16(ext[2])) | (uint32_t((r.cosAngle + 1.f) * 32767.f) << 16);
        w[6] = encn(r.dir.v);
        std::memcpy(&w[7], &r.flux, 4);
    }
}

}  // namespace orc
