// oracle_capi.cpp -- C entry points of the CPU oracle, loaded with ctypes by
// the tests, by smoke() and by bench.py's cpu_baseline leg.
//
// TEST INFRASTRUCTURE ONLY (see oracle_math.h): nothing in the product path
// links or loads this library.
#include <chrono>
#include <cstdio>
#include <exception>
#include <mutex>
#include <string>
#include <thread>
#include <random>
#include <vector>

#include "oracle_render.h"
#include "../falcor_b200/csrc/procedural.h"

using namespace orc;

namespace {
thread_local std::string g_err;
}

extern "C" {

const char* orc_last_error() { return g_err.c_str(); }

void* orc_scene_create(const fpt_scene_desc* d, const fpt_camera_data* cam) {
    try {
        return new Scene(d, cam);
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}
void orc_scene_destroy(void* s) { delete static_cast<Scene*>(s); }

// The synthetic workloads (falcor_b200/csrc/procedural.h, compiled into this
// library too), so that the oracle renders them without the CUDA library.
void* orc_procedural_scene(const fpt_procedural_params* p) {
    try {
        return build_procedural_scene(*p);
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}
const fpt_scene_desc* orc_procedural_desc(const void* h) { return &static_cast<const fpt_scene_host*>(h)->desc; }
void orc_procedural_free(void* h) { delete static_cast<fpt_scene_host*>(h); }
void orc_camera_compute(const fpt_camera* c, fpt_camera_data* out) { camera_data_from(*c, *out); }

struct orc_scene_info {
    uint32_t triangle_count, instance_count, emissive_count, active_emissive_count;
    uint32_t type_bits, instance_id_bits, primitive_index_bits, has_env;
    float alias_weight_sum;
    uint32_t imp_dim, imp_base_mip;
};
void orc_scene_get_info(const void* sp, orc_scene_info* out) {
    const Scene& s = *static_cast<const Scene*>(sp);
    out->triangle_count = uint32_t(s.triInstance.size());
    out->instance_count = uint32_t(s.instances.size());
    out->emissive_count = uint32_t(s.emissive.size());
    out->active_emissive_count = uint32_t(s.activeTriangles.size());
    out->type_bits = s.hitBits.type_bits;
    out->instance_id_bits = s.hitBits.instance_id_bits;
    out->primitive_index_bits = s.hitBits.primitive_index_bits;
    out->has_env = s.hasEnv ? 1u : 0u;
    out->alias_weight_sum = s.aliasWeightSum;
    out->imp_dim = s.impDim;
    out->imp_base_mip = s.impBaseMip;
}
// Alias table (2 uints per emissive triangle) and per-triangle flux.
// Light BVH of the oracle scene: sizes, then copies into caller arrays.
void orc_scene_light_bvh_sizes(const void* sp, uint32_t* nodes, uint32_t* tris, uint32_t* masks) {
    const Scene& s = *static_cast<const Scene*>(sp);
    *nodes = uint32_t(s.lightBvh.nodes.size() / 8);
    *tris = uint32_t(s.lightBvh.triIndices.size());
    *masks = uint32_t(s.lightBvh.bitmasks.size());
}
void orc_scene_get_light_bvh(const void* sp, uint32_t* nodes, uint32_t* tris, uint64_t* masks) {
    const Scene& s = *static_cast<const Scene*>(sp);
    std::copy(s.lightBvh.nodes.begin(), s.lightBvh.nodes.end(), nodes);
    std::copy(s.lightBvh.triIndices.begin(), s.lightBvh.triIndices.end(), tris);
    std::copy(s.lightBvh.bitmasks.begin(), s.lightBvh.bitmasks.end(), masks);
}
float orc_lbvh_selection_pdf(const void* sp, const float* posW, const float* n, int upper, uint32_t tri) {
    return lbvh_selection_pdf_f(*static_cast<const Scene*>(sp), posW, n, upper != 0, tri);
}
int orc_lbvh_select(const void* sp, const float* posW, const float* n, int upper, float u, uint32_t* tri, float* pdf) {
    return lbvh_select_f(*static_cast<const Scene*>(sp), posW, n, upper != 0, u, tri, pdf) ? 1 : 0;
}

void orc_scene_get_lights(const void* sp, uint32_t* alias, float* flux, float* area) {
    const Scene& s = *static_cast<const Scene*>(sp);
    for (size_t i = 0; i < s.emissive.size(); i++) {
        if (alias) { alias[2 * i] = s.aliasTable[2 * i]; alias[2 * i + 1] = s.aliasTable[2 * i + 1]; }
        if (flux) flux[i] = s.emissive[i].flux;
        if (area) area[i] = s.emissive[i].area;
    }
}
// Importance map mip (dim >> mip)^2 floats.
void orc_scene_get_importance(const void* sp, uint32_t mip, float* out) {
    const Scene& s = *static_cast<const Scene*>(sp);
    if (mip >= s.impMips.size()) return;
    std::copy(s.impMips[mip].begin(), s.impMips[mip].end(), out);
}

// The deterministic elementary functions (falcor_b200/csrc/fmath.h) on host
// arrays, numbered as fpt_fmath_fn.
void orc_fmath(uint32_t fn, uint32_t n, const float* x, const float* y, float* out) {
    for (uint32_t i = 0; i < n; i++) {
        const float a = x[i], b = y ? y[i] : 0.f;
        float r;
        switch (fn) {
            case 0: r = fm::sin(a); break;
            case 1: r = fm::cos(a); break;
            case 2: r = fm::atan2(a, b); break;
            case 3: r = fm::acos(a); break;
            case 4: r = fm::exp(a); break;
            case 5: r = fm::log(a); break;
            case 6: r = fm::log2(a); break;
            case 7: r = fm::exp2(a); break;
            default: r = fm::pow(a, b); break;
        }
        out[i] = r;
    }
}

void orc_vbuffer(const void* sp, uint32_t W, uint32_t H, uint32_t* out, uint32_t threads) {
    const Scene& s = *static_cast<const Scene*>(sp);
    parallel_tiles(0, 0, W, H, threads, [&](uint32_t x, uint32_t y, uint32_t) { render_vbuffer_pixel(s, W, H, x, y, out); });
}

// Per-ray closest hits: origins/dirs n*3 floats; out n*4 uint32 PackedHitInfo +
// tOut n floats.  brute != 0 tests every triangle.
void orc_trace_closest(const void* sp, uint32_t n, const float* o, const float* d, const float* tmin, const float* tmax,
                       uint32_t* out, float* tOut, int brute) {
    const Scene& s = *static_cast<const Scene*>(sp);
    for (uint32_t i = 0; i < n; i++) {
        V3<float> oo(o[3 * i], o[3 * i + 1], o[3 * i + 2]), dd(d[3 * i], d[3 * i + 1], d[3 * i + 2]);
        Hit h = brute ? s.traceClosestBrute(oo, dd, tmin[i], tmax[i]) : s.traceClosest(oo, dd, tmin[i], tmax[i], nullptr);
        pack_hit(s.hitBits, h, out + 4 * size_t(i));
        if (tOut) tOut[i] = h.valid ? h.t : -1.f;
    }
}
void orc_trace_visibility(const void* sp, uint32_t n, const float* o, const float* d, const float* tmax, uint32_t* out) {
    const Scene& s = *static_cast<const Scene*>(sp);
    for (uint32_t i = 0; i < n; i++) {
        V3<float> oo(o[3 * i], o[3 * i + 1], o[3 * i + 2]), dd(d[3 * i], d[3 * i + 1], d[3 * i + 2]);
        out[i] = s.traceVisibility(oo, dd, 0.f, tmax[i], nullptr) ? 1u : 0u;
    }
}

// MinimalPathTracer over the rectangle [x0,x1)x[y0,y1) of a W x H frame.
// out: RGBA32F for the full frame (only the rectangle is written).
// trace (optional): per pixel (maxBounces + 2) x 4 uints of per-vertex hits.
double orc_minimal_pt(const void* sp, const MinimalPTParams* p, const uint32_t* vbuffer, float* out, uint32_t* rays,
                      int fp64, uint32_t threads, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1, uint32_t* trace) {
    const Scene& s = *static_cast<const Scene*>(sp);
    auto t0 = std::chrono::steady_clock::now();
    parallel_tiles(x0, y0, x1, y1, threads, [&](uint32_t x, uint32_t y, uint32_t) {
        size_t i = size_t(y) * p->width + x;
        uint32_t r = 0;
        float* o = out + 4 * i;
        if (fp64) {
            V3<double> c = minimal_pt_pixel<double>(s, *p, x, y, vbuffer + 4 * i, &r);
            o[0] = float(c.x); o[1] = float(c.y); o[2] = float(c.z);
        } else {
            uint32_t* tr = trace ? trace + i * size_t(p->maxBounces + 2) * 4 : nullptr;
            V3<float> c = minimal_pt_pixel<float>(s, *p, x, y, vbuffer + 4 * i, &r, tr);
            o[0] = c.x; o[1] = c.y; o[2] = c.z;
        }
        o[3] = 1.f;
        if (rays) rays[i] = r;
    });
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

struct orc_counters {
    uint64_t paths, rays, closest, shadow, node_visits, tri_tests;
    uint64_t b8_nodes_closest, b8_tris_closest, b8_nodes_shadow, b8_tris_shadow, b8_mismatch;
};

static void sum_counters(const std::vector<PathCounters>& pcs, orc_counters* cnt) {
    *cnt = orc_counters{};
    for (auto& c : pcs) {
        cnt->paths += c.paths; cnt->rays += c.rays; cnt->closest += c.tc.closest; cnt->shadow += c.tc.shadow;
        cnt->node_visits += c.tc.nodeVisits; cnt->tri_tests += c.tc.triTests;
        cnt->b8_nodes_closest += c.tc.b8NodesClosest; cnt->b8_tris_closest += c.tc.b8TrisClosest;
        cnt->b8_nodes_shadow += c.tc.b8NodesShadow; cnt->b8_tris_shadow += c.tc.b8TrisShadow;
        cnt->b8_mismatch += c.tc.b8Mismatch;
    }
}

// A copy of the library's 8-wide BVH for the algorithmic traversal counts.
void orc_scene_attach_bvh8(void* sp, const void* nodes, uint32_t nodeCount, const void* tris, uint32_t triCount) {
    static_cast<Scene*>(sp)->attachBvh8(nodes, nodeCount, tris, triCount);
}

// PathTracer over a rectangle.  color: RGBA32F full frame; samples (optional):
// per pixel spp*3 floats, pixel-major over the full frame.
// trace (optional): per pixel spp x (maxSurfaceBounces + 2) x 4 uints of per-vertex hits.
double orc_path_tracer(const void* sp, const PathTracerParams* p, const uint32_t* vbuffer, float* color, float* samples,
                       int fp64, uint32_t threads, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1, orc_counters* cnt,
                       uint32_t* trace) {
    const Scene& s = *static_cast<const Scene*>(sp);
    uint32_t nthreads = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
    std::vector<PathCounters> pcs(nthreads);
    auto t0 = std::chrono::steady_clock::now();
    parallel_tiles(x0, y0, x1, y1, nthreads, [&](uint32_t x, uint32_t y, uint32_t tid) {
        size_t i = size_t(y) * p->width + x;
        float* so = samples ? samples + i * size_t(p->samplesPerPixel) * 3 : nullptr;
        if (fp64) path_tracer_pixel<double>(s, *p, x, y, vbuffer + 4 * i, so, color + 4 * i, &pcs[tid]);
        else path_tracer_pixel<float>(s, *p, x, y, vbuffer + 4 * i, so, color + 4 * i, &pcs[tid],
                                      trace ? trace + i * size_t(p->samplesPerPixel) * (p->maxSurfaceBounces + 2) * 4 : nullptr);
    });
    double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (cnt) sum_counters(pcs, cnt);
    return dt;
}

// PathTracer (FP32) over the pixels with x % stride == 0 and y % stride == 0
// of the frame, images discarded: event and traversal counts only.
double orc_path_tracer_counts(const void* sp, const PathTracerParams* p, const uint32_t* vbuffer, uint32_t stride,
                              uint32_t threads, orc_counters* cnt) {
    const Scene& s = *static_cast<const Scene*>(sp);
    uint32_t nthreads = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
    std::vector<PathCounters> pcs(nthreads);
    const uint32_t sw = (p->width + stride - 1) / stride, sh = (p->height + stride - 1) / stride;
    auto t0 = std::chrono::steady_clock::now();
    parallel_tiles(0, 0, sw, sh, nthreads, [&](uint32_t sx, uint32_t sy, uint32_t tid) {
        const uint32_t x = sx * stride, y = sy * stride;
        const size_t i = size_t(y) * p->width + x;
        float color[4];
        path_tracer_pixel<float>(s, *p, x, y, vbuffer + 4 * i, nullptr, color, &pcs[tid]);
    });
    double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (cnt) sum_counters(pcs, cnt);
    return dt;
}

// ----- Known-answer helpers (RNG, hashing, packing, ray offsets) ---------------
void orc_xoshiro(const uint32_t* seeds, uint32_t n, uint32_t dims, uint32_t* out) {
    for (uint32_t i = 0; i < n; i++) {
        Xoshiro128 r{{seeds[4 * i], seeds[4 * i + 1], seeds[4 * i + 2], seeds[4 * i + 3]}};
        for (uint32_t j = 0; j < dims; j++) out[size_t(j) * n + i] = r.next();
    }
}
void orc_splitmix(const uint32_t* seeds, uint32_t n, uint32_t dims, uint64_t* out) {
    for (uint32_t i = 0; i < n; i++) {
        SplitMix64 r = SplitMix64::create(seeds[2 * i], seeds[2 * i + 1]);
        for (uint32_t j = 0; j < dims; j++) out[size_t(j) * n + i] = r.next64();
    }
}
void orc_lcg(const uint32_t* seeds, uint32_t n, uint32_t dims, uint32_t* out) {
    for (uint32_t i = 0; i < n; i++) {
        LCG r{seeds[i]};
        for (uint32_t j = 0; j < dims; j++) out[size_t(j) * n + i] = r.next();
    }
}
void orc_jenkins(const uint32_t* in, uint32_t n, uint32_t* out) { for (uint32_t i = 0; i < n; i++) out[i] = jenkins_hash(in[i]); }
// Mirrors the five outputs of BitTricksTests.cs.slang:testBitInterleave.
void orc_bit_interleave(const uint32_t* data, uint32_t n, uint32_t* out) {
    for (uint32_t i = 0; i < n; i++) {
        uint32_t d = data[i];
        uint32_t bx = d & 0xffffu, by = d >> 16;
        uint32_t inter = interleave_32bit(bx, by);
        out[5 * i + 0] = interleave_32bit(bx ^ 0xbeef0000u, by ^ 0xbeef0000u);
        out[5 * i + 1] = interleave_16bit(bx ^ 0xbeefed00u, by ^ 0xbeefed00u);
        uint32_t x, y;
        deinterleave_16bit(inter & 0x0000ffffu, x, y);
        out[5 * i + 2] = (y << 16) | x;
        deinterleave_8bit(inter & 0x000000ffu, x, y);
        out[5 * i + 3] = (y << 16) | x;
        deinterleave_2x8bit(inter & 0x00ff00ffu, x, y);
        uint32_t tx = ((x >> 8) & 0x0f00u) | (x & 0xfu), ty = ((y >> 8) & 0x0f00u) | (y & 0xfu);
        out[5 * i + 4] = (ty << 16) | tx;
    }
}
void orc_compute_ray_origin(const float* pos, const float* nrm, uint32_t n, float* out) {
    for (uint32_t i = 0; i < n; i++) {
        V3<float> r = compute_ray_origin(V3<float>(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]),
                                         V3<float>(nrm[3 * i], nrm[3 * i + 1], nrm[3 * i + 2]));
        out[3 * i] = r.x; out[3 * i + 1] = r.y; out[3 * i + 2] = r.z;
    }
}
// First `dims` raw 32-bit outputs of a sample generator per (pixel, sampleNumber).
void orc_sample_generator(int kind, const uint32_t* px, const uint32_t* py, const uint32_t* sn, uint32_t n, uint32_t dims,
                          uint32_t* out) {
    for (uint32_t i = 0; i < n; i++) {
        if (kind == 1) {
            UniformSG g(px[i], py[i], sn[i]);
            for (uint32_t j = 0; j < dims; j++) out[size_t(i) * dims + j] = g.next();
        } else {
            TinyUniformSG g(px[i], py[i], sn[i]);
            for (uint32_t j = 0; j < dims; j++) out[size_t(i) * dims + j] = g.next();
        }
    }
}
void orc_f32tof16(const float* in, uint32_t n, uint16_t* out) { for (uint32_t i = 0; i < n; i++) out[i] = f32tof16_host(in[i]); }
void orc_f16tof32(const uint16_t* in, uint32_t n, float* out) { for (uint32_t i = 0; i < n; i++) out[i] = f16tof32(in[i]); }
void orc_logluv(const float* rgb, uint32_t n, uint32_t* enc, float* dec) {
    for (uint32_t i = 0; i < n; i++) {
        uint32_t e = encode_logluv_hdr(V3<float>(rgb[3 * i], rgb[3 * i + 1], rgb[3 * i + 2]));
        enc[i] = e;
        V3<float> d = decode_logluv_hdr(e);
        dec[3 * i] = d.x; dec[3 * i + 1] = d.y; dec[3 * i + 2] = d.z;
    }
}
uint32_t orc_intersect_triangle(const float* ro, const float* rd, const float* v, float* bary, float* t) {
    V3<float> vv[3] = {V3<float>(v[0], v[1], v[2]), V3<float>(v[3], v[4], v[5]), V3<float>(v[6], v[7], v[8])};
    V3<float> b;
    bool hit = intersect_ray_triangle(V3<float>(ro[0], ro[1], ro[2]), V3<float>(rd[0], rd[1], rd[2]), vv, b, *t);
    bary[0] = b.x; bary[1] = b.y; bary[2] = b.z;
    return hit ? 1u : 0u;
}

// StandardBSDF in the local frame, for sampling/pdf consistency tests.
// data: diffuse[3], specular[3], roughness, metallic, eta, diffTrans, specTrans.
// For each of n inputs: wi (3 floats), u (4 random uint32 words used as the
// sample generator stream).  Outputs wo, weight, pdf, lobe, valid, plus
// eval(wi, wo) and evalPdf(wi, wo) of the sampled direction.
struct ListSG {
    const uint32_t* w; uint32_t i = 0, n;
    uint32_t next() { return i < n ? w[i++] : 0u; }
};
void orc_bsdf_sample(const float* data, int lambert, uint32_t n, const float* wi, const uint32_t* words, uint32_t nwords,
                     float* wo, float* weight, float* pdf, uint32_t* lobe, uint32_t* valid, float* evalOut, float* pdfOut) {
    BSDFData<float> d;
    d.diffuse = V3<float>(data[0], data[1], data[2]);
    d.specular = V3<float>(data[3], data[4], data[5]);
    d.roughness = data[6]; d.metallic = data[7]; d.eta = data[8]; d.diffuseTransmission = data[9]; d.specularTransmission = data[10];
    d.transmission = V3<float>(1.f);
    for (uint32_t i = 0; i < n; i++) {
        V3<float> w(wi[3 * i], wi[3 * i + 1], wi[3 * i + 2]);
        StandardBSDF<float> b(w, d, false, LOBE_ALL, lambert != 0);
        ListSG sg{words + size_t(i) * nwords, 0, nwords};
        V3<float> o, wt;
        float pd;
        uint32_t lb;
        bool ok = b.sample(w, o, pd, wt, lb, sg);
        wo[3 * i] = o.x; wo[3 * i + 1] = o.y; wo[3 * i + 2] = o.z;
        weight[3 * i] = wt.x; weight[3 * i + 1] = wt.y; weight[3 * i + 2] = wt.z;
        pdf[i] = pd; lobe[i] = lb; valid[i] = ok ? 1u : 0u;
        V3<float> e = b.eval(w, o);
        evalOut[3 * i] = e.x; evalOut[3 * i + 1] = e.y; evalOut[3 * i + 2] = e.z;
        pdfOut[i] = b.eval_pdf(w, o);
    }
}


// WARDiffPathTracer over a rectangle (one path per pixel).  color: RGBA32F full
// frame (optional); dLdI: 3 floats per pixel, pixel-major (mode 1); grads: K
// doubles, sum over the rectangle of dLdI . dL/dv_k (mode 1); pert: 3 doubles
// per pixel of the perturbed radiance (mode 2).
double orc_wardiff(const void* sp, const WarDiffParams* p, int mode, int K, const double* matTangents, uint32_t matDim,
                   const double* posTangents, uint32_t posDim, const double* nrmTangents, uint32_t nrmDim,
                   const double* tanTangents, uint32_t tanDim, double eps, const float* dLdI, float* color, double* grads,
                   double* pert, uint32_t threads, uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1, uint64_t* rays,
                   const double* texTangents, uint32_t texDim) {
    const Scene& s = *static_cast<const Scene*>(sp);
    WarSeeds seeds;
    seeds.K = K;
    seeds.mat = matTangents;
    seeds.matDim = matDim;
    seeds.pos = posTangents;
    seeds.posDim = posDim;
    seeds.meshID = p->meshID;
    seeds.nrm = nrmTangents;
    seeds.nrmDim = nrmDim;
    seeds.tan = tanTangents;
    seeds.tanDim = tanDim;
    seeds.tex = texTangents;
    seeds.texDim = texDim;
    seeds.eps = eps;
    uint32_t nthreads = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
    std::vector<std::vector<double>> acc(nthreads, std::vector<double>(4, 0.0));
    std::vector<WarCounters> wcs(nthreads);
    auto t0 = std::chrono::steady_clock::now();
    parallel_tiles(x0, y0, x1, y1, nthreads, [&](uint32_t x, uint32_t y, uint32_t tid) {
        size_t i = size_t(y) * p->width + x;
        wardiff_pixel(s, *p, seeds, mode, x, y, dLdI ? dLdI + 3 * i : nullptr, color ? color + 4 * i : nullptr,
                      acc[tid].data(), pert ? pert + 3 * i : nullptr, &wcs[tid]);
    });
    double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (grads)
        for (int k = 0; k < K && k < 4; k++) {
            grads[k] = 0;
            for (auto& a : acc) grads[k] += a[k];
        }
    if (rays) {
        *rays = 0;
        for (auto& c : wcs) *rays += c.rays;
    }
    return dt;
}

// Traversal counts of the WARDiffPathTracer adjoint's rays: forward-mode
// derivatives (mode 1, K = 1, no seeded tangents) of every stride-th pixel in
// x and y, which trace the same rays as the adjoint (the path, its visibility
// rays and, with useWAR, every auxiliary ray), with the library's 8-wide BVH
// attached.  out: b8 nodes / triangles of closest-hit rays, of visibility
// rays, mismatches, rays, sampled pixels.  Returns seconds.
double orc_wardiff_traversal(const void* sp, const WarDiffParams* p, uint32_t stride, uint32_t threads, uint64_t* out) {
    const Scene& s = *static_cast<const Scene*>(sp);
    const uint32_t nthreads = threads ? threads : std::max(1u, std::thread::hardware_concurrency());
    std::vector<TraceCounters> tcs(nthreads);
    std::vector<WarCounters> wcs(nthreads);
    const uint32_t sw = (p->width + stride - 1) / stride, sh = (p->height + stride - 1) / stride;
    auto t0 = std::chrono::steady_clock::now();
    parallel_tiles(0, 0, sw, sh, nthreads, [&](uint32_t xs, uint32_t ys, uint32_t tid) {
        WarSeeds seeds;
        seeds.K = 1;
        seeds.meshID = p->meshID;
        seeds.tc = &tcs[tid];
        double acc[4] = {0, 0, 0, 0};
        const uint32_t x = xs * stride, y = ys * stride;
        const float g[3] = {1.f, 1.f, 1.f};
        wardiff_pixel(s, *p, seeds, 1, x, y, g, nullptr, acc, nullptr, &wcs[tid]);
    });
    const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int i = 0; i < 7; i++) out[i] = 0;
    for (const TraceCounters& c : tcs) {
        out[0] += c.b8NodesClosest; out[1] += c.b8TrisClosest; out[2] += c.b8NodesShadow; out[3] += c.b8TrisShadow;
        out[4] += c.b8Mismatch;
    }
    for (const WarCounters& c : wcs) out[5] += c.rays;
    out[6] = uint64_t(sw) * sh;
    return dt;
}

// Camera-jitter sample patterns of VBufferRT (Utils/SampleGenerators):
// kind 1 DirectX (DxSamplePattern.cpp:33-45), 2 Halton (HaltonSamplePattern.cpp:
// 33-64), 3 Stratified (StratifiedSamplePattern.cpp:35-95, std::mt19937 with its
// default seed, std::shuffle once per round, uniform_real_distribution<float>).
// Writes n (x, y) pairs in [-0.5, 0.5).
void orc_sample_pattern(int kind, uint32_t sampleCount, uint32_t n, float* out) {
    if (kind == 1) {
        static const float t[8][2] = {{1, -3}, {-1, 3}, {5, 1}, {-3, -5}, {-5, 5}, {-7, -1}, {3, 7}, {7, -7}};
        for (uint32_t i = 0; i < n; i++) {
            out[2 * i] = t[i % 8][0] / 16.f;
            out[2 * i + 1] = t[i % 8][1] / 16.f;
        }
        return;
    }
    if (kind == 2) {
        uint32_t cur = 0;
        auto halton = [](uint32_t index, uint32_t base) {
            float r = 0.f, f = 1.f;
            while (index > 0) {
                f /= float(base);
                r += f * float(index % base);
                index /= base;
            }
            return r;
        };
        for (uint32_t i = 0; i < n; i++) {
            float v[2] = {halton(cur, 2), halton(cur, 3)};
            cur++;
            if (sampleCount) cur %= sampleCount;
            for (int k = 0; k < 2; k++) out[2 * i + k] = (v[k] + 0.5f - std::floor(v[k] + 0.5f)) - 0.5f;
        }
        return;
    }
    const uint32_t count = std::min(std::max(sampleCount, 1u), 1024u);
    uint32_t bx = uint32_t(std::sqrt(double(count))), by = count / bx;
    while (bx * by != count) by = count / ++bx;
    std::vector<uint32_t> perm(count);
    for (uint32_t i = 0; i < count; i++) perm[i] = i;
    std::mt19937 rng;
    uint32_t cur = 0;
    for (uint32_t i = 0; i < n; i++) {
        std::uniform_real_distribution<float> u;
        if (cur == 0) std::shuffle(perm.begin(), perm.end(), rng);
        const uint32_t bin = perm[cur];
        cur = (cur + 1) % count;
        const float fx = (float(bin % bx) + u(rng)) / float(bx);
        const float fy = (float(bin / bx) + u(rng)) / float(by);
        out[2 * i] = fx - 0.5f;
        out[2 * i + 1] = fy - 0.5f;
    }
}

}  // extern "C"
