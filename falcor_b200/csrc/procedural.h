// procedural.h -- the synthetic workloads: seeded procedural scenes (box +
// icosphere, fBm heightfield + random triangle soup, displaced sphere, random
// soup, displaced grid) with their StandardMaterials, emitters, env map and
// camera.  Host-only C++ over the C-ABI's plain structs.  The library's
// fpt_procedural_scene and the CPU oracle both compile this file (every
// function has internal linkage), so both render the same inputs without the
// oracle loading the library.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/fpt.h"

struct fpt_scene_host {
    std::vector<fpt_vertex> vertices;
    std::vector<uint32_t> indices;
    std::vector<fpt_geometry_instance> instances;
    std::vector<fpt_material> materials;
    std::vector<float> envRGB;
    fpt_envmap_desc env{};
    fpt_scene_desc desc{};

    void finalize() {
        desc.vertices = vertices.data();
        desc.vertex_count = uint32_t(vertices.size());
        desc.indices = indices.data();
        desc.index_count = uint32_t(indices.size());
        desc.instances = instances.data();
        desc.instance_count = uint32_t(instances.size());
        desc.materials = materials.data();
        desc.material_count = uint32_t(materials.size());
        if (!envRGB.empty()) {
            env.rgb = envRGB.data();
            desc.envmap = &env;
        } else {
            desc.envmap = nullptr;
        }
    }
};

namespace {

struct Mesh {
    std::vector<float> pos;      // 3 per vertex
    std::vector<float> nrm;      // 3 per vertex
    std::vector<uint32_t> idx;   // 3 per triangle
};

fpt_material make_material(float r, float g, float b, float roughness, float metallic) {
    fpt_material m;
    std::memset(&m, 0, sizeof(m));
    m.base_color[0] = r; m.base_color[1] = g; m.base_color[2] = b; m.base_color[3] = 1.f;
    m.specular[0] = 0.f; m.specular[1] = roughness; m.specular[2] = metallic; m.specular[3] = 0.f;
    m.emissive_factor = 1.f;
    m.ior = 1.5f;
    m.transmission[0] = m.transmission[1] = m.transmission[2] = 1.f;
    return m;
}

// Appends a mesh as one geometry instance with its own vertex/index range.
void add_instance(fpt_scene_host& h, const Mesh& m, uint32_t material) {
    fpt_geometry_instance in;
    in.vb_offset = uint32_t(h.vertices.size());
    in.ib_offset = uint32_t(h.indices.size());
    in.triangle_count = uint32_t(m.idx.size() / 3);
    in.material_id = material;
    in.flags = 0;
    const size_t nv = m.pos.size() / 3;
    for (size_t i = 0; i < nv; i++) {
        fpt_vertex v;
        std::memset(&v, 0, sizeof(v));
        for (int k = 0; k < 3; k++) { v.position[k] = m.pos[3 * i + k]; v.normal[k] = m.nrm[3 * i + k]; }
        // No tangents: w = 0 marks an invalid tangent, the shading frame is
        // then built from the normal (ShadingFrame::orthonormalizeSafe).
        h.vertices.push_back(v);
    }
    h.indices.insert(h.indices.end(), m.idx.begin(), m.idx.end());
    h.instances.push_back(in);
}

// Quad p0,p1,p2,p3 (counter-clockwise seen from the front) with normal n.
Mesh quad(const float p[4][3], const float n[3]) {
    Mesh m;
    for (int i = 0; i < 4; i++)
        for (int k = 0; k < 3; k++) { m.pos.push_back(p[i][k]); m.nrm.push_back(n[k]); }
    m.idx = {0, 1, 2, 0, 2, 3};
    return m;
}

void normalize3(float* v) {
    float l = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (l > 0.f) { v[0] /= l; v[1] /= l; v[2] /= l; }
}

Mesh icosphere(uint32_t subdiv, float radius, const float c[3]) {
    const float t = (1.f + std::sqrt(5.f)) / 2.f;
    std::vector<float> v = {-1, t, 0, 1, t, 0, -1, -t, 0, 1, -t, 0, 0, -1, t, 0, 1, t,
                            0, -1, -t, 0, 1, -t, t, 0, -1, t, 0, 1, -t, 0, -1, -t, 0, 1};
    std::vector<uint32_t> f = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4, 11, 10, 2, 10, 7, 6, 7, 1, 8,
                               3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8, 3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    for (size_t i = 0; i < v.size(); i += 3) normalize3(&v[i]);
    for (uint32_t s = 0; s < subdiv; s++) {
        std::map<uint64_t, uint32_t> mid;
        auto midpoint = [&](uint32_t a, uint32_t b) {
            uint64_t key = (uint64_t(std::min(a, b)) << 32) | std::max(a, b);
            auto it = mid.find(key);
            if (it != mid.end()) return it->second;
            float m[3] = {(v[3 * a] + v[3 * b]) * 0.5f, (v[3 * a + 1] + v[3 * b + 1]) * 0.5f, (v[3 * a + 2] + v[3 * b + 2]) * 0.5f};
            normalize3(m);
            uint32_t id = uint32_t(v.size() / 3);
            v.insert(v.end(), m, m + 3);
            mid[key] = id;
            return id;
        };
        std::vector<uint32_t> nf;
        for (size_t i = 0; i < f.size(); i += 3) {
            uint32_t a = f[i], b = f[i + 1], cc = f[i + 2];
            uint32_t ab = midpoint(a, b), bc = midpoint(b, cc), ca = midpoint(cc, a);
            uint32_t tris[12] = {a, ab, ca, b, bc, ab, cc, ca, bc, ab, bc, ca};
            nf.insert(nf.end(), tris, tris + 12);
        }
        f.swap(nf);
    }
    Mesh m;
    for (size_t i = 0; i < v.size(); i += 3) {
        for (int k = 0; k < 3; k++) { m.pos.push_back(c[k] + radius * v[i + k]); m.nrm.push_back(v[i + k]); }
    }
    m.idx = f;
    return m;
}

// Value noise fBm for the heightfields.
struct Noise {
    std::vector<float> g;
    uint32_t n;
    explicit Noise(uint32_t seed, uint32_t size = 256) : n(size) {
        std::mt19937_64 rng(seed);
        std::uniform_real_distribution<float> u(-1.f, 1.f);
        g.resize(size_t(n) * n);
        for (auto& x : g) x = u(rng);
    }
    float at(int x, int y) const { return g[size_t((y % int(n) + int(n)) % int(n)) * n + size_t((x % int(n) + int(n)) % int(n))]; }
    float value(float x, float y) const {
        float fx = std::floor(x), fy = std::floor(y);
        float ax = x - fx, ay = y - fy;
        ax = ax * ax * (3.f - 2.f * ax);
        ay = ay * ay * (3.f - 2.f * ay);
        int ix = int(fx), iy = int(fy);
        float a = at(ix, iy), b = at(ix + 1, iy), c = at(ix, iy + 1), d = at(ix + 1, iy + 1);
        return (a * (1 - ax) + b * ax) * (1 - ay) + (c * (1 - ax) + d * ax) * ay;
    }
    float fbm(float x, float y, int octaves) const {
        float s = 0.f, amp = 0.5f, f = 1.f;
        for (int o = 0; o < octaves; o++) { s += amp * value(x * f, y * f); amp *= 0.5f; f *= 2.f; }
        return s;
    }
};

// Heightfield grid of res x res vertices over [-1,1]^2 (xz), split into
// tiles x tiles instances that share nothing.  Returns meshes in tile order.
std::vector<Mesh> heightfield(uint32_t res, uint32_t tiles, uint32_t seed, float amplitude, float freq) {
    Noise noise(seed);
    auto height = [&](uint32_t i, uint32_t j) {
        float u = float(i) / float(res - 1), v = float(j) / float(res - 1);
        return amplitude * noise.fbm(u * freq, v * freq, 6);
    };
    std::vector<float> H(size_t(res) * res);
    for (uint32_t j = 0; j < res; j++)
        for (uint32_t i = 0; i < res; i++) H[size_t(j) * res + i] = height(i, j);
    auto P = [&](uint32_t i, uint32_t j, float* out) {
        out[0] = -1.f + 2.f * float(i) / float(res - 1);
        out[1] = H[size_t(j) * res + i];
        out[2] = -1.f + 2.f * float(j) / float(res - 1);
    };
    auto N = [&](uint32_t i, uint32_t j, float* out) {
        uint32_t i0 = i > 0 ? i - 1 : i, i1 = i + 1 < res ? i + 1 : i;
        uint32_t j0 = j > 0 ? j - 1 : j, j1 = j + 1 < res ? j + 1 : j;
        float dx = (H[size_t(j) * res + i1] - H[size_t(j) * res + i0]) / (2.f * float(i1 - i0) / float(res - 1));
        float dz = (H[size_t(j1) * res + i] - H[size_t(j0) * res + i]) / (2.f * float(j1 - j0) / float(res - 1));
        out[0] = -dx; out[1] = 1.f; out[2] = -dz;
        normalize3(out);
    };
    const uint32_t quads = res - 1;
    std::vector<Mesh> meshes;
    for (uint32_t ty = 0; ty < tiles; ty++)
        for (uint32_t tx = 0; tx < tiles; tx++) {
            uint32_t q0x = quads * tx / tiles, q1x = quads * (tx + 1) / tiles;
            uint32_t q0y = quads * ty / tiles, q1y = quads * (ty + 1) / tiles;
            Mesh m;
            uint32_t w = q1x - q0x + 1;
            for (uint32_t j = q0y; j <= q1y; j++)
                for (uint32_t i = q0x; i <= q1x; i++) {
                    float p[3], n[3];
                    P(i, j, p);
                    N(i, j, n);
                    m.pos.insert(m.pos.end(), p, p + 3);
                    m.nrm.insert(m.nrm.end(), n, n + 3);
                }
            for (uint32_t j = 0; j < q1y - q0y; j++)
                for (uint32_t i = 0; i < q1x - q0x; i++) {
                    uint32_t a = j * w + i, b = a + 1, c = a + w, d = c + 1;
                    // Counter-clockwise seen from +y (front face up).
                    uint32_t t[6] = {a, c, b, b, c, d};
                    m.idx.insert(m.idx.end(), t, t + 6);
                }
            meshes.push_back(std::move(m));
        }
    return meshes;
}

// Random triangles with log-uniform edge lengths inside the box [lo, hi].
Mesh random_soup(std::mt19937_64& rng, uint32_t count, const float lo[3], const float hi[3], float emin, float emax) {
    std::uniform_real_distribution<float> u01(0.f, 1.f);
    Mesh m;
    for (uint32_t t = 0; t < count; t++) {
        float c[3];
        for (int k = 0; k < 3; k++) c[k] = lo[k] + (hi[k] - lo[k]) * u01(rng);
        float edge = std::exp(std::log(emin) + (std::log(emax) - std::log(emin)) * u01(rng));
        // Two random unit directions spanning the triangle.
        float a[3], b[3];
        for (int k = 0; k < 3; k++) { a[k] = u01(rng) * 2.f - 1.f; b[k] = u01(rng) * 2.f - 1.f; }
        normalize3(a);
        normalize3(b);
        float p0[3], p1[3], p2[3];
        for (int k = 0; k < 3; k++) {
            p0[k] = c[k];
            p1[k] = c[k] + edge * a[k];
            p2[k] = c[k] + edge * b[k];
        }
        float e1[3] = {p1[0] - p0[0], p1[1] - p0[1], p1[2] - p0[2]}, e2[3] = {p2[0] - p0[0], p2[1] - p0[1], p2[2] - p0[2]};
        float n[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
        normalize3(n);
        uint32_t base = uint32_t(m.pos.size() / 3);
        for (const float* p : {p0, p1, p2}) {
            m.pos.insert(m.pos.end(), p, p + 3);
            m.nrm.insert(m.nrm.end(), n, n + 3);
        }
        uint32_t tri[3] = {base, base + 1, base + 2};
        m.idx.insert(m.idx.end(), tri, tri + 3);
    }
    return m;
}

// Procedural sky: vertical gradient plus a sun lobe, lat-long RGB32F.
void make_envmap(fpt_scene_host& h, uint32_t W, uint32_t H) {
    h.envRGB.resize(size_t(W) * H * 3);
    const float sun[3] = {0.3f, 0.8f, -0.52f};
    float sl = std::sqrt(sun[0] * sun[0] + sun[1] * sun[1] + sun[2] * sun[2]);
    for (uint32_t y = 0; y < H; y++)
        for (uint32_t x = 0; x < W; x++) {
            // latlong_map_to_world (Utils/Math/MathHelpers.slang:126-135).
            float u = (float(x) + 0.5f) / float(W), v = (float(y) + 0.5f) / float(H);
            float phi = 3.14159265f * (2.f * u - 1.f), theta = 3.14159265f * v;
            float d[3] = {std::sin(theta) * std::sin(phi), std::cos(theta), -std::sin(theta) * std::cos(phi)};
            float up = std::max(0.f, d[1]);
            float c = (d[0] * sun[0] + d[1] * sun[1] + d[2] * sun[2]) / sl;
            float lobe = 200.f * std::pow(std::max(0.f, c), 512.f);
            float* o = &h.envRGB[(size_t(y) * W + x) * 3];
            o[0] = 0.25f + 0.35f * up + lobe;
            o[1] = 0.35f + 0.45f * up + 0.95f * lobe;
            o[2] = 0.55f + 0.60f * up + 0.85f * lobe;
            if (d[1] < 0.f) { o[0] = 0.18f; o[1] = 0.16f; o[2] = 0.14f; }
        }
    h.env.width = W;
    h.env.height = H;
    h.env.tint[0] = h.env.tint[1] = h.env.tint[2] = 1.f;
    h.env.intensity = 1.f;
}

void set_camera(fpt_scene_host& h, const float pos[3], const float target[3], float fovYDeg, float aspect) {
    fpt_camera& c = h.desc.camera;
    std::memset(&c, 0, sizeof(c));
    for (int k = 0; k < 3; k++) { c.position[k] = pos[k]; c.target[k] = target[k]; }
    c.up[0] = 0.f; c.up[1] = 1.f; c.up[2] = 0.f;
    c.frame_height = 24.f;
    // fovYToFocalLength (Utils/Math/FalcorMath.h): f = frameHeight / (2 tan(fovY/2)).
    c.focal_length = c.frame_height / (2.f * std::tan(0.5f * fovYDeg * 3.14159265358979f / 180.f));
    c.aspect_ratio = aspect;
    c.near_z = 0.1f;
    c.far_z = 1000.f;
    c.focal_distance = 10000.f;
}

// Lambertian-ish StandardMaterial library of the large scenes: baseColor U[0,1],
// roughness U[0.05,1], metallic Bernoulli(0.3).
void random_materials(fpt_scene_host& h, std::mt19937_64& rng, uint32_t count) {
    std::uniform_real_distribution<float> u01(0.f, 1.f);
    for (uint32_t i = 0; i < count; i++) {
        float r = u01(rng), g = u01(rng), b = u01(rng);
        float rough = 0.05f + 0.95f * u01(rng);
        float metal = u01(rng) < 0.3f ? 1.f : 0.f;
        h.materials.push_back(make_material(r, g, b, rough, metal));
    }
}

// Emissive triangles with power log-uniform in [pmin, pmax]: radiance is set so
// that flux = luminance(L) * area * pi equals the drawn power.
void add_emitters(fpt_scene_host& h, std::mt19937_64& rng, uint32_t count, const float lo[3], const float hi[3], float emin,
                  float emax, float pmin, float pmax) {
    std::uniform_real_distribution<float> u01(0.f, 1.f);
    for (uint32_t i = 0; i < count; i++) {
        Mesh m = random_soup(rng, 1, lo, hi, emin, emax);
        // Face downwards so that the emitters light the ground.
        const float* n = &m.nrm[0];
        if (n[1] > 0.f) {
            std::swap(m.idx[1], m.idx[2]);
            for (size_t k = 0; k < m.nrm.size(); k++) m.nrm[k] = -m.nrm[k];
        }
        float e1[3], e2[3];
        for (int k = 0; k < 3; k++) { e1[k] = m.pos[3 + k] - m.pos[k]; e2[k] = m.pos[6 + k] - m.pos[k]; }
        float cx = e1[1] * e2[2] - e1[2] * e2[1], cy = e1[2] * e2[0] - e1[0] * e2[2], cz = e1[0] * e2[1] - e1[1] * e2[0];
        float area = 0.5f * std::sqrt(cx * cx + cy * cy + cz * cz);
        float power = std::exp(std::log(pmin) + (std::log(pmax) - std::log(pmin)) * u01(rng));
        float L = power / (std::max(area, 1e-12f) * 3.14159265f);
        fpt_material mat = make_material(1.f, 1.f, 1.f, 1.f, 0.f);
        mat.emissive[0] = L; mat.emissive[1] = L; mat.emissive[2] = L;
        uint32_t mid = uint32_t(h.materials.size());
        h.materials.push_back(mat);
        add_instance(h, m, mid);
    }
}

fpt_scene_host* build_box_icosphere(const fpt_procedural_params& p) {
    auto* h = new fpt_scene_host();
    std::mt19937_64 rng(p.seed);
    std::uniform_real_distribution<float> alb(0.2f, 0.8f);
    // Room [-1,1]^3; each wall is split into two quads: 12 quads = 24 triangles,
    // one albedo per quad.  Fronts face the inside of the room.
    struct Wall { int axis; float side; };
    const Wall walls[6] = {{0, -1}, {0, 1}, {1, -1}, {1, 1}, {2, -1}, {2, 1}};
    for (const Wall& w : walls) {
        int a = w.axis, b = (a + 1) % 3, c = (a + 2) % 3;
        float n[3] = {0, 0, 0};
        n[a] = -w.side;  // inward
        for (int half = 0; half < 2; half++) {
            float b0 = half == 0 ? -1.f : 0.f, b1 = half == 0 ? 0.f : 1.f;
            float q[4][3];
            float corners[4][2] = {{b0, -1.f}, {b1, -1.f}, {b1, 1.f}, {b0, 1.f}};
            for (int k = 0; k < 4; k++) {
                q[k][a] = w.side;
                q[k][b] = corners[k][0];
                q[k][c] = corners[k][1];
            }
            // Orient counter-clockwise around the inward normal.
            float e1[3], e2[3];
            for (int k = 0; k < 3; k++) { e1[k] = q[1][k] - q[0][k]; e2[k] = q[2][k] - q[0][k]; }
            float cr[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
            if (cr[0] * n[0] + cr[1] * n[1] + cr[2] * n[2] < 0.f) {
                for (int k = 0; k < 3; k++) std::swap(q[1][k], q[3][k]);
            }
            uint32_t mid = uint32_t(h->materials.size());
            float r = alb(rng), g = alb(rng), bb = alb(rng);
            h->materials.push_back(make_material(r, g, bb, 1.f, 0.f));
            add_instance(*h, quad(q, n), mid);
        }
    }
    // Emissive ceiling quad 0.5 x 0.5, radiance 10, facing down.
    {
        const float y = 0.999f;
        float q[4][3] = {{-0.25f, y, -0.25f}, {0.25f, y, -0.25f}, {0.25f, y, 0.25f}, {-0.25f, y, 0.25f}};
        float n[3] = {0.f, -1.f, 0.f};
        // counter-clockwise around -y (cross(p1 - p0, p2 - p0) points down)
        fpt_material m = make_material(0.8f, 0.8f, 0.8f, 1.f, 0.f);
        m.emissive[0] = m.emissive[1] = m.emissive[2] = 10.f;
        uint32_t mid = uint32_t(h->materials.size());
        h->materials.push_back(m);
        add_instance(*h, quad(q, n), mid);
    }
    // Icosphere at the centre.
    {
        const float c[3] = {0.f, -0.35f, 0.f};
        uint32_t mid = uint32_t(h->materials.size());
        h->materials.push_back(make_material(alb(rng), alb(rng), alb(rng), 1.f, 0.f));
        add_instance(*h, icosphere(p.sphere_subdiv ? p.sphere_subdiv : 4, 0.45f, c), mid);
    }
    const float cam[3] = {0.f, 0.f, 0.98f}, tgt[3] = {0.f, -0.2f, 0.f};
    set_camera(*h, cam, tgt, 45.f, p.aspect_ratio > 0.f ? p.aspect_ratio : 1.f);
    return h;
}

fpt_scene_host* build_heightfield_soup(const fpt_procedural_params& p) {
    auto* h = new fpt_scene_host();
    std::mt19937_64 rng(p.seed);
    const uint32_t nmat = p.material_count ? p.material_count : 256;
    random_materials(*h, rng, nmat);
    const uint32_t res = p.grid_res ? p.grid_res : 1024;
    std::vector<Mesh> tiles = heightfield(res, 16, p.seed, 0.25f, 6.f);
    for (size_t i = 0; i < tiles.size(); i++) add_instance(*h, tiles[i], uint32_t(i % nmat));
    const uint32_t soup = p.soup_triangles;
    if (soup) {
        const float lo[3] = {-1.f, -0.1f, -1.f}, hi[3] = {1.f, 0.6f, 1.f};
        Mesh all = random_soup(rng, soup, lo, hi, 1e-3f, 1e-1f);
        const uint32_t chunks = 256;
        std::uniform_int_distribution<uint32_t> mdist(0, nmat - 1);
        for (uint32_t c = 0; c < chunks; c++) {
            uint32_t t0 = uint32_t(uint64_t(soup) * c / chunks), t1 = uint32_t(uint64_t(soup) * (c + 1) / chunks);
            Mesh m;
            m.pos.assign(all.pos.begin() + size_t(t0) * 9, all.pos.begin() + size_t(t1) * 9);
            m.nrm.assign(all.nrm.begin() + size_t(t0) * 9, all.nrm.begin() + size_t(t1) * 9);
            for (uint32_t t = 0; t < (t1 - t0) * 3; t++) m.idx.push_back(t);
            add_instance(*h, m, mdist(rng));
        }
    }
    const float elo[3] = {-0.9f, 0.7f, -0.9f}, ehi[3] = {0.9f, 0.95f, 0.9f};
    add_emitters(*h, rng, p.emissive_count ? p.emissive_count : 64, elo, ehi, 0.02f, 0.1f, 1.f, 1e3f);
    if (p.envmap_width && p.envmap_height) make_envmap(*h, p.envmap_width, p.envmap_height);
    const float cam[3] = {0.f, 1.1f, 2.1f}, tgt[3] = {0.f, 0.f, 0.f};
    set_camera(*h, cam, tgt, 45.f, p.aspect_ratio > 0.f ? p.aspect_ratio : 16.f / 9.f);
    return h;
}

// Displaced UV sphere split into up to 16 x 16 latitude/longitude patches,
// one instance and one material each (256 materials for the default 142 x 71
// grid).  sphere_subdiv = segments around (rings = segments / 2).
fpt_scene_host* build_displaced_sphere(const fpt_procedural_params& p) {
    auto* h = new fpt_scene_host();
    std::mt19937_64 rng(p.seed);
    const uint32_t nmat = p.material_count ? p.material_count : 256;
    random_materials(*h, rng, nmat);
    for (auto& m : h->materials) m.specular[2] = 0.f;  // dielectric
    Noise noise(p.seed + 7);
    const uint32_t seg = p.sphere_subdiv ? p.sphere_subdiv : 142;
    const uint32_t rings = seg / 2;
    auto disp = [&](float th, float ph) { return 0.6f + 0.05f * noise.fbm(3.f * ph, 3.f * th, 4); };
    auto vertex = [&](uint32_t r, uint32_t sIdx, Mesh& m) {
        const float th = 3.14159265f * float(r) / float(rings), ph = 2.f * 3.14159265f * float(sIdx % seg) / float(seg);
        const float d[3] = {std::sin(th) * std::cos(ph), std::cos(th), std::sin(th) * std::sin(ph)};
        const float rad = disp(th, ph);
        for (int k = 0; k < 3; k++) { m.pos.push_back(rad * d[k]); m.nrm.push_back(d[k]); }
    };
    const uint32_t pr = std::min<uint32_t>(16, rings), ps = std::min<uint32_t>(16, seg);
    uint32_t patch = 0;
    for (uint32_t a = 0; a < pr; a++)
        for (uint32_t c = 0; c < ps; c++, patch++) {
            const uint32_t r0 = rings * a / pr, r1 = rings * (a + 1) / pr, s0 = seg * c / ps, s1 = seg * (c + 1) / ps;
            Mesh m;
            const uint32_t cols = s1 - s0 + 1;
            for (uint32_t r = r0; r <= r1; r++)
                for (uint32_t sIdx = s0; sIdx <= s1; sIdx++) vertex(r, sIdx, m);
            for (uint32_t r = 0; r < r1 - r0; r++)
                for (uint32_t q = 0; q < s1 - s0; q++) {
                    const uint32_t v00 = r * cols + q, v01 = v00 + 1, v10 = v00 + cols, v11 = v10 + 1;
                    if (r + r0 != 0) { uint32_t t[3] = {v00, v01, v10}; m.idx.insert(m.idx.end(), t, t + 3); }
                    if (r + r0 + 1 != rings) { uint32_t t[3] = {v01, v11, v10}; m.idx.insert(m.idx.end(), t, t + 3); }
                }
            if (!m.idx.empty()) add_instance(*h, m, patch % nmat);
        }
    // Two emissive quads as area lights.
    const float elo[3] = {-0.8f, 1.3f, -0.8f}, ehi[3] = {0.8f, 1.5f, 0.8f};
    add_emitters(*h, rng, p.emissive_count ? p.emissive_count : 8, elo, ehi, 0.3f, 0.6f, 20.f, 60.f);
    if (p.envmap_width && p.envmap_height) make_envmap(*h, p.envmap_width, p.envmap_height);
    const float cam[3] = {0.f, 0.4f, 2.2f}, tgt[3] = {0.f, 0.f, 0.f};
    set_camera(*h, cam, tgt, 40.f, p.aspect_ratio > 0.f ? p.aspect_ratio : 1.f);
    return h;
}

fpt_scene_host* build_random_soup(const fpt_procedural_params& p) {
    auto* h = new fpt_scene_host();
    std::mt19937_64 rng(p.seed);
    const uint32_t nmat = p.material_count ? p.material_count : 256;
    random_materials(*h, rng, nmat);
    const uint32_t count = p.soup_triangles ? p.soup_triangles : 10000;
    const float lo[3] = {-1.f, -1.f, -1.f}, hi[3] = {1.f, 0.6f, 1.f};
    Mesh all = random_soup(rng, count, lo, hi, 1e-3f, 1e-1f);
    const uint32_t chunks = std::min<uint32_t>(256, count);
    std::uniform_int_distribution<uint32_t> mdist(0, nmat - 1);
    for (uint32_t c = 0; c < chunks; c++) {
        uint32_t t0 = uint32_t(uint64_t(count) * c / chunks), t1 = uint32_t(uint64_t(count) * (c + 1) / chunks);
        Mesh m;
        m.pos.assign(all.pos.begin() + size_t(t0) * 9, all.pos.begin() + size_t(t1) * 9);
        m.nrm.assign(all.nrm.begin() + size_t(t0) * 9, all.nrm.begin() + size_t(t1) * 9);
        for (uint32_t t = 0; t < (t1 - t0) * 3; t++) m.idx.push_back(t);
        add_instance(*h, m, mdist(rng));
    }
    const float elo[3] = {-0.9f, 0.7f, -0.9f}, ehi[3] = {0.9f, 0.95f, 0.9f};
    add_emitters(*h, rng, p.emissive_count ? p.emissive_count : 64, elo, ehi, 0.02f, 0.1f, 1.f, 1e3f);
    if (p.envmap_width && p.envmap_height) make_envmap(*h, p.envmap_width, p.envmap_height);
    const float cam[3] = {0.f, 0.5f, 2.6f}, tgt[3] = {0.f, -0.1f, 0.f};
    set_camera(*h, cam, tgt, 45.f, p.aspect_ratio > 0.f ? p.aspect_ratio : 1.f);
    return h;
}

fpt_scene_host* build_displaced_grid(const fpt_procedural_params& p) {
    auto* h = new fpt_scene_host();
    std::mt19937_64 rng(p.seed);
    const uint32_t nmat = p.material_count ? p.material_count : 256;
    random_materials(*h, rng, nmat);
    const uint32_t res = p.grid_res ? p.grid_res : 225;
    std::vector<Mesh> tiles = heightfield(res, 4, p.seed, 0.2f, 4.f);
    for (size_t i = 0; i < tiles.size(); i++) add_instance(*h, tiles[i], uint32_t(i % nmat));
    const float elo[3] = {-0.9f, 0.7f, -0.9f}, ehi[3] = {0.9f, 0.95f, 0.9f};
    add_emitters(*h, rng, p.emissive_count ? p.emissive_count : 64, elo, ehi, 0.02f, 0.1f, 1.f, 1e3f);
    if (p.envmap_width && p.envmap_height) make_envmap(*h, p.envmap_width, p.envmap_height);
    const float cam[3] = {0.f, 1.0f, 2.0f}, tgt[3] = {0.f, 0.f, 0.f};
    set_camera(*h, cam, tgt, 45.f, p.aspect_ratio > 0.f ? p.aspect_ratio : 1.f);
    return h;
}

// Builds a procedural scene; throws std::invalid_argument on an unknown kind.
fpt_scene_host* build_procedural_scene(const fpt_procedural_params& p) {
    fpt_scene_host* h = nullptr;
    switch (p.kind) {
        case FPT_SCENE_BOX_ICOSPHERE: h = build_box_icosphere(p); break;
        case FPT_SCENE_HEIGHTFIELD_SOUP: h = build_heightfield_soup(p); break;
        case FPT_SCENE_DISPLACED_SPHERE: h = build_displaced_sphere(p); break;
        case FPT_SCENE_RANDOM_SOUP: h = build_random_soup(p); break;
        case FPT_SCENE_DISPLACED_GRID: h = build_displaced_grid(p); break;
        default: throw std::invalid_argument("unknown procedural scene kind " + std::to_string(p.kind));
    }
    fpt_camera cam = h->desc.camera;
    h->finalize();
    h->desc.camera = cam;
    return h;
}

}  // namespace
