// oracle_scene.cpp -- scene packing, light collection, env-map importance map
// and a simple binary BVH for the CPU oracle.
//
// TEST INFRASTRUCTURE ONLY (see oracle_math.h).
#include "oracle_scene.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <stdexcept>

namespace orc {

PackedVertex pack_vertex(const fpt_vertex& v) {
    // PackedStaticVertexData::pack, HOST_CODE branch (Scene/SceneTypes.slang:236-256).
    PackedVertex p;
    for (int i = 0; i < 3; i++) p.pos[i] = v.position[i];
    p.uv[0] = v.texcoord[0];
    p.uv[1] = v.texcoord[1];
    uint32_t nx = f32tof16_host(v.normal[0]), ny = f32tof16_host(v.normal[1]), nz = f32tof16_host(v.normal[2]);
    uint32_t tw = f32tof16_host(v.tangent[3]);
    p.nxy = (ny << 16) | nx;
    p.nz_tw = (tw << 16) | nz;
    p.tangentOct = encode_normal2x16(V3<float>(v.tangent[0], v.tangent[1], v.tangent[2]));
    return p;
}

static uint32_t allocate_bits(uint32_t count) {
    // HitInfo.cpp:45-50.
    if (count <= 1) return 0;
    uint32_t maxValue = count - 1, b = 0;
    while (maxValue >> b) b++;
    return b;
}

void generate_alias_table(std::vector<float> weights, std::vector<uint32_t>& table, float& weightSum) {
    const uint32_t N = uint32_t(weights.size());
    table.assign(size_t(N) * 2, 0u);
    if (N == 0) { weightSum = 0.f; return; }
    std::mt19937 rng;  // EmissivePowerSampler::mAliasTableRng, default seed
    std::uniform_int_distribution<uint32_t> rngDist;
    double sum = 0.0;
    for (float f : weights) sum += f;
    for (float& f : weights) f *= N / float(sum);
    std::vector<uint32_t> permutation(N);
    for (uint32_t i = 0; i < N; ++i) permutation[i] = i;
    std::sort(permutation.begin(), permutation.end(), [&](uint32_t a, uint32_t b) { return weights[a] < weights[b]; });
    std::vector<float> thresholds(N);
    std::vector<uint32_t> redirect(N);
    uint32_t head = 0, tail = N - 1;
    while (head != tail) {
        int i = int(permutation[head]);
        int j = int(permutation[tail]);
        thresholds[i] = weights[i];
        redirect[i] = uint32_t(j);
        weights[j] -= 1.0f - weights[i];
        if (head == tail - 1) {
            thresholds[j] = 1.0f;
            redirect[j] = uint32_t(j);
            break;
        } else if (weights[j] < 1.0f) {
            std::swap(permutation[head], permutation[tail]);
            tail--;
        } else {
            head++;
        }
    }
    for (uint32_t i = 0; i < N; ++i) permutation[i] = i;
    for (uint32_t i = 0; i < N; ++i) {
        uint32_t dst = i + (rngDist(rng) % (N - i));
        std::swap(thresholds[i], thresholds[dst]);
        std::swap(redirect[i], redirect[dst]);
        std::swap(permutation[i], permutation[dst]);
    }
    for (uint32_t i = 0; i < N; ++i) {
        uint32_t prob = uint32_t(f32tof16_host(thresholds[i])) << 16u;
        uint32_t lx = redirect[i] & 0xFFFFFFu, ly = permutation[i] & 0xFFFFFFu;
        table[2 * i + 0] = prob | ((lx >> 8u) & 0xFFFFu);
        table[2 * i + 1] = ((lx & 0xFFu) << 24u) | ly;
    }
    weightSum = float(sum);
}

// Camera::calculateCameraParameters (Scene/Camera/Camera.cpp:112-195), the
// ray-tracing vectors only: frame height preserved, fovY from
// focalLengthToFovY (Utils/Math/FalcorMath.h:123-126), 0 focal length = 0 FOV.
void camera_data_from(const fpt_camera& c, fpt_camera_data& o) {
    const float fovY = c.focal_length == 0.0f ? 0.0f : 2.0f * std::atan(0.5f * c.frame_height / c.focal_length);
    const V3<float> posW(c.position[0], c.position[1], c.position[2]);
    const V3<float> target(c.target[0], c.target[1], c.target[2]);
    const V3<float> up(c.up[0], c.up[1], c.up[2]);
    const V3<float> camW = normalize(target - posW) * c.focal_distance;
    V3<float> camU = normalize(cross(camW, up));
    V3<float> camV = normalize(cross(camU, camW));
    const float ulen = c.focal_distance * std::tan(fovY * 0.5f) * c.aspect_ratio;
    camU = camU * ulen;
    const float vlen = c.focal_distance * std::tan(fovY * 0.5f);
    camV = camV * vlen;
    const V3<float>* vs[4] = {&posW, &camU, &camV, &camW};
    float* outs[4] = {o.posW, o.cameraU, o.cameraV, o.cameraW};
    for (int k = 0; k < 4; k++) { outs[k][0] = vs[k]->x; outs[k][1] = vs[k]->y; outs[k][2] = vs[k]->z; }
    o.nearZ = c.near_z;
    o.farZ = c.far_z;
    o.jitterX = c.jitter_x;
    o.jitterY = c.jitter_y;
}

Scene::Scene(const fpt_scene_desc* d, const fpt_camera_data* cam, uint32_t aliasSeed) {
    if (!d) throw std::runtime_error("null scene");
    if (cam) camera = *cam;
    else camera_data_from(d->camera, camera);
    vertices.resize(d->vertex_count);
    for (uint32_t i = 0; i < d->vertex_count; i++) vertices[i] = pack_vertex(d->vertices[i]);
    indices.assign(d->indices, d->indices + d->index_count);
    instances.assign(d->instances, d->instances + d->instance_count);
    materials.resize(d->material_count);
    for (uint32_t m = 0; m < d->material_count; m++) {
        const fpt_material& s = d->materials[m];
        Material& o = materials[m];
        for (int i = 0; i < 4; i++) { o.baseColor[i] = quantize_f16(s.base_color[i]); o.specular[i] = quantize_f16(s.specular[i]); }
        for (int i = 0; i < 3; i++) { o.emissive[i] = s.emissive[i]; o.transmission[i] = quantize_f16(s.transmission[i]); }
        o.emissiveFactor = s.emissive_factor;
        o.ior = quantize_f16(s.ior);
        o.specTrans = quantize_f16(s.specular_transmission);
        o.diffTrans = quantize_f16(s.diffuse_transmission);
        o.doubleSided = (s.flags & FPT_MATERIAL_DOUBLE_SIDED) != 0;
        o.thinSurface = (s.flags & FPT_MATERIAL_THIN_SURFACE) != 0;
        o.activeLobes = LOBE_ALL;
        V3<float> e = V3<float>(o.emissive[0], o.emissive[1], o.emissive[2]) * o.emissiveFactor;
        o.emissiveNonZero = any_pos(e);
        if (d->base_color_textures && d->base_color_textures[m]) o.baseColorTexture = int32_t(d->base_color_textures[m]) - 1;
    }
    // Material textures (StandardMaterial base colour), texels decoded once.
    float srgb[256];
    fpt_tex::srgb_decode_table(srgb);
    textures.resize(d->texture_count);
    for (uint32_t t = 0; t < d->texture_count; t++) {
        const fpt_texture_desc& td = d->textures[t];
        TextureO& o = textures[t];
        o.width = td.width;
        o.height = td.height;
        o.format = td.format;
        o.texelBase = texelCount;
        const size_t n = size_t(td.width) * td.height;
        texelCount += uint32_t(n);
        o.rgb.resize(n * 3);
        for (size_t i = 0; i < n; i++)
            for (int c = 0; c < 3; c++) {
                if (td.format == FPT_TEXTURE_RGBA32_FLOAT) o.rgb[3 * i + c] = static_cast<const float*>(td.texels)[4 * i + c];
                else {
                    const uint8_t b = static_cast<const uint8_t*>(td.texels)[4 * i + c];
                    o.rgb[3 * i + c] = td.format == FPT_TEXTURE_RGBA8_UNORM_SRGB ? srgb[b] : fpt_tex::unorm8(b);
                }
            }
    }
    // Global triangle numbering: instance-major, primitive-minor.
    uint32_t total = 0, maxTris = 0;
    instanceTriOffset.resize(instances.size());
    for (size_t i = 0; i < instances.size(); i++) {
        instanceTriOffset[i] = total;
        total += instances[i].triangle_count;
        maxTris = std::max(maxTris, instances[i].triangle_count);
    }
    triInstance.resize(total);
    triPrim.resize(total);
    triV.resize(size_t(total) * 3);
    for (uint32_t i = 0; i < instances.size(); i++) {
        for (uint32_t p = 0; p < instances[i].triangle_count; p++) {
            uint32_t g = instanceTriOffset[i] + p;
            triInstance[g] = i;
            triPrim[g] = p;
            uint32_t idx[3];
            getTriangleVertexIndices(i, p, idx);
            for (int k = 0; k < 3; k++) {
                const float* q = vertices[idx[k]].pos;
                triV[size_t(g) * 3 + k] = V3<float>(q[0], q[1], q[2]);
            }
        }
    }
    hitBits.type_bits = allocate_bits(7);  // HitType::Count
    hitBits.instance_id_bits = allocate_bits(uint32_t(instances.size()));
    hitBits.primitive_index_bits = allocate_bits(maxTris);
    buildBVH();
    buildLights(aliasSeed);
    buildEnv(d->envmap);
}

void Scene::getTriangleVertexIndices(uint32_t instanceID, uint32_t prim, uint32_t idx[3]) const {
    // Scene::getIndices with 32-bit indexed vertices (Scene/Scene.slang:276-332).
    const fpt_geometry_instance& in = instances[instanceID];
    for (int k = 0; k < 3; k++) idx[k] = indices[in.ib_offset + prim * 3 + k] + in.vb_offset;
}

StaticVertex Scene::getVertex(uint32_t gi) const {
    // PackedStaticVertexData::unpack (Scene/SceneTypes.slang:276-294).
    const PackedVertex& p = vertices[gi];
    StaticVertex v;
    v.position = V3<float>(p.pos[0], p.pos[1], p.pos[2]);
    v.uv = V2<float>(p.uv[0], p.uv[1]);
    v.normal = normalize(V3<float>(f16tof32(p.nxy & 0xffffu), f16tof32(p.nxy >> 16), f16tof32(p.nz_tw & 0xffffu)));
    V3<float> t = decode_normal2x16(p.tangentOct);
    float tw = f16tof32(p.nz_tw >> 16);
    v.tangent[0] = t.x; v.tangent[1] = t.y; v.tangent[2] = t.z; v.tangent[3] = sgn(tw);
    return v;
}

void Scene::buildLights(uint32_t) {
    // LightCollection: emissive triangles of every instance with an emissive
    // material, in instance order (LightCollection.cpp), positions and
    // area/normal from Scene::computeFaceNormalAndAreaW (Scene/Scene.slang:392-407),
    // packed with PackedEmissiveTriangle::pack and flux from
    // FinalizeIntegration.cs.slang:103-111.
    instanceEmissiveOffset.assign(instances.size(), 0xffffffffu);
    emissive.clear();
    for (uint32_t i = 0; i < instances.size(); i++) {
        const Material& m = materials[instances[i].material_id];
        if (!m.emissiveNonZero) continue;
        instanceEmissiveOffset[i] = uint32_t(emissive.size());
        for (uint32_t p = 0; p < instances[i].triangle_count; p++) {
            uint32_t idx[3];
            getTriangleVertexIndices(i, p, idx);
            EmissiveTri t;
            for (int k = 0; k < 3; k++) {
                const PackedVertex& pv = vertices[idx[k]];
                t.posW[k] = V3<float>(pv.pos[0], pv.pos[1], pv.pos[2]);
                t.uv[k] = V2<float>(quantize_f16(pv.uv[0]), quantize_f16(pv.uv[1]));
            }
            V3<float> e0 = t.posW[1] - t.posW[0], e1 = t.posW[2] - t.posW[0];
            V3<float> N = cross(e0, e1);
            t.area = 0.5f * length(N);
            if (instances[i].flags & FPT_INSTANCE_FRONT_FACE_CW) N = -N;
            t.normalEnc = encode_normal2x16(normalize(N));
            t.normal = decode_normal2x16(t.normalEnc);
            t.materialID = instances[i].material_id;
            V3<float> avg(m.emissive[0], m.emissive[1], m.emissive[2]);
            t.averageRadiance = avg * m.emissiveFactor;
            t.flux = luminance(t.averageRadiance) * t.area * float(3.14159265358979323846);
            emissive.push_back(t);
        }
    }
    activeTriangles.clear();
    std::vector<float> w(emissive.size());
    for (uint32_t k = 0; k < emissive.size(); k++) {
        if (emissive[k].flux > 0.f) activeTriangles.push_back(k);
        w[k] = emissive[k].flux;
    }
    generate_alias_table(w, aliasTable, aliasWeightSum);
    // LightBVHBuilder::build on the light collection's CPU copy, whose normals are
    // the unpacked octahedral ones decoded by the host code (normalize = v * rsqrt).
    std::vector<float> lv, ln, lf;
    for (const EmissiveTri& t : emissive) {
        for (int k = 0; k < 3; k++) { lv.push_back(t.posW[k].x); lv.push_back(t.posW[k].y); lv.push_back(t.posW[k].z); }
        const V2<float> o = unpack_snorm2x16(t.normalEnc);
        V3<float> n(o.x, o.y, 1.f - std::fabs(o.x) - std::fabs(o.y));
        if (n.z < 0.f) { V2<float> wv = oct_wrap(V2<float>(n.x, n.y)); n.x = wv.x; n.y = wv.y; }
        n = n * (1.f / std::sqrt(dot(n, n)));
        ln.push_back(n.x); ln.push_back(n.y); ln.push_back(n.z);
        lf.push_back(t.flux);
    }
    build_light_bvh_oracle(lv, ln, lf, [](float v) { return f32tof16_host(v); },
                           [](const float* d) { return encode_normal2x16(V3<float>(d[0], d[1], d[2])); }, lightBvh);
}

void Scene::buildEnv(const fpt_envmap_desc* env) {
    hasEnv = env && env->rgb && env->width && env->height;
    if (!hasEnv) return;
    envW = env->width; envH = env->height;
    envRGB.assign(env->rgb, env->rgb + size_t(envW) * envH * 3);
    for (int i = 0; i < 3; i++) envScale[i] = env->intensity * env->tint[i];
    // EnvMapSampler::createImportanceMap (EnvMapSampler.cpp:74-109) with the
    // default 512^2 texels x 64 samples, base mip from EnvMapSamplerSetup.cs.slang,
    // then a 2x2 box-filtered mip chain down to 1x1.
    impDim = 512;
    const uint32_t samplesX = 8, samplesY = 8;
    const float invSamples = 1.f / float(samplesX * samplesY);
    const uint32_t dimS = impDim * samplesX;
    uint32_t mips = 0;
    while ((1u << mips) < impDim) mips++;
    impBaseMip = mips;
    impMips.assign(mips + 1, {});
    impMips[0].resize(size_t(impDim) * impDim);
    for (uint32_t py = 0; py < impDim; py++) {
        for (uint32_t px = 0; px < impDim; px++) {
            float L = 0.f;
            for (uint32_t y = 0; y < samplesY; y++) {
                for (uint32_t x = 0; x < samplesX; x++) {
                    float sx = float(px * samplesX + x), sy = float(py * samplesY + y);
                    V2<float> p((sx + 0.5f) / float(dimS), (sy + 0.5f) / float(dimS));
                    V3<float> dir = oct_to_ndir_equal_area_unorm(p);
                    V2<float> uv = world_to_latlong_map(dir);
                    // gEnvMap.SampleLevel without intensity: bilinear texel fetch.
                    float fx = uv.x * float(envW) - 0.5f, fy = uv.y * float(envH) - 0.5f;
                    float x0f = std::floor(fx), y0f = std::floor(fy);
                    float ax = fx - x0f, ay = fy - y0f;
                    int x0 = int(x0f), y0 = int(y0f);
                    int W = int(envW), H = int(envH);
                    int xa = ((x0 % W) + W) % W, xb = (((x0 + 1) % W) + W) % W;
                    int ya = std::min(std::max(y0, 0), H - 1), yb = std::min(std::max(y0 + 1, 0), H - 1);
                    V3<float> rad(0.f);
                    const float* T = envRGB.data();
                    auto tex = [&](int xx, int yy) { const float* q = T + (size_t(yy) * W + xx) * 3; return V3<float>(q[0], q[1], q[2]); };
                    rad = tex(xa, ya) * ((1.f - ax) * (1.f - ay)) + tex(xb, ya) * (ax * (1.f - ay)) +
                          tex(xa, yb) * ((1.f - ax) * ay) + tex(xb, yb) * (ax * ay);
                    L += luminance(rad);
                }
            }
            impMips[0][size_t(py) * impDim + px] = L * invSamples;
        }
    }
    for (uint32_t m = 1; m <= mips; m++) {
        uint32_t d = impDim >> m, ds = impDim >> (m - 1);
        impMips[m].resize(size_t(d) * d);
        for (uint32_t y = 0; y < d; y++)
            for (uint32_t x = 0; x < d; x++) {
                const std::vector<float>& s = impMips[m - 1];
                float a = s[size_t(2 * y) * ds + 2 * x], b = s[size_t(2 * y) * ds + 2 * x + 1];
                float c = s[size_t(2 * y + 1) * ds + 2 * x], e = s[size_t(2 * y + 1) * ds + 2 * x + 1];
                impMips[m][size_t(y) * d + x] = (a + b + c + e) * 0.25f;
            }
    }
}

template <class R> static V3<R> env_bilinear(const Scene& s, V2<R> uv) {
    R fx = uv.x * R(s.envW) - R(0.5f), fy = uv.y * R(s.envH) - R(0.5f);
    R x0f = std::floor(fx), y0f = std::floor(fy);
    R ax = fx - x0f, ay = fy - y0f;
    int x0 = int(x0f), y0 = int(y0f);
    int W = int(s.envW), H = int(s.envH);
    int xa = ((x0 % W) + W) % W, xb = (((x0 + 1) % W) + W) % W;
    int ya = std::min(std::max(y0, 0), H - 1), yb = std::min(std::max(y0 + 1, 0), H - 1);
    auto tex = [&](int xx, int yy) {
        const float* q = s.envRGB.data() + (size_t(yy) * W + xx) * 3;
        return V3<R>(R(q[0]), R(q[1]), R(q[2]));
    };
    V3<R> c = tex(xa, ya) * ((R(1) - ax) * (R(1) - ay)) + tex(xb, ya) * (ax * (R(1) - ay)) +
              tex(xa, yb) * ((R(1) - ax) * ay) + tex(xb, yb) * (ax * ay);
    return c * V3<R>(R(s.envScale[0]), R(s.envScale[1]), R(s.envScale[2]));
}

V3<float> Scene::envEval(V3<float> dir) const {
    if (!hasEnv) return V3<float>(0.f);
    return env_bilinear<float>(*this, world_to_latlong_map(dir));
}
V3<double> Scene::envEvalD(V3<double> dir) const {
    if (!hasEnv) return V3<double>(0.0);
    return env_bilinear<double>(*this, world_to_latlong_map(dir));
}

// ---------------------------------------------------------------------------
// Binary BVH (median split on the longest centroid axis).  Its shape does not
// matter for the results: closest hits are defined by the watertight test,
// the [tMin, tMax] interval and the tie-break on the global triangle index.
// ---------------------------------------------------------------------------
void Scene::buildBVH() {
    const uint32_t n = uint32_t(triInstance.size());
    order.resize(n);
    std::iota(order.begin(), order.end(), 0u);
    nodes.clear();
    nodes.reserve(size_t(n) * 2 + 1);
    std::vector<float> cen(size_t(n) * 3);
    for (uint32_t i = 0; i < n; i++)
        for (int a = 0; a < 3; a++)
            cen[size_t(i) * 3 + a] = (triV[size_t(i) * 3][a] + triV[size_t(i) * 3 + 1][a] + triV[size_t(i) * 3 + 2][a]) * (1.f / 3.f);
    struct Item { uint32_t node, first, count; };
    std::vector<Item> stack;
    nodes.push_back(Node{});
    stack.push_back({0, 0, n});
    while (!stack.empty()) {
        Item it = stack.back();
        stack.pop_back();
        Node nd;
        for (int a = 0; a < 3; a++) { nd.lo[a] = 1e30f; nd.hi[a] = -1e30f; }
        float clo[3] = {1e30f, 1e30f, 1e30f}, chi[3] = {-1e30f, -1e30f, -1e30f};
        for (uint32_t k = it.first; k < it.first + it.count; k++) {
            uint32_t t = order[k];
            for (int v = 0; v < 3; v++)
                for (int a = 0; a < 3; a++) {
                    nd.lo[a] = std::min(nd.lo[a], triV[size_t(t) * 3 + v][a]);
                    nd.hi[a] = std::max(nd.hi[a], triV[size_t(t) * 3 + v][a]);
                }
            for (int a = 0; a < 3; a++) {
                clo[a] = std::min(clo[a], cen[size_t(t) * 3 + a]);
                chi[a] = std::max(chi[a], cen[size_t(t) * 3 + a]);
            }
        }
        nd.left = nd.right = 0;
        nd.first = it.first;
        nd.count = it.count;
        if (it.count > 4) {
            int axis = 0;
            for (int a = 1; a < 3; a++)
                if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
            uint32_t mid = it.first + it.count / 2;
            std::nth_element(order.begin() + it.first, order.begin() + mid, order.begin() + it.first + it.count,
                             [&](uint32_t x, uint32_t y) {
                                 float cx = cen[size_t(x) * 3 + axis], cy = cen[size_t(y) * 3 + axis];
                                 return cx < cy || (cx == cy && x < y);
                             });
            nd.left = uint32_t(nodes.size());
            nodes.push_back(Node{});
            nd.right = uint32_t(nodes.size());
            nodes.push_back(Node{});
            nd.count = 0;
            stack.push_back({nd.right, mid, it.first + it.count - mid});
            stack.push_back({nd.left, it.first, mid - it.first});
        }
        nodes[it.node] = nd;
    }
}

template <class R>
Hit Scene::traceImpl(V3<R> o, V3<R> d, R tMin, R tMax, bool anyHit, TraceCounters* c) const {
    Hit best;
    R bestT = tMax;
    uint32_t bestTri = 0xffffffffu;
    R bestU = 0, bestV = 0;
    // Conservative slab test: every interval is widened by a few ulps so that
    // no box that the ray touches within [tMin, tMax] is culled.
    V3<R> inv(R(1) / d.x, R(1) / d.y, R(1) / d.z);
    uint32_t stack[128];
    int sp = 0;
    stack[sp++] = 0;
    if (c) { if (anyHit) c->shadow++; else c->closest++; }
    while (sp > 0) {
        const Node& nd = nodes[stack[--sp]];
        R t0 = tMin, t1 = bestT;
        bool miss = false;
        for (int a = 0; a < 3; a++) {
            R ta = (R(nd.lo[a]) - o[a]) * inv[a], tb = (R(nd.hi[a]) - o[a]) * inv[a];
            if (std::isnan(ta) || std::isnan(tb)) { ta = -std::numeric_limits<R>::infinity(); tb = std::numeric_limits<R>::infinity(); }
            if (ta > tb) std::swap(ta, tb);
            ta = ta - std::fabs(ta) * R(1e-5) - R(1e-30);
            tb = tb + std::fabs(tb) * R(1e-5) + R(1e-30);
            t0 = std::max(t0, ta);
            t1 = std::min(t1, tb);
            if (t0 > t1) { miss = true; break; }
        }
        if (miss) continue;
        if (nd.count == 0) {
            stack[sp++] = nd.left;
            stack[sp++] = nd.right;
            continue;
        }
        for (uint32_t k = nd.first; k < nd.first + nd.count; k++) {
            uint32_t tri = order[k];
            V3<R> v[3] = {cvt3<R>(triV[size_t(tri) * 3]), cvt3<R>(triV[size_t(tri) * 3 + 1]), cvt3<R>(triV[size_t(tri) * 3 + 2])};
            V3<R> bary;
            R t;
            if (c) c->triTests++;
            if (!intersect_ray_triangle(o, d, v, bary, t)) continue;
            if (!(t >= tMin && t <= bestT)) continue;
            if (t == bestT && tri > bestTri) continue;
            bestT = t;
            bestTri = tri;
            bestU = bary.y;
            bestV = bary.z;
            if (anyHit) {
                best.valid = true;
                return best;
            }
        }
    }
    if (bestTri != 0xffffffffu) {
        best.valid = true;
        best.globalTri = bestTri;
        best.instanceID = triInstance[bestTri];
        best.primitiveIndex = triPrim[bestTri];
        best.baryX = float(bestU);
        best.baryY = float(bestV);
        best.t = float(bestT);
    }
    return best;
}

void Scene::attachBvh8(const void* nodes, uint32_t nodeCount, const void* tris, uint32_t triCount) {
    b8nodes.resize(nodeCount);
    b8tris.resize(triCount);
    if (nodeCount) std::memcpy(b8nodes.data(), nodes, size_t(nodeCount) * sizeof(Bvh8NodeO));
    if (triCount) std::memcpy(b8tris.data(), tris, size_t(triCount) * sizeof(Bvh8TriO));
}

// Exact traversal of the attached 8-wide BVH: child boxes decoded in double,
// exact slab tests against [tMin, best t], hit children visited nearest entry
// first (a child whose entry lies beyond the best hit found meanwhile is
// skipped when popped).  Counts every node visited and every triangle tested:
// the algorithmic work of a closest-hit (any-hit) query on this tree.
Hit Scene::traceBvh8(V3<float> o, V3<float> d, float tMin, float tMax, bool anyHit, uint64_t& nodes, uint64_t& tris) const {
    Hit best;
    float bestT = tMax;
    uint32_t bestTri = 0xffffffffu;
    float bestU = 0.f, bestV = 0.f;
    if (b8nodes.empty()) return best;
    const double inv[3] = {1.0 / double(d.x), 1.0 / double(d.y), 1.0 / double(d.z)};
    const double org[3] = {o.x, o.y, o.z};
    struct Entry { uint32_t node; double t; };
    std::vector<Entry> stack;
    stack.reserve(128);
    stack.push_back({0u, double(tMin)});
    while (!stack.empty()) {
        const Entry e = stack.back();
        stack.pop_back();
        if (e.t > double(bestT)) continue;
        const Bvh8NodeO& n = b8nodes[e.node];
        nodes++;
        Entry kids[8];
        int nk = 0;
        uint32_t rank = 0;
        for (int k = 0; k < 8; k++) {
            const bool internal = (n.imask >> k) & 1u;
            const uint32_t childRank = internal ? rank++ : 0u;
            const uint32_t meta = n.meta[k];
            if (!internal && meta == 0) continue;  // empty slot
            double t0 = double(tMin), t1 = double(bestT);
            for (int a = 0; a < 3 && t0 <= t1; a++) {
                const double s = std::ldexp(1.0, int(n.e[a]) - 127);
                const double lo = double(n.p[a]) + double(n.qlo[a][k]) * s, hi = double(n.p[a]) + double(n.qhi[a][k]) * s;
                double ta = (lo - org[a]) * inv[a], tb = (hi - org[a]) * inv[a];
                if (std::isnan(ta) || std::isnan(tb)) { ta = -INFINITY; tb = INFINITY; }
                if (ta > tb) std::swap(ta, tb);
                t0 = std::max(t0, ta);
                t1 = std::min(t1, tb);
            }
            if (t0 > t1) continue;
            if (internal) {
                kids[nk++] = {n.childBase + childRank, t0};
                continue;
            }
            // Leaf slot: its triangles are tested now (nearest-first order
            // matters only across internal children).
            const uint32_t first = n.triBase + (meta & 31u), count = meta >> 5;
            for (uint32_t i = 0; i < count; i++) {
                const Bvh8TriO& tr = b8tris[first + i];
                V3<float> v[3] = {V3<float>(tr.v0[0], tr.v0[1], tr.v0[2]), V3<float>(tr.v1[0], tr.v1[1], tr.v1[2]),
                                  V3<float>(tr.v2[0], tr.v2[1], tr.v2[2])};
                V3<float> bary;
                float t;
                tris++;
                if (!intersect_ray_triangle(o, d, v, bary, t)) continue;
                if (!(t >= tMin && t <= bestT)) continue;
                if (t == bestT && tr.globalTri > bestTri) continue;
                bestT = t;
                bestTri = tr.globalTri;
                bestU = bary.y;
                bestV = bary.z;
                if (anyHit) {
                    best.valid = true;
                    return best;
                }
            }
        }
        // Push far to near so that the nearest child is popped first.
        for (int i = 1; i < nk; i++)  // insertion sort, descending t (at most 8 entries)
            for (int j = i; j > 0 && kids[j - 1].t < kids[j].t; j--) std::swap(kids[j - 1], kids[j]);
        for (int i = 0; i < nk; i++) stack.push_back(kids[i]);
    }
    if (bestTri != 0xffffffffu) {
        best.valid = true;
        best.globalTri = bestTri;
        best.baryX = bestU;
        best.baryY = bestV;
        best.t = bestT;
    }
    return best;
}

Hit Scene::traceClosest(V3<float> o, V3<float> d, float tMin, float tMax, TraceCounters* c) const {
    Hit h = traceImpl<float>(o, d, tMin, tMax, false, c);
    if (c && !b8nodes.empty()) {
        const Hit g = traceBvh8(o, d, tMin, tMax, false, c->b8NodesClosest, c->b8TrisClosest);
        if (g.valid != h.valid || (h.valid && (g.globalTri != h.globalTri || g.t != h.t))) c->b8Mismatch++;
    }
    return h;
}
bool Scene::traceVisibility(V3<float> o, V3<float> d, float tMin, float tMax, TraceCounters* c) const {
    const bool vis = !traceImpl<float>(o, d, tMin, tMax, true, c).valid;
    if (c && !b8nodes.empty()) {
        const Hit g = traceBvh8(o, d, tMin, tMax, true, c->b8NodesShadow, c->b8TrisShadow);
        if (g.valid == vis) c->b8Mismatch++;
    }
    return vis;
}
Hit Scene::traceClosestD(V3<double> o, V3<double> d, double tMin, double tMax) const {
    return traceImpl<double>(o, d, tMin, tMax, false, nullptr);
}
bool Scene::traceVisibilityD(V3<double> o, V3<double> d, double tMin, double tMax) const {
    return !traceImpl<double>(o, d, tMin, tMax, true, nullptr).valid;
}

Hit Scene::traceClosestBrute(V3<float> o, V3<float> d, float tMin, float tMax) const {
    Hit best;
    float bestT = tMax;
    uint32_t bestTri = 0xffffffffu;
    float bu = 0, bv = 0;
    for (uint32_t tri = 0; tri < triInstance.size(); tri++) {
        V3<float> v[3] = {triV[size_t(tri) * 3], triV[size_t(tri) * 3 + 1], triV[size_t(tri) * 3 + 2]};
        V3<float> bary;
        float t;
        if (!intersect_ray_triangle(o, d, v, bary, t)) continue;
        if (!(t >= tMin && t <= bestT)) continue;
        if (t == bestT && tri > bestTri) continue;
        bestT = t; bestTri = tri; bu = bary.y; bv = bary.z;
    }
    if (bestTri != 0xffffffffu) {
        best.valid = true;
        best.globalTri = bestTri;
        best.instanceID = triInstance[bestTri];
        best.primitiveIndex = triPrim[bestTri];
        best.baryX = bu; best.baryY = bv; best.t = bestT;
    }
    return best;
}

}  // namespace orc
