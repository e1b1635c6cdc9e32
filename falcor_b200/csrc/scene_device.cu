// scene_device.cu -- device scene creation: BVH build, vertex/material
// packing, light collection with the power-sampler alias table, environment
// map upload and the env-map importance map (built on the GPU).
//
// Replaces Scene (Scene/Scene.cpp), its driver-built BLAS/TLAS
// (Scene::buildBlas Scene.cpp:3376), LightCollection (LightCollection.cpp,
// UpdateTriangleVertices.cs.slang, FinalizeIntegration.cs.slang),
// EmissivePowerSampler::generateAliasTable (EmissivePowerSampler.cpp:86-175)
// and EnvMapSampler::createImportanceMap (EnvMapSampler.cpp:74-109).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <random>
#include <string>

#include "f16.h"
#include "scene_device.h"

namespace fpt {

namespace {

// Env-map importance map base mip (EnvMapSamplerSetup.cs.slang:46-70):
// 512^2 texels x 8x8 samples of the bilinearly filtered env map luminance.
__global__ void importance_base_kernel(const float4* env, uint32_t envW, uint32_t envH, uint32_t dim, uint32_t spx,
                                       float* out) {
    using namespace dev;
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= dim || y >= dim) return;
    const float invSamples = 1.f / float(spx * spx);
    const float dimS = float(dim * spx);
    float L = 0.f;
    for (uint32_t sy = 0; sy < spx; sy++)
        for (uint32_t sx = 0; sx < spx; sx++) {
            const float2 p = make_float2((float(x * spx + sx) + 0.5f) / dimS, (float(y * spx + sy) + 0.5f) / dimS);
            const float3 dir = oct_to_ndir_equal_area_unorm(p);
            const float2 uv = world_to_latlong_map(dir);
            const float fx = uv.x * float(envW) - 0.5f, fy = uv.y * float(envH) - 0.5f;
            const float x0f = floorf(fx), y0f = floorf(fy);
            const float ax = fx - x0f, ay = fy - y0f;
            const int x0 = int(x0f), y0 = int(y0f), W = int(envW), H = int(envH);
            const int xa = ((x0 % W) + W) % W, xb = (((x0 + 1) % W) + W) % W;
            const int ya = min(max(y0, 0), H - 1), yb = min(max(y0 + 1, 0), H - 1);
            auto tex = [&](int xx, int yy) { const float4 t = env[size_t(yy) * W + xx]; return make_float3(t.x, t.y, t.z); };
            const float3 r = tex(xa, ya) * ((1.f - ax) * (1.f - ay)) + tex(xb, ya) * (ax * (1.f - ay)) +
                             tex(xa, yb) * ((1.f - ax) * ay) + tex(xb, yb) * (ax * ay);
            L += luminance(r);
        }
    out[size_t(y) * dim + x] = L * invSamples;
}

// 2x2 box-filtered mip level (the reference relies on generateMips()).
__global__ void importance_mip_kernel(const float* src, uint32_t srcDim, float* dst) {
    const uint32_t d = srcDim / 2;
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= d || y >= d) return;
    const float a = src[size_t(2 * y) * srcDim + 2 * x], b = src[size_t(2 * y) * srcDim + 2 * x + 1];
    const float c = src[size_t(2 * y + 1) * srcDim + 2 * x], e = src[size_t(2 * y + 1) * srcDim + 2 * x + 1];
    dst[size_t(y) * d + x] = (a + b + c + e) * 0.25f;
}

float luminance_host(const float c[3]) { return c[0] * 0.2126f + c[1] * 0.7152f + c[2] * 0.0722f; }

// EmissivePowerSampler::generateAliasTable (EmissivePowerSampler.cpp:86-175):
// Vose-style pairing over weights sorted ascending, then a random permutation
// of the table drawn from a default-seeded std::mt19937, packed as an fp16
// threshold plus two 24-bit indices.
void build_alias_table(std::vector<float> weights, std::vector<uint32_t>& table, float& weightSum) {
    const uint32_t N = uint32_t(weights.size());
    table.assign(size_t(N) * 2, 0u);
    weightSum = 0.f;
    if (N == 0) return;
    std::mt19937 rng;
    std::uniform_int_distribution<uint32_t> dist;
    double sum = 0.0;
    for (float f : weights) sum += f;
    for (float& f : weights) f *= N / float(sum);
    std::vector<uint32_t> perm(N);
    for (uint32_t i = 0; i < N; i++) perm[i] = i;
    std::sort(perm.begin(), perm.end(), [&](uint32_t a, uint32_t b) { return weights[a] < weights[b]; });
    std::vector<float> thr(N, 0.f);
    std::vector<uint32_t> redir(N, 0u);
    uint32_t head = 0, tail = N - 1;
    while (head != tail) {
        const uint32_t i = perm[head], j = perm[tail];
        thr[i] = weights[i];
        redir[i] = j;
        weights[j] -= 1.0f - weights[i];
        if (head == tail - 1) { thr[j] = 1.0f; redir[j] = j; break; }
        if (weights[j] < 1.0f) { std::swap(perm[head], perm[tail]); tail--; }
        else head++;
    }
    for (uint32_t i = 0; i < N; i++) perm[i] = i;
    for (uint32_t i = 0; i < N; i++) {
        const uint32_t dst = i + (dist(rng) % (N - i));
        std::swap(thr[i], thr[dst]);
        std::swap(redir[i], redir[dst]);
        std::swap(perm[i], perm[dst]);
    }
    for (uint32_t i = 0; i < N; i++) {
        const uint32_t prob = uint32_t(f32_to_f16_host(thr[i])) << 16;
        const uint32_t lx = redir[i] & 0xFFFFFFu, ly = perm[i] & 0xFFFFFFu;
        table[2 * i] = prob | ((lx >> 8) & 0xFFFFu);
        table[2 * i + 1] = ((lx & 0xFFu) << 24) | ly;
    }
    weightSum = float(sum);
}

template <class T>
fpt_status upload(DeviceBuffers& b, const std::vector<T>& v, const T*& out) {
    out = nullptr;
    if (v.empty()) return FPT_OK;
    void* p = nullptr;
    const size_t bytes = v.size() * sizeof(T);
    if (cudaMalloc(&p, bytes) != cudaSuccess) return set_error(FPT_ERR_OOM, "cudaMalloc failed (" + std::to_string(bytes) + " bytes)");
    b.ptrs.push_back(p);
    b.bytes += bytes;
    if (cudaMemcpy(p, v.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess) return set_error(FPT_ERR_CUDA, "cudaMemcpy failed");
    out = static_cast<const T*>(p);
    return FPT_OK;
}

}  // namespace

DeviceBuffers::~DeviceBuffers() {
    for (void* p : ptrs) cudaFree(p);
}

// BasicMaterialData packing of a StandardMaterial (fp16 fields quantised on
// the host like Falcor's float16_t, Utils/Math/Float16.cpp:56-169).
DevMaterial pack_material(const fpt_material& s0, uint32_t baseColorTexture) {
    DevMaterial o;
    std::memset(&o, 0, sizeof(o));
    for (int k = 0; k < 4; k++) { o.baseColor[k] = f32_to_f16_host(s0.base_color[k]); o.specular[k] = f32_to_f16_host(s0.specular[k]); }
    for (int k = 0; k < 3; k++) { o.emissive[k] = s0.emissive[k]; o.transmission[k] = f32_to_f16_host(s0.transmission[k]); }
    o.emissiveFactor = s0.emissive_factor;
    o.ior = f32_to_f16_host(s0.ior);
    o.specTrans = f32_to_f16_host(s0.specular_transmission);
    o.diffTrans = f32_to_f16_host(s0.diffuse_transmission);
    o.flags = uint16_t((s0.flags & FPT_MATERIAL_DOUBLE_SIDED ? 1u : 0u) | (s0.flags & FPT_MATERIAL_THIN_SURFACE ? 2u : 0u));
    o.activeLobes = 0xff;
    if (baseColorTexture) {
        o.flags |= kMatFlagBaseColorTexture;
        o.baseColorTexture = baseColorTexture - 1;
    }
    return o;
}

// Host-side checks of a scene description, before any device work: the
// arrays exist, positions are finite and within |x| <= 1e15 (the traversal's
// conservative box test needs |coordinate| * |1/d| to stay finite), every
// index, material and texture reference is in range.
fpt_status validate_desc(const fpt_scene_desc& d) {
    if (d.vertex_count && !d.vertices) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_create: vertices is NULL");
    if (d.index_count && !d.indices) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_create: indices is NULL");
    if (d.instance_count && !d.instances) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_create: instances is NULL");
    if (d.material_count == 0 || !d.materials) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_create: no materials");
    for (uint32_t i = 0; i < d.vertex_count; i++)
        for (int a = 0; a < 3; a++)
            if (!(std::fabs(d.vertices[i].position[a]) <= 1e15f))
                return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_create: vertex " + std::to_string(i) +
                                                          " has a non-finite or out-of-range (|x| > 1e15) position");
    for (uint32_t i = 0; i < d.instance_count; i++) {
        const fpt_geometry_instance& in = d.instances[i];
        if (in.material_id >= d.material_count) return set_error(FPT_ERR_INVALID_ARG, "instance material_id out of range");
        if (uint64_t(in.ib_offset) + uint64_t(in.triangle_count) * 3 > d.index_count)
            return set_error(FPT_ERR_INVALID_ARG, "instance index range out of bounds");
        for (uint64_t k = 0; k < uint64_t(in.triangle_count) * 3; k++)
            if (uint64_t(d.indices[in.ib_offset + k]) + in.vb_offset >= d.vertex_count)
                return set_error(FPT_ERR_INVALID_ARG, "vertex index out of bounds");
    }
    if (d.texture_count && !d.textures) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_create: textures is NULL");
    for (uint32_t t = 0; t < d.texture_count; t++) {
        const fpt_texture_desc& td = d.textures[t];
        if (!td.texels || td.width == 0 || td.height == 0 || td.width > 65536 || td.height > 65536 || td.format > FPT_TEXTURE_RGBA32_FLOAT)
            return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_create: texture " + std::to_string(t) +
                                                      " needs texels, a size in [1, 65536]^2 and a known format");
    }
    if (d.base_color_textures)
        for (uint32_t m = 0; m < d.material_count; m++)
            if (d.base_color_textures[m] > d.texture_count)
                return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_create: material " + std::to_string(m) + " names a missing texture");
    return FPT_OK;
}

fpt_status create_scene(const fpt_scene_desc& d, fpt_scene*& out) {
    const fpt_status vs = validate_desc(d);
    if (vs != FPT_OK) return vs;
    int devCount = 0;
    if (cudaGetDeviceCount(&devCount) != cudaSuccess || devCount == 0)
        return set_error(FPT_ERR_NO_DEVICE, "fpt_scene_create: no CUDA device");
    auto sc = std::make_unique<fpt_scene>();
    fpt_scene& s = *sc;
    compute_camera(d.camera, s.info.camera);
    s.info.hit_bits = compute_hit_bits(d);
    if (s.info.hit_bits.primitive_index_bits > 32 || s.info.hit_bits.type_bits + s.info.hit_bits.instance_id_bits > 32)
        return set_error(FPT_ERR_UNSUPPORTED, "scene requires > 64 bits of HitInfo header");

    // Global triangle list (instance-major) with world-space vertices.
    uint32_t total = 0;
    for (uint32_t i = 0; i < d.instance_count; i++) {
        const fpt_geometry_instance& in = d.instances[i];
        if (in.material_id >= d.material_count) return set_error(FPT_ERR_INVALID_ARG, "instance material_id out of range");
        if (uint64_t(in.ib_offset) + uint64_t(in.triangle_count) * 3 > d.index_count)
            return set_error(FPT_ERR_INVALID_ARG, "instance index range out of bounds");
        total += in.triangle_count;
    }
    std::vector<float> triVerts(size_t(total) * 9);
    std::vector<uint32_t> triInst(total), triPrim(total);
    bool hasTransmission = false;
    {
        uint32_t g = 0;
        for (uint32_t i = 0; i < d.instance_count; i++) {
            const fpt_geometry_instance& in = d.instances[i];
            for (uint32_t t = 0; t < in.triangle_count; t++, g++) {
                for (int k = 0; k < 3; k++) {
                    const uint32_t vi = d.indices[in.ib_offset + t * 3 + k] + in.vb_offset;
                    if (vi >= d.vertex_count) return set_error(FPT_ERR_INVALID_ARG, "vertex index out of bounds");
                    std::memcpy(&triVerts[size_t(g) * 9 + size_t(k) * 3], d.vertices[vi].position, 12);
                }
                triInst[g] = i;
                triPrim[g] = t;
            }
        }
    }
    try {
        build_bvh8(triVerts, triInst, triPrim, s.bvh);
    } catch (const std::exception& e) {
        return set_error(FPT_ERR_INVALID_ARG, std::string("BVH build failed: ") + e.what());
    }
    if (s.bvh.maxDepth > uint32_t(dev::kStackSize))
        return set_error(FPT_ERR_UNSUPPORTED, "BVH depth " + std::to_string(s.bvh.maxDepth) + " exceeds the traversal stack");

    // Packed vertices (PackedStaticVertexData::pack, Scene/SceneTypes.slang:236-256).
    std::vector<PackedVertex> pv(d.vertex_count);
    for (uint32_t i = 0; i < d.vertex_count; i++) {
        const fpt_vertex& v = d.vertices[i];
        PackedVertex& p = pv[i];
        std::memcpy(p.pos, v.position, 12);
        p.uv[0] = v.texcoord[0];
        p.uv[1] = v.texcoord[1];
        const uint32_t nx = f32_to_f16_host(v.normal[0]), ny = f32_to_f16_host(v.normal[1]), nz = f32_to_f16_host(v.normal[2]);
        const uint32_t tw = f32_to_f16_host(v.tangent[3]);
        p.nxy = (ny << 16) | nx;
        p.nz_tw = (tw << 16) | nz;
        p.tangentOct = encode_normal_2x16_host(v.tangent);
    }
    std::vector<DevInstance> inst(d.instance_count);
    for (uint32_t i = 0; i < d.instance_count; i++)
        inst[i] = DevInstance{d.instances[i].vb_offset, d.instances[i].ib_offset, d.instances[i].material_id, d.instances[i].flags};
    std::vector<DevMaterial> mats(d.material_count);
    std::vector<bool> emissiveMat(d.material_count, false);
    s.materials.assign(d.materials, d.materials + d.material_count);
    s.baseColorTex.assign(d.material_count, 0u);
    if (d.base_color_textures) s.baseColorTex.assign(d.base_color_textures, d.base_color_textures + d.material_count);
    for (uint32_t m = 0; m < d.material_count; m++) {
        const fpt_material& s0 = d.materials[m];
        DevMaterial& o = mats[m];
        o = pack_material(s0, s.baseColorTex[m]);
        if (f16_to_f32_host(o.specTrans) > 0.f || f16_to_f32_host(o.diffTrans) > 0.f) hasTransmission = true;
        emissiveMat[m] = (s0.emissive[0] * s0.emissive_factor > 0.f) || (s0.emissive[1] * s0.emissive_factor > 0.f) ||
                         (s0.emissive[2] * s0.emissive_factor > 0.f);
    }

    // Light collection (instance order), flux and alias table.
    std::vector<DevEmissiveTri> em;
    std::vector<float> flux;
    std::vector<uint32_t> instOff(d.instance_count, 0xffffffffu), active;
    std::vector<float> emVerts, emNormals;  // light BVH input
    for (uint32_t i = 0; i < d.instance_count; i++) {
        const fpt_geometry_instance& in = d.instances[i];
        if (!emissiveMat[in.material_id]) continue;
        instOff[i] = uint32_t(em.size());
        const fpt_material& m = d.materials[in.material_id];
        for (uint32_t t = 0; t < in.triangle_count; t++) {
            DevEmissiveTri e;
            std::memset(&e, 0, sizeof(e));
            float P[3][3];
            uint32_t uvp[3];
            for (int k = 0; k < 3; k++) {
                const fpt_vertex& v = d.vertices[d.indices[in.ib_offset + t * 3 + k] + in.vb_offset];
                std::memcpy(P[k], v.position, 12);
                uvp[k] = (uint32_t(f32_to_f16_host(v.texcoord[1])) << 16) | f32_to_f16_host(v.texcoord[0]);
            }
            std::memcpy(e.p0, P[0], 12); e.uv0 = uvp[0];
            std::memcpy(e.p1, P[1], 12); e.uv1 = uvp[1];
            std::memcpy(e.p2, P[2], 12); e.uv2 = uvp[2];
            // Scene::computeFaceNormalAndAreaW (Scene/Scene.slang:392-407).
            const float e0[3] = {P[1][0] - P[0][0], P[1][1] - P[0][1], P[1][2] - P[0][2]};
            const float e1[3] = {P[2][0] - P[0][0], P[2][1] - P[0][1], P[2][2] - P[0][2]};
            float N[3] = {e0[1] * e1[2] - e0[2] * e1[1], e0[2] * e1[0] - e0[0] * e1[2], e0[0] * e1[1] - e0[1] * e1[0]};
            const float len = std::sqrt(N[0] * N[0] + N[1] * N[1] + N[2] * N[2]);
            e.area = 0.5f * len;
            if (in.flags & FPT_INSTANCE_FRONT_FACE_CW) { N[0] = -N[0]; N[1] = -N[1]; N[2] = -N[2]; }
            const float nn[3] = {N[0] / len, N[1] / len, N[2] / len};
            e.normal = encode_normal_2x16_host(nn);
            for (int k = 0; k < 3; k++)
                for (int a = 0; a < 3; a++) emVerts.push_back(P[k][a]);
            // The builder sees the light collection's unpacked (decoded) normal
            // (LightCollection::syncCPUData, LightCollection.cpp:680-689).
            float dn[3];
            decode_normal_2x16_host(e.normal, dn);
            for (int a = 0; a < 3; a++) emNormals.push_back(dn[a]);
            e.materialID = in.material_id;
            e.lightIdx = i;
            // FinalizeIntegration.cs.slang:103-111.
            const float avg[3] = {m.emissive[0] * m.emissive_factor, m.emissive[1] * m.emissive_factor, m.emissive[2] * m.emissive_factor};
            const float f = luminance_host(avg) * e.area * float(3.14159265358979323846);
            if (f > 0.f) active.push_back(uint32_t(em.size()));
            em.push_back(e);
            flux.push_back(f);
        }
    }
    build_alias_table(flux, s.aliasTable, s.aliasWeightSum);
    try {
        build_light_bvh(emVerts, emNormals, flux, s.lightBvh);
    } catch (const std::exception& ex) {
        return set_error(FPT_ERR_UNSUPPORTED, std::string("light BVH build failed: ") + ex.what());
    }
    s.meshVertexCount.assign(d.instance_count, 0);
    s.meshTriCount.assign(d.instance_count, 0);
    s.meshEmissive.assign(d.instance_count, 0);
    for (uint32_t i = 0; i < d.instance_count; i++) {
        const fpt_geometry_instance& in = d.instances[i];
        uint32_t nv = 0;
        for (uint32_t k = 0; k < in.triangle_count * 3; k++) nv = std::max(nv, d.indices[in.ib_offset + k] + 1);
        s.meshVertexCount[i] = nv;
        s.meshTriCount[i] = in.triangle_count;
        s.meshEmissive[i] = instOff[i] != 0xffffffffu ? 1 : 0;
    }
    std::vector<uint2> alias(em.size());
    for (size_t i = 0; i < em.size(); i++) alias[i] = make_uint2(s.aliasTable[2 * i], s.aliasTable[2 * i + 1]);

    DevScene& ds = s.dev;
    std::memset(&ds, 0, sizeof(ds));
    DeviceBuffers& B = s.buffers;
    fpt_status st;
    const BVH8Node* nodesPtr;
    const TriRecord* trisPtr;
    if ((st = upload(B, s.bvh.nodes, nodesPtr)) != FPT_OK) return st;
    if ((st = upload(B, s.bvh.tris, trisPtr)) != FPT_OK) return st;
    ds.nodes = reinterpret_cast<const uint4*>(nodesPtr);
    ds.tris = reinterpret_cast<const float4*>(trisPtr);
    if ((st = upload(B, pv, ds.vertices)) != FPT_OK) return st;
    std::vector<uint32_t> idx(d.indices, d.indices + d.index_count);
    if ((st = upload(B, idx, ds.indices)) != FPT_OK) return st;
    if ((st = upload(B, inst, ds.instances)) != FPT_OK) return st;
    if ((st = upload(B, mats, ds.materials)) != FPT_OK) return st;
    if ((st = upload(B, em, ds.emissive)) != FPT_OK) return st;
    if ((st = upload(B, flux, ds.flux)) != FPT_OK) return st;
    if ((st = upload(B, alias, ds.alias)) != FPT_OK) return st;
    if ((st = upload(B, instOff, ds.instEmissiveOffset)) != FPT_OK) return st;
    if ((st = upload(B, active, ds.activeTris)) != FPT_OK) return st;
    {
        const LightBVHNode* ln;
        if ((st = upload(B, s.lightBvh.nodes, ln)) != FPT_OK) return st;
        ds.lbvhNodes = reinterpret_cast<const uint4*>(ln);
        if ((st = upload(B, s.lightBvh.triIndices, ds.lbvhTriIndices)) != FPT_OK) return st;
        std::vector<uint2> masks(s.lightBvh.bitmasks.size());
        for (size_t i = 0; i < masks.size(); i++)
            masks[i] = make_uint2(uint32_t(s.lightBvh.bitmasks[i]), uint32_t(s.lightBvh.bitmasks[i] >> 32));
        if ((st = upload(B, masks, ds.lbvhBitmasks)) != FPT_OK) return st;
        ds.lbvhNodeCount = uint32_t(s.lightBvh.nodes.size());
    }
    ds.emissiveCount = uint32_t(em.size());
    ds.activeCount = uint32_t(active.size());
    ds.invWeightSum = s.aliasWeightSum > 0.f ? 1.0f / s.aliasWeightSum : 0.f;
    ds.hasEmissive = em.empty() ? 0u : 1u;
    ds.hasTransmission = hasTransmission ? 1u : 0u;
    ds.nodeCount = uint32_t(s.bvh.nodes.size());
    ds.triCount = uint32_t(s.bvh.tris.size());  // triangle records (spatial splits repeat a triangle)
    ds.bvhDepth = s.bvh.maxDepth;
    for (int a = 0; a < 3; a++) {
        ds.sceneLo[a] = s.bvh.lo[a];
        const float ext = s.bvh.hi[a] - s.bvh.lo[a];
        ds.sceneInvExtent[a] = ext > 0.f ? 1.f / ext : 0.f;
    }
    ds.materialCount = d.material_count;
    ds.camera = s.info.camera;
    ds.bits = s.info.hit_bits;

    // Environment map and importance map.
    const fpt_envmap_desc* env = d.envmap;
    if (env && env->rgb && env->width && env->height) {
        std::vector<float4> texels(size_t(env->width) * env->height);
        for (size_t i = 0; i < texels.size(); i++) texels[i] = make_float4(env->rgb[3 * i], env->rgb[3 * i + 1], env->rgb[3 * i + 2], 0.f);
        if ((st = upload(B, texels, ds.env)) != FPT_OK) return st;
        ds.envW = env->width;
        ds.envH = env->height;
        for (int k = 0; k < 3; k++) ds.envScale[k] = env->intensity * env->tint[k];
        ds.hasEnv = 1;
        const uint32_t dim = 512, spx = 8;
        uint32_t mips = 0;
        while ((1u << mips) < dim) mips++;
        ds.impDim = dim;
        ds.impBaseMip = mips;
        size_t totalFloats = 0;
        for (uint32_t m = 0; m <= mips; m++) { ds.impMipOffset[m] = uint32_t(totalFloats); totalFloats += size_t(dim >> m) * (dim >> m); }
        void* imp = nullptr;
        if (cudaMalloc(&imp, totalFloats * sizeof(float)) != cudaSuccess) return set_error(FPT_ERR_OOM, "cudaMalloc importance map");
        B.ptrs.push_back(imp);
        B.bytes += totalFloats * sizeof(float);
        float* impf = static_cast<float*>(imp);
        dim3 blk(16, 16);
        importance_base_kernel<<<dim3((dim + 15) / 16, (dim + 15) / 16), blk>>>(ds.env, ds.envW, ds.envH, dim, spx, impf);
        for (uint32_t m = 1; m <= mips; m++) {
            const uint32_t dd = dim >> m;
            importance_mip_kernel<<<dim3((dd + 15) / 16, (dd + 15) / 16), blk>>>(impf + ds.impMipOffset[m - 1], dim >> (m - 1),
                                                                               impf + ds.impMipOffset[m]);
        }
        if (cudaDeviceSynchronize() != cudaSuccess) return set_error(FPT_ERR_CUDA, std::string("importance map: ") + cudaGetErrorString(cudaGetLastError()));
        ds.impMips = impf;
    }
    // Material textures: one texel buffer (each texture 16-byte aligned), the
    // texture table and the sRGB decode table.
    if (d.texture_count) {
        std::vector<DevTexture> tex(d.texture_count);
        uint64_t bytes = 0;
        uint32_t texels = 0;
        for (uint32_t t = 0; t < d.texture_count; t++) {
            const fpt_texture_desc& td = d.textures[t];
            DevTexture& o = tex[t];
            std::memset(&o, 0, sizeof(o));
            o.offset = bytes;
            o.width = td.width;
            o.height = td.height;
            o.format = td.format;
            o.texelBase = texels;
            const uint64_t n = uint64_t(td.width) * td.height;
            if (uint64_t(texels) + n > 0x7fffffffull) return set_error(FPT_ERR_UNSUPPORTED, "fpt_scene_create: more than 2^31 texels");
            texels += uint32_t(n);
            bytes += (n * fpt_tex::texel_bytes(td.format) + 15u) & ~uint64_t(15);
        }
        std::vector<uint8_t> data(bytes, 0);
        for (uint32_t t = 0; t < d.texture_count; t++)
            std::memcpy(data.data() + tex[t].offset, d.textures[t].texels,
                        size_t(tex[t].width) * tex[t].height * fpt_tex::texel_bytes(tex[t].format));
        if ((st = upload(B, data, ds.texData)) != FPT_OK) return st;
        if ((st = upload(B, tex, ds.textures)) != FPT_OK) return st;
        float lut[256];
        fpt_tex::srgb_decode_table(lut);
        std::vector<float> lutv(lut, lut + 256);
        if ((st = upload(B, lutv, ds.srgbDecode)) != FPT_OK) return st;
        ds.textureCount = d.texture_count;
        s.textures = tex;
    }
    void* err = nullptr;
    if (cudaMalloc(&err, sizeof(uint32_t)) != cudaSuccess) return set_error(FPT_ERR_OOM, "cudaMalloc error word");
    B.ptrs.push_back(err);
    cudaMemset(err, 0, sizeof(uint32_t));
    ds.errorWord = static_cast<uint32_t*>(err);

    s.info.triangle_count = total;
    s.info.instance_count = d.instance_count;
    s.info.material_count = d.material_count;
    s.info.emissive_triangle_count = uint32_t(em.size());
    s.info.bvh_node_count = uint32_t(s.bvh.nodes.size());
    s.info.has_envmap = ds.hasEnv;
    s.info.bvh_build_seconds = s.bvh.buildSeconds;
    s.info.device_bytes = B.bytes;
    out = sc.release();
    return FPT_OK;
}

// Refreshes the host copy of the materials from the device after device-side
// updates (the device holds the fp16 values of the updated fields).
fpt_status sync_materials_from_device(fpt_scene& scene) {
    if (!scene.materialsOnDevice) return FPT_OK;
    std::vector<DevMaterial> dm(scene.materials.size());
    if (cudaMemcpy(dm.data(), scene.dev.materials, dm.size() * sizeof(DevMaterial), cudaMemcpyDeviceToHost) != cudaSuccess)
        return set_error(FPT_ERR_CUDA, "material parameters: download failed");
    for (size_t i = 0; i < dm.size(); i++) {
        fpt_material& m = scene.materials[i];
        for (int k = 0; k < 3; k++) {
            m.base_color[k] = f16_to_f32_host(dm[i].baseColor[k]);
            m.transmission[k] = f16_to_f32_host(dm[i].transmission[k]);
        }
        m.specular[1] = f16_to_f32_host(dm[i].specular[1]);
        m.specular[2] = f16_to_f32_host(dm[i].specular[2]);
        m.ior = f16_to_f32_host(dm[i].ior);
        m.specular_transmission = f16_to_f32_host(dm[i].specTrans);
        m.diffuse_transmission = f16_to_f32_host(dm[i].diffTrans);
    }
    scene.materialsOnDevice = false;
    return FPT_OK;
}

// setMaterialParams on the device: the differentiable fields of material
// ids[i] (i when ids is null) from params[i * 20 ...], packed like the host
// packer; emissive entries are ignored (the light collection is fixed).
__global__ void set_material_params_kernel(DevMaterial* mats, const uint32_t* ids, uint32_t count, const float* params) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t id = ids ? ids[i] : i;
        const float* v = params + size_t(i) * 20;
        DevMaterial& m = mats[id];
        for (int k = 0; k < 3; k++) {
            m.baseColor[k] = f32_to_f16_bits(v[k]);
            m.transmission[k] = f32_to_f16_bits(v[6 + k]);
        }
        m.specular[2] = f32_to_f16_bits(v[3]);
        m.specular[1] = f32_to_f16_bits(v[4]);
        m.ior = f32_to_f16_bits(v[5]);
        m.diffTrans = f32_to_f16_bits(v[9]);
        m.specTrans = f32_to_f16_bits(v[10]);
    }
}

}  // namespace fpt

using namespace fpt;

extern "C" {

FPT_API int fpt_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    int ok = 0;
    for (int i = 0; i < n; i++) {
        cudaDeviceProp p;
        if (cudaGetDeviceProperties(&p, i) == cudaSuccess && p.major == 10) ok++;
    }
    return ok;
}

FPT_API fpt_status fpt_scene_create(const fpt_scene_desc* desc, fpt_scene** out) {
    if (!desc || !out) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_create: null argument");
    *out = nullptr;
    try {
        return create_scene(*desc, *out);
    } catch (const std::exception& e) {
        return set_error(FPT_ERR_OOM, std::string("fpt_scene_create: ") + e.what());
    }
}

FPT_API void fpt_scene_destroy(fpt_scene* scene) { delete scene; }

FPT_API fpt_status fpt_scene_get_info(const fpt_scene* scene, fpt_scene_info* out) {
    if (!scene || !out) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_get_info: null argument");
    *out = scene->info;
    return FPT_OK;
}

FPT_API fpt_status fpt_scene_set_camera(fpt_scene* scene, const fpt_camera* camera) {
    if (!scene || !camera) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_set_camera: null argument");
    fpt_camera_data cd;
    compute_camera(*camera, cd);
    // A change of the jitter alone does not restart accumulation (Camera::Changes::Jitter).
    fpt_camera_data a = scene->info.camera, b = cd;
    a.jitterX = a.jitterY = b.jitterX = b.jitterY = 0.f;
    if (std::memcmp(&a, &b, sizeof(a)) != 0) scene->resetVersion++;
    scene->info.camera = cd;
    scene->dev.camera = cd;
    scene->version++;
    return FPT_OK;
}

// Serialized material parameters (Scene/Material/StandardMaterialParamLayout.slang:32-42,
// Material::serializeParams / deserializeParams): baseColor 0-2, metallic 3,
// roughness 4, ior 5, transmissionColor 6-8, diffuseTransmission 9,
// specularTransmission 10, emissiveColor 11-13, emissiveFactor 14, 15-19 unused.
FPT_API fpt_status fpt_scene_set_material_params_device(fpt_scene* scene, const uint32_t* ids, uint32_t count, const float* params,
                                                        void* stream) {
    if (!scene || (count && !params)) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_set_material_params_device: null argument");
    if (count == 0) return FPT_OK;
    const uint32_t nm = uint32_t(scene->materials.size());
    if (!ids && count > nm)
        return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_set_material_params_device: more parameter rows than materials");
    for (uint32_t i = 0; ids && i < count; i++)
        if (ids[i] >= nm) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_set_material_params_device: material ID out of range");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t* dIds = nullptr;
    if (ids) {
        if (scene->materialIdCapacity < count) {
            void* p = nullptr;
            if (cudaMalloc(&p, size_t(count) * 4) != cudaSuccess)
                return set_error(FPT_ERR_OOM, "fpt_scene_set_material_params_device: allocation failed");
            scene->buffers.ptrs.push_back(p);
            scene->materialIds = static_cast<uint32_t*>(p);
            scene->materialIdCapacity = count;
        }
        if (cudaMemcpyAsync(scene->materialIds, ids, size_t(count) * 4, cudaMemcpyHostToDevice, st) != cudaSuccess)
            return set_error(FPT_ERR_CUDA, "fpt_scene_set_material_params_device: ID upload failed");
        dIds = scene->materialIds;
    }
    const uint32_t grid = std::min<uint32_t>((count + 127) / 128, 1024);
    set_material_params_kernel<<<grid, 128, 0, st>>>(const_cast<DevMaterial*>(scene->dev.materials), dIds, count, params);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, std::string("fpt_scene_set_material_params_device: ") + cudaGetErrorString(e));
    // Transmission values are not read back: the transmission-capable kernels
    // (which render materials without transmission identically) are used from now on.
    scene->dev.hasTransmission = 1u;
    scene->materialsOnDevice = true;
    scene->version++;
    scene->resetVersion++;
    return FPT_OK;
}

FPT_API fpt_status fpt_scene_get_material_params(const fpt_scene* cscene, const uint32_t* ids, uint32_t count, float* params) {
    const fpt_scene* scene = cscene;
    if (!scene || (count && (!ids || !params))) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_get_material_params: null argument");
    if (scene->materialsOnDevice) {
        const fpt_status s = sync_materials_from_device(*const_cast<fpt_scene*>(scene));
        if (s != FPT_OK) return s;
    }
    for (uint32_t i = 0; i < count; i++) {
        if (ids[i] >= scene->materials.size()) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_get_material_params: material ID out of range");
        const fpt_material& m = scene->materials[ids[i]];
        float* o = params + size_t(i) * 20;
        std::memset(o, 0, 20 * sizeof(float));
        for (int k = 0; k < 3; k++) { o[k] = m.base_color[k]; o[6 + k] = m.transmission[k]; o[11 + k] = m.emissive[k]; }
        o[3] = m.specular[2];
        o[4] = m.specular[1];
        o[5] = m.ior;
        o[9] = m.diffuse_transmission;
        o[10] = m.specular_transmission;
        o[14] = m.emissive_factor;
    }
    return FPT_OK;
}

FPT_API fpt_status fpt_scene_set_material_params(fpt_scene* scene, const uint32_t* ids, uint32_t count, const float* params) {
    if (!scene || (count && (!ids || !params))) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_set_material_params: null argument");
    if (scene->materialsOnDevice) {
        const fpt_status st = sync_materials_from_device(*scene);
        if (st != FPT_OK) return st;
    }
    for (uint32_t i = 0; i < count; i++)
        if (ids[i] >= scene->materials.size()) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_set_material_params: material ID out of range");
    std::vector<fpt_material> next = scene->materials;
    for (uint32_t i = 0; i < count; i++) {
        fpt_material& m = next[ids[i]];
        const float* v = params + size_t(i) * 20;
        for (int k = 0; k < 3; k++) { m.base_color[k] = v[k]; m.transmission[k] = v[6 + k]; }
        m.specular[2] = v[3];
        m.specular[1] = v[4];
        m.ior = v[5];
        m.diffuse_transmission = v[9];
        m.specular_transmission = v[10];
        const fpt_material& cur = scene->materials[ids[i]];
        if (v[11] != cur.emissive[0] || v[12] != cur.emissive[1] || v[13] != cur.emissive[2] || v[14] != cur.emissive_factor)
            return set_error(FPT_ERR_UNSUPPORTED, "fpt_scene_set_material_params: emissive parameters are fixed (the light collection is not rebuilt)");
    }
    bool hasTransmission = false;
    for (uint32_t i = 0; i < count; i++) {
        const DevMaterial dm = pack_material(next[ids[i]], scene->baseColorTex[ids[i]]);
        if (cudaMemcpy(const_cast<DevMaterial*>(scene->dev.materials) + ids[i], &dm, sizeof(dm), cudaMemcpyHostToDevice) != cudaSuccess)
            return set_error(FPT_ERR_CUDA, "fpt_scene_set_material_params: upload failed");
    }
    for (const fpt_material& m : next)
        if (f16_to_f32_host(f32_to_f16_host(m.specular_transmission)) > 0.f || f16_to_f32_host(f32_to_f16_host(m.diffuse_transmission)) > 0.f)
            hasTransmission = true;
    scene->materials.swap(next);
    scene->dev.hasTransmission = hasTransmission ? 1u : 0u;
    scene->version++;
    scene->resetVersion++;
    return FPT_OK;
}

FPT_API fpt_status fpt_scene_set_texture_device(fpt_scene* scene, uint32_t index, const void* texels, void* stream) {
    if (!scene || !texels) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_set_texture_device: null argument");
    if (index >= scene->textures.size()) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_set_texture_device: texture index out of range");
    const DevTexture& t = scene->textures[index];
    const size_t bytes = size_t(t.width) * t.height * fpt_tex::texel_bytes(t.format);
    const cudaError_t e = cudaMemcpyAsync(const_cast<uint8_t*>(scene->dev.texData) + t.offset, texels, bytes, cudaMemcpyDeviceToDevice,
                                          static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, std::string("fpt_scene_set_texture_device: ") + cudaGetErrorString(e));
    scene->version++;
    scene->resetVersion++;
    return FPT_OK;
}

FPT_API fpt_status fpt_scene_get_bvh(const fpt_scene* scene, fpt_bvh_view* out) {
    if (!scene || !out) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_get_bvh: null argument");
    out->nodes = scene->bvh.nodes.data();
    out->node_count = uint32_t(scene->bvh.nodes.size());
    out->tris = scene->bvh.tris.data();
    out->tri_count = uint32_t(scene->bvh.tris.size());
    for (int a = 0; a < 3; a++) { out->scene_lo[a] = scene->bvh.lo[a]; out->scene_hi[a] = scene->bvh.hi[a]; }
    return FPT_OK;
}

FPT_API fpt_status fpt_scene_get_light_bvh(const fpt_scene* scene, fpt_light_bvh_view* out) {
    if (!scene || !out) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_get_light_bvh: null argument");
    const LightBVH& b = scene->lightBvh;
    out->nodes = b.nodes.empty() ? nullptr : b.nodes[0].w;
    out->node_count = uint32_t(b.nodes.size());
    out->triangle_indices = b.triIndices.data();
    out->triangle_index_count = uint32_t(b.triIndices.size());
    out->bitmasks = b.bitmasks.data();
    out->bitmask_count = uint32_t(b.bitmasks.size());
    return FPT_OK;
}

FPT_API fpt_status fpt_scene_get_alias_table(const fpt_scene* scene, uint32_t* pairs, uint32_t capacity, float* invWeightSum) {
    if (!scene) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_get_alias_table: null scene");
    const uint32_t n = uint32_t(scene->aliasTable.size() / 2);
    if (pairs) {
        if (capacity < n) return set_error(FPT_ERR_INVALID_ARG, "fpt_scene_get_alias_table: capacity too small");
        std::memcpy(pairs, scene->aliasTable.data(), size_t(n) * 8);
    }
    if (invWeightSum) *invWeightSum = scene->dev.invWeightSum;
    return FPT_OK;
}

}  // extern "C"
