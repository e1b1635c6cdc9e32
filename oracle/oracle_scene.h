// oracle_scene.h -- the oracle's own copy of the scene as the reference shaders
// see it: packed vertices, fp16-quantised materials, the emissive light
// collection, the power-sampler alias table and the env-map importance map,
// plus a simple binary BVH used only to find closest hits quickly.
//
// TEST INFRASTRUCTURE ONLY (see oracle_math.h).
#pragma once

#include <vector>
#include <cstdint>
#include "oracle_math.h"
#include "oracle_lightbvh.h"
#include "../include/fpt.h"
#include "../falcor_b200/csrc/texture.h"

namespace orc {

// PackedStaticVertexData (Scene/SceneTypes.slang:226-294), host pack + device unpack.
struct PackedVertex {
    float pos[3];
    uint32_t nxy;        // fp16 normal.x | normal.y << 16
    uint32_t nz_tw;      // fp16 normal.z | fp16 tangent sign << 16
    uint32_t tangentOct; // encodeNormal2x16(tangent.xyz)
    float uv[2];
};

struct StaticVertex {  // StaticVertexData after unpack()
    V3<float> position, normal;
    float tangent[4];
    V2<float> uv;
};

// BasicMaterialData fields used by StandardMaterial (fp16 where the reference stores fp16).
struct Material {
    float baseColor[4];  // fp16-quantised
    float specular[4];   // fp16-quantised: occlusion, roughness, metallic
    float emissive[3];
    float emissiveFactor;
    float ior;           // fp16-quantised (MaterialHeader IoR)
    float specTrans, diffTrans;  // fp16-quantised
    float transmission[3];       // fp16-quantised
    bool doubleSided, thinSurface;
    uint32_t activeLobes;
    bool emissiveNonZero;
    int32_t baseColorTexture = -1;  // texture index, or -1 for the uniform baseColor
};

// A material texture with its texels decoded to linear rgb as the kernels
// decode them (sRGB table, c / 255, or the float value).
struct TextureO {
    uint32_t width = 0, height = 0, format = 0, texelBase = 0;
    std::vector<float> rgb;  // 3 floats per texel, row-major
};

// EmissiveTriangle after PackedEmissiveTriangle::unpack (LightCollectionShared.slang:41-135).
struct EmissiveTri {
    V3<float> posW[3];
    V2<float> uv[3];     // fp16-quantised
    V3<float> normal;    // decoded from the 2x16 octahedral encoding
    uint32_t normalEnc;  // the 2x16 octahedral encoding
    float area;
    uint32_t materialID;
    float flux;          // FinalizeIntegration.cs.slang:103-111
    V3<float> averageRadiance;
};

struct Hit {
    bool valid = false;
    uint32_t instanceID = 0, primitiveIndex = 0, globalTri = 0;
    float baryX = 0, baryY = 0;  // DXR-style barycentrics (weights of v1, v2)
    float t = 0;
};

struct TraceCounters {
    uint64_t closest = 0, shadow = 0, nodeVisits = 0, triTests = 0;
    // Exact nearest-first traversal of the library's 8-wide BVH (attachBvh8):
    // node visits and triangle tests of closest-hit and visibility rays, and
    // rays whose result differs from the oracle's own tree.
    uint64_t b8NodesClosest = 0, b8TrisClosest = 0, b8NodesShadow = 0, b8TrisShadow = 0, b8Mismatch = 0;
};

// The library's compressed 8-wide BVH node and triangle record, as
// falcor_b200/csrc/common.h lays them out (80 and 48 bytes): box slot k
// spans p + q{lo,hi}[k] 2^(e - 127) per axis; meta[k] = (count << 5) | offset
// of a leaf slot; internal children are contiguous from childBase in slot order.
struct Bvh8NodeO {
    float p[3];
    uint8_t e[3];
    uint8_t imask;
    uint32_t childBase, triBase;
    uint8_t meta[8];
    uint8_t qlo[3][8], qhi[3][8];
};
static_assert(sizeof(Bvh8NodeO) == 80, "Bvh8NodeO must be 80 bytes");
struct Bvh8TriO {
    float v0[3]; uint32_t globalTri;
    float v1[3]; uint32_t instanceID;
    float v2[3]; uint32_t primIndex;
};
static_assert(sizeof(Bvh8TriO) == 48, "Bvh8TriO must be 48 bytes");

// Camera::calculateCameraParameters ray-tracing vectors (Scene/Camera/Camera.cpp:112-195).
void camera_data_from(const fpt_camera& c, fpt_camera_data& o);

class Scene {
public:
    // cam == nullptr: the camera vectors are computed from d->camera here.
    Scene(const fpt_scene_desc* d, const fpt_camera_data* cam, uint32_t aliasSeedDefault = 1);

    // geometry
    std::vector<PackedVertex> vertices;
    std::vector<uint32_t> indices;
    std::vector<fpt_geometry_instance> instances;
    std::vector<uint32_t> triInstance, triPrim;     // global triangle -> (instance, primitive)
    std::vector<uint32_t> instanceTriOffset;        // instance -> first global triangle
    std::vector<V3<float>> triV;                    // 3 world-space positions per global triangle
    std::vector<Material> materials;
    fpt_camera_data camera;
    fpt_hitinfo_bits hitBits;

    // lights
    std::vector<EmissiveTri> emissive;
    std::vector<uint32_t> instanceEmissiveOffset;   // perMeshInstanceOffset, 0xffffffff if none
    std::vector<uint32_t> activeTriangles;
    std::vector<uint32_t> aliasTable;               // 2 uints per emissive triangle
    LightBvhOracle lightBvh;                        // LightBVH sampler data
    float aliasWeightSum = 0.f;

    // environment
    bool hasEnv = false;
    uint32_t envW = 0, envH = 0;
    std::vector<float> envRGB;
    float envScale[3] = {1, 1, 1};                  // intensity * tint
    uint32_t impDim = 0, impBaseMip = 0;
    std::vector<std::vector<float>> impMips;        // mip 0 = impDim^2

    // material textures
    std::vector<TextureO> textures;
    uint32_t texelCount = 0;

    // helpers
    StaticVertex getVertex(uint32_t globalIndex) const;
    void getTriangleVertexIndices(uint32_t instanceID, uint32_t prim, uint32_t idx[3]) const;
    uint32_t emissiveIndex(uint32_t instanceID, uint32_t prim) const {
        uint32_t o = instanceEmissiveOffset[instanceID];
        return o == 0xffffffffu ? 0xffffffffu : o + prim;
    }
    V3<float> envEval(V3<float> dir) const;         // EnvMap::eval (bilinear, wrap u, clamp v)
    V3<double> envEvalD(V3<double> dir) const;

    // traversal
    Hit traceClosest(V3<float> o, V3<float> d, float tMin, float tMax, TraceCounters* c) const;
    bool traceVisibility(V3<float> o, V3<float> d, float tMin, float tMax, TraceCounters* c) const;
    Hit traceClosestD(V3<double> o, V3<double> d, double tMin, double tMax) const;
    bool traceVisibilityD(V3<double> o, V3<double> d, double tMin, double tMax) const;

    // brute-force closest hit over all triangles (for traversal tests)
    Hit traceClosestBrute(V3<float> o, V3<float> d, float tMin, float tMax) const;
    // Attaches a copy of the library's 8-wide BVH: the FP32 traces then also
    // traverse it (exactly, nearest child first) to count the algorithmic node
    // visits and triangle tests into TraceCounters::b8*.
    void attachBvh8(const void* nodes, uint32_t nodeCount, const void* tris, uint32_t triCount);
    std::vector<Bvh8NodeO> b8nodes;
    std::vector<Bvh8TriO> b8tris;

private:
    struct Node { float lo[3], hi[3]; uint32_t left, right, first, count; };
    std::vector<Node> nodes;
    std::vector<uint32_t> order;
    void buildBVH();
    void buildLights(uint32_t aliasSeed);
    void buildEnv(const fpt_envmap_desc* env);
    template <class R> Hit traceImpl(V3<R> o, V3<R> d, R tMin, R tMax, bool anyHit, TraceCounters* c) const;
    Hit traceBvh8(V3<float> o, V3<float> d, float tMin, float tMax, bool anyHit, uint64_t& nodes, uint64_t& tris) const;
};

// MaterialSystem::sampleTexture with ExplicitLodTextureSampler(0)
// (MaterialSystem.slang:308-320): bilinear at mip 0 with wrap addressing
// (texture.h), accumulated in R in the kernels' order.
template <class R> V3<R> tex_sample(const Scene& s, uint32_t tex, float u, float v) {
    const TextureO& t = s.textures[tex];
    const fpt_tex::Bilinear b = fpt_tex::bilinear(u, v, t.width, t.height);
    auto texel = [&](uint32_t x, uint32_t y) {
        const float* c = &t.rgb[(size_t(y) * t.width + x) * 3];
        return V3<R>(R(c[0]), R(c[1]), R(c[2]));
    };
    V3<R> c = texel(b.x0, b.y0) * R(b.w[0]);
    c += texel(b.x1, b.y0) * R(b.w[1]);
    c += texel(b.x0, b.y1) * R(b.w[2]);
    c += texel(b.x1, b.y1) * R(b.w[3]);
    return c;
}

// Packs one vertex like PackedStaticVertexData::pack on the host.
PackedVertex pack_vertex(const fpt_vertex& v);

// EmissivePowerSampler::generateAliasTable (EmissivePowerSampler.cpp:86-175).
void generate_alias_table(std::vector<float> weights, std::vector<uint32_t>& table, float& weightSum);

}  // namespace orc
