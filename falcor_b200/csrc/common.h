// common.h -- internal declarations shared by the host C++ and the CUDA
// translation units of libfpt: error reporting, host math for camera and
// HitInfo set-up, and the device data layouts.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/fpt.h"

namespace fpt {

// Thread-local error message; returns `code` for convenient `return set_error(...)`.
fpt_status set_error(fpt_status code, const std::string& msg);
void log_warning(const std::string& msg);

// Camera::calculateCameraParameters ray-tracing vectors (Scene/Camera/Camera.cpp:112-195).
void compute_camera(const fpt_camera& cam, fpt_camera_data& out);

// HitInfo::init bit allocation (Scene/HitInfo.cpp:52-108), uncompressed format.
fpt_hitinfo_bits compute_hit_bits(const fpt_scene_desc& d);

// fp16 quantisation as done by the host scene packer (Utils/Math/Float16.cpp:56-169).
uint16_t f32_to_f16_host(float v);
float f16_to_f32_host(uint16_t h);
uint32_t encode_normal_2x16_host(const float n[3]);
void decode_normal_2x16_host(uint32_t p, float n[3]);

// ---------------------------------------------------------------------------
// Device data layouts (all 16-byte aligned).
// ---------------------------------------------------------------------------

// Compressed 8-wide BVH node, 80 bytes = 5 x 16-byte loads.
//   p[3]          origin of the quantisation grid
//   e[3]          per-axis scale exponents (scale = 2^(e - 127))
//   imask         bit k set: child slot k is an internal node
//   childBase     index of the first internal child (children are contiguous,
//                 in slot order of the internal slots)
//   triBase       index of the first triangle record of the leaf slots
//   meta[k]       leaf slot: (count << 5) | offset relative to triBase
//   q{lo,hi}{x,y,z}[k]  quantised child boxes; empty slots have lo > hi
struct alignas(16) BVH8Node {
    float p[3];
    uint8_t e[3];
    uint8_t imask;
    uint32_t childBase;
    uint32_t triBase;
    uint8_t meta[8];
    uint8_t qlox[8], qloy[8], qloz[8];
    uint8_t qhix[8], qhiy[8], qhiz[8];
};
static_assert(sizeof(BVH8Node) == 80, "BVH8Node must be 80 bytes");

// Triangle record in BVH leaf order, 48 bytes: three float4 with the
// world-space vertices in xyz and (globalTriangle, instanceID, primitiveIndex)
// in the w components (as integer bits).
struct alignas(16) TriRecord {
    float v0[3]; uint32_t globalTri;
    float v1[3]; uint32_t instanceID;
    float v2[3]; uint32_t primIndex;
};
static_assert(sizeof(TriRecord) == 48, "TriRecord must be 48 bytes");

// PackedStaticVertexData (Scene/SceneTypes.slang:226-294), 32 bytes.
struct alignas(16) PackedVertex {
    float pos[3];
    uint32_t nxy;         // fp16 normal.x | normal.y << 16
    uint32_t nz_tw;       // fp16 normal.z | fp16 tangent sign << 16
    uint32_t tangentOct;  // 2x16 snorm octahedral tangent
    float uv[2];
};
static_assert(sizeof(PackedVertex) == 32, "PackedVertex must be 32 bytes");

// GeometryInstanceData subset, 16 bytes.
struct alignas(16) DevInstance {
    uint32_t vbOffset, ibOffset, materialID, flags;
};

// StandardMaterial parameters as the shaders read them (fp16 where the
// reference stores fp16), 64 bytes; the shading code reads the first 48 bytes
// as three 16-byte loads.
struct alignas(16) DevMaterial {
    uint16_t baseColor[4];    // fp16 rgb + opacity
    uint16_t specular[4];     // fp16 occlusion, roughness, metallic, -
    float emissive[3];
    float emissiveFactor;
    uint16_t ior;             // fp16
    uint16_t specTrans;       // fp16
    uint16_t diffTrans;       // fp16
    uint16_t transmission[3]; // fp16
    uint16_t flags;           // bit0 double-sided, bit1 thin surface, bit2 base-colour texture
    uint16_t activeLobes;
    uint32_t baseColorTexture; // texture index when flags bit2 is set (the fourth 16-byte load)
    uint32_t pad[3];
};
static_assert(sizeof(DevMaterial) == 64, "DevMaterial must be 64 bytes");

constexpr uint16_t kMatFlagBaseColorTexture = 4;

// A material texture in the scene's texel buffer, 32 bytes.
struct alignas(16) DevTexture {
    uint64_t offset;     // byte offset of texel (0, 0) in the texel buffer
    uint32_t width, height;
    uint32_t format;     // fpt_texture_format
    uint32_t texelBase;  // texels of the textures before this one (gradient index base)
    uint32_t pad[2];
};
static_assert(sizeof(DevTexture) == 32, "DevTexture must be 32 bytes");

// PackedEmissiveTriangle (Scene/Lights/LightCollectionShared.slang:77-135), 64 bytes.
struct alignas(16) DevEmissiveTri {
    float p0[3]; uint32_t uv0;
    float p1[3]; uint32_t uv1;
    float p2[3]; uint32_t uv2;
    uint32_t normal;     // 2x16 snorm octahedral
    float area;
    uint32_t materialID;
    uint32_t lightIdx;
};
static_assert(sizeof(DevEmissiveTri) == 64, "DevEmissiveTri must be 64 bytes");

// Host-side BVH8 build result.
struct BVH8 {
    std::vector<BVH8Node> nodes;
    std::vector<TriRecord> tris;
    uint32_t maxDepth = 0;
    float lo[3], hi[3];
    double buildSeconds = 0;
};

// Builds a binned-SAH binary BVH with spatial splits (a triangle may be
// referenced by several leaves, each with its own record), collapses it to
// 8-wide nodes with octant slot ordering and quantises the child boxes
// conservatively.
void build_bvh8(const std::vector<float>& triVerts,  // 9 floats per global triangle
                const std::vector<uint32_t>& triInstance, const std::vector<uint32_t>& triPrim, BVH8& out);

// Light BVH (Rendering/Lights/LightBVH*.{cpp,slang}): 32-byte compressed
// PackedNode (LightBVHTypes.slang:102-200), the emissive-triangle index list of
// the leaves, and per emissive triangle the bit path to its leaf (all ones:
// culled, zero flux).
struct LightBVHNode {
    uint32_t w[8];
};
struct LightBVH {
    std::vector<LightBVHNode> nodes;
    std::vector<uint32_t> triIndices;
    std::vector<uint64_t> bitmasks;
};
// triVerts: 9 floats, triNormals: 3 floats (unit face normal), flux: 1 float per
// emissive triangle of the light collection.
void build_light_bvh(const std::vector<float>& triVerts, const std::vector<float>& triNormals, const std::vector<float>& flux,
                     LightBVH& out);

// Decodes a quantised child box exactly as the device does (fmaf(q, scale, p)).
void decode_child_box(const BVH8Node& n, int slot, float lo[3], float hi[3]);

}  // namespace fpt
