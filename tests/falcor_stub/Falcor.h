// Stand-in for the slice of Falcor's C++ API that the FalcorB200 render-pass
// plugin (falcor_b200/plugin/FalcorB200Passes.cpp) uses, so that the plugin
// compiles and runs in this repository (Falcor itself needs its Slang and
// graphics toolchain).  Names and signatures follow the reference headers
// (Core/Plugin.h, Core/Object.h, Core/Error.h, Utils/Properties.h,
// RenderGraph/RenderPass.h, RenderPassHelpers.h, RenderPassReflection.h,
// Core/API/{Device,Buffer,Texture,CopyContext,Formats}.h, Core/Pass/ComputePass.h,
// Scene/{Scene,SceneTypes,Camera,EnvMap}.h, Scene/Material/StandardMaterial.h).
// Resources live in CUDA device memory; ComputePass runs C++ stand-ins of the
// plugin's two Slang programs.
//
// TEST INFRASTRUCTURE ONLY.
#pragma once

#include "Utils/CudaRuntime.h"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <sstream>
#include <stdexcept>
#include <string>
#include <string_view>
#include <utility>
#include <vector>

#define FALCOR_API_EXPORT __attribute__((visibility("default")))

namespace Falcor {

// ----- Core/Object.h -----------------------------------------------------------
template <class T> using ref = std::shared_ptr<T>;
template <class T, class... A> ref<T> make_ref(A&&... a) { return std::make_shared<T>(std::forward<A>(a)...); }
template <class T, class U> ref<T> dynamic_ref_cast(const ref<U>& p) { return std::dynamic_pointer_cast<T>(p); }

// ----- Core/Error.h / Utils/Logger.h (fmt-style "{}" formatting) ------------------
namespace detail {
inline void format_into(std::ostringstream& o, std::string_view f) { o << f; }
template <class T, class... A> void format_into(std::ostringstream& o, std::string_view f, const T& v, const A&... a) {
    const size_t p = f.find("{}");
    if (p == std::string_view::npos) { o << f; return; }
    o << f.substr(0, p) << v;
    format_into(o, f.substr(p + 2), a...);
}
template <class... A> std::string format(std::string_view f, const A&... a) {
    std::ostringstream o;
    format_into(o, f, a...);
    return o.str();
}
}  // namespace detail
inline std::vector<std::string>& warnings() { static std::vector<std::string> w; return w; }
template <class... A> void logWarning(std::string_view f, const A&... a) { warnings().push_back(detail::format(f, a...)); }
#define FALCOR_THROW(...) throw std::runtime_error(::Falcor::detail::format(__VA_ARGS__))

// ----- math ---------------------------------------------------------------------
struct float2 { float x = 0, y = 0; };
struct uint2 { uint32_t x = 0, y = 0; };
struct uint3 { uint32_t x = 0, y = 0, z = 0; };
struct float3 {
    float x = 0, y = 0, z = 0;
    float3() = default;
    float3(float a, float b, float c) : x(a), y(b), z(c) {}
};
struct float4 {
    float x = 0, y = 0, z = 0, w = 0;
    float4() = default;
    float4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    float3 xyz() const { return {x, y, z}; }
};
struct float4x4 {
    float m[4][4] = {{1, 0, 0, 0}, {0, 1, 0, 0}, {0, 0, 1, 0}, {0, 0, 0, 1}};  // row-major, column vectors
    static float4x4 identity() { return float4x4(); }
    // matrix::operator== (Utils/Math/MatrixTypes.h:167): bitwise.
    bool operator==(const float4x4& o) const { return std::memcmp(m, o.m, sizeof(m)) == 0; }
};
struct float3x3 {
    float m[3][3] = {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    float3x3() = default;
    explicit float3x3(const float4x4& a) {
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) m[r][c] = a.m[r][c];
    }
};
inline float4x4 transpose(const float4x4& a) {
    float4x4 t;
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) t.m[r][c] = a.m[c][r];
    return t;
}
inline float4x4 inverse(const float4x4& a) {  // Gauss-Jordan in double
    double w[4][8];
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 8; c++) w[r][c] = c < 4 ? a.m[r][c] : (c - 4 == r ? 1.0 : 0.0);
    for (int c = 0; c < 4; c++) {
        int p = c;
        for (int r = c + 1; r < 4; r++)
            if (std::fabs(w[r][c]) > std::fabs(w[p][c])) p = r;
        for (int k = 0; k < 8; k++) std::swap(w[c][k], w[p][k]);
        const double d = w[c][c];
        for (int k = 0; k < 8; k++) w[c][k] /= d;
        for (int r = 0; r < 4; r++)
            if (r != c) {
                const double f = w[r][c];
                for (int k = 0; k < 8; k++) w[r][k] -= f * w[c][k];
            }
    }
    float4x4 o;
    for (int r = 0; r < 4; r++)
        for (int c = 0; c < 4; c++) o.m[r][c] = float(w[r][c + 4]);
    return o;
}
inline float3 mul(const float3x3& a, const float3& v) {
    return {a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z, a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z,
            a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z};
}
inline float3 transformPoint(const float4x4& a, const float3& v) {
    return {a.m[0][0] * v.x + a.m[0][1] * v.y + a.m[0][2] * v.z + a.m[0][3],
            a.m[1][0] * v.x + a.m[1][1] * v.y + a.m[1][2] * v.z + a.m[1][3],
            a.m[2][0] * v.x + a.m[2][1] * v.y + a.m[2][2] * v.z + a.m[2][3]};
}
inline float3 normalize(const float3& v) {
    const float l = std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z);
    return {v.x / l, v.y / l, v.z / l};
}

// ----- Core/API: formats, flags, resources ---------------------------------------
enum class ResourceFormat { Unknown, RGBA32Float, RGBA32Uint, RG32Float, R32Float, R32Uint, RGBA8Unorm, RGBA8UnormSrgb };
inline bool isIntegerFormat(ResourceFormat f) { return f == ResourceFormat::RGBA32Uint || f == ResourceFormat::R32Uint; }
inline uint32_t getFormatBytesPerBlock(ResourceFormat f) {
    switch (f) {
        case ResourceFormat::RGBA32Float:
        case ResourceFormat::RGBA32Uint: return 16;
        case ResourceFormat::RG32Float: return 8;
        default: return 4;
    }
}
enum class ResourceBindFlags : uint32_t { None = 0, ShaderResource = 1, UnorderedAccess = 2, RenderTarget = 4, Shared = 8 };
inline ResourceBindFlags operator|(ResourceBindFlags a, ResourceBindFlags b) { return ResourceBindFlags(uint32_t(a) | uint32_t(b)); }
enum class MemoryType { DeviceLocal };

inline void cudaCheck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) FALCOR_THROW("{}: {}", what, cudaGetErrorString(e));
}

namespace cuda_utils {
// Utils/CudaUtils.h: ExternalMemory::getMappedData.
struct ExternalMemory {
    void* ptr = nullptr;
    void* getMappedData() const { return ptr; }
};
}  // namespace cuda_utils

class Resource {
public:
    virtual ~Resource() { if (mem.ptr) cudaFree(mem.ptr); }
    void* data() const { return mem.ptr; }
    size_t bytes = 0;
    cuda_utils::ExternalMemory mem;
};

class Buffer : public Resource {
public:
    Buffer(size_t size, uint32_t structSize) : elementSize(structSize) {
        bytes = size;
        cudaCheck(cudaMalloc(&mem.ptr, size ? size : 4), "cudaMalloc");
        cudaCheck(cudaMemset(mem.ptr, 0, size ? size : 4), "cudaMemset");
    }
    cuda_utils::ExternalMemory* getCudaMemory() const { return const_cast<cuda_utils::ExternalMemory*>(&mem); }
    template <class T> std::vector<T> getElements() const {
        std::vector<T> out(bytes / sizeof(T));
        cudaCheck(cudaMemcpy(out.data(), mem.ptr, out.size() * sizeof(T), cudaMemcpyDeviceToHost), "getElements");
        return out;
    }
    uint64_t getSize() const { return bytes; }
    uint32_t elementSize = 1;
};

class Texture : public Resource {
public:
    Texture(uint32_t w, uint32_t h, ResourceFormat f) : width(w), height(h), format(f) {
        bytes = size_t(w) * h * getFormatBytesPerBlock(f);
        cudaCheck(cudaMalloc(&mem.ptr, bytes), "cudaMalloc");
        cudaCheck(cudaMemset(mem.ptr, 0, bytes), "cudaMemset");
    }
    ResourceFormat getFormat() const { return format; }
    uint32_t getWidth() const { return width; }
    uint32_t getHeight() const { return height; }
    uint32_t width, height;
    ResourceFormat format;
};

// Core/API/CopyContext.h / RenderContext.h: CUDA interop fences and read-back.
class RenderContext {
public:
    void waitForCuda(cudaStream_t stream = 0) { cudaCheck(cudaStreamSynchronize(stream), "waitForCuda"); }
    void waitForFalcor(cudaStream_t stream = 0) { cudaCheck(cudaDeviceSynchronize(), "waitForFalcor"); }
    std::vector<uint8_t> readTextureSubresource(const Texture* t, uint32_t) {
        std::vector<uint8_t> out(t->bytes);
        cudaCheck(cudaMemcpy(out.data(), t->data(), t->bytes, cudaMemcpyDeviceToHost), "readTextureSubresource");
        return out;
    }
};

class Device {
public:
    ref<Buffer> createBuffer(size_t size, ResourceBindFlags = ResourceBindFlags::ShaderResource | ResourceBindFlags::UnorderedAccess,
                             MemoryType = MemoryType::DeviceLocal, const void* init = nullptr) {
        auto b = make_ref<Buffer>(size, 1);
        if (init) cudaCheck(cudaMemcpy(b->data(), init, size, cudaMemcpyHostToDevice), "createBuffer");
        return b;
    }
    ref<Buffer> createStructuredBuffer(uint32_t structSize, uint32_t elementCount,
                                       ResourceBindFlags = ResourceBindFlags::ShaderResource | ResourceBindFlags::UnorderedAccess,
                                       MemoryType = MemoryType::DeviceLocal, const void* init = nullptr, bool = false) {
        auto b = make_ref<Buffer>(size_t(structSize) * elementCount, structSize);
        if (init) cudaCheck(cudaMemcpy(b->data(), init, b->bytes, cudaMemcpyHostToDevice), "createStructuredBuffer");
        return b;
    }
    ref<Texture> createTexture2D(uint32_t w, uint32_t h, ResourceFormat f) { return make_ref<Texture>(w, h, f); }
    RenderContext* getRenderContext() { return &renderContext; }
    RenderContext renderContext;
};

// ----- Utils/Properties.h (JSON-backed) -------------------------------------------
class Properties {
public:
    // nlohmann::ordered_json stand-in: the JSON text of an object.
    struct json {
        std::string text;
        static json parse(const char* s) { return json{s}; }
    };
    Properties() = default;
    Properties(const json& j) : mText(j.text), mParsed(false) {}
    template <class T> void set(std::string_view name, const T& value) {
        std::ostringstream o;
        if constexpr (std::is_same_v<T, bool>) o << (value ? "true" : "false");
        else if constexpr (std::is_arithmetic_v<T>) o << value;
        else o << '"' << value << '"';
        put(std::string(name), o.str());
    }
    void set(std::string_view name, const char* value) { set(name, std::string(value)); }
    bool has(std::string_view name) const { return dump().find("\"" + std::string(name) + "\"") != std::string::npos; }
    std::string dump(int = -1) const {
        if (!mParsed) return mText;
        std::string s = "{";
        for (size_t i = 0; i < mItems.size(); i++) s += (i ? ", \"" : "\"") + mItems[i].first + "\": " + mItems[i].second;
        return s + "}";
    }

private:
    void put(const std::string& k, const std::string& v) {
        for (auto& kv : mItems)
            if (kv.first == k) { kv.second = v; return; }
        mItems.emplace_back(k, v);
    }
    std::string mText;
    bool mParsed = true;
    std::vector<std::pair<std::string, std::string>> mItems;
};

// ----- Core/Program: shader variables, defines, ComputePass -------------------------
struct DefineList : std::map<std::string, std::string> {};

class ComputePass;
// A named variable of a fake program: "CB.gWidth", "gBuf", "gLoader.normals".
struct ShaderVar {
    std::map<std::string, uint32_t>* constants;
    std::map<std::string, ref<Resource>>* resources;
    std::map<std::string, const void*>* blocks;
    std::string name;
    ShaderVar operator[](std::string_view sub) const { return {constants, resources, blocks, name.empty() ? std::string(sub) : name + "." + std::string(sub)}; }
    void operator=(uint32_t v) const { (*constants)[name] = v; }
    void operator=(const ref<Buffer>& b) const { (*resources)[name] = b; }
    void operator=(const ref<Texture>& t) const { (*resources)[name] = t; }
};

class ComputePass {
public:
    using Program = std::function<void(ComputePass&, uint32_t, uint32_t, uint32_t)>;
    // Stand-ins of the compute programs by "file:entry" (set by the test host).
    static std::map<std::string, Program>& programs() { static std::map<std::string, Program> p; return p; }
    static ref<ComputePass> create(const ref<Device>&, const std::string& path, const std::string& entry, const DefineList& = {}) {
        auto p = make_ref<ComputePass>();
        const size_t slash = path.find_last_of('/');
        p->key = (slash == std::string::npos ? path : path.substr(slash + 1)) + ":" + entry;
        return p;
    }
    ShaderVar getRootVar() { return {&constants, &resources, &blocks, ""}; }
    void execute(RenderContext*, uint32_t x, uint32_t y, uint32_t z = 1) {
        auto it = programs().find(key);
        if (it == programs().end()) FALCOR_THROW("no stand-in for compute program {}", key);
        it->second(*this, x, y, z);
    }
    std::string key;
    std::map<std::string, uint32_t> constants;
    std::map<std::string, ref<Resource>> resources;
    std::map<std::string, const void*> blocks;
};

// ----- RenderGraph ------------------------------------------------------------------
class RenderPassReflection {
public:
    class Field {
    public:
        enum class Flags { None = 0, Optional = 1 };
        Field& format(ResourceFormat f) { fmt = f; return *this; }
        Field& bindFlags(ResourceBindFlags f) { bind = f; return *this; }
        Field& flags(Flags f) { optional = f == Flags::Optional; return *this; }
        Field& texture2D(uint32_t = 0, uint32_t = 0, uint32_t = 1, uint32_t = 1, uint32_t = 1) { return *this; }
        std::string name, desc;
        bool isInput = false, optional = false;
        ResourceFormat fmt = ResourceFormat::Unknown;
        ResourceBindFlags bind = ResourceBindFlags::None;
    };
    Field& addInput(const std::string& name, const std::string& desc) { return add(name, desc, true); }
    Field& addOutput(const std::string& name, const std::string& desc) { return add(name, desc, false); }
    std::vector<std::unique_ptr<Field>> fields;

private:
    Field& add(const std::string& name, const std::string& desc, bool in) {
        fields.push_back(std::make_unique<Field>());
        fields.back()->name = name;
        fields.back()->desc = desc;
        fields.back()->isInput = in;
        return *fields.back();
    }
};

struct ChannelDesc {
    std::string name;
    std::string texname;
    std::string desc;
    bool optional = false;
    ResourceFormat format = ResourceFormat::Unknown;
};
using ChannelList = std::vector<ChannelDesc>;
inline void addRenderPassInputs(RenderPassReflection& r, const ChannelList& channels,
                                ResourceBindFlags bindFlags = ResourceBindFlags::ShaderResource) {
    for (const auto& c : channels) {
        auto& f = r.addInput(c.name, c.desc).bindFlags(bindFlags);
        if (c.format != ResourceFormat::Unknown) f.format(c.format);
        if (c.optional) f.flags(RenderPassReflection::Field::Flags::Optional);
    }
}
inline void addRenderPassOutputs(RenderPassReflection& r, const ChannelList& channels,
                                 ResourceBindFlags bindFlags = ResourceBindFlags::UnorderedAccess) {
    for (const auto& c : channels) {
        auto& f = r.addOutput(c.name, c.desc).bindFlags(bindFlags);
        if (c.format != ResourceFormat::Unknown) f.format(c.format);
        if (c.optional) f.flags(RenderPassReflection::Field::Flags::Optional);
    }
}

class RenderData {
public:
    ref<Texture> getTexture(const std::string_view name) const {
        auto it = textures.find(std::string(name));
        return it == textures.end() ? nullptr : it->second;
    }
    const uint2& getDefaultTextureDims() const { return dims; }
    std::map<std::string, ref<Texture>> textures;
    uint2 dims;
};

// ----- Scene ---------------------------------------------------------------------
struct MeshID {
    uint32_t id = 0;
    uint32_t get() const { return id; }
};
struct MaterialID {
    uint32_t id = 0;
    MaterialID() = default;
    explicit MaterialID(uint32_t v) : id(v) {}
};
enum class GeometryType : uint32_t { None, TriangleMesh, DisplacedTriangleMesh, Curve };
struct MeshDesc {
    uint32_t vbOffset = 0, ibOffset = 0, vertexCount = 0, indexCount = 0, skinningVbOffset = 0, prevVbOffset = 0, materialID = 0,
             flags = 0;
    uint32_t getTriangleCount() const { return (indexCount > 0 ? indexCount : vertexCount) / 3; }
};
struct GeometryInstanceData {
    uint32_t flags = 0, globalMatrixID = 0, materialID = 0, geometryID = 0;
    GeometryType type = GeometryType::TriangleMesh;
    GeometryType getType() const { return type; }
};

class Material {
public:
    virtual ~Material() = default;
    const std::string& getName() const { return name; }
    virtual bool isDoubleSided() const { return doubleSided; }
    virtual bool isThinSurface() const { return thinSurface; }
    virtual float getIndexOfRefraction() const { return ior; }
    std::string name;
    bool doubleSided = false, thinSurface = false;
    float ior = 1.5f;
};
class StandardMaterial : public Material {
public:
    float4 getBaseColor() const { return baseColor; }
    float4 getSpecularParams() const { return specular; }
    float3 getEmissiveColor() const { return emissive; }
    float getEmissiveFactor() const { return emissiveFactor; }
    float getSpecularTransmission() const { return specTrans; }
    float getDiffuseTransmission() const { return diffTrans; }
    float3 getTransmissionColor() const { return transmission; }
    // BasicMaterial::getBaseColorTexture (Scene/Material/BasicMaterial.h).
    ref<Texture> getBaseColorTexture() const { return baseColorTexture; }
    ref<Texture> baseColorTexture;
    float4 baseColor, specular;
    float3 emissive, transmission;
    float emissiveFactor = 1.f, specTrans = 0.f, diffTrans = 0.f;
};
class Camera {
public:
    float3 getPosition() const { return position; }
    float3 getTarget() const { return target; }
    float3 getUpVector() const { return up; }
    float getFocalLength() const { return focalLength; }
    float getFrameHeight() const { return frameHeight; }
    float getAspectRatio() const { return aspectRatio; }
    float getNearPlane() const { return nearZ; }
    float getFarPlane() const { return farZ; }
    float getFocalDistance() const { return focalDistance; }
    float getJitterX() const { return jitterX; }
    float getJitterY() const { return jitterY; }
    float3 position, target, up;
    float focalLength = 21.f, frameHeight = 24.f, aspectRatio = 1.f, nearZ = 0.1f, farZ = 1000.f, focalDistance = 10000.f;
    float jitterX = 0.f, jitterY = 0.f;
};
class EnvMap {
public:
    const ref<Texture>& getEnvMap() const { return texture; }
    float3 getTint() const { return tint; }
    float getIntensity() const { return intensity; }
    ref<Texture> texture;
    float3 tint{1.f, 1.f, 1.f};
    float intensity = 1.f;
};
class AnimationController {
public:
    const std::vector<float4x4>& getGlobalMatrices() const { return globalMatrices; }
    std::vector<float4x4> globalMatrices;
};

// Host-side scene of the stand-in: mesh data in host arrays.
class Scene {
public:
    uint32_t getMeshCount() const { return uint32_t(meshes.size()); }
    const MeshDesc& getMesh(MeshID id) const { return meshes[id.get()]; }
    uint32_t getGeometryInstanceCount() const { return uint32_t(instances.size()); }
    const GeometryInstanceData& getGeometryInstance(uint32_t i) const { return instances[i]; }
    uint32_t getMaterialCount() const { return uint32_t(materials.size()); }
    const ref<Material>& getMaterial(MaterialID id) const { return materials[id.id]; }
    const ref<Camera>& getCamera() const { return camera; }
    const ref<EnvMap>& getEnvMap() const { return envMap; }
    AnimationController* getAnimationController() { return &animation; }
    DefineList getSceneDefines() const { return {}; }
    void bindShaderData(const ShaderVar& var) const { (*var.blocks)[var.name] = this; }
    // Scene::getMeshVerticesAndIndices (Scene.cpp:4291-4312): positions and
    // texcrds (float3) per vertex, triangleIndices (uint3) per triangle.
    void getMeshVerticesAndIndices(MeshID id, const std::map<std::string, ref<Buffer>>& buffers) {
        const MeshDesc& m = meshes[id.get()];
        std::vector<float> pos(size_t(m.vertexCount) * 3), tex(size_t(m.vertexCount) * 3);
        for (uint32_t v = 0; v < m.vertexCount; v++)
            for (int k = 0; k < 3; k++) {
                pos[size_t(v) * 3 + k] = positions[(size_t(m.vbOffset) + v) * 3 + k];
                tex[size_t(v) * 3 + k] = k < 2 ? texcrds[(size_t(m.vbOffset) + v) * 2 + k] : 0.f;
            }
        std::vector<uint32_t> idx(indices.begin() + m.ibOffset, indices.begin() + m.ibOffset + m.indexCount);
        auto put = [&](const char* n, const void* src, size_t bytes) {
            auto it = buffers.find(n);
            if (it == buffers.end()) FALCOR_THROW("Mesh data buffer '{}' is missing.", n);
            cudaCheck(cudaMemcpy(it->second->data(), src, bytes, cudaMemcpyHostToDevice), "getMeshVerticesAndIndices");
        };
        put("positions", pos.data(), pos.size() * 4);
        put("texcrds", tex.data(), tex.size() * 4);
        put("triangleIndices", idx.data(), idx.size() * 4);
    }
    std::vector<MeshDesc> meshes;
    std::vector<GeometryInstanceData> instances;
    std::vector<ref<Material>> materials;
    std::vector<float> positions, normals, tangents, texcrds;  // global vertex arrays (3, 3, 4, 2 floats)
    std::vector<uint32_t> indices;                           // mesh-local indices
    ref<Camera> camera;
    ref<EnvMap> envMap;
    AnimationController animation;
};

// ----- Core/Plugin.h and RenderGraph/RenderPass.h -------------------------------------
struct PluginInfo {
    std::string desc;
};
#define FALCOR_PLUGIN_CLASS(cls, type, info)                                        \
public:                                                                             \
    static inline const std::string kPluginType{type};                              \
    static inline const ::Falcor::PluginInfo kPluginInfo{info};                     \
    virtual const std::string& getPluginType() const final { return kPluginType; } \
    virtual const ::Falcor::PluginInfo& getPluginInfo() const final { return kPluginInfo; }

struct CompileData {
    uint2 defaultTexDims;
};

class RenderPass {
public:
    using PluginCreate = std::function<ref<RenderPass>(ref<Device>, const Properties&)>;
    explicit RenderPass(ref<Device> pDevice) : mpDevice(std::move(pDevice)) {}
    virtual ~RenderPass() = default;
    virtual const std::string& getPluginType() const = 0;
    virtual const PluginInfo& getPluginInfo() const = 0;
    const std::string& getType() const { return getPluginType(); }
    const std::string& getDesc() const { return getPluginInfo().desc; }
    virtual RenderPassReflection reflect(const CompileData& compileData) = 0;
    virtual void execute(RenderContext* pRenderContext, const RenderData& renderData) = 0;
    virtual void setProperties(const Properties&) {}
    virtual Properties getProperties() const { return {}; }
    virtual void setScene(RenderContext*, const ref<Scene>&) {}
    // RenderPass::create (RenderPass.cpp:53-60): by type name through the plugin registry.
    static ref<RenderPass> create(std::string_view type, ref<Device> pDevice, const Properties& props = {});

protected:
    ref<Device> mpDevice;
};

class PluginRegistry {
public:
    template <class Base, class T> void registerClass() {
        factories()[T::kPluginType] = [](ref<Device> d, const Properties& p) -> ref<Base> { return T::create(d, p); };
    }
    static std::map<std::string, RenderPass::PluginCreate>& factories() {
        static std::map<std::string, RenderPass::PluginCreate> f;
        return f;
    }
};

inline ref<RenderPass> RenderPass::create(std::string_view type, ref<Device> pDevice, const Properties& props) {
    auto& f = PluginRegistry::factories();
    auto it = f.find(std::string(type));
    if (it == f.end()) FALCOR_THROW("Can't create render pass of type '{}'. No render pass with that name is registered.", type);
    return it->second(pDevice, props);
}

}  // namespace Falcor
