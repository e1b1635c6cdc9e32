// Stand-in for Falcor's Testing/UnitTest.h (Source/Falcor/Testing/UnitTest.h)
// that lets the reference's own unit-test sources compile on the CPU.
//
// TEST INFRASTRUCTURE ONLY.  GPU_TEST bodies run unchanged; where they would
// dispatch a Slang compute program, the fake context runs the oracle's C++
// restatement of that program (oracle/kat_main.cpp), and the reference's
// EXPECT_* checks then compare the oracle against the reference's embedded
// CPU implementations.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <filesystem>
#include <functional>
#include <iterator>
#include <map>
#include <memory>
#include <sstream>
#include <string>
#include <vector>

namespace Falcor {

template <class T> using ref = std::shared_ptr<T>;

#define FALCOR_ASSERT(x) ((void)0)

struct float2 {
    float x = 0, y = 0;
    float2() = default;
    float2(float a, float b) : x(a), y(b) {}
    explicit float2(float a) : x(a), y(a) {}
};
inline float2 operator+(float2 a, float2 b) { return {a.x + b.x, a.y + b.y}; }
inline float2 operator-(float2 a, float2 b) { return {a.x - b.x, a.y - b.y}; }
inline float2 operator*(float2 a, float s) { return {a.x * s, a.y * s}; }
inline float2 operator*(float s, float2 a) { return {a.x * s, a.y * s}; }
inline float2 operator*(float2 a, float2 b) { return {a.x * b.x, a.y * b.y}; }
inline float2 operator/(float2 a, float2 b) { return {a.x / b.x, a.y / b.y}; }
inline bool operator==(float2 a, float2 b) { return a.x == b.x && a.y == b.y; }
struct float3 {
    float x = 0, y = 0, z = 0;
    float3() = default;
    float3(float a, float b, float c) : x(a), y(b), z(c) {}
    float3(float2 v, float c) : x(v.x), y(v.y), z(c) {}
    explicit float3(float a) : x(a), y(a), z(a) {}
};
namespace math {
inline float lerp(float a, float b, float t) { return a + t * (b - a); }
}
struct float4 {
    float x = 0, y = 0, z = 0, w = 0;
    float4() = default;
    float4(float a, float b, float c, float d) : x(a), y(b), z(c), w(d) {}
    float4(float3 v, float d) : x(v.x), y(v.y), z(v.z), w(d) {}
};
inline float2 min(float2 a, float2 b) { return {std::fmin(a.x, b.x), std::fmin(a.y, b.y)}; }
inline float2 max(float2 a, float2 b) { return {std::fmax(a.x, b.x), std::fmax(a.y, b.y)}; }
struct int3 {
    int x = 0, y = 0, z = 0;
    int3() = default;
    int3(int a, int b, int c) : x(a), y(b), z(c) {}
};
struct uint2 {
    uint32_t x = 0, y = 0;
    uint2() = default;
    uint2(uint32_t a, uint32_t b) : x(a), y(b) {}
};
struct uint4 {
    uint32_t x = 0, y = 0, z = 0, w = 0;
    uint4() = default;
    explicit uint4(uint32_t a) : x(a), y(a), z(a), w(a) {}
};
inline float3 operator+(float3 a, float3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline float3 operator-(float3 a, float3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline float3 operator*(float3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
inline float3 operator*(float s, float3 a) { return {a.x * s, a.y * s, a.z * s}; }
inline bool operator==(float3 a, float3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline std::ostream& operator<<(std::ostream& o, float3 a) { return o << "(" << a.x << "," << a.y << "," << a.z << ")"; }
inline float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float3 normalize(float3 a) { float l = std::sqrt(dot(a, a)); return {a.x / l, a.y / l, a.z / l}; }
inline float asfloat(int32_t i) { float f; std::memcpy(&f, &i, 4); return f; }
inline float asfloat(uint32_t i) { float f; std::memcpy(&f, &i, 4); return f; }
inline int32_t asint(float f) { int32_t i; std::memcpy(&i, &f, 4); return i; }

enum class ResourceBindFlags { None = 0, ShaderResource = 1, UnorderedAccess = 2 };
inline ResourceBindFlags operator|(ResourceBindFlags a, ResourceBindFlags b) { return ResourceBindFlags(int(a) | int(b)); }
enum class MemoryType { DeviceLocal };
enum class SlangCompilerFlags { None = 0, FloatingPointModePrecise = 1 };
struct DefineList {
    std::map<std::string, std::string> values;
    DefineList& add(const std::string& name, const std::string& value = "") { values[name] = value; return *this; }
};
enum class ResourceFormat { RGB32Float };
// Image output of a test (histogram dumps); not used by the shimmed runs.
struct Bitmap {
    enum class FileFormat { ExrFile };
    enum class ExportFlags { None };
    static void saveImage(const std::filesystem::path&, uint32_t, uint32_t, FileFormat, ExportFlags, ResourceFormat, bool, void*) {}
};

class Buffer {
public:
    std::vector<uint8_t> data;
    size_t elementSize = 0;
    size_t elementCount = 0;
    template <class T> void setElement(size_t i, const T& v) {
        if (elementSize == 0) elementSize = sizeof(T);
        if (data.size() < (i + 1) * sizeof(T)) data.resize((i + 1) * sizeof(T));
        std::memcpy(data.data() + i * sizeof(T), &v, sizeof(T));
    }
    template <class T> std::vector<T> getElements() const {
        std::vector<T> out(data.size() / sizeof(T));
        if (!out.empty()) std::memcpy(out.data(), data.data(), out.size() * sizeof(T));
        return out;
    }
    size_t getElementCount() const { return elementCount; }
    struct View { Buffer* b; Buffer* get() const { return b; } };
    View getUAV() { return View{this}; }
};

class RenderContext {
public:
    void clearUAV(Buffer* b, uint4 v) { std::fill(b->data.begin(), b->data.end(), uint8_t(v.x)); }
};

class GPUUnitTestContext;
// A named shader variable of the fake program ("CB.sz", "gSamplingTest.testWi").
struct ShaderVar {
    GPUUnitTestContext* ctx;
    std::string name;
    ShaderVar operator[](const char* sub) const { return ShaderVar{ctx, name + "." + sub}; }
    const ShaderVar& operator=(const ref<Buffer>& b) const;
    const ShaderVar& operator=(uint32_t v) const;
    const ShaderVar& operator=(uint2 v) const;
    std::string leaf() const { const size_t p = name.rfind('.'); return p == std::string::npos ? name : name.substr(p + 1); }
};

class Device {
public:
    enum class Type { Default, D3D12, Vulkan };
    RenderContext renderContext;
    RenderContext* getRenderContext() { return &renderContext; }
    // Structured buffer typed by the shader variable it is created for; the
    // element size comes from the oracle's restatement of that program.
    ref<Buffer> createStructuredBuffer(const ShaderVar& var, uint32_t n,
                                       ResourceBindFlags = ResourceBindFlags::ShaderResource, MemoryType = MemoryType::DeviceLocal,
                                       const void* init = nullptr);
    ref<Buffer> createBuffer(size_t size, ResourceBindFlags, MemoryType, const void* init) {
        auto b = std::make_shared<Buffer>();
        b->data.resize(size);
        if (init) std::memcpy(b->data.data(), init, size);
        b->elementSize = 1;
        b->elementCount = size;
        return b;
    }
    ref<Buffer> createStructuredBuffer(size_t elemSize, uint32_t n, ResourceBindFlags, MemoryType, const void* init, bool) {
        auto b = std::make_shared<Buffer>();
        b->data.resize(elemSize * n);
        if (init) std::memcpy(b->data.data(), init, elemSize * n);
        b->elementSize = elemSize;
        b->elementCount = n;
        return b;
    }
    template <class T> ref<Buffer> createTypedBuffer(size_t n, ResourceBindFlags = ResourceBindFlags::ShaderResource) {
        auto b = std::make_shared<Buffer>();
        b->data.assign(n * sizeof(T), 0);
        b->elementSize = sizeof(T);
        b->elementCount = n;
        return b;
    }
};

}  // namespace Falcor

namespace kat {
// Element size of a structured-buffer variable of a shimmed program (by leaf name).
size_t element_size(const std::string& leaf);
// The oracle-side implementation of a Slang test program (kat_main.cpp).
using Program = std::function<void(Falcor::GPUUnitTestContext&, uint32_t, uint32_t, uint32_t)>;
Program find_program(const std::string& entry);
// Programs of the BSDF sampling and scene-gradient tests (kat_bsdf.cpp).
Program find_program_bsdf(const std::string& entry);
struct Failure { std::string test, expr, file; int line; };
void record(bool ok, const char* expr, const char* file, int line);
struct Expect {
    bool ok;
    std::ostringstream msg;
    Expect(bool o, const char* expr, const char* file, int line) : ok(o) { record(o, expr, file, line); }
    template <class T> Expect& operator<<(const T& v) { if (!ok) msg << v; return *this; }
};
struct Options { bool disabled = false; };
inline Options options() { return {}; }
inline Options options(int) { return {}; }
inline Options options(int, Falcor::Device::Type) { return {}; }
inline Options options(int, const char*) { Options o; o.disabled = true; return o; }
void register_gpu(const char* name, void (*fn)(Falcor::GPUUnitTestContext&), Options o);
struct CPUUnitTestContext {};
void register_cpu(const char* name, void (*fn)(CPUUnitTestContext&), Options o);
struct GpuReg { GpuReg(const char* n, void (*f)(Falcor::GPUUnitTestContext&), Options o) { register_gpu(n, f, o); } };
struct CpuReg { CpuReg(const char* n, void (*f)(CPUUnitTestContext&), Options o) { register_cpu(n, f, o); } };
}  // namespace kat

namespace Falcor {

class GPUUnitTestContext {
public:
    using Var = ShaderVar;
    std::map<std::string, ref<Buffer>> buffers;
    std::map<std::string, uint32_t> constants;
    std::map<std::string, std::string> defines;
    std::map<std::string, const void*> blocks;  // parameter blocks bound by host objects (SceneGradients)
    std::string entry;
    Device device;

    ref<Device> getDevice() { return ref<Device>(&device, [](Device*) {}); }
    RenderContext* getRenderContext() { return device.getRenderContext(); }
    void createProgram(const std::string&, const std::string& e, DefineList d = {}, SlangCompilerFlags = SlangCompilerFlags::None) {
        entry = e;
        defines = d.values;
    }
    void allocateStructuredBuffer(const std::string& name, uint32_t n, const void* init = nullptr, size_t size = 0) {
        auto b = std::make_shared<Buffer>();
        b->elementCount = n;
        if (init) { b->data.resize(size); std::memcpy(b->data.data(), init, size); }
        buffers[name] = b;
    }
    Var operator[](const char* name) { return Var{this, name}; }
    void runProgram(uint32_t x, uint32_t y = 1, uint32_t z = 1);
    template <class T> std::vector<T> readBuffer(const std::string& name) { return buffers.at(name)->getElements<T>(); }
};

inline const ShaderVar& ShaderVar::operator=(const ref<Buffer>& b) const { ctx->buffers[name] = b; return *this; }
inline const ShaderVar& ShaderVar::operator=(uint32_t v) const { ctx->constants[name] = v; return *this; }
inline const ShaderVar& ShaderVar::operator=(uint2 v) const {
    ctx->constants[name + ".x"] = v.x;
    ctx->constants[name + ".y"] = v.y;
    return *this;
}
inline ref<Buffer> Device::createStructuredBuffer(const ShaderVar& var, uint32_t n, ResourceBindFlags, MemoryType, const void* init) {
    const size_t es = kat::element_size(var.leaf());
    auto b = std::make_shared<Buffer>();
    b->data.assign(es * n, 0);
    if (init) std::memcpy(b->data.data(), init, es * n);
    b->elementSize = es;
    b->elementCount = n;
    return b;
}

}  // namespace Falcor

#define KAT_CAT2(a, b) a##b
#define KAT_CAT(a, b) KAT_CAT2(a, b)
#define GPU_TEST(name, ...)                                                                              \
    static void KAT_CAT(kat_gpu_, name)(::Falcor::GPUUnitTestContext & ctx);                            \
    static ::kat::GpuReg KAT_CAT(kat_gpu_reg_, name)(#name, &KAT_CAT(kat_gpu_, name),                   \
                                                      ::kat::options(0 __VA_OPT__(, ) __VA_ARGS__));     \
    static void KAT_CAT(kat_gpu_, name)(::Falcor::GPUUnitTestContext & ctx)
#define CPU_TEST(name, ...)                                                                              \
    static void KAT_CAT(kat_cpu_, name)(::kat::CPUUnitTestContext & ctx);                               \
    static ::kat::CpuReg KAT_CAT(kat_cpu_reg_, name)(#name, &KAT_CAT(kat_cpu_, name),                   \
                                                      ::kat::options(0 __VA_OPT__(, ) __VA_ARGS__));     \
    static void KAT_CAT(kat_cpu_, name)(::kat::CPUUnitTestContext & ctx)
#define EXPECT_EQ(a, b) ::kat::Expect(((a) == (b)), #a " == " #b, __FILE__, __LINE__)
#define EXPECT_NE(a, b) ::kat::Expect(((a) != (b)), #a " != " #b, __FILE__, __LINE__)
#define EXPECT_GT(a, b) ::kat::Expect(((a) > (b)), #a " > " #b, __FILE__, __LINE__)
#define EXPECT_LT(a, b) ::kat::Expect(((a) < (b)), #a " < " #b, __FILE__, __LINE__)
#define EXPECT_GE(a, b) ::kat::Expect(((a) >= (b)), #a " >= " #b, __FILE__, __LINE__)
#define EXPECT_LE(a, b) ::kat::Expect(((a) <= (b)), #a " <= " #b, __FILE__, __LINE__)
#define EXPECT(a) ::kat::Expect(bool(a), #a, __FILE__, __LINE__)
#define EXPECT_TRUE(a) ::kat::Expect(bool(a), #a, __FILE__, __LINE__)
#define EXPECT_FALSE(a) ::kat::Expect(!bool(a), "!" #a, __FILE__, __LINE__)
