// kat_main.cpp -- known-answer harness that runs the reference's own unit
// tests (compiled from Source/Tools/FalcorTest/Tests/... under the reference
// tree, see ref.mk) against the CPU oracle, plus an exhaustive comparison of
// the oracle's fp16 conversions with the reference's Utils/Math/Float16.cpp.
//
// TEST INFRASTRUCTURE ONLY.  Each "program" below restates the compute shader
// the reference test dispatches (Tests/.../*.cs.slang) with oracle functions.
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "Testing/UnitTest.h"
#include "Utils/Math/Float16.h"
#include "oracle_math.h"

namespace kat {

namespace {
struct TestEntry { std::string name; void (*gpu)(Falcor::GPUUnitTestContext&); void (*cpu)(CPUUnitTestContext&); Options opt; };
std::vector<TestEntry>& tests() { static std::vector<TestEntry> t; return t; }
uint64_t g_checks = 0, g_fail = 0;
std::string g_current;
bool g_missingProgram = false;
}  // namespace

void register_gpu(const char* name, void (*fn)(Falcor::GPUUnitTestContext&), Options o) { tests().push_back({name, fn, nullptr, o}); }
void register_cpu(const char* name, void (*fn)(CPUUnitTestContext&), Options o) { tests().push_back({name, nullptr, fn, o}); }

void record(bool ok, const char* expr, const char* file, int line) {
    g_checks++;
    if (!ok) {
        if (g_fail < 20) std::fprintf(stderr, "  FAIL %s: %s (%s:%d)\n", g_current.c_str(), expr, file, line);
        g_fail++;
    }
}

// ----- Oracle restatements of the test shaders ------------------------------
template <class T> static T load(const Falcor::ref<Falcor::Buffer>& b, size_t i) {
    T v;
    std::memcpy(&v, b->data.data() + i * sizeof(T), sizeof(T));
    return v;
}

Program find_program(const std::string& entry) {
    using Ctx = Falcor::GPUUnitTestContext;
    // Tests/Sampling/PseudorandomTests.cs.slang
    if (entry == "testXoshiro")
        return [](Ctx& c, uint32_t nx, uint32_t, uint32_t) {
            auto seed = c.buffers.at("seed");
            auto out = c.buffers.at("result");
            for (uint32_t i = 0; i < nx; i++) {
                orc::Xoshiro128 r{{load<uint32_t>(seed, 4 * i), load<uint32_t>(seed, 4 * i + 1), load<uint32_t>(seed, 4 * i + 2),
                                   load<uint32_t>(seed, 4 * i + 3)}};
                for (uint32_t j = 0; j < 64; j++) out->setElement<uint32_t>(size_t(j) * nx + i, r.next());
            }
        };
    if (entry == "testSplitMix")
        return [](Ctx& c, uint32_t nx, uint32_t, uint32_t) {
            auto seed = c.buffers.at("seed");
            auto out = c.buffers.at("result64");
            for (uint32_t i = 0; i < nx; i++) {
                orc::SplitMix64 r = orc::SplitMix64::create(load<uint32_t>(seed, 2 * i), load<uint32_t>(seed, 2 * i + 1));
                for (uint32_t j = 0; j < 64; j++) out->setElement<uint64_t>(size_t(j) * nx + i, r.next64());
            }
        };
    if (entry == "testLCG")
        return [](Ctx& c, uint32_t nx, uint32_t, uint32_t) {
            auto seed = c.buffers.at("seed");
            auto out = c.buffers.at("result");
            for (uint32_t i = 0; i < nx; i++) {
                orc::LCG r{load<uint32_t>(seed, i)};
                for (uint32_t j = 0; j < 64; j++) out->setElement<uint32_t>(size_t(j) * nx + i, r.next());
            }
        };
    // Tests/Utils/HashUtilsTests.cs.slang
    if (entry == "testJenkinsHash")
        return [](Ctx& c, uint32_t nx, uint32_t ny, uint32_t) {
            auto out = c.buffers.at("result");
            for (uint32_t y = 0; y < ny; y++)
                for (uint32_t x = 0; x < nx; x++) {
                    const uint32_t i = (y << 16) | x;
                    out->setElement<uint32_t>(i, orc::jenkins_hash(i));
                }
        };
    // Tests/Utils/BitTricksTests.cs.slang
    if (entry == "testBitInterleave")
        return [](Ctx& c, uint32_t nx, uint32_t, uint32_t) {
            auto data = c.buffers.at("testData");
            auto out = c.buffers.at("result");
            auto pack = [](uint32_t x, uint32_t y) { return (y << 16) | x; };
            for (uint32_t idx = 0; idx < nx; idx++) {
                const uint32_t d = load<uint32_t>(data, idx);
                const uint32_t bx = d & 0xffffu, by = d >> 16;
                const uint32_t inter = orc::interleave_32bit(bx, by);
                out->setElement<uint32_t>(5 * idx + 0, orc::interleave_32bit(bx ^ 0xbeef0000u, by ^ 0xbeef0000u));
                out->setElement<uint32_t>(5 * idx + 1, orc::interleave_16bit(bx ^ 0xbeefed00u, by ^ 0xbeefed00u));
                uint32_t x, y;
                orc::deinterleave_16bit(inter & 0x0000ffffu, x, y);
                out->setElement<uint32_t>(5 * idx + 2, pack(x, y));
                orc::deinterleave_8bit(inter & 0x000000ffu, x, y);
                out->setElement<uint32_t>(5 * idx + 3, pack(x, y));
                orc::deinterleave_2x8bit(inter & 0x00ff00ffu, x, y);
                out->setElement<uint32_t>(5 * idx + 4, pack(((x >> 8) & 0x0f00u) | (x & 0xfu), ((y >> 8) & 0x0f00u) | (y & 0xfu)));
            }
        };
    // Tests/Utils/GeometryHelpersTests.cs.slang: testComputeRayOrigin
    if (entry == "testComputeRayOrigin")
        return [](Ctx& c, uint32_t nx, uint32_t, uint32_t) {
            auto pos = c.buffers.at("pos"), nrm = c.buffers.at("normal"), out = c.buffers.at("result");
            const uint32_t n = c.constants.at("CB.n");
            for (uint32_t i = 0; i < nx && i < n; i++) {
                const Falcor::float3 p = load<Falcor::float3>(pos, i), q = load<Falcor::float3>(nrm, i);
                const orc::V3<float> r = orc::compute_ray_origin(orc::V3<float>(p.x, p.y, p.z), orc::V3<float>(q.x, q.y, q.z));
                out->setElement<Falcor::float3>(i, Falcor::float3(r.x, r.y, r.z));
            }
        };
    return find_program_bsdf(entry);
}

}  // namespace kat

void Falcor::GPUUnitTestContext::runProgram(uint32_t x, uint32_t y, uint32_t z) {
    kat::Program p = kat::find_program(entry);
    if (!p) {
        kat::g_missingProgram = true;
        throw std::runtime_error("no oracle program for " + entry);
    }
    p(*this, x, y, z);
}

// Exhaustive fp16 -> fp32 and stratified fp32 -> fp16 comparison with the
// reference's host conversion (Utils/Math/Float16.cpp).
static void check_float16() {
    kat::g_current = "Float16 (reference Float16.cpp vs oracle)";
    for (uint32_t h = 0; h < 65536; h++) {
        const float a = Falcor::math::float16ToFloat32(uint16_t(h)), b = orc::f16tof32(h);
        uint32_t ua, ub;
        std::memcpy(&ua, &a, 4);
        std::memcpy(&ub, &b, 4);
        kat::record(ua == ub, "float16ToFloat32 bit-exact", __FILE__, __LINE__);
    }
    auto check = [](uint32_t bits) {
        float f;
        std::memcpy(&f, &bits, 4);
        kat::record(Falcor::math::float32ToFloat16(f) == orc::f32tof16_host(f), "float32ToFloat16 bit-exact", __FILE__, __LINE__);
    };
    const uint32_t lows[] = {0u, 1u, 0x0fffu, 0x1000u, 0x1001u, 0x1fffu, 0x0800u, 0x17ffu};
    for (uint32_t hi = 0; hi < (1u << 19); hi++)
        for (uint32_t lo : lows) check((hi << 13) | lo);
    std::mt19937 rng(1234);
    for (int i = 0; i < (1 << 22); i++) check(rng());
}

// Usage: kat_runner [substring ...] -- runs the tests whose names contain one
// of the substrings (all tests and the fp16 check without arguments).
int main(int argc, char** argv) {
    int failedTests = 0, passed = 0, skipped = 0;
    auto selected = [&](const std::string& name) {
        if (argc < 2) return true;
        for (int i = 1; i < argc; i++)
            if (name.find(argv[i]) != std::string::npos) return true;
        return false;
    };
    for (auto& t : kat::tests()) {
        if (!selected(t.name)) continue;
        if (t.opt.disabled) {
            std::printf("SKIP %-36s (disabled in the reference)\n", t.name.c_str());
            skipped++;
            continue;
        }
        kat::g_current = t.name;
        const uint64_t f0 = kat::g_fail, c0 = kat::g_checks;
        kat::g_missingProgram = false;
        try {
            if (t.gpu) {
                Falcor::GPUUnitTestContext ctx;
                t.gpu(ctx);
            } else {
                kat::CPUUnitTestContext ctx;
                t.cpu(ctx);
            }
        } catch (const std::exception& e) {
            if (kat::g_missingProgram || std::string(e.what()).find("no oracle restatement") != std::string::npos) {
                std::printf("SKIP %-36s (%s)\n", t.name.c_str(), e.what());
                skipped++;
                continue;
            }
            std::printf("FAIL %-36s exception %s\n", t.name.c_str(), e.what());
            failedTests++;
            continue;
        }
        const uint64_t nf = kat::g_fail - f0, nc = kat::g_checks - c0;
        std::printf("%s %-36s %llu checks, %llu failed\n", nf ? "FAIL" : "PASS", t.name.c_str(), (unsigned long long)nc,
                    (unsigned long long)nf);
        if (nf) failedTests++; else passed++;
    }
    if (!selected("Float16Conversions")) {
        std::printf("SUMMARY passed=%d failed=%d skipped=%d\n", passed, failedTests, skipped);
        return failedTests ? 1 : 0;
    }
    const uint64_t f0 = kat::g_fail, c0 = kat::g_checks;
    check_float16();
    const uint64_t nf = kat::g_fail - f0;
    std::printf("%s %-36s %llu checks, %llu failed\n", nf ? "FAIL" : "PASS", "Float16Conversions",
                (unsigned long long)(kat::g_checks - c0), (unsigned long long)nf);
    if (nf) failedTests++; else passed++;
    std::printf("SUMMARY passed=%d failed=%d skipped=%d\n", passed, failedTests, skipped);
    return failedTests ? 1 : 0;
}
