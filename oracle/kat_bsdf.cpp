// kat_bsdf.cpp -- oracle restatements of the compute programs that the
// reference's Tests/Scene/Material/BSDFTests.cpp and
// Tests/DiffRendering/SceneGradientsTest.cpp dispatch
// (BSDFTests.cs.slang, SceneGradientsTest.cs.slang), so that those tests'
// own chi^2, weight/pdf and aggregation checks judge the oracle's BSDF lobes
// and gradient accumulation.
//
// TEST INFRASTRUCTURE ONLY.  BSDFs off the hot path (DisneyDiffuseBRDF,
// OrenNayarBRDF, SheenBSDF, DiffuseSpecularBRDF) have no restatement: their
// tests are reported as skipped.
#include <algorithm>
#include <atomic>
#include <cstring>
#include <regex>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "Testing/UnitTest.h"
#include "oracle_gradients.h"
#include "oracle_math.h"

namespace kat {

size_t element_size(const std::string& leaf) {
    if (leaf == "testWi") return 12;
    if (leaf == "testParams") return 16;
    if (leaf == "histogramPdf") return 8;
    return 4;  // histogramSampling, histogramWeightError, histogramPdfError, result
}

namespace {

using Ctx = Falcor::GPUUnitTestContext;
using orc::V3;

constexpr float kCosThetaMargin = 1e-3f;  // SamplingTest::kCosThetaMargin
constexpr float kOneOver2Pi = 0.159154943091895335768883763372514362f;
constexpr float k2Pi = 6.28318530717958647692528676655900576f;

// One lobe of StandardBSDF as the test shader's TEST_BSDF, with the fields its
// TEST_BSDF_INIT line sets (BSDFTests.cpp:300-470).
struct LobeUnderTest {
    enum Kind { Frostbite, LambertBRDF, LambertBTDF, MicrofacetBRDF } kind;
    orc::StandardBSDF<float> b;

    template <class SG> bool sample(V3<float> wi, V3<float>& wo, float& pdf, V3<float>& weight, uint32_t& lobe, SG& sg) const {
        switch (kind) {
            case Frostbite:
            case LambertBRDF: return b.diffuse_sample(wi, wo, pdf, weight, lobe, sg);
            case LambertBTDF: return b.difftrans_sample(wi, wo, pdf, weight, lobe, sg);
            default: return b.spec_sample(wi, wo, pdf, weight, lobe, sg);
        }
    }
    V3<float> eval(V3<float> wi, V3<float> wo) const {
        switch (kind) {
            case Frostbite:
            case LambertBRDF: return b.diffuse_eval(wi, wo);
            case LambertBTDF: return b.difftrans_eval(wi, wo);
            default: return b.spec_eval(wi, wo);
        }
    }
    float evalPdf(V3<float> wi, V3<float> wo) const {
        switch (kind) {
            case Frostbite:
            case LambertBRDF: return b.diffuse_pdf(wi, wo);
            case LambertBTDF: return b.difftrans_pdf(wi, wo);
            default: return b.spec_pdf(wi, wo);
        }
    }
};

// Reads a "bsdf.<field> = <number>f" assignment of the TEST_BSDF_INIT line.
bool init_number(const std::string& init, const std::string& field, float& out) {
    std::smatch m;
    if (std::regex_search(init, m, std::regex("bsdf\\." + field + " = ([0-9.]+)f"))) {
        out = std::stof(m[1].str());
        return true;
    }
    return false;
}

LobeUnderTest make_lobe(const Ctx& c, const Falcor::float4& params) {
    const std::string name = c.defines.count("TEST_BSDF") ? c.defines.at("TEST_BSDF") : "";
    const std::string init = c.defines.count("TEST_BSDF_INIT") ? c.defines.at("TEST_BSDF_INIT") : "";
    LobeUnderTest t{};
    t.b.lambert = false;
    t.b.diffAlbedo = t.b.transAlbedo = t.b.specAlbedo = V3<float>(1.f);  // "bsdf.albedo = float3(1.f)"
    t.b.diffRoughness = 0.f;
    t.b.activeLobes = 0;
    if (name == "FrostbiteDiffuseBRDF") {
        t.kind = LobeUnderTest::Frostbite;
        if (!init_number(init, "roughness", t.b.diffRoughness)) throw std::runtime_error("FrostbiteDiffuseBRDF: roughness not set");
    } else if (name == "LambertDiffuseBRDF") {
        t.kind = LobeUnderTest::LambertBRDF;
        t.b.lambert = true;
    } else if (name == "LambertDiffuseBTDF") {
        t.kind = LobeUnderTest::LambertBTDF;
    } else if (name == "SpecularMicrofacetBRDF") {
        t.kind = LobeUnderTest::MicrofacetBRDF;
        if (init.find("bsdf.activeLobes = 0xff") != std::string::npos) t.b.activeLobes = 0xffu;
        if (init.find("bsdf.alpha = params.x") == std::string::npos) throw std::runtime_error("SpecularMicrofacetBRDF: alpha not set");
        t.b.alpha = params.x;
    } else {
        throw std::runtime_error("no oracle restatement of " + name + " (not on the hot path)");
    }
    return t;
}

template <class T> T load(const Falcor::ref<Falcor::Buffer>& b, size_t i) {
    T v;
    std::memcpy(&v, b->data.data() + i * sizeof(T), sizeof(T));
    return v;
}

// Runs fn(x, z, worker) for x < nx, z < nz on all host cores.
template <class F> void parallel(uint32_t nx, uint32_t nz, F fn, uint32_t workers) {
    std::atomic<uint64_t> next{0};
    const uint64_t total = uint64_t(nx) * nz;
    std::vector<std::thread> th;
    for (uint32_t w = 0; w < workers; w++)
        th.emplace_back([&, w] {
            for (uint64_t k = next++; k < total; k = next++) fn(uint32_t(k % nx), uint32_t(k / nx), w);
        });
    for (auto& t : th) t.join();
}

uint32_t bin_index(const Ctx& c, const V3<float>& wo, uint32_t testIndex) {
    const uint32_t phiBins = c.constants.at("SamplingTestCB.gSamplingTest.phiBinCount");
    const uint32_t cosBins = c.constants.at("SamplingTestCB.gSamplingTest.cosThetaBinCount");
    // clamp((uint)floor(((double)wo.z * 0.5 + 0.5) * cosThetaBinCount), 0, cosThetaBinCount - 1)
    const uint32_t cosBin = std::min(uint32_t(std::floor((double(wo.z) * 0.5 + 0.5) * cosBins)), cosBins - 1);
    float scaledPhi = orc::el_atan2(wo.y, wo.x) * kOneOver2Pi;
    if (scaledPhi < 0.f) scaledPhi += 1.f;
    const uint32_t phiBin = std::min(uint32_t(std::floor(scaledPhi * float(phiBins))), phiBins - 1);
    return testIndex * (phiBins * cosBins) + cosBin * phiBins + phiBin;
}

uint32_t workers() { return std::max(1u, std::thread::hardware_concurrency()); }

// SamplingTest::tabulateHistogram and ::tabulateWeightAndPdfError (BSDFTests.cs.slang).
void sampling_program(Ctx& c, uint32_t nx, uint32_t, uint32_t nz, bool errors) {
    const std::string P = "SamplingTestCB.gSamplingTest.";
    const uint32_t testCount = c.constants.at(P + "testCount");
    const uint32_t sampleCount = c.constants.at(P + "sampleCount");
    const uint32_t threadSampleCount = c.constants.at(P + "threadSampleCount");
    const uint32_t bins = c.constants.at(P + "phiBinCount") * c.constants.at(P + "cosThetaBinCount");
    const uint32_t threadCount = sampleCount / threadSampleCount;
    auto wiBuf = c.buffers.at(P + "testWi");
    auto parBuf = c.buffers.at(P + "testParams");
    const uint32_t W = workers();
    // Per-worker histograms (atomics in the shader), merged afterwards.
    std::vector<std::vector<uint32_t>> hist(W), werr(W), perr(W);
    for (uint32_t w = 0; w < W; w++) {
        if (errors) {
            werr[w].assign(size_t(testCount) * bins, 0u);
            perr[w].assign(size_t(testCount) * bins, 0u);
        } else {
            hist[w].assign(size_t(testCount) * bins, 0u);
        }
    }
    std::vector<LobeUnderTest> lobes;
    for (uint32_t t = 0; t < testCount; t++) lobes.push_back(make_lobe(c, load<Falcor::float4>(parBuf, t)));
    parallel(std::min(nx, threadCount), std::min(nz, testCount), [&](uint32_t x, uint32_t testIndex, uint32_t w) {
        const Falcor::float3 f = load<Falcor::float3>(wiBuf, testIndex);
        const V3<float> wi = orc::normalize(V3<float>(f.x, f.y, f.z));
        const LobeUnderTest& bsdf = lobes[testIndex];
        orc::UniformSG sg(x, 0, 0);  // UniformSampleGenerator(threadId.xy, 0)
        for (uint32_t i = 0; i < threadSampleCount; i++) {
            V3<float> wo, weight;
            float pdf;
            uint32_t lobe;
            if (!bsdf.sample(wi, wo, pdf, weight, lobe, sg)) continue;
            if (!errors) {
                if (wo.z < -1.f + kCosThetaMargin || wo.z > 1.f - kCosThetaMargin) continue;
                hist[w][bin_index(c, wo, testIndex)]++;
                continue;
            }
            const V3<float> value = bsdf.eval(wi, wo);
            const float pdfRef = bsdf.evalPdf(wi, wo);
            const V3<float> weightRef = pdfRef > 0.f ? value / pdfRef : V3<float>(0.f);
            const float ex = std::fabs(weight.x - weightRef.x) / (weightRef.x > 0.f ? weightRef.x : 1.f);
            const float ey = std::fabs(weight.y - weightRef.y) / (weightRef.y > 0.f ? weightRef.y : 1.f);
            const float ez = std::fabs(weight.z - weightRef.z) / (weightRef.z > 0.f ? weightRef.z : 1.f);
            const float weightError = std::max(std::max(ex, ey), ez);
            const float pdfError = std::fabs(pdf - pdfRef) / (pdfRef > 0.f ? pdfRef : 1.f);
            const uint32_t bi = bin_index(c, wo, testIndex);
            uint32_t a, b;
            std::memcpy(&a, &weightError, 4);
            std::memcpy(&b, &pdfError, 4);
            werr[w][bi] = std::max(werr[w][bi], a);  // InterlockedMax(asuint(...))
            perr[w][bi] = std::max(perr[w][bi], b);
        }
    }, W);
    if (!errors) {
        auto out = c.buffers.at(P + "histogramSampling");
        for (size_t i = 0; i < size_t(testCount) * bins; i++) {
            uint32_t s = load<uint32_t>(out, i);
            for (uint32_t w = 0; w < W; w++) s += hist[w][i];
            out->setElement<uint32_t>(i, s);
        }
    } else {
        auto ow = c.buffers.at(P + "histogramWeightError"), op = c.buffers.at(P + "histogramPdfError");
        for (size_t i = 0; i < size_t(testCount) * bins; i++) {
            uint32_t a = load<uint32_t>(ow, i), b = load<uint32_t>(op, i);
            for (uint32_t w = 0; w < W; w++) {
                a = std::max(a, werr[w][i]);
                b = std::max(b, perr[w][i]);
            }
            ow->setElement<uint32_t>(i, a);
            op->setElement<uint32_t>(i, b);
        }
    }
}

float hlsl_lerp(float a, float b, float t) { return a + t * (b - a); }

// SamplingTest::tabulatePdf (BSDFTests.cs.slang): midpoint integral of
// evalPdf over each (phi, cos theta) bin.
void pdf_program(Ctx& c, uint32_t nx, uint32_t ny, uint32_t nz) {
    const std::string P = "SamplingTestCB.gSamplingTest.";
    const uint32_t testCount = c.constants.at(P + "testCount");
    const uint32_t phiBins = c.constants.at(P + "phiBinCount");
    const uint32_t cosBins = c.constants.at(P + "cosThetaBinCount");
    const uint32_t sampleCount = c.constants.at(P + "sampleCount");
    const uint32_t binSamples = c.constants.at(P + "binSampleCount");
    auto wiBuf = c.buffers.at(P + "testWi");
    auto parBuf = c.buffers.at(P + "testParams");
    auto out = c.buffers.at(P + "histogramPdf");
    std::vector<LobeUnderTest> lobes;
    for (uint32_t t = 0; t < testCount; t++) lobes.push_back(make_lobe(c, load<Falcor::float4>(parBuf, t)));
    std::vector<double> res(size_t(testCount) * phiBins * cosBins, 0.0);
    const uint32_t nPhi = std::min(nx, phiBins), nCos = std::min(ny, cosBins), nT = std::min(nz, testCount);
    parallel(nPhi * nCos, nT, [&](uint32_t xy, uint32_t testIndex, uint32_t) {
        const uint32_t phiBin = xy % nPhi, cosBin = xy / nPhi;
        const Falcor::float3 f = load<Falcor::float3>(wiBuf, testIndex);
        const V3<float> wi = orc::normalize(V3<float>(f.x, f.y, f.z));
        const LobeUnderTest& bsdf = lobes[testIndex];
        const float phiStart = float(phiBin) * k2Pi / float(phiBins);
        const float phiEnd = float(phiBin + 1) * k2Pi / float(phiBins);
        float cosStart = -1.f + float(cosBin) * 2.f / float(cosBins);
        float cosEnd = -1.f + float(cosBin + 1) * 2.f / float(cosBins);
        cosStart = std::max(cosStart, -1.f + kCosThetaMargin);
        cosEnd = std::min(cosEnd, 1.f - kCosThetaMargin);
        float pdf = 0.f;
        for (uint32_t ix = 0; ix < binSamples; ix++)
            for (uint32_t iy = 0; iy < binSamples; iy++) {
                const float phi = hlsl_lerp(phiStart, phiEnd, (float(ix) + 0.5f) / float(binSamples));
                const float cosTheta = hlsl_lerp(cosStart, cosEnd, (float(iy) + 0.5f) / float(binSamples));
                const float sinTheta = std::sqrt(1.f - cosTheta * cosTheta);
                const V3<float> wo = orc::normalize(V3<float>(sinTheta * orc::el_cos(phi), sinTheta * orc::el_sin(phi), cosTheta));
                pdf += bsdf.evalPdf(wi, wo);
            }
        pdf *= (cosEnd - cosStart) * (phiEnd - phiStart) / float(binSamples * binSamples);
        res[size_t(testIndex) * phiBins * cosBins + size_t(cosBin) * phiBins + phiBin] = double(pdf) * double(sampleCount);
    }, workers());
    for (size_t i = 0; i < res.size(); i++) out->setElement<double>(i, res[i]);
}

}  // namespace

// Programs of BSDFTests.cs.slang and SceneGradientsTest.cs.slang.
Program find_program_bsdf(const std::string& entry) {
    if (entry == "tabulateHistogram")
        return [](Ctx& c, uint32_t x, uint32_t y, uint32_t z) { sampling_program(c, x, y, z, false); };
    if (entry == "tabulateWeightAndPdfError")
        return [](Ctx& c, uint32_t x, uint32_t y, uint32_t z) { sampling_program(c, x, y, z, true); };
    if (entry == "tabulatePdf") return [](Ctx& c, uint32_t x, uint32_t y, uint32_t z) { pdf_program(c, x, y, z); };
    // SceneGradientsTest.cs.slang: atomicAdd / testAggregateGradients.
    if (entry == "atomicAdd")
        return [](Ctx& c, uint32_t nx, uint32_t ny, uint32_t) {
            auto* g = static_cast<orc::SceneGradientsOracle*>(const_cast<void*>(c.blocks.at("gSceneGradients")));
            const uint32_t sx = c.constants.at("CB.sz.x"), sy = c.constants.at("CB.sz.y"), hash = c.constants.at("CB.hashSize");
            for (uint32_t y = 0; y < ny && y < sy; y++)
                for (uint32_t x = 0; x < nx && x < sx; x++) g->atomic_add(0, x, y % hash, orc::el_pow(10.f, float(x)));
        };
    if (entry == "testAggregateGradients")
        return [](Ctx& c, uint32_t nx, uint32_t, uint32_t) {
            auto grads = c.buffers.at("grads");
            auto out = c.buffers.at("result");
            const uint32_t sx = c.constants.at("CB.sz.x");
            for (uint32_t x = 0; x < nx && x < sx; x++) out->setElement<float>(x, load<float>(grads, x));
        };
    return nullptr;
}

}  // namespace kat
