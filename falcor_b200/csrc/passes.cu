// passes.cu -- render-pass objects of the C-ABI: properties with the
// reference names and defaults, channel reflection, and execute().
//
//   MinimalPathTracer  RenderPasses/MinimalPathTracer/MinimalPathTracer.cpp:60-200
//   PathTracer         RenderPasses/PathTracer/PathTracer.cpp:155-415,1329-1598
//   VBufferRT          RenderPasses/GBuffer/VBuffer/VBufferRT.cpp
//   WARDiffPathTracer  RenderPasses/WARDiffPathTracer/WARDiffPathTracer.cpp:53-144 (adjoint.cu)
//   AccumulatePass, ToneMapper, ColorMapPass, RenderToViewportPass (image_passes.cu)
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cctype>
#include <cstdlib>
#include <cstring>
#include <map>
#include <sstream>
#include <string>

#include "image_passes.h"
#include "kernels.cuh"
#include "passes.h"
#include "scene_device.h"
#include "wardiff.h"

namespace fpt {

namespace {

struct ChannelSpec { const char* name; const char* desc; bool input; bool optional; const char* format; };

const ChannelSpec kMinimalChannels[] = {
    {"vbuffer", "Visibility buffer in packed format", true, false, "PackedHitInfo"},
    {"viewW", "World-space view direction (xyz float format)", true, true, "RGBA32Float"},
    {"color", "Output color (sum of direct and indirect)", false, false, "RGBA32Float"},
};
const ChannelSpec kPathTracerChannels[] = {
    {"vbuffer", "Visibility buffer in packed format", true, false, "PackedHitInfo"},
    {"mvec", "Motion vector buffer (float format)", true, true, "RG32Float"},
    {"viewW", "World-space view direction (xyz float format)", true, true, "RGBA32Float"},
    {"sampleCount", "Sample count buffer (integer format)", true, true, "R8Uint"},
    {"color", "Output color (linear)", false, true, "RGBA32Float"},
    {"albedo", "Output albedo (linear)", false, true, "RGBA8Unorm"},
    {"specularAlbedo", "Output specular albedo (linear)", false, true, "RGBA8Unorm"},
    {"indirectAlbedo", "Output indirect albedo (linear)", false, true, "RGBA8Unorm"},
    {"guideNormal", "Output guide normal (linear)", false, true, "RGBA16Float"},
    {"reflectionPosW", "Output reflection pos (world space)", false, true, "RGBA32Float"},
    {"rayCount", "Per-pixel ray count", false, true, "R32Uint"},
    {"pathLength", "Per-pixel path length", false, true, "R32Uint"},
};
const ChannelSpec kVBufferChannels[] = {
    {"vbuffer", "Visibility buffer in packed format", false, false, "PackedHitInfo"},
    {"depth", "Depth buffer (NDC)", false, true, "R32Float"},
    {"mvec", "Motion vector", false, true, "RG32Float"},
    {"viewW", "View direction in world space", false, true, "RGBA32Float"},
    {"mask", "Mask", false, true, "R32Float"},
};
const ChannelSpec kAccumulateChannels[] = {
    {"input", "Input data to be temporally accumulated", true, false, "RGBA32Float"},
    {"output", "Output data that is temporally accumulated", false, false, "RGBA32Float"},
};
const ChannelSpec kToneMapperChannels[] = {
    {"src", "Source texture", true, false, "RGBA32Float"},
    {"dst", "Tone-mapped output texture", false, false, "RGBA32Float"},
};
const ChannelSpec kColorMapChannels[] = {
    {"input", "Input image", true, false, "RGBA32Float"},
    {"output", "Output image", false, false, "RGBA32Float"},
};
const ChannelSpec kViewportChannels[] = {
    {"input", "input", true, false, "RGBA32Float"},
    {"output", "output", false, false, "RGBA32Float"},
};

bool is_image_pass(const std::string& t) {
    return t == "AccumulatePass" || t == "ToneMapper" || t == "ColorMapPass" || t == "RenderToViewportPass";
}
const ChannelSpec kWARDiffChannels[] = {
    {"color", "Output color (linear)", false, false, "RGBA32Float"},
    {"dColor", "Output gradient of color w.r.t. the debug variable", false, true, "RGBA32Float"},
};

void set_defaults(fpt_pass& p) {
    auto& d = p.props;
    if (p.type == "MinimalPathTracer") {
        d["maxBounces"] = PropValue::num(3);
        d["computeDirect"] = PropValue::num(1);
        d["useImportanceSampling"] = PropValue::num(1);
        d["diffuseBrdf"] = PropValue::str("Frostbite");
    } else if (p.type == "PathTracer") {
        d["samplesPerPixel"] = PropValue::num(1);
        d["maxSurfaceBounces"] = PropValue::num(0);
        d["maxDiffuseBounces"] = PropValue::num(3);
        d["maxSpecularBounces"] = PropValue::num(3);
        d["maxTransmissionBounces"] = PropValue::num(10);
        d["sampleGenerator"] = PropValue::num(0);
        d["fixedSeed"] = PropValue::num(1);
        d["useBSDFSampling"] = PropValue::num(1);
        d["useRussianRoulette"] = PropValue::num(0);
        d["useNEE"] = PropValue::num(1);
        d["useMIS"] = PropValue::num(1);
        d["misHeuristic"] = PropValue::str("Balance");
        d["misPowerExponent"] = PropValue::num(2);
        d["emissiveSampler"] = PropValue::str("LightBVH");
        d["useRTXDI"] = PropValue::num(0);
        d["useAlphaTest"] = PropValue::num(1);
        d["adjustShadingNormals"] = PropValue::num(0);
        d["maxNestedMaterials"] = PropValue::num(2);
        d["useLightsInDielectricVolumes"] = PropValue::num(0);
        d["disableCaustics"] = PropValue::num(0);
        d["specularRoughnessThreshold"] = PropValue::num(0.25);
        d["primaryLodMode"] = PropValue::str("Mip0");
        d["lodBias"] = PropValue::num(0);
        d["useNRDDemodulation"] = PropValue::num(1);
        d["useSER"] = PropValue::num(1);
        d["outputSize"] = PropValue::str("Default");
        d["colorFormat"] = PropValue::str("LogLuvHDR");
        d["diffuseBrdf"] = PropValue::str("Frostbite");
        // Scheduling of this implementation (no reference counterpart):
        // "Wavefront" (default) or "Megakernel"; the most paths in flight per
        // wave.  A 1920x1080 16-spp frame (33.2 M paths) fits one wave of 2^25
        // paths (6.2 GB of path state at 184 B per path): every bounce then
        // runs once per frame, which on that frame is 1.5x faster than four
        // waves of 2^23.  Smaller frames allocate only what they use.
        d["scheduler"] = PropValue::str("Wavefront");
        d["wavefrontCapacity"] = PropValue::num(1 << 25);
        // CUDA-event timing of each wavefront kernel category (fpt_pass_get_kernel_times).
        d["profileKernels"] = PropValue::num(0);
        // Wavefront: counting-sort each secondary shade queue by material (hits
        // grouped per material, misses last) before shading.  Off by default: on
        // the 1080p heightfield frame it made shading 3.7 % faster but cost
        // 3.2 ms per frame and slowed the extension rays that follow (net -6 %).
        d["sortShadeQueue"] = PropValue::num(0);
        // Wavefront: the extension kernel queues hits and misses apart; misses
        // (environment emission) are shaded by their own small kernel.  Off by
        // default: on the 1080p heightfield frame shading got 5 % faster but the
        // queue pushes made the extension kernel 10 % slower (net -2 %).
        d["splitMisses"] = PropValue::num(0);
        // Wavefront: counting-sort each extension queue by origin cell (4 x 4 x 4
        // grid over the scene) and direction octant before traversal, so that
        // the lanes of a warp trace similar rays; the bin order also becomes the
        // next shade queue's order.
        d["sortExtensionRays"] = PropValue::num(0);
        // The same binning for the visibility rays of NEE (their origin cell and
        // direction octant), before the shadow kernel.
        d["sortShadowRays"] = PropValue::num(0);
        // Wavefront: trace a bounce's visibility rays on a second stream while
        // its extension rays trace on the caller's stream.  The two kernels
        // touch disjoint path-state fields, so the samples are the same; the
        // second kernel fills the SMs that the first one's last rays leave idle.
        d["overlapTraces"] = PropValue::num(1);
    } else if (p.type == "VBufferRT") {
        // GBufferBase.h:96-98.
        d["samplePattern"] = PropValue::str("Center");
        d["sampleCount"] = PropValue::num(16);
        d["useAlphaTest"] = PropValue::num(1);
        // Accepted for graph-script compatibility; the traversal is always the
        // build's own, never culls and has no depth of field.
        d["outputSize"] = PropValue::str("Default");
        d["useTraceRayInline"] = PropValue::num(0);
        d["useDOF"] = PropValue::num(1);
        d["adjustShadingNormals"] = PropValue::num(0);
        d["forceCullMode"] = PropValue::num(0);
        d["cull"] = PropValue::str("Back");
    } else if (p.type == "AccumulatePass") {
        // AccumulatePass.h:135-150.
        d["enabled"] = PropValue::num(1);
        d["autoReset"] = PropValue::num(1);
        d["precisionMode"] = PropValue::str("Single");
        d["maxFrameCount"] = PropValue::num(0);
        d["overflowMode"] = PropValue::str("Stop");
        d["outputSize"] = PropValue::str("Default");
        d["outputFormat"] = PropValue::str("Unknown");
    } else if (p.type == "ToneMapper") {
        // ToneMapper.h:121-169.
        d["outputSize"] = PropValue::str("Default");
        d["outputFormat"] = PropValue::str("Unknown");
        d["useSceneMetadata"] = PropValue::num(1);
        d["exposureCompensation"] = PropValue::num(0);
        d["autoExposure"] = PropValue::num(0);
        d["exposureValue"] = PropValue::num(0);
        d["filmSpeed"] = PropValue::num(100);
        d["whiteBalance"] = PropValue::num(0);
        d["whitePoint"] = PropValue::num(6500);
        d["operator"] = PropValue::str("Aces");
        d["clamp"] = PropValue::num(1);
        d["whiteMaxLuminance"] = PropValue::num(1);
        d["whiteScale"] = PropValue::num(11.199999809265137);
        d["fNumber"] = PropValue::num(1);
        d["shutter"] = PropValue::num(1);
        d["exposureMode"] = PropValue::str("AperturePriority");
    } else if (p.type == "ColorMapPass") {
        // ColorMapPass.h:52-56.
        d["colorMap"] = PropValue::str("Jet");
        d["channel"] = PropValue::num(0);
        d["autoRange"] = PropValue::num(1);
        d["minValue"] = PropValue::num(0);
        d["maxValue"] = PropValue::num(1);
    } else if (p.type == "WARDiffPathTracer") {
        d["samplesPerPixel"] = PropValue::num(1);
        d["maxBounces"] = PropValue::num(0);
        d["diffMode"] = PropValue::str("ForwardDiffDebug");
        d["diffVarName"] = PropValue::str("");
        d["sampleGenerator"] = PropValue::num(0);
        d["fixedSeed"] = PropValue::num(1);
        d["useBSDFSampling"] = PropValue::num(1);
        d["useNEE"] = PropValue::num(1);
        d["useMIS"] = PropValue::num(1);
        d["useWAR"] = PropValue::num(1);
        d["auxSampleCount"] = PropValue::num(16);
        d["Log10vMFConcentration"] = PropValue::num(5);
        d["Log10vMFConcentrationScreen"] = PropValue::num(5);
        d["boundaryTermBeta"] = PropValue::num(0.01);
        d["useAntitheticSampling"] = PropValue::num(1);
        d["diffuseBrdf"] = PropValue::str("Frostbite");
        // WARDiffPathTracerParams.runBackward (Params.slang:51) and the mesh of
        // InverseOptimizationParams (set_mesh_to_optimize).
        d["runBackward"] = PropValue::num(1);
        d["meshToOptimize"] = PropValue::num(0);
        // "Wavefront" (default) or "Megakernel" (one thread per pixel); paths per wave.
        d["scheduler"] = PropValue::str("Wavefront");
        d["wavefrontCapacity"] = PropValue::num(1 << 22);
        // "Replay" (re-trace the frame in the adjoint) or "Checkpoint" (the forward
        // render stores the path vertices; the adjoint of the same frame reads them).
        d["adjointMode"] = PropValue::str("Replay");
    }
}

const std::map<std::string, int> kMISHeuristics = {{"Balance", 0}, {"PowerTwo", 1}, {"PowerExp", 2}};
const std::map<std::string, int> kEmissiveSamplers = {{"Uniform", 0}, {"LightBVH", 1}, {"Power", 2}};
const std::map<std::string, int> kColorFormats = {{"RGBA32F", 0}, {"LogLuvHDR", 1}};
const std::map<std::string, int> kDiffModes = {{"Primal", 0}, {"BackwardDiff", 1}, {"ForwardDiffDebug", 2}, {"BackwardDiffDebug", 3}};
const std::map<std::string, int> kSamplePatterns = {{"Center", 0}, {"DirectX", 1}, {"Halton", 2}, {"Stratified", 3}};

// Enum-valued string properties: the accepted names (and integer values).
const std::map<std::string, int>* enum_map(const std::string& k) {
    if (k == "misHeuristic") return &kMISHeuristics;
    if (k == "emissiveSampler") return &kEmissiveSamplers;
    if (k == "colorFormat") return &kColorFormats;
    if (k == "diffMode") return &kDiffModes;
    if (k == "samplePattern") return &kSamplePatterns;
    if (k == "operator") return &kToneMapOperators;
    if (k == "exposureMode") return &kToneMapExposureModes;
    if (k == "colorMap") return &kColorMaps;
    if (k == "precisionMode") return &kPrecisionModes;
    if (k == "overflowMode") return &kOverflowModes;
    return nullptr;
}

// ToneMapper setters (ToneMapper.cpp:405-510): clamping and the exposure
// value tied to the shutter and f-number.  Float arithmetic as in the reference.
void tone_mapper_set(fpt_pass& p, const std::string& k, double value) {
    const float kShutterMin = 0.1f, kShutterMax = 10000.f, kFNumberMin = 0.1f, kFNumberMax = 100.f;
    const float kEVMin = std::log2(kShutterMin * kFNumberMin * kFNumberMin), kEVMax = std::log2(kShutterMax * kFNumberMax * kFNumberMax);
    auto& d = p.props;
    float v = float(value);
    auto updateEV = [&]() {
        const float sh = float(d["shutter"].n), fN = float(d["fNumber"].n);
        d["exposureValue"].n = std::log2(sh * fN * fN);
    };
    if (k == "exposureCompensation") d[k].n = std::clamp(v, -12.f, 12.f);
    else if (k == "filmSpeed") d[k].n = std::clamp(v, 1.f, 6400.f);
    else if (k == "whitePoint") d[k].n = std::clamp(v, 1905.f, 25000.f);
    else if (k == "whiteScale") d[k].n = std::max(0.001f, v);
    else if (k == "fNumber") { d[k].n = std::clamp(v, kFNumberMin, kFNumberMax); updateEV(); }
    else if (k == "shutter") { d[k].n = std::clamp(v, kShutterMin, kShutterMax); updateEV(); }
    else if (k == "exposureValue") {
        const float ev = std::clamp(v, kEVMin, kEVMax);
        if (d["exposureMode"].s == "ShutterPriority") {
            const float sh = float(d["shutter"].n);
            d["fNumber"].n = std::clamp(std::sqrt(std::pow(2.f, ev) / sh), kFNumberMin, kFNumberMax);
        } else {
            const float fN = float(d["fNumber"].n);
            d["shutter"].n = std::clamp(std::pow(2.f, ev) / (fN * fN), kShutterMin, kShutterMax);
        }
        updateEV();
    } else d[k].n = value;
}

std::string json_escape(const std::string& s) {
    std::string o;
    for (char c : s) {
        if (c == '"' || c == '\\') o += '\\';
        o += c;
    }
    return o;
}

fpt_status write_json(const std::string& s, char* buf, size_t cap) {
    if (!buf || cap < s.size() + 1) return set_error(FPT_ERR_INVALID_ARG, "buffer too small for JSON (" + std::to_string(s.size() + 1) + " bytes)");
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return FPT_OK;
}

}  // namespace
}  // namespace fpt

double fpt_pass::num(const std::string& k) const {
    auto it = props.find(k);
    return it == props.end() ? 0.0 : it->second.n;
}
std::string fpt_pass::str(const std::string& k) const {
    auto it = props.find(k);
    return it == props.end() ? std::string() : it->second.s;
}

namespace fpt {

fpt_status ensure_scratch(fpt_pass& p) {
    if (p.scratch) return FPT_OK;
    if (cudaMalloc(&p.scratch, kScratchBytes) != cudaSuccess) return set_error(FPT_ERR_OOM, "cudaMalloc pass scratch");
    cudaMemset(p.scratch, 0, kScratchBytes);
    return FPT_OK;
}

// The camera jitter of VBufferRT's sample pattern (GBufferBase.cpp:202-229,
// Camera.cpp:50-58): the next pattern sample x (1/width, 1/height) becomes the
// scene camera's jitter for this frame; "Center" leaves the camera unjittered.
//   DirectX     Utils/SampleGenerators/DxSamplePattern.cpp (8 positions)
//   Halton      HaltonSamplePattern.cpp: bases 2 and 3, frac(v + 0.5) - 0.5
//   Stratified  StratifiedSamplePattern.cpp: binsX x binsY strata, a fresh
//               std::shuffle of the strata per round, std::mt19937 (default
//               seed) and std::uniform_real_distribution<float> for the offsets
void vbuffer_apply_jitter(fpt_pass& p, uint32_t width, uint32_t height) {
    auto it = kSamplePatterns.find(p.str("samplePattern"));
    const int pattern = it == kSamplePatterns.end() ? 0 : it->second;
    fpt_scene* sc = p.scene;
    if (p.patternBinsX == 0) {
        // (Re)create the generator (GBufferBase::updateSamplePattern).
        p.patternIndex = 0;
        p.patternRng = std::mt19937();
        p.patternBinsX = p.patternBinsY = 1;
        p.patternPermutation.clear();
        uint32_t count = uint32_t(std::max(0.0, p.num("sampleCount")));
        if (pattern == 1) {
            if (count != 8) log_warning("DxSamplePattern() currently requires sampleCount = 8. Using that number.");
            p.props["sampleCount"].n = 8;
        } else if (pattern == 3) {
            count = std::clamp(count, 1u, 1024u);
            uint32_t bx = uint32_t(std::sqrt(double(count))), by = count / bx;
            while (bx * by != count) {
                bx++;
                by = count / bx;
            }
            p.patternBinsX = bx;
            p.patternBinsY = by;
            p.patternPermutation.resize(count);
            for (uint32_t i = 0; i < count; i++) p.patternPermutation[i] = i;
            p.props["sampleCount"].n = count;
        }
        if (pattern == 0 && (sc->dev.camera.jitterX != 0.f || sc->dev.camera.jitterY != 0.f)) {
            sc->info.camera.jitterX = sc->info.camera.jitterY = 0.f;
            sc->dev.camera = sc->info.camera;
            sc->version++;
        }
    }
    if (pattern == 0) return;
    float jx = 0.f, jy = 0.f;
    if (pattern == 1) {
        static const float kDx[8][2] = {{1.f / 16.f, -3.f / 16.f}, {-1.f / 16.f, 3.f / 16.f}, {5.f / 16.f, 1.f / 16.f},
                                        {-3.f / 16.f, -5.f / 16.f}, {-5.f / 16.f, 5.f / 16.f}, {-7.f / 16.f, -1.f / 16.f},
                                        {3.f / 16.f, 7.f / 16.f}, {7.f / 16.f, -7.f / 16.f}};
        jx = kDx[p.patternIndex % 8][0];
        jy = kDx[p.patternIndex % 8][1];
        p.patternIndex++;
    } else if (pattern == 2) {
        auto radical = [](uint32_t index, uint32_t base) {
            float result = 0.f, factor = 1.f;
            for (; index > 0; index /= base) {
                factor /= float(base);
                result += factor * float(index % base);
            }
            return result;
        };
        const float hx = radical(p.patternIndex, 2), hy = radical(p.patternIndex, 3);
        const uint32_t count = uint32_t(std::max(0.0, p.num("sampleCount")));
        p.patternIndex++;
        if (count != 0) p.patternIndex %= count;
        auto frac = [](float v) { return v - std::floor(v); };
        jx = frac(hx + 0.5f) - 0.5f;
        jy = frac(hy + 0.5f) - 0.5f;
    } else {
        std::uniform_real_distribution<float> dist;
        if (p.patternIndex == 0) std::shuffle(p.patternPermutation.begin(), p.patternPermutation.end(), p.patternRng);
        const uint32_t bin = p.patternPermutation[p.patternIndex];
        const uint32_t i = bin % p.patternBinsX, j = bin / p.patternBinsX;
        p.patternIndex = (p.patternIndex + 1) % uint32_t(p.patternPermutation.size());
        const float x = (float(i) + dist(p.patternRng)) / float(p.patternBinsX);
        const float y = (float(j) + dist(p.patternRng)) / float(p.patternBinsY);
        jx = x - 0.5f;
        jy = y - 0.5f;
    }
    sc->info.camera.jitterX = jx * (1.f / float(width));
    sc->info.camera.jitterY = jy * (1.f / float(height));
    sc->dev.camera = sc->info.camera;
    sc->version++;
}

// Fills the PathTracer parameters after PathTracer::validateOptions (PathTracer.cpp:370-415).
void path_tracer_params(fpt_pass& p, FrameParams& fp) {
    fp.spp = uint32_t(std::clamp(p.num("samplesPerPixel"), 1.0, 16.0));
    auto clampB = [](double v) { return uint32_t(std::clamp(v, 0.0, 254.0)); };
    uint32_t surface = clampB(p.num("maxSurfaceBounces"));
    fp.maxDiffuseBounces = clampB(p.num("maxDiffuseBounces"));
    fp.maxSpecularBounces = clampB(p.num("maxSpecularBounces"));
    fp.maxTransmissionBounces = clampB(p.num("maxTransmissionBounces"));
    // PathTracer::parseProperties (PathTracer.cpp:336-350): an explicit
    // maxSurfaceBounces initialises the per-type counts that were not set;
    // otherwise it is the largest of them.  validateOptions (:398-401) then
    // raises it to at least each per-type count.
    if (p.explicitKeys.count("maxSurfaceBounces")) {
        if (!p.explicitKeys.count("maxDiffuseBounces")) fp.maxDiffuseBounces = surface;
        if (!p.explicitKeys.count("maxSpecularBounces")) fp.maxSpecularBounces = surface;
        if (!p.explicitKeys.count("maxTransmissionBounces")) fp.maxTransmissionBounces = surface;
    }
    const uint32_t typeMax = std::max(fp.maxDiffuseBounces, std::max(fp.maxSpecularBounces, fp.maxTransmissionBounces));
    fp.maxSurfaceBounces = p.explicitKeys.count("maxSurfaceBounces") ? std::max(surface, typeMax) : typeMax;
    fp.sampleGenerator = uint32_t(p.num("sampleGenerator")) == 1 ? 1u : 0u;
    fp.useBSDFSampling = p.num("useBSDFSampling") != 0;
    fp.useNEE = p.num("useNEE") != 0;
    fp.useMIS = p.num("useMIS") != 0;
    auto mh = kMISHeuristics.find(p.str("misHeuristic"));
    fp.misHeuristic = mh == kMISHeuristics.end() ? 0u : uint32_t(mh->second);
    fp.misPowerExponent = float(p.num("misPowerExponent"));
    auto es = kEmissiveSamplers.find(p.str("emissiveSampler"));
    const int sampler = es == kEmissiveSamplers.end() ? 1 : es->second;
    fp.emissiveSampler = uint32_t(sampler);
    fp.specularRoughnessThreshold = float(std::clamp(p.num("specularRoughnessThreshold"), 0.0, 1.0));
    auto cf = kColorFormats.find(p.str("colorFormat"));
    fp.colorFormat = cf == kColorFormats.end() ? 1u : uint32_t(cf->second);
    fp.seed = p.useFixedSeed ? uint32_t(p.num("fixedSeed")) : p.frameCount;
    fp.lambert = p.str("diffuseBrdf") == "Lambert";
    fp.sortMaterials = p.num("sortShadeQueue") != 0 ? 1u : 0u;
    fp.splitMisses = p.num("splitMisses") != 0 ? 1u : 0u;
    fp.sortRays = p.num("sortExtensionRays") != 0 ? 1u : 0u;
    fp.sortShadowRays = p.num("sortShadowRays") != 0 ? 1u : 0u;
    fp.overlapTraces = p.num("overlapTraces") != 0 ? 1u : 0u;
}

}  // namespace fpt

using namespace fpt;

extern "C" {

FPT_API fpt_status fpt_pass_create(const char* type_name, fpt_pass** out) {
    if (!type_name || !out) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_create: null argument");
    std::string t(type_name);
    if (t != "MinimalPathTracer" && t != "PathTracer" && t != "VBufferRT" && t != "WARDiffPathTracer" && !is_image_pass(t))
        return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_create: unknown render pass type '" + t + "'");
    auto* p = new fpt_pass();
    p->type = t;
    set_defaults(*p);
    *out = p;
    return FPT_OK;
}

FPT_API void fpt_pass_destroy(fpt_pass* pass) {
    if (!pass) return;
    if (pass->scratch) cudaFree(pass->scratch);
    if (pass->adjointScratch) cudaFree(pass->adjointScratch);
    if (pass->checkpoint) cudaFree(pass->checkpoint);
    if (pass->accumSum) cudaFree(pass->accumSum);
    if (pass->accumCorr) cudaFree(pass->accumCorr);
    if (pass->imageScratch) cudaFree(pass->imageScratch);
    delete pass;
}

FPT_API fpt_status fpt_pass_set_property_int(fpt_pass* pass, const char* key, int64_t value) {
    return fpt_pass_set_property_float(pass, key, double(value));
}

FPT_API fpt_status fpt_pass_set_property_float(fpt_pass* pass, const char* key, double value) {
    if (!pass || !key) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_set_property: null argument");
    std::string k(key);
    if (pass->type == "AccumulatePass" && k == "enableAccumulation") {
        // AccumulatePass.cpp:87-92.
        log_warning("'enableAccumulation' is deprecated. Use 'enabled' instead.");
        k = "enabled";
    }
    auto it = pass->props.find(k);
    if (it == pass->props.end()) {
        log_warning("Unknown property '" + k + "' in " + pass->type + " properties.");
        return FPT_OK;
    }
    if (it->second.isString) {
        // Enum-valued properties also accept their integer value.
        const std::map<std::string, int>* m = enum_map(k);
        if (!m) return set_error(FPT_ERR_INVALID_ARG, "property '" + k + "' expects a string");
        for (auto& kv : *m)
            if (kv.second == int(value)) return fpt_pass_set_property_string(pass, k.c_str(), kv.first.c_str());
        return set_error(FPT_ERR_INVALID_ARG, "invalid value for property '" + k + "'");
    }
    if (k == "fixedSeed") pass->useFixedSeed = true;
    pass->explicitKeys.insert(k);
    if (pass->type == "ToneMapper") {
        tone_mapper_set(*pass, k, value);
        return FPT_OK;
    }
    if (pass->type == "AccumulatePass" && k == "enabled" && (value != 0) != (it->second.n != 0)) pass->frameCount = 0;
    if (pass->type == "VBufferRT" && k == "sampleCount") pass->patternBinsX = 0;  // re-create the pattern
    it->second.n = value;
    return FPT_OK;
}

FPT_API fpt_status fpt_pass_set_property_string(fpt_pass* pass, const char* key, const char* value) {
    if (!pass || !key || !value) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_set_property_string: null argument");
    auto it = pass->props.find(key);
    if (it == pass->props.end()) {
        log_warning("Unknown property '" + std::string(key) + "' in " + pass->type + " properties.");
        return FPT_OK;
    }
    if (!it->second.isString) return set_error(FPT_ERR_INVALID_ARG, "property '" + std::string(key) + "' expects a number");
    std::string k(key), v(value);
    const std::map<std::string, int>* m = enum_map(k);
    if (m && m->find(v) == m->end()) return set_error(FPT_ERR_INVALID_ARG, "invalid value '" + v + "' for property '" + k + "'");
    if (k == "samplePattern") pass->patternBinsX = 0;  // re-create the pattern
    pass->explicitKeys.insert(k);
    if (k == "diffuseBrdf" && v != "Frostbite" && v != "Lambert")
        return set_error(FPT_ERR_INVALID_ARG, "diffuseBrdf must be 'Frostbite' or 'Lambert'");
    if (k == "scheduler" && v != "Wavefront" && v != "Megakernel")
        return set_error(FPT_ERR_INVALID_ARG, "scheduler must be 'Wavefront' or 'Megakernel'");
    if (k == "adjointMode" && v != "Replay" && v != "Checkpoint")
        return set_error(FPT_ERR_INVALID_ARG, "adjointMode must be 'Replay' or 'Checkpoint'");
    it->second.s = v;
    return FPT_OK;
}

FPT_API fpt_status fpt_pass_set_properties_json(fpt_pass* pass, const char* json) {
    if (!pass || !json) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_set_properties_json: null argument");
    // A flat JSON object (Properties::dump): strings, numbers and booleans are
    // applied like the typed setters; nested objects, arrays and null are
    // skipped with a warning (sub-option blocks such as lightBVHOptions).
    const char* c = json;
    auto ws = [&] { while (*c == ' ' || *c == '\t' || *c == '\n' || *c == '\r') c++; };
    auto fail = [&](const std::string& what) {
        return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_set_properties_json: " + what + " at offset " + std::to_string(c - json));
    };
    auto parse_string = [&](std::string& out) -> bool {
        if (*c != '"') return false;
        c++;
        out.clear();
        while (*c && *c != '"') {
            if (*c == '\\') {
                c++;
                switch (*c) {
                    case '"': out += '"'; break;
                    case '\\': out += '\\'; break;
                    case '/': out += '/'; break;
                    case 'b': out += '\b'; break;
                    case 'f': out += '\f'; break;
                    case 'n': out += '\n'; break;
                    case 'r': out += '\r'; break;
                    case 't': out += '\t'; break;
                    case 'u': {
                        unsigned v = 0;
                        for (int k = 1; k <= 4; k++) {
                            const char h = c[k];
                            if (!std::isxdigit(static_cast<unsigned char>(h))) return false;
                            v = v * 16 + unsigned(std::isdigit(static_cast<unsigned char>(h)) ? h - '0' : (std::tolower(h) - 'a' + 10));
                        }
                        c += 4;
                        if (v < 0x80) out += char(v);
                        else if (v < 0x800) { out += char(0xc0 | (v >> 6)); out += char(0x80 | (v & 0x3f)); }
                        else { out += char(0xe0 | (v >> 12)); out += char(0x80 | ((v >> 6) & 0x3f)); out += char(0x80 | (v & 0x3f)); }
                        break;
                    }
                    default: return false;
                }
                c++;
            } else {
                out += *c++;
            }
        }
        if (*c != '"') return false;
        c++;
        return true;
    };
    // Skips a nested value (object or array), honouring strings.
    auto skip_nested = [&]() -> bool {
        int depth = 0;
        std::string tmp;
        do {
            if (*c == '"') {
                if (!parse_string(tmp)) return false;
                continue;
            }
            if (*c == '{' || *c == '[') depth++;
            else if (*c == '}' || *c == ']') depth--;
            else if (!*c) return false;
            c++;
        } while (depth > 0);
        return true;
    };
    ws();
    if (*c != '{') return fail("expected '{'");
    c++;
    ws();
    if (*c == '}') return FPT_OK;
    for (;;) {
        ws();
        std::string key;
        if (!parse_string(key)) return fail("expected a key");
        ws();
        if (*c != ':') return fail("expected ':'");
        c++;
        ws();
        fpt_status st = FPT_OK;
        if (*c == '"') {
            std::string v;
            if (!parse_string(v)) return fail("bad string");
            st = fpt_pass_set_property_string(pass, key.c_str(), v.c_str());
        } else if (!std::strncmp(c, "true", 4) || !std::strncmp(c, "false", 5)) {
            const bool b = *c == 't';
            c += b ? 4 : 5;
            st = fpt_pass_set_property_int(pass, key.c_str(), b ? 1 : 0);
        } else if (!std::strncmp(c, "null", 4)) {
            c += 4;
            log_warning("Property '" + key + "' is null; ignored.");
        } else if (*c == '{' || *c == '[') {
            if (!skip_nested()) return fail("bad nested value");
            log_warning("Property '" + key + "' (a nested object or array) is not supported by " + pass->type + "; ignored.");
        } else {
            char* end = nullptr;
            const double v = std::strtod(c, &end);
            if (end == c) return fail("bad value");
            c = end;
            st = fpt_pass_set_property_float(pass, key.c_str(), v);
        }
        if (st != FPT_OK) return st;
        ws();
        if (*c == ',') {
            c++;
            continue;
        }
        if (*c == '}') break;
        return fail("expected ',' or '}'");
    }
    return FPT_OK;
}

FPT_API fpt_status fpt_pass_get_properties_json(const fpt_pass* pass, char* buf, size_t cap) {
    if (!pass) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_get_properties_json: null pass");
    std::map<std::string, PropValue> props = pass->props;
    if (pass->type == "PathTracer") {
        // PathTracer::getProperties reports the bounce counts after parsing and validation.
        FrameParams fp;
        std::memset(&fp, 0, sizeof(fp));
        fpt_pass tmp;
        tmp.props = pass->props;
        tmp.explicitKeys = pass->explicitKeys;
        path_tracer_params(tmp, fp);
        props["maxSurfaceBounces"].n = fp.maxSurfaceBounces;
        props["maxDiffuseBounces"].n = fp.maxDiffuseBounces;
        props["maxSpecularBounces"].n = fp.maxSpecularBounces;
        props["maxTransmissionBounces"].n = fp.maxTransmissionBounces;
    }
    std::ostringstream os;
    os << "{";
    bool first = true;
    for (auto& kv : props) {
        if (!first) os << ", ";
        first = false;
        os << "\"" << json_escape(kv.first) << "\": ";
        if (kv.second.isString) os << "\"" << json_escape(kv.second.s) << "\"";
        else {
            char tmp[64];
            std::snprintf(tmp, sizeof(tmp), "%.17g", kv.second.n);
            os << tmp;
        }
    }
    os << "}";
    return write_json(os.str(), buf, cap);
}

FPT_API fpt_status fpt_pass_reflect_json(const fpt_pass* pass, char* buf, size_t cap) {
    if (!pass) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_reflect_json: null pass");
    const ChannelSpec* ch = nullptr;
    size_t n = 0;
    if (pass->type == "MinimalPathTracer") { ch = kMinimalChannels; n = sizeof(kMinimalChannels) / sizeof(ChannelSpec); }
    else if (pass->type == "PathTracer") { ch = kPathTracerChannels; n = sizeof(kPathTracerChannels) / sizeof(ChannelSpec); }
    else if (pass->type == "VBufferRT") { ch = kVBufferChannels; n = sizeof(kVBufferChannels) / sizeof(ChannelSpec); }
    else if (pass->type == "AccumulatePass") { ch = kAccumulateChannels; n = 2; }
    else if (pass->type == "ToneMapper") { ch = kToneMapperChannels; n = 2; }
    else if (pass->type == "ColorMapPass") { ch = kColorMapChannels; n = 2; }
    else if (pass->type == "RenderToViewportPass") { ch = kViewportChannels; n = 2; }
    else { ch = kWARDiffChannels; n = sizeof(kWARDiffChannels) / sizeof(ChannelSpec); }
    std::ostringstream os;
    os << "{\"inputs\": [";
    bool first = true;
    for (size_t i = 0; i < n; i++) {
        if (!ch[i].input) continue;
        os << (first ? "" : ", ") << "{\"name\": \"" << ch[i].name << "\", \"desc\": \"" << ch[i].desc << "\", \"optional\": "
           << (ch[i].optional ? "true" : "false") << ", \"format\": \"" << ch[i].format << "\"}";
        first = false;
    }
    os << "], \"outputs\": [";
    first = true;
    for (size_t i = 0; i < n; i++) {
        if (ch[i].input) continue;
        os << (first ? "" : ", ") << "{\"name\": \"" << ch[i].name << "\", \"desc\": \"" << ch[i].desc << "\", \"optional\": "
           << (ch[i].optional ? "true" : "false") << ", \"format\": \"" << ch[i].format << "\"}";
        first = false;
    }
    os << "]}";
    return write_json(os.str(), buf, cap);
}

FPT_API fpt_status fpt_pass_set_scene(fpt_pass* pass, fpt_scene* scene) {
    if (!pass) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_set_scene: null pass");
    pass->scene = scene;
    pass->frameCount = 0;
    pass->havePrevCamera = false;
    if (scene) pass->accumSceneVersion = scene->resetVersion;
    return FPT_OK;
}

FPT_API fpt_status fpt_pass_reset(fpt_pass* pass) {
    if (!pass) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_reset: null pass");
    pass->frameCount = 0;
    return FPT_OK;
}

FPT_API fpt_status fpt_pass_execute(fpt_pass* pass, const fpt_frame_io* io, void* stream) {
    if (!pass || !io) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_execute: null argument");
    if (io->width == 0 || io->height == 0 || io->width > 16384 || io->height > 16384)
        return set_error(FPT_ERR_INVALID_ARG, pass->type + ": invalid frame size");
    if (is_image_pass(pass->type)) return image_pass_execute(*pass, io, static_cast<cudaStream_t>(stream));
    if (!pass->scene) return set_error(FPT_ERR_NO_SCENE, pass->type + ": no scene set");
    if (pass->type == "PathTracer" && (io->width > 4096 || io->height > 4096))
        return set_error(FPT_ERR_INVALID_ARG, "PathTracer: frame dimension exceeds kMaxFrameDimension (4096)");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    fpt_status s = ensure_scratch(*pass);
    if (s != FPT_OK) return s;
    const DevScene& ds = pass->scene->dev;
    FrameParams fp;
    std::memset(&fp, 0, sizeof(fp));
    fp.width = io->width;
    fp.height = io->height;
    fp.frameIndex = io->frame_index;
    fp.prngDimension = io->prng_dimension;
    fp.vbuffer = reinterpret_cast<const uint4*>(io->vbuffer);
    fp.color = reinterpret_cast<float4*>(io->color);
    fp.rayCount = io->ray_count;
    fp.pathLength = io->path_length;
    fp.sampleColor = io->sample_color;
    fp.hitTrace = reinterpret_cast<uint4*>(io->hit_trace);
    fp.vbufferOut = reinterpret_cast<uint4*>(io->vbuffer_out);
    fp.counters = reinterpret_cast<unsigned long long*>(pass->scratch);
    fp.workCounter = reinterpret_cast<uint32_t*>(static_cast<char*>(pass->scratch) + kWorkCounterOffset);
    fp.workItems = io->width * io->height;
    cudaError_t e = cudaMemsetAsync(pass->scratch, 0, kNumCounters * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, cudaGetErrorString(e));
    pass->launches = 1;
    if (pass->type == "VBufferRT") {
        if (!io->vbuffer_out) return set_error(FPT_ERR_INVALID_ARG, "VBufferRT: output 'vbuffer' not connected");
        vbuffer_apply_jitter(*pass, io->width, io->height);
        fp.depthOut = io->depth;
        fp.mvecOut = reinterpret_cast<float2*>(io->mvec);
        fp.viewWOut = reinterpret_cast<float4*>(io->view_w);
        fp.maskOut = io->mask;
        fp.prevCamera = pass->havePrevCamera ? pass->prevCamera : pass->scene->dev.camera;
        pass->prevCamera = pass->scene->dev.camera;
        pass->havePrevCamera = true;
        e = launch_vbuffer(pass->scene->dev, fp, st);
    } else if (pass->type == "MinimalPathTracer") {
        if (!io->vbuffer || !io->color) return set_error(FPT_ERR_INVALID_ARG, "MinimalPathTracer: 'vbuffer' and 'color' are required");
        fp.maxBounces = uint32_t(std::max(0.0, pass->num("maxBounces")));
        fp.computeDirect = pass->num("computeDirect") != 0;
        fp.useImportanceSampling = pass->num("useImportanceSampling") != 0;
        fp.lambert = pass->str("diffuseBrdf") == "Lambert";
        fp.frameIndex = io->frame_index;
        e = launch_minimal_pt(ds, fp, st);
    } else if (pass->type == "PathTracer") {
        if (!io->vbuffer || !io->color) return set_error(FPT_ERR_INVALID_ARG, "PathTracer: 'vbuffer' and 'color' are required");
        path_tracer_params(*pass, fp);
        if (pass->str("scheduler") == "Megakernel") {
            pass->launches = 2;
            e = launch_path_tracer(ds, fp, st);
        } else {
            // Path state grows to the largest wave this pass has rendered, up to
            // wavefrontCapacity (184 B per path): a small frame holds little memory.
            const uint32_t cap = uint32_t(std::max(1.0, pass->num("wavefrontCapacity")));
            const uint64_t framePaths = uint64_t(fp.width) * fp.height * fp.spp;
            const uint32_t need = uint32_t(std::min<uint64_t>(cap, std::max<uint64_t>(framePaths, fp.spp)));
            e = pass->wavefront.ensure(std::max<uint32_t>(need, fp.spp));
            if (e != cudaSuccess) return set_error(FPT_ERR_OOM, std::string("PathTracer: wavefront buffers: ") + cudaGetErrorString(e));
            pass->timer.enabled = pass->num("profileKernels") != 0;
            e = launch_path_tracer_wavefront(ds, fp, pass->wavefront, st, &pass->timer);
            const uint32_t wavePixels = std::max<uint32_t>(1, std::min<uint32_t>(fp.width * fp.height, pass->wavefront.capacity / fp.spp));
            const uint32_t waves = (fp.width * fp.height + wavePixels - 1) / wavePixels;
            const bool binRays = fp.sortRays && !fp.splitMisses;
            pass->launches = waves * (4 * (fp.maxSurfaceBounces + 2) + 3 +
                                      (binRays ? 3 * (fp.maxSurfaceBounces + 2) : (fp.sortMaterials ? 3 * (fp.maxSurfaceBounces + 1) : 0)) +
                                      (fp.sortShadowRays ? 3 * (fp.maxSurfaceBounces + 2) : 0) +
                                      (fp.splitMisses ? fp.maxSurfaceBounces + 1 : 0));
        }
        pass->frameCount++;
    } else {
        return wardiff_execute(*pass, io, nullptr, nullptr, st);
    }
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, pass->type + ": kernel launch failed: " + cudaGetErrorString(e));
    return FPT_OK;
}

FPT_API fpt_status fpt_pass_backward(fpt_pass* pass, const fpt_frame_io* io, const float* dLdI, const fpt_grad_buffers* grads,
                                     void* stream) {
    if (!pass || !io || !dLdI || !grads) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_backward: null argument");
    if (pass->type != "WARDiffPathTracer") return set_error(FPT_ERR_UNSUPPORTED, "fpt_pass_backward: only WARDiffPathTracer is differentiable");
    if (!pass->scene) return set_error(FPT_ERR_NO_SCENE, "WARDiffPathTracer: no scene set");
    fpt_status s = ensure_scratch(*pass);
    if (s != FPT_OK) return s;
    return wardiff_execute(*pass, io, dLdI, grads, static_cast<cudaStream_t>(stream));
}

FPT_API fpt_status fpt_pass_set_scene_gradients(fpt_pass* pass, fpt_scene_gradients* grads) {
    if (!pass) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_set_scene_gradients: null pass");
    if (pass->type != "WARDiffPathTracer") return set_error(FPT_ERR_UNSUPPORTED, "scene_gradients: only WARDiffPathTracer has scene gradients");
    pass->sceneGradients = grads;
    return FPT_OK;
}

FPT_API fpt_status fpt_pass_set_diff_debug_params(fpt_pass* pass, uint32_t var_type, uint32_t id_x, uint32_t id_y,
                                                  uint32_t offset, const float grad[4]) {
    if (!pass || !grad) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_set_diff_debug_params: null argument");
    if (var_type > FPT_DIFF_VAR_GEOMETRY_TRANSLATION)
        return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_set_diff_debug_params: invalid variable type");
    if (var_type == FPT_DIFF_VAR_MATERIAL && offset >= 20)
        return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_set_diff_debug_params: material offset must be < 20");
    pass->diffDebugExplicit = true;
    pass->diffDebugType = var_type;
    pass->diffDebugId[0] = id_x;
    pass->diffDebugId[1] = id_y;
    pass->diffDebugOffset = offset;
    for (int i = 0; i < 4; i++) pass->diffDebugGrad[i] = grad[i];
    return FPT_OK;
}

FPT_API fpt_status fpt_pass_set_dLdI(fpt_pass* pass, const float* dLdI) {
    if (!pass) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_set_dLdI: null pass");
    if (pass->type != "WARDiffPathTracer") return set_error(FPT_ERR_UNSUPPORTED, "dL_dI: only WARDiffPathTracer takes dL_dI");
    pass->dLdI = dLdI;
    return FPT_OK;
}

FPT_API fpt_status fpt_pass_get_stats(fpt_pass* pass, fpt_pass_stats* out, void* stream) {
    if (!pass || !out) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_get_stats: null argument");
    std::memset(out, 0, sizeof(*out));
    if (!pass->scratch || !pass->scene) return FPT_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned long long c[2] = {0, 0};
    uint32_t err = 0;
    cudaError_t e = cudaMemcpyAsync(c, pass->scratch, 16, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&err, pass->scene->dev.errorWord, 4, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, cudaGetErrorString(e));
    out->paths = c[0];
    out->rays = c[1];
    out->device_error = err;
    out->kernel_launches = pass->launches;
    out->adjoint_checkpointed = pass->lastAdjointCheckpointed ? 1u : 0u;
    out->checkpoint_bytes = pass->checkpointBytes;
    return err ? set_error(FPT_ERR_DEVICE, "device error word 0x" + std::to_string(err)) : FPT_OK;
}

FPT_API fpt_status fpt_pass_get_kernel_times(fpt_pass* pass, double* ms, uint64_t* launches, uint32_t count, int reset) {
    if (!pass || !ms || !launches) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_get_kernel_times: null argument");
    cudaError_t e = pass->timer.collect();
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, cudaGetErrorString(e));
    for (uint32_t i = 0; i < count; i++) {
        ms[i] = i < uint32_t(KC_COUNT) ? pass->timer.ms[i] : 0.0;
        launches[i] = i < uint32_t(KC_COUNT) ? pass->timer.launches[i] : 0;
    }
    if (reset) pass->timer.reset();
    return FPT_OK;
}

FPT_API fpt_status fpt_pass_get_counters(fpt_pass* pass, uint64_t* out, uint32_t count, void* stream) {
    if (!pass || !out) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_get_counters: null argument");
    const uint32_t n = std::min<uint32_t>(count, uint32_t(kNumCounters));
    std::memset(out, 0, size_t(count) * sizeof(uint64_t));
    if (!pass->scratch) return FPT_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemcpyAsync(out, pass->scratch, size_t(n) * sizeof(uint64_t), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, cudaGetErrorString(e));
    return FPT_OK;
}

}  // extern "C"
