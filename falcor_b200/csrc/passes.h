// passes.h -- the render-pass object behind the fpt_pass handle.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <random>
#include <set>
#include <string>
#include <vector>

#include "common.h"
#include "wavefront.h"

namespace fpt {

struct PropValue {
    double n = 0.0;
    std::string s;
    bool isString = false;
    static PropValue num(double v) { PropValue p; p.n = v; return p; }
    static PropValue str(const std::string& v) { PropValue p; p.s = v; p.isString = true; return p; }
};

}  // namespace fpt

struct fpt_pass {
    std::string type;
    std::map<std::string, fpt::PropValue> props;
    std::set<std::string> explicitKeys;  // properties set by the caller (Properties::has)
    fpt_scene* scene = nullptr;
    void* scratch = nullptr;          // counters (16 B) + work counter (4 B)
    void* adjointScratch = nullptr;   // checkpointed path vertices (adjoint)
    size_t adjointScratchBytes = 0;
    uint32_t frameCount = 0;
    bool useFixedSeed = false;
    uint32_t launches = 0;
    fpt::WavefrontBuffers wavefront;  // path state of the wavefront scheduler
    fpt::KernelTimer timer;           // per-category kernel timing ("profileKernels")
    fpt_scene_gradients* sceneGradients = nullptr;  // WARDiffPathTracer::scene_gradients (not owned)
    const float* dLdI = nullptr;                    // WARDiffPathTracer::dL_dI (device, float3 per pixel)
    // WARDiffPathTracer::setDiffDebugParams (explicit) or the diffVarName presets.
    bool diffDebugExplicit = false;
    uint32_t diffDebugType = 0, diffDebugId[2] = {0, 0}, diffDebugOffset = 0;
    float diffDebugGrad[4] = {0.f, 0.f, 0.f, 0.f};
    // WARDiffPathTracer adjointMode "Checkpoint": the path vertices of the last
    // forward frame and the state they belong to.
    void* checkpoint = nullptr;
    size_t checkpointBytes = 0;
    bool checkpointValid = false, lastAdjointCheckpointed = false;
    uint64_t checkpointKey[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    // AccumulatePass: running sums (double4 or float4 per pixel), the Kahan
    // correction, the frame size they belong to and the scene state seen last.
    void* accumSum = nullptr;
    float4* accumCorr = nullptr;
    size_t accumSumBytes = 0, accumCorrBytes = 0;
    int accumPrecision = -1;
    uint32_t accumW = 0, accumH = 0;
    uint64_t accumSceneVersion = 0;
    // ToneMapper / ColorMapPass reduction scratch; ColorMapPass auto range.
    void* imageScratch = nullptr;
    size_t imageScratchBytes = 0;
    double autoMin = 0.0, autoMax = 0.0;
    bool reductionAvailable = false;
    // VBufferRT camera-jitter pattern (GBufferBase.cpp:202-229) and the camera
    // of the previous frame (motion vectors).
    uint32_t patternIndex = 0;
    uint32_t patternBinsX = 1, patternBinsY = 1;
    std::vector<uint32_t> patternPermutation;
    std::mt19937 patternRng;
    bool havePrevCamera = false;
    fpt_camera_data prevCamera{};

    double num(const std::string& k) const;
    std::string str(const std::string& k) const;
};

namespace fpt {
fpt_status ensure_scratch(fpt_pass& p);
// PathTracer properties -> kernel parameters (PathTracer.cpp:253-415 parsing and validation).
void path_tracer_params(fpt_pass& p, FrameParams& fp);
// WARDiffPathTracer primal (dLdI == nullptr) or adjoint.
fpt_status wardiff_execute(fpt_pass& p, const fpt_frame_io* io, const float* dLdI, const fpt_grad_buffers* grads,
                           cudaStream_t st);
}  // namespace fpt
