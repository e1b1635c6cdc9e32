// kernels.cuh -- launch parameters and host-side launchers of the render-pass
// kernels (VBufferRT, MinimalPathTracer, PathTracer).
#pragma once

#include <cuda_runtime.h>

#include "device_scene.cuh"

namespace fpt {

constexpr int kNumCounters = 13;       // see Counters in path_logic.cuh
constexpr size_t kWorkCounterOffset = 128;  // byte offset of the work counter in the pass scratch
constexpr size_t kScratchBytes = 256;

struct FrameParams {
    uint32_t width, height;
    uint32_t frameIndex;       // gFrameCount (MinimalPathTracer)
    uint32_t prngDimension;    // gPRNGDimension
    const uint4* vbuffer;      // PackedHitInfo per pixel
    float4* color;             // RGBA32F output
    uint32_t* rayCount;        // optional per-pixel ray count
    uint32_t* pathLength;      // optional per-pixel path length
    float* sampleColor;        // optional per-sample radiance (3 floats)
    uint4* hitTrace;           // optional per-sample hit of every path vertex (fpt_frame_io::hit_trace)
    uint4* vbufferOut;         // VBufferRT output
    // VBufferRT optional outputs (VBufferRT.slang:69-143) and the camera of the
    // previous frame for the motion vectors.
    float* depthOut;
    float2* mvecOut;
    float4* viewWOut;
    float* maskOut;
    fpt_camera_data prevCamera;
    // MinimalPathTracer
    uint32_t maxBounces, computeDirect, useImportanceSampling;
    // PathTracer
    uint32_t spp, maxSurfaceBounces, maxDiffuseBounces, maxSpecularBounces, maxTransmissionBounces;
    uint32_t sampleGenerator, useBSDFSampling, useNEE, useMIS, misHeuristic;
    float misPowerExponent;
    uint32_t emissiveSampler;
    float specularRoughnessThreshold;
    uint32_t colorFormat;
    uint32_t seed;
    uint32_t lambert;          // DiffuseBrdf = Lambert (instead of Frostbite)
    uint32_t sortMaterials;    // wavefront: sort each secondary shade queue by material
    uint32_t splitMisses;      // wavefront: shade misses in their own kernel
    uint32_t sortRays;         // wavefront: bin each extension queue by origin cell and octant
    uint32_t sortShadowRays;   // wavefront: bin each visibility queue the same way
    uint32_t overlapTraces;    // wavefront: visibility rays on a second stream, beside the extension rays
    // bookkeeping
    unsigned long long* counters;  // [0] paths, [1] rays
    uint32_t* workCounter;         // persistent scheduling counter (zeroed by the launcher)
    uint32_t workItems;            // number of work items (pixels)
};

// Launchers (stream-ordered).  Return cudaGetLastError() of the launch.
cudaError_t launch_vbuffer(const DevScene& s, const FrameParams& p, cudaStream_t st);
cudaError_t launch_minimal_pt(const DevScene& s, const FrameParams& p, cudaStream_t st);
cudaError_t launch_path_tracer(const DevScene& s, const FrameParams& p, cudaStream_t st, int blockSize = 0);
int path_tracer_grid_blocks(int blockSize);

}  // namespace fpt
