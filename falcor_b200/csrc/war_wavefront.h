// war_wavefront.h -- launch parameters of the WARDiffPathTracer kernels and
// the wavefront launcher (war_wavefront.cu).
#pragma once

#include <cuda_runtime.h>

#include "device_scene.cuh"
#include "wavefront.h"

namespace fpt {

struct WarParams {
    uint32_t width, height, maxBounces;
    uint32_t useBSDFSampling, useNEE, useMIS, useAntithetic;
    uint32_t frameSeed, lambert, meshID;
    float4* color;               // primal output
    const float* dLdI;           // float3 per pixel (adjoint)
    float* gradMat;              // [hash][matDim]
    uint32_t matDim, matHash;
    float* gradPos;              // [hash][posDim]
    uint32_t posDim, posHash;
    float* gradNrm;              // [hash][nrmDim] vertex normals of the mesh (MeshNormal)
    uint32_t nrmDim, nrmHash;
    float* gradTan;              // [hash][tanDim] vertex tangents of the mesh (MeshTangent)
    uint32_t tanDim, tanHash;
    float* gradTex;              // [texDim] base-colour texels, 3 floats each (no hashing)
    uint32_t texDim;
    unsigned long long* counters;  // [0] paths, [1] rays
    // Warped-area reparameterisation (adjoint with position gradients only).
    uint32_t useWAR, auxCount;
    float kappa, kappaScreen;    // 10^Log10vMFConcentration, 10^Log10vMFConcentrationScreen
    // Debug gradient image (ForwardDiffDebug / BackwardDiffDebug): d(color.r)/d(variable)
    // accumulated into dbgColor[pixel].x; dLdI is then null (adjoint (1, 0, 0) per pixel).
    float4* dbgColor;
    uint32_t dbgType, dbgId, dbgOffset;  // kDbg*, material or mesh, material read offset
    float4 dbgGrad;                      // tangent of the read floats / translation velocity
};

// Bytes of adjoint scratch (pending NEE gradients + per-vertex records) for a
// wave of `capacity` paths.
size_t war_adjoint_bytes(uint32_t capacity, uint32_t maxBounces, bool war);

// Checkpointed path vertices (adjointMode "Checkpoint"): the forward render
// stores the hit of every extension ray and the outcome of every visibility
// ray; the adjoint of the same frame reads them instead of tracing, and
// recomputes the shading.
struct WarCheckpoint {
    uint4* hits;        // [bounce][pixel]: instance, primitive, baryX, baryY (instance kCkMiss: missed)
    uint32_t* visible;  // [pixel]: bit b set when bounce b's visibility ray found the light
    uint32_t pixels;
    int mode;           // 0 off, 1 record (forward), 2 read (adjoint)
};
constexpr uint32_t kCkMiss = 0xffffffffu;
size_t war_checkpoint_bytes(uint32_t pixels, uint32_t maxBounces);

// Primal (backward = false) or adjoint of one frame; `launches` counts kernels.
cudaError_t launch_war_wavefront(const DevScene& s, const WarParams& p, WavefrontBuffers& b, void* adjointScratch, bool backward,
                                 cudaStream_t st, uint32_t& launches, const WarCheckpoint* ck = nullptr);

}  // namespace fpt
