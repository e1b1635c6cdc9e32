// oracle_render.h -- declarations of the CPU restatement of the render passes.
//
// TEST INFRASTRUCTURE ONLY (see oracle_math.h).
#pragma once

#include <functional>
#include "oracle_scene.h"

namespace orc {

struct MinimalPTParams {        // MinimalPathTracer properties + CB
    uint32_t width, height;
    uint32_t frameCount;        // gFrameCount
    uint32_t prngDimension;     // gPRNGDimension
    uint32_t maxBounces;        // default 3
    uint32_t computeDirect;     // default 1
    uint32_t useImportanceSampling;  // default 1
    uint32_t lambert;           // DiffuseBrdf = Lambert instead of Frostbite
};

struct PathTracerParams {       // PathTracer static + runtime parameters
    uint32_t width, height;
    uint32_t samplesPerPixel;
    uint32_t maxSurfaceBounces, maxDiffuseBounces, maxSpecularBounces, maxTransmissionBounces;
    uint32_t sampleGenerator;   // 0 tiny uniform (default), 1 uniform
    uint32_t useBSDFSampling, useNEE, useMIS;
    uint32_t misHeuristic;      // 0 balance, 1 power two, 2 power exp
    float misPowerExponent;
    uint32_t emissiveSampler;   // 0 uniform, 2 power
    float specularRoughnessThreshold;
    uint32_t colorFormat;       // 0 RGBA32F, 1 LogLuvHDR
    uint32_t seed;              // params.seed (fixedSeed or frame count)
    uint32_t lambert;
};

struct PathCounters {
    uint64_t paths = 0, rays = 0;
    TraceCounters tc;
};

// WARDiffPathTracer (oracle_wardiff.inl).
struct WarDiffParams {           // WARDiffPathTracer static + runtime parameters
    uint32_t width, height;
    uint32_t maxBounces;         // default 0
    uint32_t useBSDFSampling, useNEE, useMIS;
    uint32_t useAntithetic;      // default 1
    uint32_t seed;               // frame seed (fixedSeed or frame count)
    uint32_t lambert;
    uint32_t meshID;             // mesh whose vertex positions are differentiated (0xffffffff: all)
    uint32_t useWAR;             // warped-area reparameterisation (pass default 1)
    uint32_t auxSampleCount;     // auxiliary rays per reparameterisation (default 16)
    float log10Kappa;            // Log10vMFConcentration (default 5)
    float log10KappaScreen;      // Log10vMFConcentrationScreen (default 5)
};

struct WarSeeds {
    int K = 0;                       // number of seeded directions
    const double* mat = nullptr;     // K x matDim tangents of material parameters (materialID * 20 + offset)
    uint32_t matDim = 0;
    const double* pos = nullptr;     // K x posDim tangents of the positions of mesh `meshID` (localVertex * 3 + axis)
    uint32_t posDim = 0;
    uint32_t meshID = 0xffffffffu;
    const double* nrm = nullptr;     // K x nrmDim tangents of the (normalised) vertex normals of mesh `meshID`
    uint32_t nrmDim = 0;
    const double* tan = nullptr;     // K x tanDim tangents of the (normalised) vertex tangents of mesh `meshID`
    uint32_t tanDim = 0;
    const double* tex = nullptr;     // K x texDim tangents of the texels' linear rgb ((texelBase + texel) * 3 + channel)
    uint32_t texDim = 0;
    TraceCounters* tc = nullptr;     // traversal counters of every ray traced (per thread)
    double eps = 0;                  // Shadow: perturbation scale
};

struct WarCounters { uint64_t rays = 0, hits = 0; };

// mode 0: FP32 primal into colorOut (RGBA); 1: forward-mode derivatives along
// the K <= 4 seeded directions, gradAcc[k] += dLdI . dL/dv_k; 2: the path with
// the seeded parameters offset by eps * v_0, perturbed radiance into pertOut (FP64);
// 3: the per-pixel derivative dL/dv_0 into pertOut (FP64).
void wardiff_pixel(const Scene& s, const WarDiffParams& p, const WarSeeds& seeds, int mode, uint32_t x, uint32_t y,
                   const float* dLdI, float* colorOut, double* gradAcc, double* pertOut, WarCounters* wc);

// LightBVHSampler selection pdf of emissive triangle `tri` and one traversal
// sample (tri, pdf) from shading point posW with normal n (FP32).
float lbvh_selection_pdf_f(const Scene& s, const float posW[3], const float n[3], bool upper, uint32_t tri);
bool lbvh_select_f(const Scene& s, const float posW[3], const float n[3], bool upper, float u, uint32_t* tri, float* pdf);

void pack_hit(const fpt_hitinfo_bits& b, const Hit& h, uint32_t out[4]);
Hit unpack_hit(const fpt_hitinfo_bits& b, const uint32_t in[4]);

void render_vbuffer_pixel(const Scene& s, uint32_t W, uint32_t H, uint32_t x, uint32_t y, uint32_t* out);
void render_vbuffer(const Scene& s, uint32_t W, uint32_t H, uint32_t* out, uint32_t y0, uint32_t y1, TraceCounters* c);

// trace (optional): the hit of every path vertex, 4 uints per entry
// (instanceID + 1, primitiveIndex, bary.x bits, bary.y bits; zeros for a miss),
// maxBounces + 2 (MinimalPathTracer) or maxSurfaceBounces + 2 (PathTracer)
// entries per sample, samples of the pixel one after the other.
template <class R>
V3<R> minimal_pt_pixel(const Scene& s, const MinimalPTParams& p, uint32_t x, uint32_t y, const uint32_t* vbufferPixel,
                       uint32_t* rays, uint32_t* trace = nullptr);

template <class R>
void path_tracer_pixel(const Scene& s, const PathTracerParams& p, uint32_t x, uint32_t y, const uint32_t* vbufferPixel,
                       float* sampleOut, float* colorOut, PathCounters* pc, uint32_t* trace = nullptr);

void parallel_tiles(uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1, uint32_t threads,
                    const std::function<void(uint32_t, uint32_t, uint32_t)>& fn);

}  // namespace orc
