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

void pack_hit(const fpt_hitinfo_bits& b, const Hit& h, uint32_t out[4]);
Hit unpack_hit(const fpt_hitinfo_bits& b, const uint32_t in[4]);

void render_vbuffer_pixel(const Scene& s, uint32_t W, uint32_t H, uint32_t x, uint32_t y, uint32_t* out);
void render_vbuffer(const Scene& s, uint32_t W, uint32_t H, uint32_t* out, uint32_t y0, uint32_t y1, TraceCounters* c);

template <class R>
V3<R> minimal_pt_pixel(const Scene& s, const MinimalPTParams& p, uint32_t x, uint32_t y, const uint32_t* vbufferPixel,
                       uint32_t* rays);

template <class R>
void path_tracer_pixel(const Scene& s, const PathTracerParams& p, uint32_t x, uint32_t y, const uint32_t* vbufferPixel,
                       float* sampleOut, float* colorOut, PathCounters* pc);

void parallel_tiles(uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1, uint32_t threads,
                    const std::function<void(uint32_t, uint32_t, uint32_t)>& fn);

}  // namespace orc
