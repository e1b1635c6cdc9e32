// noalloc.cu -- PathTracer execute that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a host that has reserved the GPU's
// memory for its own pool (a fixed memory budget that forbids stray device
// allocations), or a frame loop that must not take the implicit device-wide
// synchronisation of cudaMalloc/cudaFree while other work is in flight.
// For them this entry point runs the wavefront PathTracer with all of its
// scratch -- path state, queues, queue counts and event counters -- in one
// file-scope device array.  The array is part of the library image: every GPU
// that loads the library holds it until the process exits.
#include <cstring>
#include <string>

#include "kernels.cuh"
#include "passes.h"
#include "scene_device.h"
#include "wavefront.h"

namespace fpt {

namespace {

// Paths in flight per wave.  Frames of any size are processed in waves of
// kNoAllocPaths / spp pixels.
constexpr uint32_t kNoAllocPaths = 16384;
constexpr size_t kHeaderBytes = 256;  // event counters, work counter
constexpr size_t kNoAllocBytes = kHeaderBytes + WavefrontBuffers::bytes_for(kNoAllocPaths);  // 2.88 MiB
constexpr uint32_t kNoAllocMaxDim = 4096;  // PathTracer kMaxFrameDimension (Params.slang:68)
constexpr uint32_t kMaxSpp = 16;           // PathTracer kMaxSamplesPerPixel (Params.slang:67)
static_assert(kMaxSpp <= kNoAllocPaths, "one pixel's samples must fit one wave");
static_assert(kWorkCounterOffset + sizeof(uint32_t) <= kHeaderBytes, "work counter inside the header");

__device__ __align__(256) unsigned char g_noallocScratch[kNoAllocBytes];

// Device address of the scratch array on the current device.  The array's
// name in host code is only a host-side stand-in, so the address comes from
// cudaGetSymbolAddress with the calling device current.  It is looked up on
// every call (a host-side query, no stream work), so it stays valid after a
// cudaDeviceReset reloads the module.  The first call on a device loads the
// library's module there; make it before any stream capture.
fpt_status scratch_address(void** out) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noallocScratch);
    if (e != cudaSuccess || !p) return set_error(FPT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    *out = p;
    return FPT_OK;
}

}  // namespace

void path_tracer_params(fpt_pass& p, FrameParams& fp);

}  // namespace fpt

using namespace fpt;

extern "C" {

FPT_API fpt_status fpt_pass_execute_noalloc(fpt_pass* pass, const fpt_frame_io* io, void* stream) {
    if (!pass || !io) return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_execute_noalloc: null argument");
    if (pass->type != "PathTracer") return set_error(FPT_ERR_UNSUPPORTED, "fpt_pass_execute_noalloc: only PathTracer passes");
    if (!pass->scene) return set_error(FPT_ERR_NO_SCENE, "PathTracer: no scene set");
    if (!io->vbuffer || !io->color) return set_error(FPT_ERR_INVALID_ARG, "PathTracer: 'vbuffer' and 'color' are required");
    if (io->width == 0 || io->height == 0 || io->width > kNoAllocMaxDim || io->height > kNoAllocMaxDim)
        return set_error(FPT_ERR_INVALID_ARG, "fpt_pass_execute_noalloc: frame " + std::to_string(io->width) + "x" +
                                                  std::to_string(io->height) + " exceeds the maximum of " +
                                                  std::to_string(kNoAllocMaxDim) + "x" + std::to_string(kNoAllocMaxDim));
    if (pass->str("scheduler") == "Megakernel")
        return set_error(FPT_ERR_UNSUPPORTED, "fpt_pass_execute_noalloc: the Megakernel scheduler is not available without allocation");
    void* scratch = nullptr;
    fpt_status s = scratch_address(&scratch);
    if (s != FPT_OK) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
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
    fp.counters = static_cast<unsigned long long*>(scratch);
    fp.workCounter = reinterpret_cast<uint32_t*>(static_cast<char*>(scratch) + kWorkCounterOffset);
    fp.workItems = io->width * io->height;
    path_tracer_params(*pass, fp);
    // sortShadeQueue, splitMisses and sortExtensionRays need pass-owned queues;
    // they only reorder work (the samples are the same), so the static layout
    // runs without them.
    fp.sortMaterials = false;
    fp.splitMisses = false;
    fp.sortRays = false;
    fp.sortShadowRays = false;
    fp.overlapTraces = false;  // the second stream and its events are pass-owned objects
    // The event counters start at zero; the queue counts are cleared per wave.
    cudaError_t e = cudaMemsetAsync(scratch, 0, kHeaderBytes, st);
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, cudaGetErrorString(e));
    WavefrontBuffers view;
    view.view(static_cast<char*>(scratch) + kHeaderBytes, kNoAllocPaths);
    e = launch_path_tracer_wavefront(pass->scene->dev, fp, view, st);
    view.base = nullptr;  // the view never frees the static array
    if (e != cudaSuccess) return set_error(FPT_ERR_CUDA, std::string("PathTracer (no-alloc): ") + cudaGetErrorString(e));
    pass->frameCount++;
    return FPT_OK;
}

}  // extern "C"
