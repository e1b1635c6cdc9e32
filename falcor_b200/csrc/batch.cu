// batch.cu -- batched uneven forward rendering: many PathTracer requests
// (each its own scene, resolution, sample count, bounce limit and seed)
// rendered by one CUDA graph of wavefront launches whose waves pack whole
// pixel tiles of several requests, next to the plain per-request launches it
// is compared with.  No reference counterpart: the reference renders one
// render-graph execution per request.
//
// Each request is split into frames of at most 16 samples per pixel (the
// PathTracer's kMaxSamplesPerPixel, PathTracer/Params.slang:37); frame f uses
// the fixed seed request.seed * 64 + f and its image is weighted by its
// sample count.  Both launch modes evaluate exactly the same frames with the
// same kernel parameters (built by the PathTracer property code), so their
// images agree bit for bit.
#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "kernels.cuh"
#include "passes.h"
#include "scene_device.h"
#include "wavefront.h"

using namespace fpt;

namespace {

constexpr uint32_t kFrameSpp = 16;

__global__ void batch_average(const float4* const* frames, const float* weights, uint32_t count, float4* out, uint32_t pixels) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < pixels; i += gridDim.x * blockDim.x) {
        float3 c = make_float3(0.f, 0.f, 0.f);
        for (uint32_t f = 0; f < count; f++) {
            const float4 v = frames[f][i];
            c.x += v.x * weights[f];
            c.y += v.y * weights[f];
            c.z += v.z * weights[f];
        }
        out[i] = make_float4(c.x, c.y, c.z, 1.f);
    }
}

}  // namespace

struct fpt_batch {
    struct Request {
        fpt_batch_request r;
        uint32_t firstFrame = 0, frameCount = 0;
        uint4* vbuffer = nullptr;            // batch-owned V-buffer
        std::vector<float4*> frameColors;    // batch-owned when frameCount > 1
        float4** frameColorsDev = nullptr;
        float* weightsDev = nullptr;
    };
    std::vector<Request> reqs;
    std::vector<FrameParams> frames;         // one per frame (PathTracer kernel parameters)
    std::vector<uint32_t> frameReq;          // frame -> request
    fpt_pass* ptDefaults = nullptr;          // PathTracer pass holding the property defaults
    // tuning
    uint32_t capacity = 1u << 24;
    int shadeScale = 1;
    uint32_t fetchChunk = 0;                 // 0: the kernels' default
    bool tuned = false;
    // device state of the batched launch
    DevScene* scenesDev = nullptr;           // one per frame
    FrameParams* framesDev = nullptr;
    BatchTile* tilesDev = nullptr;
    uint32_t* slotTile = nullptr;
    unsigned long long* counters = nullptr;
    std::vector<BatchWave> waves;
    WavefrontBuffers wb;
    bool uniformSG = false, hasT = false;
    bool built = false;
    // graph
    cudaStream_t capStream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    uint32_t launchesPerRun = 0;
    // sequential baseline
    WavefrontBuffers seqWb;

    void free_device() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        cudaFree(scenesDev);
        cudaFree(framesDev);
        cudaFree(tilesDev);
        cudaFree(slotTile);
        scenesDev = nullptr;
        framesDev = nullptr;
        tilesDev = nullptr;
        slotTile = nullptr;
        built = false;
    }
    ~fpt_batch() {
        free_device();
        for (auto& q : reqs) {
            cudaFree(q.vbuffer);
            for (float4* c : q.frameColors) cudaFree(c);
            cudaFree(q.frameColorsDev);
            cudaFree(q.weightsDev);
        }
        cudaFree(counters);
        if (capStream) cudaStreamDestroy(capStream);
        if (ptDefaults) fpt_pass_destroy(ptDefaults);
    }
};

namespace {

fpt_status cuda_fail(const char* what, cudaError_t e) {
    return set_error(FPT_ERR_CUDA, std::string("fpt_batch: ") + what + ": " + cudaGetErrorString(e));
}

// Tiles every frame into whole-pixel tiles of at most `capacity` paths and
// packs them, in frame order, into waves of at most `capacity` paths.
void build_waves(fpt_batch& b, std::vector<BatchTile>& tiles) {
    tiles.clear();
    b.waves.clear();
    BatchWave cur{0, 0, 0, 0, 0};
    auto flush = [&]() {
        if (cur.tileCount) b.waves.push_back(cur);
        cur = BatchWave{uint32_t(tiles.size()), 0, 0, 0, 0};
    };
    for (uint32_t f = 0; f < b.frames.size(); f++) {
        const FrameParams& fp = b.frames[f];
        const uint32_t pixels = fp.width * fp.height;
        for (uint32_t p0 = 0; p0 < pixels;) {
            uint32_t room = (b.capacity - cur.paths) / fp.spp;
            if (room == 0) {
                flush();
                room = b.capacity / fp.spp;  // >= 1: capacity >= 16 >= spp
            }
            const uint32_t n = std::min(room, pixels - p0);
            tiles.push_back(BatchTile{f, p0, n, cur.paths, cur.pixels, fp.spp});
            cur.tileCount++;
            cur.paths += n * fp.spp;
            cur.pixels += n;
            cur.maxIter = std::max(cur.maxIter, fp.maxSurfaceBounces + 2);
            p0 += n;
        }
    }
    flush();
}

fpt_status build_batch(fpt_batch& b, cudaStream_t st) {
    b.free_device();
    std::vector<DevScene> scenes(b.frames.size());
    b.hasT = false;
    for (uint32_t f = 0; f < b.frames.size(); f++) {
        scenes[f] = b.reqs[b.frameReq[f]].r.scene->dev;
        b.hasT |= scenes[f].hasTransmission != 0;
    }
    std::vector<BatchTile> tiles;
    build_waves(b, tiles);
    cudaError_t e;
    if ((e = cudaMalloc(&b.scenesDev, scenes.size() * sizeof(DevScene))) != cudaSuccess) return cuda_fail("alloc", e);
    if ((e = cudaMalloc(&b.framesDev, b.frames.size() * sizeof(FrameParams))) != cudaSuccess) return cuda_fail("alloc", e);
    if ((e = cudaMalloc(&b.tilesDev, std::max<size_t>(1, tiles.size()) * sizeof(BatchTile))) != cudaSuccess) return cuda_fail("alloc", e);
    if ((e = cudaMalloc(&b.slotTile, size_t(b.capacity) * sizeof(uint32_t))) != cudaSuccess) return cuda_fail("alloc", e);
    cudaMemcpy(b.scenesDev, scenes.data(), scenes.size() * sizeof(DevScene), cudaMemcpyHostToDevice);
    cudaMemcpy(b.framesDev, b.frames.data(), b.frames.size() * sizeof(FrameParams), cudaMemcpyHostToDevice);
    if (!tiles.empty()) cudaMemcpy(b.tilesDev, tiles.data(), tiles.size() * sizeof(BatchTile), cudaMemcpyHostToDevice);
    if ((e = b.wb.ensure(b.capacity)) != cudaSuccess) return cuda_fail("wavefront buffers", e);
    // overlapTraces (the requests' PathTracer property): the visibility rays'
    // stream exists before the capture starts; without it the traversals stay
    // sequential.
    bool overlap = false;
    for (const FrameParams& f : b.frames) overlap = overlap || f.overlapTraces != 0;
    if (overlap && b.wb.ensure_aux() != cudaSuccess) cudaGetLastError();
    if (!overlap) b.wb.release_aux();
    if (!b.capStream && (e = cudaStreamCreateWithFlags(&b.capStream, cudaStreamNonBlocking)) != cudaSuccess)
        return cuda_fail("stream", e);
    // Capture V-buffers, all waves and the frame averaging in one graph.
    BatchDevice bd;
    bd.scenes = b.scenesDev;
    bd.frames = b.framesDev;
    bd.tiles = b.tilesDev;
    bd.slotTile = b.slotTile;
    bd.counters = b.counters;
    bd.fetchChunk = b.fetchChunk;
    uint32_t launches = 0;
    if ((e = cudaStreamBeginCapture(b.capStream, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) return cuda_fail("capture", e);
    cudaError_t le = cudaSuccess;
    for (auto& q : b.reqs) {  // one V-buffer per request
        if (le != cudaSuccess) break;
        FrameParams vp = b.frames[q.firstFrame];
        vp.vbufferOut = q.vbuffer;
        le = launch_vbuffer(q.r.scene->dev, vp, b.capStream);
        launches++;
    }
    if (le == cudaSuccess) {
        uint32_t wl = 0;
        le = launch_batch_wavefront(bd, b.waves, b.uniformSG, b.hasT, b.wb, b.shadeScale, b.capStream, wl);
        launches += wl;
    }
    for (auto& q : b.reqs) {
        if (le != cudaSuccess || q.frameCount <= 1) continue;
        const uint32_t pixels = q.r.width * q.r.height;
        batch_average<<<std::min<uint32_t>((pixels + 255) / 256, 4096), 256, 0, b.capStream>>>(
            q.frameColorsDev, q.weightsDev, q.frameCount, reinterpret_cast<float4*>(q.r.color), pixels);
        launches++;
    }
    e = cudaStreamEndCapture(b.capStream, &b.graph);
    if (le != cudaSuccess) return cuda_fail("launch during capture", le);
    if (e != cudaSuccess) return cuda_fail("end capture", e);
    if ((e = cudaGraphInstantiate(&b.exec, b.graph, 0)) != cudaSuccess) return cuda_fail("graph instantiate", e);
    b.launchesPerRun = launches;
    b.built = true;
    (void)st;
    return FPT_OK;
}

fpt_status run_batched(fpt_batch& b, cudaStream_t st) {
    if (!b.built) {
        fpt_status s = build_batch(b, st);
        if (s != FPT_OK) return s;
    }
    cudaError_t e = cudaMemsetAsync(b.counters, 0, kNumCounters * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return cuda_fail("memset", e);
    if ((e = cudaGraphLaunch(b.exec, st)) != cudaSuccess) return cuda_fail("graph launch", e);
    return FPT_OK;
}

}  // namespace

extern "C" {

FPT_API fpt_status fpt_batch_create(fpt_batch** out) {
    if (!out) return set_error(FPT_ERR_INVALID_ARG, "fpt_batch_create: null argument");
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return set_error(FPT_ERR_NO_DEVICE, "fpt_batch_create: no CUDA device");
    auto* b = new fpt_batch();
    fpt_status s = fpt_pass_create("PathTracer", &b->ptDefaults);
    if (s != FPT_OK) { delete b; return s; }
    if (cudaMalloc(&b->counters, kNumCounters * sizeof(unsigned long long)) != cudaSuccess) {
        delete b;
        return set_error(FPT_ERR_OOM, "fpt_batch_create: out of device memory");
    }
    *out = b;
    return FPT_OK;
}

FPT_API void fpt_batch_destroy(fpt_batch* batch) { delete batch; }

FPT_API fpt_status fpt_batch_add(fpt_batch* b, const fpt_batch_request* req) {
    if (!b || !req || !req->scene || !req->color) return set_error(FPT_ERR_INVALID_ARG, "fpt_batch_add: null argument");
    if (req->width == 0 || req->height == 0 || req->width > 4096 || req->height > 4096 || req->spp == 0)
        return set_error(FPT_ERR_INVALID_ARG, "fpt_batch_add: invalid resolution or sample count");
    fpt_batch::Request q;
    q.r = *req;
    q.firstFrame = uint32_t(b->frames.size());
    q.frameCount = (req->spp + kFrameSpp - 1) / kFrameSpp;
    const size_t pixels = size_t(req->width) * req->height;
    if (cudaMalloc(&q.vbuffer, pixels * sizeof(uint4)) != cudaSuccess) return set_error(FPT_ERR_OOM, "fpt_batch_add: out of device memory");
    std::vector<float> weights;
    for (uint32_t f = 0; f < q.frameCount; f++) {
        const uint32_t spp = std::min(kFrameSpp, req->spp - f * kFrameSpp);
        fpt_pass& pt = *b->ptDefaults;
        pt.props["samplesPerPixel"] = PropValue::num(spp);
        pt.props["maxSurfaceBounces"] = PropValue::num(req->max_bounces);
        pt.props["maxDiffuseBounces"] = PropValue::num(req->max_bounces);
        pt.props["maxSpecularBounces"] = PropValue::num(req->max_bounces);
        pt.explicitKeys.insert({"maxSurfaceBounces", "maxDiffuseBounces", "maxSpecularBounces"});
        pt.props["emissiveSampler"] = PropValue::str("Power");
        pt.props["fixedSeed"] = PropValue::num(double(req->seed) * 64.0 + f);
        pt.useFixedSeed = true;
        FrameParams fp;
        std::memset(&fp, 0, sizeof(fp));
        path_tracer_params(pt, fp);
        fp.width = req->width;
        fp.height = req->height;
        fp.vbuffer = q.vbuffer;
        fp.counters = b->counters;
        fp.workItems = uint32_t(pixels);
        float4* color = reinterpret_cast<float4*>(req->color);
        if (q.frameCount > 1) {
            if (cudaMalloc(&color, pixels * sizeof(float4)) != cudaSuccess) return set_error(FPT_ERR_OOM, "fpt_batch_add: out of device memory");
            q.frameColors.push_back(color);
        }
        fp.color = color;
        weights.push_back(float(spp) / float(req->spp));
        b->uniformSG = fp.sampleGenerator == 1;
        b->frames.push_back(fp);
        b->frameReq.push_back(uint32_t(b->reqs.size()));
    }
    if (q.frameCount > 1) {
        if (cudaMalloc(&q.frameColorsDev, q.frameCount * sizeof(float4*)) != cudaSuccess ||
            cudaMalloc(&q.weightsDev, q.frameCount * sizeof(float)) != cudaSuccess)
            return set_error(FPT_ERR_OOM, "fpt_batch_add: out of device memory");
        cudaMemcpy(q.frameColorsDev, q.frameColors.data(), q.frameCount * sizeof(float4*), cudaMemcpyHostToDevice);
        cudaMemcpy(q.weightsDev, weights.data(), q.frameCount * sizeof(float), cudaMemcpyHostToDevice);
    }
    b->reqs.push_back(q);
    b->free_device();
    return FPT_OK;
}

FPT_API fpt_status fpt_batch_set_tuning(fpt_batch* b, uint32_t wave_capacity, uint32_t shade_grid_scale) {
    if (!b) return set_error(FPT_ERR_INVALID_ARG, "fpt_batch_set_tuning: null batch");
    if (wave_capacity) b->capacity = std::max<uint32_t>(wave_capacity, kFrameSpp);
    if (shade_grid_scale) b->shadeScale = int(std::min<uint32_t>(shade_grid_scale, 8));
    b->free_device();
    return FPT_OK;
}

FPT_API fpt_status fpt_batch_get_tuning(const fpt_batch* b, uint32_t* wave_capacity, uint32_t* shade_grid_scale) {
    if (!b) return set_error(FPT_ERR_INVALID_ARG, "fpt_batch_get_tuning: null batch");
    if (wave_capacity) *wave_capacity = b->capacity;
    if (shade_grid_scale) *shade_grid_scale = uint32_t(b->shadeScale);
    return FPT_OK;
}

FPT_API fpt_status fpt_batch_set_tuning_ex(fpt_batch* b, const fpt_batch_tuning* t) {
    if (!b || !t) return set_error(FPT_ERR_INVALID_ARG, "fpt_batch_set_tuning_ex: null argument");
    if (t->fetch_chunk && (t->fetch_chunk > 1024 || (t->fetch_chunk & 31u)))
        return set_error(FPT_ERR_INVALID_ARG, "fpt_batch_set_tuning_ex: fetch_chunk must be a multiple of 32 up to 1024");
    if (t->wave_capacity) b->capacity = std::max<uint32_t>(t->wave_capacity, kFrameSpp);
    if (t->shade_grid_scale) b->shadeScale = int(std::min<uint32_t>(t->shade_grid_scale, 8));
    b->fetchChunk = t->fetch_chunk;
    b->free_device();
    return FPT_OK;
}

FPT_API fpt_status fpt_batch_get_tuning_ex(const fpt_batch* b, fpt_batch_tuning* t) {
    if (!b || !t) return set_error(FPT_ERR_INVALID_ARG, "fpt_batch_get_tuning_ex: null argument");
    t->wave_capacity = b->capacity;
    t->shade_grid_scale = uint32_t(b->shadeScale);
    t->fetch_chunk = b->fetchChunk ? b->fetchChunk : 32u;
    return FPT_OK;
}

FPT_API fpt_status fpt_batch_autotune(fpt_batch* b, void* stream) {
    if (!b || b->reqs.empty()) return set_error(FPT_ERR_INVALID_ARG, "fpt_batch_autotune: empty batch");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const uint32_t caps[] = {1u << 21, 1u << 22, 1u << 23, 1u << 24, 1u << 25};
    const int scales[] = {1, 2};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    uint32_t bestCap = b->capacity;
    int bestScale = b->shadeScale;
    for (uint32_t cap : caps) {
        for (int sc : scales) {
            b->capacity = cap;
            b->shadeScale = sc;
            b->free_device();
            fpt_status s = run_batched(*b, st);  // builds and warms up
            if (s != FPT_OK) { cudaEventDestroy(e0); cudaEventDestroy(e1); return s; }
            cudaEventRecord(e0, st);
            for (int r = 0; r < 2 && s == FPT_OK; r++) s = run_batched(*b, st);
            cudaEventRecord(e1, st);
            cudaEventSynchronize(e1);
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (s == FPT_OK && ms < best) { best = ms; bestCap = cap; bestScale = sc; }
        }
    }
    // Then the queue depth per warp claim at the best capacity and grid.
    b->capacity = bestCap;
    b->shadeScale = bestScale;
    uint32_t bestChunk = b->fetchChunk;
    for (uint32_t chunk : {32u, 64u, 128u}) {
        b->fetchChunk = chunk;
        b->free_device();
        fpt_status s = run_batched(*b, st);
        if (s != FPT_OK) { cudaEventDestroy(e0); cudaEventDestroy(e1); return s; }
        cudaEventRecord(e0, st);
        for (int r = 0; r < 2 && s == FPT_OK; r++) s = run_batched(*b, st);
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (s == FPT_OK && ms < best) { best = ms; bestChunk = chunk; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->fetchChunk = bestChunk;
    b->free_device();
    b->tuned = true;
    return FPT_OK;
}

FPT_API fpt_status fpt_batch_launch(fpt_batch* b, void* stream) {
    if (!b || b->reqs.empty()) return set_error(FPT_ERR_INVALID_ARG, "fpt_batch_launch: empty batch");
    return run_batched(*b, static_cast<cudaStream_t>(stream));
}

FPT_API fpt_status fpt_batch_launch_sequential(fpt_batch* b, void* stream) {
    if (!b || b->reqs.empty()) return set_error(FPT_ERR_INVALID_ARG, "fpt_batch_launch_sequential: empty batch");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(b->counters, 0, kNumCounters * sizeof(unsigned long long), st);
    if (e != cudaSuccess) return cuda_fail("memset", e);
    // One plain launch per request: VBufferRT, then the PathTracer wavefront per frame.
    if ((e = b->seqWb.ensure(b->capacity)) != cudaSuccess) return cuda_fail("wavefront buffers", e);
    for (auto& q : b->reqs) {
        FrameParams vp = b->frames[q.firstFrame];
        vp.vbufferOut = q.vbuffer;
        if ((e = launch_vbuffer(q.r.scene->dev, vp, st)) != cudaSuccess) return cuda_fail("vbuffer", e);
        for (uint32_t f = q.firstFrame; f < q.firstFrame + q.frameCount; f++)
            if ((e = launch_path_tracer_wavefront(q.r.scene->dev, b->frames[f], b->seqWb, st)) != cudaSuccess) return cuda_fail("path tracer", e);
        if (q.frameCount > 1) {
            const uint32_t pixels = q.r.width * q.r.height;
            batch_average<<<std::min<uint32_t>((pixels + 255) / 256, 4096), 256, 0, st>>>(
                q.frameColorsDev, q.weightsDev, q.frameCount, reinterpret_cast<float4*>(q.r.color), pixels);
        }
    }
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail("launch", e);
    return FPT_OK;
}

FPT_API fpt_status fpt_batch_get_stats(fpt_batch* b, fpt_pass_stats* out, void* stream) {
    if (!b || !out) return set_error(FPT_ERR_INVALID_ARG, "fpt_batch_get_stats: null argument");
    std::memset(out, 0, sizeof(*out));
    unsigned long long c[2] = {0, 0};
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaMemcpyAsync(c, b->counters, sizeof(c), cudaMemcpyDeviceToHost, st);
    cudaStreamSynchronize(st);
    out->paths = c[0];
    out->rays = c[1];
    uint32_t err = 0;
    for (auto& q : b->reqs) {
        uint32_t w = 0;
        cudaMemcpy(&w, q.r.scene->dev.errorWord, 4, cudaMemcpyDeviceToHost);
        err |= w;
    }
    out->device_error = err;
    out->kernel_launches = b->launchesPerRun;
    return FPT_OK;
}

}  // extern "C"
