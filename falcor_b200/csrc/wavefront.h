// wavefront.h -- path-state buffers and launcher of the wavefront PathTracer.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "kernels.cuh"

namespace fpt {

// Structure-of-arrays path state for `capacity` paths in flight, allocated
// once per pass and reused by every frame (scratch owned by the pass).
struct WavefrontBuffers {
    static constexpr int kFloat4Arrays = 10;
    void* base = nullptr;
    uint32_t capacity = 0;
    size_t bytesAllocated = 0;
    bool owning = true;            // false after view(): the memory belongs to someone else
    float4* arrays = nullptr;      // kFloat4Arrays x capacity float4
    float* sampleL = nullptr;      // 3 floats per path
    uint32_t* queueA = nullptr;
    uint32_t* queueB = nullptr;
    uint32_t* shadowQueue = nullptr;
    uint32_t* counts = nullptr;    // [0] shade, [1] extension, [2] shadow
    // Material sort of the shade queue (allocated on first use, owning mode
    // only): per-position keys, the sorted queue, bin counts and cursors.
    void* sortBase = nullptr;
    uint32_t sortCapacity = 0;
    uint32_t* sortKeys = nullptr;
    uint32_t* sortQueue = nullptr;
    uint32_t* sortBins = nullptr;  // kMaxSortBins counts + kMaxSortBins cursors
    uint32_t* shadowKeys = nullptr;    // visibility-ray binning: keys and the sorted queue
    uint32_t* shadowSorted = nullptr;
    static constexpr uint32_t kMaxSortBins = 1024;
    // Hit/miss split of the shade stage (owning mode only): the extension
    // kernel pushes hits and misses into separate next-bounce queues.
    void* splitBase = nullptr;
    uint32_t splitCapacity = 0;
    uint32_t* missQueue = nullptr;
    uint32_t* nextHitQueue = nullptr;
    uint32_t* nextMissQueue = nullptr;
    // overlapTraces (owning mode only): the visibility rays' stream
    // (non-blocking, created on first use on the current device) and the
    // fork / join events between it and the caller's stream.
    cudaStream_t aux = nullptr;
    cudaEvent_t forkEv = nullptr;
    cudaEvent_t joinEv = nullptr;
    int auxDevice = -1;
    float4* f4(int k) const { return arrays + size_t(k) * capacity; }
    cudaError_t ensure(uint32_t capacity);
    cudaError_t ensure_sort();
    cudaError_t ensure_split();
    cudaError_t ensure_aux();
    void release();
    void release_aux();
    ~WavefrontBuffers() { release(); release_aux(); }

    // Bytes needed for `capacity` paths in flight.
    static constexpr size_t bytes_for(uint32_t cap) {
        return kFloat4Arrays * size_t(cap) * 16 + size_t(cap) * 3 * sizeof(float) + 3 * size_t(cap) * sizeof(uint32_t) + 256;
    }
    // Lays the buffers out over `mem` (at least bytes_for(capacity) bytes,
    // 256-byte aligned) without allocating; the view never frees `mem`.
    void view(void* mem, uint32_t capacity);
};

// Kernel categories timed by KernelTimer.
// KC_TRACE (overlapTraces only): the span of a bounce's visibility and
// extension traversals, from the fork to the join of their two streams; the
// two kernels' own spans overlap inside it.
enum KernelCategory { KC_GENERATE = 0, KC_SHADE = 1, KC_SHADOW = 2, KC_EXTEND = 3, KC_RESOLVE = 4, KC_SORT = 5, KC_TRACE = 6, KC_COUNT = 7 };

// Optional CUDA-event timing of each kernel launch, by category (the
// equivalent of Falcor's FALCOR_PROFILE scopes, Utils/Timing/Profiler.h).
struct KernelTimer {
    bool enabled = false;
    std::vector<cudaEvent_t> events;   // pool, reused
    std::vector<int> pendingCat;       // category of each recorded pair
    std::vector<char> ended;           // whether each pair's end was recorded
    size_t used = 0;                   // events in use (pairs * 2)
    double ms[KC_COUNT] = {0};
    uint64_t launches[KC_COUNT] = {0};
    // begin records a pair's start on `st` and returns the pair (-1 when
    // disabled); end records its end.  Pairs may nest and may be ended on
    // another stream than the one they began on.
    int begin(int cat, cudaStream_t st);
    void end(int pair, cudaStream_t st);
    // Waits for the recorded events and folds them into ms/launches.
    cudaError_t collect();
    void reset();
    ~KernelTimer();
};

cudaError_t launch_path_tracer_wavefront(const DevScene& s, const FrameParams& p, WavefrontBuffers& b, cudaStream_t st,
                                         KernelTimer* timer = nullptr);

// Batched PathTracer: one wave holds whole pixel tiles of several requests.
// Tile t covers pixels [firstPixel, firstPixel + numPixels) of request `req`,
// all `spp` samples, at wave slots [slotOffset, slotOffset + numPixels * spp)
// (sample-major) and resolved pixels [pixelOffset, pixelOffset + numPixels).
struct BatchTile {
    uint32_t req, firstPixel, numPixels, slotOffset, pixelOffset, spp;
};
struct BatchWave {
    uint32_t firstTile, tileCount, paths, pixels, maxIter;
};
// Device arrays of a batch: per-request scenes and frame parameters, all
// tiles, and a per-slot tile index (capacity entries).
struct BatchDevice {
    const DevScene* scenes = nullptr;
    const FrameParams* frames = nullptr;
    const BatchTile* tiles = nullptr;
    uint32_t* slotTile = nullptr;
    unsigned long long* counters = nullptr;
    uint32_t fetchChunk = 0;     // trace-kernel queue entries per warp claim (0: default)
};
// Enqueues every wave of the batch (uniform sample generator type and
// transmission variant across requests); shadeScale multiplies the shade grid.
cudaError_t launch_batch_wavefront(const BatchDevice& bd, const std::vector<BatchWave>& waves, bool uniformSG, bool hasT,
                                   WavefrontBuffers& b, int shadeScale, cudaStream_t st, uint32_t& launches);

}  // namespace fpt
