// oracle_gradients.h -- CPU restatement of SceneGradients: hashed scratch
// gradients and their aggregation (DiffRendering/SceneGradients.slang:50-57,
// SceneGradients.cpp:42-135, AggregateGradients.cs.slang:50-73).
//
// TEST INFRASTRUCTURE ONLY: the checker of the CUDA gradient accumulation and
// the stand-in for the reference's SceneGradients in its own unit test.
#pragma once

#include <algorithm>
#include <cstdint>
#include <vector>

namespace orc {

struct SceneGradientsOracle {
    static constexpr int kTypes = 4;  // GradientType::Material .. MeshTangent (SharedTypes.slang:53-60)
    struct Entry {
        bool active = false;
        uint32_t dim = 0, hashSize = 0;
        std::vector<float> tmp;    // hashSize rows of dim floats
        std::vector<float> grads;  // dim floats
    };
    Entry e[kTypes];

    void configure(uint32_t type, uint32_t dim, uint32_t hashSize) {
        Entry& x = e[type];
        x.active = true;
        x.dim = dim;
        x.hashSize = hashSize;
        x.tmp.assign(size_t(dim) * hashSize, 0.f);
        x.grads.assign(dim, 0.f);
    }
    // atomicAddGrad: ignored beyond the dimension.
    void atomic_add(uint32_t type, uint32_t gradIndex, uint32_t hashIndex, float value) {
        Entry& x = e[type];
        if (gradIndex < x.dim) x.tmp[size_t(hashIndex) * x.dim + gradIndex] += value;
    }
    // clearGrads: zero scratch and result.
    void clear(uint32_t type) {
        Entry& x = e[type];
        if (!x.active) return;
        std::fill(x.tmp.begin(), x.tmp.end(), 0.f);
        std::fill(x.grads.begin(), x.grads.end(), 0.f);
    }
    // aggregateGrads in the default HashGrid mode: every scratch row added into
    // the result (rows in order; the reference adds them with float atomics).
    void aggregate(uint32_t type) {
        Entry& x = e[type];
        if (!x.active) return;
        for (uint32_t h = 0; h < x.hashSize; h++)
            for (uint32_t i = 0; i < x.dim; i++) x.grads[i] += x.tmp[size_t(h) * x.dim + i];
    }
};

}  // namespace orc
