// Stand-in for Falcor's DiffRendering/SceneGradients.h
// (Source/Falcor/DiffRendering/SceneGradients.h) over the oracle's
// restatement (oracle/oracle_gradients.h), so that the reference's
// Tests/DiffRendering/SceneGradientsTest.cpp compiles on the CPU.
//
// TEST INFRASTRUCTURE ONLY.
#pragma once

#include <memory>
#include <vector>

#include "Testing/UnitTest.h"
#include "oracle_gradients.h"

namespace Falcor {

enum class GradientType : uint32_t { Material, MeshPosition, MeshNormal, MeshTangent, Count };

class SceneGradients {
public:
    struct GradConfig {
        GradientType type = GradientType::Material;
        uint32_t dim = 0;
        uint32_t hashSize = 0;
        GradConfig() {}
        GradConfig(GradientType t, uint32_t d, uint32_t h) : type(t), dim(d), hashSize(h) {}
    };
    SceneGradients(ref<Device>, const std::vector<GradConfig>& configs) {
        for (const GradConfig& c : configs) impl.configure(uint32_t(c.type), c.dim, c.hashSize);
        for (int t = 0; t < orc::SceneGradientsOracle::kTypes; t++) {
            grads[t] = std::make_shared<Buffer>();
            grads[t]->elementSize = 4;
        }
    }
    // The fake program reaches the oracle object through the context.
    void bindShaderData(const ShaderVar& var) const { var.ctx->blocks[var.name] = &impl; }
    void clearGrads(RenderContext*, GradientType t) { impl.clear(uint32_t(t)); sync(t); }
    void aggregateGrads(RenderContext*, GradientType t) { impl.aggregate(uint32_t(t)); sync(t); }
    const ref<Buffer>& getGradsBuffer(GradientType t) const { return grads[size_t(t)]; }

    mutable orc::SceneGradientsOracle impl;

private:
    void sync(GradientType t) {
        const auto& g = impl.e[size_t(t)].grads;
        grads[size_t(t)]->data.resize(g.size() * 4);
        if (!g.empty()) std::memcpy(grads[size_t(t)]->data.data(), g.data(), g.size() * 4);
        grads[size_t(t)]->elementCount = g.size();
    }
    ref<Buffer> grads[orc::SceneGradientsOracle::kTypes];
};

}  // namespace Falcor
