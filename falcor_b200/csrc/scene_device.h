// scene_device.h -- the device scene object behind the fpt_scene handle.
#pragma once

#include <memory>
#include <vector>

#include "device_scene.cuh"

namespace fpt {

struct DeviceBuffers {
    std::vector<void*> ptrs;
    size_t bytes = 0;
    DeviceBuffers() = default;
    DeviceBuffers(const DeviceBuffers&) = delete;
    DeviceBuffers& operator=(const DeviceBuffers&) = delete;
    ~DeviceBuffers();
};

fpt_status create_scene(const fpt_scene_desc& d, fpt_scene*& out);
// baseColorTexture: 1 + texture index, or 0 for the uniform base colour.
DevMaterial pack_material(const fpt_material& m, uint32_t baseColorTexture = 0);

}  // namespace fpt

struct fpt_scene {
    fpt::DevScene dev;
    fpt::DeviceBuffers buffers;
    fpt::BVH8 bvh;                    // host copy of the acceleration structure
    std::vector<uint32_t> aliasTable; // host copy of the alias table
    std::vector<fpt_material> materials;  // host copy of the material parameters
    std::vector<uint32_t> baseColorTex;   // per material: 1 + base-colour texture index, or 0
    std::vector<fpt::DevTexture> textures; // host copy of the texture table
    fpt::LightBVH lightBvh;               // host copy of the light BVH
    float aliasWeightSum = 0.f;
    fpt_scene_info info{};
    uint64_t version = 0;             // bumped by every change that can change a path (camera, materials, vertices)
    // Bumped by the changes that restart progressive accumulation: all of the
    // above except camera jitter (AccumulatePass.cpp:150-168).
    uint64_t resetVersion = 0;
    // Per mesh (= geometry instance): vertex and triangle counts, emissive flag.
    std::vector<uint32_t> meshVertexCount, meshTriCount;
    std::vector<uint8_t> meshEmissive;
    // BVH refit after vertex updates: node index range of each tree level
    // (breadth-first order), a node-box buffer and a device status word.
    std::vector<uint32_t> levelStart;
    float* nodeBoxes = nullptr;
    uint32_t* refitStatus = nullptr;
    // Material parameters last written on the device (fpt_scene_set_material_params_device):
    // the host copy is refreshed from the device before it is read.
    bool materialsOnDevice = false;
    uint32_t* materialIds = nullptr;     // device copy of the IDs of a device-side update
    uint32_t materialIdCapacity = 0;
};
