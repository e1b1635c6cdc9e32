// wardiff.h -- SceneGradients behind the fpt_scene_gradients handle
// (DiffRendering/SceneGradients.h:40-120): per gradient type a result buffer
// of `dim` floats and a scratch buffer of `dim * hash_size` floats that the
// adjoint scatters into (row = jenkinsHash(pixelID) % hash_size), summed into
// the result by fpt_scene_gradients_aggregate.
#pragma once

#include "common.h"

struct fpt_scene_gradients {
    struct Entry {
        bool active = false;
        uint32_t dim = 0, hash = 0;
        float* grads = nullptr;
        float* tmp = nullptr;
    };
    Entry e[FPT_GRAD_TYPE_COUNT];
    fpt_scene_gradients() = default;
    fpt_scene_gradients(const fpt_scene_gradients&) = delete;
    fpt_scene_gradients& operator=(const fpt_scene_gradients&) = delete;
    ~fpt_scene_gradients();
};
