// host_scene.cpp -- host-side scene tools of the C-ABI: procedural synthetic
// scenes (the benchmark workloads, defined in procedural.h), camera vectors
// and HitInfo bit allocation.  No CUDA here: these run on any machine.
#include <string>

#include "common.h"
#include "procedural.h"

using namespace fpt;

extern "C" {

FPT_API fpt_status fpt_procedural_scene(const fpt_procedural_params* params, fpt_scene_host** out) {
    if (!params || !out) return set_error(FPT_ERR_INVALID_ARG, "fpt_procedural_scene: null argument");
    try {
        *out = build_procedural_scene(*params);
        return FPT_OK;
    } catch (const std::invalid_argument& e) {
        return set_error(FPT_ERR_INVALID_ARG, std::string("fpt_procedural_scene: ") + e.what());
    } catch (const std::exception& e) {
        return set_error(FPT_ERR_OOM, std::string("fpt_procedural_scene: ") + e.what());
    }
}

FPT_API const fpt_scene_desc* fpt_scene_host_desc(const fpt_scene_host* h) { return h ? &h->desc : nullptr; }
FPT_API void fpt_scene_host_free(fpt_scene_host* h) { delete h; }

FPT_API fpt_status fpt_camera_compute(const fpt_camera* cam, fpt_camera_data* out) {
    if (!cam || !out) return set_error(FPT_ERR_INVALID_ARG, "fpt_camera_compute: null argument");
    compute_camera(*cam, *out);
    return FPT_OK;
}

FPT_API fpt_status fpt_hitinfo_compute_bits(const fpt_scene_desc* desc, fpt_hitinfo_bits* out) {
    if (!desc || !out) return set_error(FPT_ERR_INVALID_ARG, "fpt_hitinfo_compute_bits: null argument");
    *out = compute_hit_bits(*desc);
    return FPT_OK;
}

}  // extern "C"
