// batch.cu -- batched uneven forward rendering (persistent launch).
#include "kernels.cuh"
#include "passes.h"
#include "scene_device.h"

using namespace fpt;

extern "C" {
FPT_API fpt_status fpt_batch_create(fpt_batch** out) {
    if (out) *out = nullptr;
    return set_error(FPT_ERR_UNSUPPORTED, "fpt_batch_create: not available in this build");
}
FPT_API void fpt_batch_destroy(fpt_batch*) {}
FPT_API fpt_status fpt_batch_add(fpt_batch*, const fpt_batch_request*) { return set_error(FPT_ERR_UNSUPPORTED, "batch"); }
FPT_API fpt_status fpt_batch_set_tuning(fpt_batch*, uint32_t, uint32_t) { return set_error(FPT_ERR_UNSUPPORTED, "batch"); }
FPT_API fpt_status fpt_batch_autotune(fpt_batch*, void*) { return set_error(FPT_ERR_UNSUPPORTED, "batch"); }
FPT_API fpt_status fpt_batch_launch(fpt_batch*, void*) { return set_error(FPT_ERR_UNSUPPORTED, "batch"); }
FPT_API fpt_status fpt_batch_launch_sequential(fpt_batch*, void*) { return set_error(FPT_ERR_UNSUPPORTED, "batch"); }
FPT_API fpt_status fpt_batch_get_stats(fpt_batch*, fpt_pass_stats*, void*) { return set_error(FPT_ERR_UNSUPPORTED, "batch"); }
}
