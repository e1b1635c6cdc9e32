// adjoint.cu -- WARDiffPathTracer primal and adjoint.
#include "kernels.cuh"
#include "passes.h"
#include "scene_device.h"

namespace fpt {

fpt_status wardiff_execute(fpt_pass& p, const fpt_frame_io* io, const float* dLdI, const fpt_grad_buffers* grads,
                           cudaStream_t st) {
    (void)p; (void)io; (void)dLdI; (void)grads; (void)st;
    return set_error(FPT_ERR_UNSUPPORTED, "WARDiffPathTracer: not available in this build");
}

}  // namespace fpt
