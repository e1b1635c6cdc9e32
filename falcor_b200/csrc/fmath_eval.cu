// fmath_eval.cu -- evaluates the path's elementary functions on device arrays:
// the deterministic single-precision implementations the kernels use
// (fmath.h), or CUDA's own functions for comparison.  A test hook of the
// C-ABI; nothing on the rendering path calls it.
#include <cuda_runtime.h>

#include <string>

#include "common.h"
#include "fmath.h"

namespace {

__global__ void fmath_kernel(uint32_t fn, uint32_t cudaLibm, uint32_t n, const float* __restrict__ x,
                             const float* __restrict__ y, float* __restrict__ out) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float a = x[i];
        const float b = y ? y[i] : 0.f;
        float r = 0.f;
        if (cudaLibm) {
            switch (fn) {
                case FPT_FMATH_SIN: r = sinf(a); break;
                case FPT_FMATH_COS: r = cosf(a); break;
                case FPT_FMATH_ATAN2: r = atan2f(a, b); break;
                case FPT_FMATH_ACOS: r = acosf(a); break;
                case FPT_FMATH_EXP: r = expf(a); break;
                case FPT_FMATH_LOG: r = logf(a); break;
                case FPT_FMATH_LOG2: r = log2f(a); break;
                case FPT_FMATH_EXP2: r = exp2f(a); break;
                default: r = powf(a, b); break;
            }
        } else {
            switch (fn) {
                case FPT_FMATH_SIN: r = fm::sin(a); break;
                case FPT_FMATH_COS: r = fm::cos(a); break;
                case FPT_FMATH_ATAN2: r = fm::atan2(a, b); break;
                case FPT_FMATH_ACOS: r = fm::acos(a); break;
                case FPT_FMATH_EXP: r = fm::exp(a); break;
                case FPT_FMATH_LOG: r = fm::log(a); break;
                case FPT_FMATH_LOG2: r = fm::log2(a); break;
                case FPT_FMATH_EXP2: r = fm::exp2(a); break;
                default: r = fm::pow(a, b); break;
            }
        }
        out[i] = r;
    }
}

}  // namespace

extern "C" {

FPT_API fpt_status fpt_fmath_eval(uint32_t fn, uint32_t cuda_libm, uint32_t n, const float* x, const float* y, float* out,
                                  void* stream) {
    if (fn > FPT_FMATH_POW) return fpt::set_error(FPT_ERR_INVALID_ARG, "fpt_fmath_eval: unknown function");
    if (n == 0) return FPT_OK;
    if (!x || !out) return fpt::set_error(FPT_ERR_INVALID_ARG, "fpt_fmath_eval: null array");
    if ((fn == FPT_FMATH_ATAN2 || fn == FPT_FMATH_POW) && !y)
        return fpt::set_error(FPT_ERR_INVALID_ARG, "fpt_fmath_eval: atan2 and pow take two arrays");
    const uint32_t block = 256;
    const uint32_t grid = (n + block - 1) / block < 148u * 16u ? (n + block - 1) / block : 148u * 16u;
    fmath_kernel<<<grid, block, 0, static_cast<cudaStream_t>(stream)>>>(fn, cuda_libm, n, x, y, out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fpt::set_error(FPT_ERR_CUDA, std::string("fpt_fmath_eval: ") + cudaGetErrorString(e));
    return FPT_OK;
}

}  // extern "C"
