// image_passes.h -- AccumulatePass, ToneMapper, ColorMapPass and
// RenderToViewportPass (image_passes.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <string>

#include "common.h"

struct fpt_pass;

namespace fpt {

// ToneMapper parameters: the colour transform (white balance x exposure, row
// major), the ToneMapperOperator (Linear, Reinhard, ReinhardModified,
// HejiHableAlu, HableUc2, Aces) and the switches.
struct ToneMapArgs {
    float m[9];
    float whiteScale, whiteMaxLuminance;
    uint32_t lumTexels;  // texels of the luminance target (auto exposure)
    int op;
    bool clamp, autoExposure;
};

// Enum-valued properties (ToneMapperOperator, ColorMap, AccumulatePass::Precision
// and OverflowMode), in the reference's enum order.
const std::map<std::string, int> kToneMapOperators = {{"Linear", 0}, {"Reinhard", 1}, {"ReinhardModified", 2},
                                                      {"HejiHableAlu", 3}, {"HableUc2", 4}, {"Aces", 5}};
const std::map<std::string, int> kToneMapExposureModes = {{"AperturePriority", 0}, {"ShutterPriority", 1}};
const std::map<std::string, int> kColorMaps = {{"Grey", 0}, {"Jet", 1}, {"Viridis", 2}, {"Plasma", 3}, {"Magma", 4}, {"Inferno", 5}};
const std::map<std::string, int> kPrecisionModes = {{"Double", 0}, {"Single", 1}, {"SingleCompensated", 2}};
const std::map<std::string, int> kOverflowModes = {{"Stop", 0}, {"Reset", 1}, {"EMA", 2}};

// precision: 0 Double, 1 Single, 2 SingleCompensated.  sum: double[4 n] for
// Double, float4[n] otherwise; corr: float4[n] for SingleCompensated.
cudaError_t launch_accumulate(int precision, const float4* cur, float4* out, void* sum, float4* corr, uint32_t n, uint32_t count,
                              bool accumulate, bool ema, cudaStream_t st);
cudaError_t launch_blit(const float4* src, uint32_t sw, uint32_t sh, float4* dst, uint32_t dw, uint32_t dh, cudaStream_t st);
// scratch: 1 + 148 doubles (auto exposure).
cudaError_t launch_tone_map(const float4* src, uint32_t sw, uint32_t sh, float4* dst, uint32_t dw, uint32_t dh, ToneMapArgs a,
                            double* scratch, cudaStream_t st);
// The ToneMapper colour transform of the pass's current properties (row major).
void tone_map_color_transform(const fpt_pass& p, float m[9]);
// execute() of the four image pass types.
fpt_status image_pass_execute(fpt_pass& p, const fpt_frame_io* io, cudaStream_t st);

}  // namespace fpt
