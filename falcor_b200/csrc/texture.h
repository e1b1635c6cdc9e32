// texture.h -- the StandardMaterial base-colour texture lookup, shared by the
// kernels and the CPU oracle so that both evaluate the same FP32 operations.
//
// The PathTracer's default texture LOD mode (TexLODMode::Mip0) samples every
// material texture with ExplicitLodTextureSampler(0) (PathTracer.slang:799-814)
// through MaterialSystem::sampleTexture (MaterialSystem.slang:308-320): a
// bilinear SampleLevel at mip 0 with the material sampler's wrap addressing.
// The texture unit filters RGBA8 texels after decoding them (sRGB formats
// decode rgb to linear first); here the filter runs in FP32 in software with
// exact weights, and the sRGB decode is a 256-entry table computed in double.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define FPT_TEX_HD __host__ __device__ __forceinline__
#else
#define FPT_TEX_HD inline
#endif

namespace fpt_tex {

enum Format : uint32_t { kRGBA8Srgb = 0, kRGBA8Unorm = 1, kRGBA32Float = 2 };

FPT_TEX_HD uint32_t texel_bytes(uint32_t format) { return format == kRGBA32Float ? 16u : 4u; }

// IEC 61966-2-1 sRGB to linear of the 8-bit code i (the decode of the
// RGBA8UnormSrgb formats), rounded once from double.
inline void srgb_decode_table(float (&lut)[256]) {
    for (int i = 0; i < 256; i++) {
        const double c = double(i) / 255.0;
        const double l = c <= 0.04045 ? c / 12.92 : std::pow((c + 0.055) / 1.055, 2.4);
        lut[i] = float(l);
    }
}

// UNORM8 to float (D3D/Vulkan: c / 255, correctly rounded).
FPT_TEX_HD float unorm8(uint32_t c) { return float(c) / 255.f; }

// Texel coordinates and weights of one bilinear lookup at mip 0 with wrap
// addressing: texel centres at (i + 0.5) / size, weights (1 - ax, ax) x
// (1 - ay, ay) on (x0, x1) x (y0, y1).  Non-finite or huge coordinates
// (|u * size| >= 1e9) fall back to texel 0.
struct Bilinear {
    uint32_t x0, x1, y0, y1;
    float w[4];  // (x0, y0), (x1, y0), (x0, y1), (x1, y1)
};

FPT_TEX_HD uint32_t wrap_index(float f, uint32_t n) {
    const long long i = (long long)f % (long long)n;
    return uint32_t(i < 0 ? i + (long long)n : i);
}

FPT_TEX_HD Bilinear bilinear(float u, float v, uint32_t W, uint32_t H) {
    float fx = u * float(W) - 0.5f, fy = v * float(H) - 0.5f;
    if (!(fabsf(fx) < 1.0e9f)) fx = 0.f;
    if (!(fabsf(fy) < 1.0e9f)) fy = 0.f;
    const float x0f = floorf(fx), y0f = floorf(fy);
    const float ax = fx - x0f, ay = fy - y0f;
    Bilinear b;
    b.x0 = wrap_index(x0f, W);
    b.y0 = wrap_index(y0f, H);
    b.x1 = b.x0 + 1u == W ? 0u : b.x0 + 1u;
    b.y1 = b.y0 + 1u == H ? 0u : b.y0 + 1u;
    const float bx = 1.f - ax, by = 1.f - ay;
    b.w[0] = bx * by;
    b.w[1] = ax * by;
    b.w[2] = bx * ay;
    b.w[3] = ax * ay;
    return b;
}

}  // namespace fpt_tex
