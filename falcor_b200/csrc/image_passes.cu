// image_passes.cu -- the image passes around the path tracers in the
// reference's render graphs, each a streaming kernel over RGBA32F pixels:
//
//   AccumulatePass        RenderPasses/AccumulatePass/Accumulate.cs.slang:54-205,
//                         AccumulatePass.cpp:138-290,375-420
//   ToneMapper            RenderPasses/ToneMapper/ToneMapping.ps.slang:38-190,
//                         Luminance.ps.slang, ToneMapper.cpp:200-555
//   ColorMapPass          RenderPasses/DebugPasses/ColorMapPass/ColorMapPass.ps.slang,
//                         ColorMapPass.cpp:97-225, Utils/Color/ColorMap.slang
//   RenderToViewportPass  RenderPasses/Viewport/RenderToViewportPass.cpp (headless: a blit)
//
// All four are HBM-bound (16 B read + 16 B written per pixel, plus the
// accumulation buffers); one thread per pixel, grid-stride, 256 threads.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "image_passes.h"
#include "passes.h"
#include "scene_device.h"

namespace fpt {

namespace {

__device__ __forceinline__ float4 f4add(float4 a, float4 b) { return make_float4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }
__device__ __forceinline__ float4 f4sub(float4 a, float4 b) { return make_float4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w); }
__device__ __forceinline__ float4 f4mul(float4 a, float s) { return make_float4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ float4 f4div(float4 a, float s) { return make_float4(a.x / s, a.y / s, a.z / s, a.w / s); }

// accumulateSingle (Accumulate.cs.slang:54-90).
__global__ void accumulate_single(const float4* cur, float4* out, float4* sum, uint32_t n, uint32_t count, bool accumulate, bool ema) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 c = cur[i];
        float4 o;
        if (accumulate) {
            const float w = 1.f / float(count + 1);
            if (ema) {
                const float4 s = sum[i];
                o = f4add(s, f4mul(f4sub(c, s), w));  // lerp(sum, cur, w)
                sum[i] = o;
            } else {
                const float4 s = f4add(sum[i], c);
                o = f4mul(s, w);
                sum[i] = s;
            }
        } else {
            o = c;
        }
        out[i] = o;
    }
}

// accumulateSingleCompensated (Accumulate.cs.slang:92-126): Kahan summation.
// The build compiles without fast-math reassociation, so the compensation
// term survives as written.
__global__ void accumulate_kahan(const float4* cur, float4* out, float4* sum, float4* corr, uint32_t n, uint32_t count, bool accumulate) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 c = cur[i];
        float4 o;
        if (accumulate) {
            const float4 s = sum[i];
            const float4 k = corr[i];
            const float4 y = f4sub(c, k);
            const float4 next = f4add(s, y);
            o = f4div(next, float(count + 1));
            sum[i] = next;
            corr[i] = f4sub(f4sub(next, s), y);
        } else {
            o = c;
        }
        out[i] = o;
    }
}

// accumulateDouble (Accumulate.cs.slang:128-205); the sum is held as double4
// instead of the reference's lo/hi uint4 texture pair (same 64-bit values).
__global__ void accumulate_double(const float4* cur, float4* out, double* sum, uint32_t n, uint32_t count, bool accumulate, bool ema) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 c = cur[i];
        float4 o;
        if (accumulate) {
            const double w = 1.0 / double(count + 1);
            const float cv[4] = {c.x, c.y, c.z, c.w};
            float ov[4];
            for (int k = 0; k < 4; k++) {
                double s = sum[4 * size_t(i) + k];
                if (ema) {
                    s = s * (1.0 - w) + double(cv[k]) * w;
                    ov[k] = float(s);
                } else {
                    s += double(cv[k]);
                    ov[k] = float(s * w);
                }
                sum[4 * size_t(i) + k] = s;
            }
            o = make_float4(ov[0], ov[1], ov[2], ov[3]);
        } else {
            o = c;
        }
        out[i] = o;
    }
}

// Bilinear fetch at texture coordinate (u, v) in [0,1]^2 with clamped texel
// indices (RenderContext::blit with a linear filter, and the luminance pass's
// linear sampler).  Weights are full FP32 (the hardware filter quantises them).
__device__ float4 bilinear(const float4* img, uint32_t w, uint32_t h, float u, float v) {
    const float x = u * float(w) - 0.5f, y = v * float(h) - 0.5f;
    const float fx0 = floorf(x), fy0 = floorf(y);
    const float fx = x - fx0, fy = y - fy0;
    const int x0 = int(fx0), y0 = int(fy0);
    auto cl = [](int a, uint32_t n) { return uint32_t(min(max(a, 0), int(n) - 1)); };
    const uint32_t xa = cl(x0, w), xb = cl(x0 + 1, w), ya = cl(y0, h), yb = cl(y0 + 1, h);
    const float4 a = img[size_t(ya) * w + xa], b = img[size_t(ya) * w + xb];
    const float4 c = img[size_t(yb) * w + xa], d = img[size_t(yb) * w + xb];
    const float4 top = f4add(f4mul(a, 1.f - fx), f4mul(b, fx));
    const float4 bot = f4add(f4mul(c, 1.f - fx), f4mul(d, fx));
    return f4add(f4mul(top, 1.f - fy), f4mul(bot, fy));
}

// RenderContext::blit (linear filter): copy when the sizes match, else a bilinear resample.
__global__ void blit_kernel(const float4* src, uint32_t sw, uint32_t sh, float4* dst, uint32_t dw, uint32_t dh) {
    const uint32_t n = dw * dh;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (sw == dw && sh == dh) { dst[i] = src[i]; continue; }
        const uint32_t x = i % dw, y = i / dw;
        dst[i] = bilinear(src, sw, sh, (float(x) + 0.5f) / float(dw), (float(y) + 0.5f) / float(dh));
    }
}

__device__ __forceinline__ float luminance601(float3 c) { return c.x * 0.299f + c.y * 0.587f + c.z * 0.114f; }

// Luminance.ps.slang over the bit_floor(W) x bit_floor(H) luminance target
// (ToneMapper::createLuminanceFbo, ToneMapper.cpp:264-287): each target texel
// samples the source bilinearly at its centre and stores
// log2(max(1e-4, luminance)); the mip chain the tone-map pass reads at
// kLuminanceLod is the mean of that target, summed here per block in double.
__global__ void log_luminance_sum(const float4* src, uint32_t sw, uint32_t sh, uint32_t lw, uint32_t lh, double* partial) {
    __shared__ double red[256];
    double acc = 0.0;
    const uint32_t n = lw * lh;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t x = i % lw, y = i / lw;
        float4 c;
        if (lw == sw && lh == sh) c = src[i];
        else c = bilinear(src, sw, sh, (float(x) + 0.5f) / float(lw), (float(y) + 0.5f) / float(lh));
        acc += double(log2f(fmaxf(0.0001f, luminance601(make_float3(c.x, c.y, c.z)))));
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (uint32_t s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

// Folds the per-block partial sums (one block).
__global__ void sum_partials(const double* partial, int count, double* out) {
    __shared__ double red[256];
    double acc = 0.0;
    for (int i = threadIdx.x; i < count; i += blockDim.x) acc += partial[i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (uint32_t s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// John Hable's filmic curve with the Uncharted 2 constants (ToneMapping.ps.slang:87-100).
__device__ float uc2(float x) {
    const float A = 0.22f, B = 0.3f, C = 0.1f, D = 0.2f, E = 0.01f, F = 0.3f;
    return ((x * (A * x + C * B) + D * E) / (x * (A * x + B) + D * F)) - E / F;
}
__device__ __forceinline__ float sat(float v) { return fminf(fmaxf(v, 0.f), 1.f); }

// toneMap (ToneMapping.ps.slang:52-161) and main (:163-190).  The source is
// read with a point sampler at the destination texel centre.
__global__ void tone_map_kernel(const float4* src, uint32_t sw, uint32_t sh, float4* dst, uint32_t dw, uint32_t dh, ToneMapArgs a,
                                const double* logLumSum) {
    float exposure = 1.f;
    if (a.autoExposure) {
        const float avgLuminance = exp2f(float(*logLumSum / double(a.lumTexels)));
        exposure = 0.042f / avgLuminance;  // kExposureKey
    }
    const uint32_t n = dw * dh;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 c0;
        if (sw == dw && sh == dh) {
            c0 = src[i];
        } else {
            const uint32_t x = i % dw, y = i / dw;
            const uint32_t sx = min(uint32_t((float(x) + 0.5f) / float(dw) * float(sw)), sw - 1);
            const uint32_t sy = min(uint32_t((float(y) + 0.5f) / float(dh) * float(sh)), sh - 1);
            c0 = src[size_t(sy) * sw + sx];
        }
        float3 c = make_float3(c0.x, c0.y, c0.z);
        if (a.autoExposure) c = make_float3(c.x * exposure, c.y * exposure, c.z * exposure);
        c = make_float3(a.m[0] * c.x + a.m[1] * c.y + a.m[2] * c.z, a.m[3] * c.x + a.m[4] * c.y + a.m[5] * c.z,
                        a.m[6] * c.x + a.m[7] * c.y + a.m[8] * c.z);
        switch (a.op) {
        case 0:  // Linear
            break;
        case 1: {  // Reinhard: luminance-preserving l / (l + 1)
            const float l = luminance601(c);
            const float s = (l / (l + 1.f)) / l;
            c = make_float3(c.x * s, c.y * s, c.z * s);
            break;
        }
        case 2: {  // ReinhardModified: the reference multiplies by (1 + l) where
                   // Reinhard et al. 2002 divide; kept as the reference computes it
            const float l = luminance601(c);
            const float s = (l * (1.f + l / (a.whiteMaxLuminance * a.whiteMaxLuminance)) * (1.f + l)) / l;
            c = make_float3(c.x * s, c.y * s, c.z * s);
            break;
        }
        case 3: {  // HejiHableAlu (output already gamma corrected; linearised with 2.2)
            auto f = [](float x) {
                x = fmaxf(0.f, x - 0.004f);
                x = (x * (6.2f * x + 0.5f)) / (x * (6.2f * x + 1.7f) + 0.06f);
                return powf(x, 2.2f);
            };
            c = make_float3(f(c.x), f(c.y), f(c.z));
            break;
        }
        case 4: {  // HableUc2: exposure bias 2, normalised by the curve at whiteScale
            const float ws = 1.f / uc2(a.whiteScale);
            c = make_float3(uc2(2.f * c.x) * ws, uc2(2.f * c.y) * ws, uc2(2.f * c.z) * ws);
            break;
        }
        default: {  // Aces (Narkowicz's fit, input scaled by 0.6)
            const float A = 2.51f, B = 0.03f, C = 2.43f, D = 0.59f, E = 0.14f;
            auto f = [&](float x) {
                x *= 0.6f;
                return sat((x * (A * x + B)) / (x * (C * x + D) + E));
            };
            c = make_float3(f(c.x), f(c.y), f(c.z));
            break;
        }
        }
        if (a.clamp) c = make_float3(sat(c.x), sat(c.y), sat(c.z));
        dst[i] = make_float4(c.x, c.y, c.z, c0.w);
    }
}

// Utils/Color/ColorMap.slang: grey, jet, and the sixth-order polynomial fits
// of the matplotlib viridis / plasma / magma / inferno maps.
__constant__ float kColorMapPoly[4][7][3] = {
    {{0.2777273272234177f, 0.005407344544966578f, 0.3340998053353061f},
     {0.1050930431085774f, 1.404613529898575f, 1.384590162594685f},
     {-0.3308618287255563f, 0.214847559468213f, 0.09509516302823659f},
     {-4.634230498983486f, -5.799100973351585f, -19.33244095627987f},
     {6.228269936347081f, 14.17993336680509f, 56.69055260068105f},
     {4.776384997670288f, -13.74514537774601f, -65.35303263337234f},
     {-5.435455855934631f, 4.645852612178535f, 26.3124352495832f}},
    {{0.05873234392399702f, 0.02333670892565664f, 0.5433401826748754f},
     {2.176514634195958f, 0.2383834171260182f, 0.7539604599784036f},
     {-2.689460476458034f, -7.455851135738909f, 3.110799939717086f},
     {6.130348345893603f, 42.3461881477227f, -28.51885465332158f},
     {-11.10743619062271f, -82.66631109428045f, 60.13984767418263f},
     {10.02306557647065f, 71.41361770095349f, -54.07218655560067f},
     {-3.658713842777788f, -22.93153465461149f, 18.19190778539828f}},
    {{-0.002136485053939582f, -0.000749655052795221f, -0.005386127855323933f},
     {0.2516605407371642f, 0.6775232436837668f, 2.494026599312351f},
     {8.353717279216625f, -3.577719514958484f, 0.3144679030132573f},
     {-27.66873308576866f, 14.26473078096533f, -13.64921318813922f},
     {52.17613981234068f, -27.94360607168351f, 12.94416944238394f},
     {-50.76852536473588f, 29.04658282127291f, 4.23415299384598f},
     {18.65570506591883f, -11.48977351997711f, -5.601961508734096f}},
    {{0.0002189403691192265f, 0.001651004631001012f, -0.01948089843709184f},
     {0.1065134194856116f, 0.5639564367884091f, 3.932712388889277f},
     {11.60249308247187f, -3.972853965665698f, -15.9423941062914f},
     {-41.70399613139459f, 17.43639888205313f, 44.35414519872813f},
     {77.162935699427f, -33.40235894210092f, -81.80730925738993f},
     {-71.31942824499214f, 32.62606426397723f, 73.20951985803202f},
     {25.13112622477341f, -12.24266895238567f, -23.07032500287172f}},
};

__device__ float3 apply_color_map(int map, float x) {
    if (map == 0) {
        const float v = sat(x);
        return make_float3(v, v, v);
    }
    if (map == 1) {
        const float s = 4.f * sat(x);
        return make_float3(sat(1.5f - fabsf(s - 3.f)), sat(1.5f - fabsf(s - 2.f)), sat(1.5f - fabsf(s - 1.f)));
    }
    if (map < 2 || map > 5) return make_float3(0.f, 0.f, 0.f);
    const float(*c)[3] = kColorMapPoly[map - 2];
    x = sat(x);
    float r[3];
    for (int k = 0; k < 3; k++)
        r[k] = sat(c[0][k] + x * (c[1][k] + x * (c[2][k] + x * (c[3][k] + x * (c[4][k] + x * (c[5][k] + x * c[6][k]))))));
    return make_float3(r[0], r[1], r[2]);
}

// ColorMapPass.ps.slang main: Load at the destination pixel (zero outside the
// source), normalise to [min, max], colourise, alpha 1.
__global__ void color_map_kernel(const float4* src, uint32_t sw, uint32_t sh, float4* dst, uint32_t dw, uint32_t dh, int map,
                                 int channel, float minValue, float maxValue) {
    const uint32_t n = dw * dh;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t x = i % dw, y = i / dw;
        float value = 0.f;
        if (x < sw && y < sh) {
            const float4 s = src[size_t(y) * sw + x];
            value = channel == 0 ? s.x : channel == 1 ? s.y : channel == 2 ? s.z : s.w;
        }
        const float t = minValue == maxValue ? 0.f : sat((value - minValue) / (maxValue - minValue));
        const float3 c = apply_color_map(map, t);
        dst[i] = make_float4(c.x, c.y, c.z, 1.f);
    }
}

// Per-block min/max of one channel (ParallelReduction::Type::MinMax for the
// ColorMapPass auto range); partial[2b] = min, partial[2b+1] = max.
__global__ void channel_min_max(const float4* src, uint32_t n, int channel, float* partial) {
    __shared__ float mn[256], mx[256];
    float lo = INFINITY, hi = -INFINITY;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 s = src[i];
        const float v = channel == 0 ? s.x : channel == 1 ? s.y : channel == 2 ? s.z : s.w;
        lo = fminf(lo, v);
        hi = fmaxf(hi, v);
    }
    mn[threadIdx.x] = lo;
    mx[threadIdx.x] = hi;
    __syncthreads();
    for (uint32_t s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            mn[threadIdx.x] = fminf(mn[threadIdx.x], mn[threadIdx.x + s]);
            mx[threadIdx.x] = fmaxf(mx[threadIdx.x], mx[threadIdx.x + s]);
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        partial[2 * blockIdx.x] = mn[0];
        partial[2 * blockIdx.x + 1] = mx[0];
    }
}

__global__ void fold_min_max(const float* partial, int count, float* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    float lo = INFINITY, hi = -INFINITY;
    for (int i = 0; i < count; i++) {
        lo = fminf(lo, partial[2 * i]);
        hi = fmaxf(hi, partial[2 * i + 1]);
    }
    out[0] = lo;
    out[1] = hi;
}

constexpr int kReduceBlocks = 148;

int grid(uint32_t n) { return int(std::max<uint32_t>(1, std::min<uint32_t>((n + 255) / 256, 148u * 8u))); }

uint32_t bit_floor(uint32_t v) {
    uint32_t r = 1;
    while ((r << 1) != 0 && (r << 1) <= v) r <<= 1;
    return r;
}

// ---- host-side colour transforms (ToneMapper.cpp:520-555, Utils/Color/ColorUtils.h) ----

struct M3 { float m[3][3]; };
M3 mul3(const M3& a, const M3& b) {
    M3 r;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) r.m[i][j] = a.m[i][0] * b.m[0][j] + a.m[i][1] * b.m[1][j] + a.m[i][2] * b.m[2][j];
    return r;
}

// Rec.709 primaries with the D65 white (IEC 61966-2-1) and CIECAM02's CAT02 LMS matrix.
const M3 kRGBtoXYZ = {{{0.4123907992659595f, 0.3575843393838780f, 0.1804807884018343f},
                       {0.2126390058715104f, 0.7151686787677559f, 0.0721923153607337f},
                       {0.0193308187155918f, 0.1191947797946259f, 0.9505321522496608f}}};
const M3 kXYZtoRGB = {{{3.2409699419045213f, -1.5373831775700935f, -0.4986107602930033f},
                       {-0.9692436362808798f, 1.8759675015077206f, 0.0415550574071756f},
                       {0.0556300796969936f, -0.2039769588889765f, 1.0569715142428784f}}};
const M3 kXYZtoLMS = {{{0.7328f, 0.4296f, -0.1624f}, {-0.7036f, 1.6975f, 0.0061f}, {0.0030f, 0.0136f, 0.9834f}}};
const M3 kLMStoXYZ = {{{1.096123820835514f, -0.278869000218287f, 0.182745179382773f},
                       {0.454369041975359f, 0.473533154307412f, 0.072097803717229f},
                       {-0.009627608738429f, -0.005698031216113f, 1.015325639954543f}}};

// Blackbody chromaticity by Kang et al. 2002's piecewise rational fits, in
// double, returned as XYZ with Y = 1 (ColorUtils.h colorTemperatureToXYZ).
void color_temperature_xyz(float T, float out[3]) {
    const double t = T, t2 = t * t, t3 = t2 * t;
    const double xc = T < 4000.f ? -0.2661239e9 / t3 - 0.2343580e6 / t2 + 0.8776956e3 / t + 0.179910
                                 : -3.0258469e9 / t3 + 2.1070379e6 / t2 + 0.2226347e3 / t + 0.240390;
    const double x = xc, x2 = x * x, x3 = x2 * x;
    double yc;
    if (T < 2222.f) yc = -1.1063814 * x3 - 1.34811020 * x2 + 2.18555832 * x - 0.20219683;
    else if (T < 4000.f) yc = -0.9549476 * x3 - 1.37418593 * x2 + 2.09137015 * x - 0.16748867;
    else yc = 3.0817580 * x3 - 5.87338670 * x2 + 3.75112997 * x - 0.37001483;
    const float xf = float(xc), yf = float(yc);
    out[0] = xf * 1.f / yf;
    out[1] = 1.f;
    out[2] = (1.f - xf - yf) * 1.f / yf;
}

// von Kries adaptation in CAT02 LMS from white T to the D65 white (6500 K).
M3 white_balance_rgb709(float T) {
    const M3 MA = mul3(kXYZtoLMS, kRGBtoXYZ), invMA = mul3(kXYZtoRGB, kLMStoXYZ);
    float xyzD[3], xyzS[3];
    color_temperature_xyz(6500.f, xyzD);
    color_temperature_xyz(T, xyzS);
    float wd[3], ws[3];
    for (int i = 0; i < 3; i++) {
        wd[i] = kXYZtoLMS.m[i][0] * xyzD[0] + kXYZtoLMS.m[i][1] * xyzD[1] + kXYZtoLMS.m[i][2] * xyzD[2];
        ws[i] = kXYZtoLMS.m[i][0] * xyzS[0] + kXYZtoLMS.m[i][1] * xyzS[1] + kXYZtoLMS.m[i][2] * xyzS[2];
    }
    M3 D = {{{wd[0] / ws[0], 0.f, 0.f}, {0.f, wd[1] / ws[1], 0.f}, {0.f, 0.f, wd[2] / ws[2]}}};
    return mul3(mul3(invMA, D), MA);
}

cudaError_t ensure_image_scratch(fpt_pass& p, size_t bytes) {
    if (p.imageScratch && p.imageScratchBytes >= bytes) return cudaSuccess;
    if (p.imageScratch) cudaFree(p.imageScratch);
    p.imageScratch = nullptr;
    p.imageScratchBytes = 0;
    cudaError_t e = cudaMalloc(&p.imageScratch, bytes);
    if (e == cudaSuccess) p.imageScratchBytes = bytes;
    return e;
}

fpt_status cuda_fail(const std::string& who, cudaError_t e) {
    return set_error(e == cudaErrorMemoryAllocation ? FPT_ERR_OOM : FPT_ERR_CUDA, who + ": " + cudaGetErrorString(e));
}

}  // namespace

cudaError_t launch_accumulate(int precision, const float4* cur, float4* out, void* sum, float4* corr, uint32_t n, uint32_t count,
                              bool accumulate, bool ema, cudaStream_t st) {
    if (precision == 0) accumulate_double<<<grid(n), 256, 0, st>>>(cur, out, static_cast<double*>(sum), n, count, accumulate, ema);
    else if (precision == 1) accumulate_single<<<grid(n), 256, 0, st>>>(cur, out, static_cast<float4*>(sum), n, count, accumulate, ema);
    else accumulate_kahan<<<grid(n), 256, 0, st>>>(cur, out, static_cast<float4*>(sum), corr, n, count, accumulate);
    return cudaGetLastError();
}

cudaError_t launch_blit(const float4* src, uint32_t sw, uint32_t sh, float4* dst, uint32_t dw, uint32_t dh, cudaStream_t st) {
    blit_kernel<<<grid(dw * dh), 256, 0, st>>>(src, sw, sh, dst, dw, dh);
    return cudaGetLastError();
}

cudaError_t launch_tone_map(const float4* src, uint32_t sw, uint32_t sh, float4* dst, uint32_t dw, uint32_t dh, ToneMapArgs a,
                            double* scratch, cudaStream_t st) {
    if (a.autoExposure) {
        const uint32_t lw = bit_floor(sw), lh = bit_floor(sh);
        a.lumTexels = lw * lh;
        log_luminance_sum<<<kReduceBlocks, 256, 0, st>>>(src, sw, sh, lw, lh, scratch + 1);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        sum_partials<<<1, 256, 0, st>>>(scratch + 1, kReduceBlocks, scratch);
    }
    tone_map_kernel<<<grid(dw * dh), 256, 0, st>>>(src, sw, sh, dst, dw, dh, a, scratch);
    return cudaGetLastError();
}

void tone_map_color_transform(const fpt_pass& p, float m[9]) {
    // ToneMapper::updateWhiteBalanceTransform / updateColorTransform (ToneMapper.cpp:520-555).
    M3 wb = {{{1.f, 0.f, 0.f}, {0.f, 1.f, 0.f}, {0.f, 0.f, 1.f}}};
    if (p.num("whiteBalance") != 0) wb = white_balance_rgb709(float(p.num("whitePoint")));
    const float exposureScale = std::pow(2.f, float(p.num("exposureCompensation")));
    float manual = 1.f;
    if (p.num("autoExposure") == 0) {
        const float fN = float(p.num("fNumber")), sh = float(p.num("shutter"));
        manual = (1.f / 100.f * float(p.num("filmSpeed"))) / (sh * fN * fN);
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) m[3 * i + j] = wb.m[i][j] * exposureScale * manual;
}

fpt_status image_pass_execute(fpt_pass& p, const fpt_frame_io* io, cudaStream_t st) {
    const float4* src = reinterpret_cast<const float4*>(io->src);
    float4* dst = reinterpret_cast<float4*>(io->dst);
    const uint32_t dw = io->width, dh = io->height;
    const uint32_t sw = io->src_width ? io->src_width : dw, sh = io->src_height ? io->src_height : dh;
    if (!src || !dst)
        return set_error(FPT_ERR_INVALID_ARG, p.type + (p.type == "ToneMapper" ? ": 'src' and 'dst' are required" : ": 'input' and 'output' are required"));
    if (sw == 0 || sh == 0 || sw > 16384 || sh > 16384) return set_error(FPT_ERR_INVALID_ARG, p.type + ": invalid source size");
    cudaError_t e = cudaSuccess;
    p.launches = 1;

    if (p.type == "RenderToViewportPass") {
        e = launch_blit(src, sw, sh, dst, dw, dh, st);
        return e == cudaSuccess ? FPT_OK : cuda_fail(p.type, e);
    }

    if (p.type == "ToneMapper") {
        if (sw != dw || sh != dh) log_warning("ToneMapper pass I/O has different dimensions. The image will be resampled.");
        ToneMapArgs a;
        std::memset(&a, 0, sizeof(a));
        tone_map_color_transform(p, a.m);
        a.whiteScale = float(p.num("whiteScale"));
        a.whiteMaxLuminance = float(p.num("whiteMaxLuminance"));
        auto it = kToneMapOperators.find(p.str("operator"));
        a.op = it == kToneMapOperators.end() ? 5 : it->second;
        a.clamp = p.num("clamp") != 0;
        a.autoExposure = p.num("autoExposure") != 0;
        e = ensure_image_scratch(p, (1 + kReduceBlocks) * sizeof(double));
        if (e != cudaSuccess) return cuda_fail(p.type, e);
        e = launch_tone_map(src, sw, sh, dst, dw, dh, a, static_cast<double*>(p.imageScratch), st);
        p.launches = a.autoExposure ? 3 : 1;
        return e == cudaSuccess ? FPT_OK : cuda_fail(p.type, e);
    }

    if (p.type == "ColorMapPass") {
        const int channel = int(std::clamp(p.num("channel"), 0.0, 3.0));
        auto it = kColorMaps.find(p.str("colorMap"));
        const int map = it == kColorMaps.end() ? 1 : it->second;
        e = ensure_image_scratch(p, 2 * kReduceBlocks * sizeof(float) + 2 * sizeof(float));
        if (e != cudaSuccess) return cuda_fail(p.type, e);
        float* partial = static_cast<float*>(p.imageScratch);
        float* result = partial + 2 * kReduceBlocks;
        if (p.num("autoRange") != 0) {
            // AutoRanging::getMinMax (ColorMapPass.cpp:183-225): the reduction of
            // the previous frame sets this frame's range; a reduction of this
            // frame is issued for the next one.
            if (p.reductionAvailable) {
                float mm[2];
                e = cudaMemcpyAsync(mm, result, sizeof(mm), cudaMemcpyDeviceToHost, st);
                if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                if (e != cudaSuccess) return cuda_fail(p.type, e);
                p.autoMin = std::min(p.autoMin, double(mm[0]));
                p.autoMax = std::max(p.autoMax, double(mm[1]));
                const double alpha = 0.01;
                p.autoMin = p.autoMin + (double(mm[0]) - p.autoMin) * alpha;
                p.autoMax = p.autoMax + (double(mm[1]) - p.autoMax) * alpha;
                p.props["minValue"].n = double(float(p.autoMin));
                p.props["maxValue"].n = double(float(p.autoMax));
                p.reductionAvailable = false;
            } else {
                p.autoMin = p.num("minValue");
                p.autoMax = p.num("maxValue");
            }
            channel_min_max<<<kReduceBlocks, 256, 0, st>>>(src, sw * sh, channel, partial);
            fold_min_max<<<1, 32, 0, st>>>(partial, kReduceBlocks, result);
            e = cudaGetLastError();
            if (e != cudaSuccess) return cuda_fail(p.type, e);
            p.reductionAvailable = true;
            p.launches = 3;
        } else {
            p.reductionAvailable = false;
        }
        color_map_kernel<<<grid(dw * dh), 256, 0, st>>>(src, sw, sh, dst, dw, dh, map, channel, float(p.num("minValue")),
                                                        float(p.num("maxValue")));
        e = cudaGetLastError();
        return e == cudaSuccess ? FPT_OK : cuda_fail(p.type, e);
    }

    // AccumulatePass::execute (AccumulatePass.cpp:138-212) and accumulate (:214-290).
    if (p.num("autoReset") != 0) {
        if (io->refresh) p.frameCount = 0;
        if (p.scene && p.scene->resetVersion != p.accumSceneVersion) {
            p.accumSceneVersion = p.scene->resetVersion;
            p.frameCount = 0;
        }
    }
    const uint32_t maxFrames = uint32_t(std::max(0.0, p.num("maxFrameCount")));
    if (maxFrames > 0 && p.frameCount == maxFrames) {
        const std::string om = p.str("overflowMode");
        if (om == "Stop") return FPT_OK;
        if (om == "Reset") p.frameCount = 0;
    }
    if (sw != p.accumW || sh != p.accumH) {
        p.accumW = sw;
        p.accumH = sh;
        p.frameCount = 0;
    }
    const bool match = sw == dw && sh == dh;
    if (p.num("enabled") != 0 && !match) {
        log_warning("AccumulatePass I/O sizes don't match. The pass will be disabled.");
        p.props["enabled"].n = 0;
    }
    if (p.num("enabled") == 0) {
        e = launch_blit(src, sw, sh, dst, dw, dh, st);
        return e == cudaSuccess ? FPT_OK : cuda_fail(p.type, e);
    }
    auto pm = kPrecisionModes.find(p.str("precisionMode"));
    const int precision = pm == kPrecisionModes.end() ? 1 : pm->second;
    const size_t n = size_t(sw) * sh;
    const size_t sumBytes = n * (precision == 0 ? 32 : 16);
    const size_t corrBytes = precision == 2 ? n * 16 : 0;
    if (p.accumPrecision != precision || p.accumSumBytes != sumBytes || p.accumCorrBytes != corrBytes) {
        // prepareAccumulation (AccumulatePass.cpp:380-420): (re)create and reset.
        if (p.accumSum) cudaFree(p.accumSum);
        if (p.accumCorr) cudaFree(p.accumCorr);
        p.accumSum = nullptr;
        p.accumCorr = nullptr;
        p.accumSumBytes = p.accumCorrBytes = 0;
        p.accumPrecision = -1;
        e = cudaMalloc(&p.accumSum, sumBytes);
        if (e == cudaSuccess && corrBytes) e = cudaMalloc(reinterpret_cast<void**>(&p.accumCorr), corrBytes);
        if (e != cudaSuccess) return cuda_fail("AccumulatePass: accumulation buffers", e);
        p.accumSumBytes = sumBytes;
        p.accumCorrBytes = corrBytes;
        p.accumPrecision = precision;
        p.frameCount = 0;
    }
    if (p.frameCount == 0) {
        e = cudaMemsetAsync(p.accumSum, 0, sumBytes, st);
        if (e == cudaSuccess && corrBytes) e = cudaMemsetAsync(p.accumCorr, 0, corrBytes, st);
        if (e != cudaSuccess) return cuda_fail(p.type, e);
    }
    const uint32_t count = p.frameCount;
    const bool ema = maxFrames > 0;
    if (maxFrames == 0 || precision == 2 || p.frameCount < maxFrames) p.frameCount++;
    e = launch_accumulate(precision, src, dst, p.accumSum, p.accumCorr, uint32_t(n), count, true, ema, st);
    return e == cudaSuccess ? FPT_OK : cuda_fail(p.type, e);
}

}  // namespace fpt
