// bsdf_probe.cu -- statistical probes of the device StandardBSDF lobes: the
// three programs of the reference's BSDF unit test
// (Tools/FalcorTest/Tests/Scene/Material/BSDFTests.cs.slang) run on the
// kernels' own StandardBSDF code: a histogram of sampled directions over
// (phi, cos theta) bins, the per-bin integral of evalPdf, and the per-bin
// largest relative error of the sampled weight and pdf against eval / evalPdf.
// A test hook of the C-ABI; nothing on the rendering path calls it.
#include <cuda_runtime.h>

#include <string>

#include "common.h"
#include "device_math.cuh"

namespace {

using namespace fpt::dev;

constexpr float kCosThetaMargin = 1e-3f;
constexpr float kOneOver2Pi = 0.159154943091895335768883763372514362f;
constexpr float k2PiF = 6.28318530717958647692528676655900576f;

struct Probe {
    uint32_t lobe;
    float3 wi;
    float4 params;
    uint32_t threadCount, threadSampleCount, phiBins, cosBins, binSamples, sampleCount;
};

// One lobe of StandardBSDF alone: the mixture with that lobe's selection
// probability 1 (the fields the reference test's TEST_BSDF_INIT sets: albedo 1,
// roughness params.x for the Frostbite lobe, alpha params.x for the
// microfacet lobe).
template <bool HAS_T>
__device__ StandardBSDF<HAS_T> make_lobe(const Probe& p) {
    StandardBSDF<HAS_T> b;
    b.diffAlbedo = b.transAlbedo = b.specAlbedo = make_float3(1.f, 1.f, 1.f);
    b.diffRoughness = 0.f;
    b.alpha = b.stAlpha = 0.f;
    b.eta = 1.f;
    b.diffTrans = b.specTrans = 0.f;
    b.pDR = b.pDT = b.pSR = b.pST = 0.f;
    b.activeLobes = 0u;
    b.lambert = false;
    switch (p.lobe) {
        case FPT_PROBE_FROSTBITE_BRDF: b.diffRoughness = p.params.x; b.pDR = 1.f; break;
        case FPT_PROBE_LAMBERT_BRDF: b.lambert = true; b.pDR = 1.f; break;
        case FPT_PROBE_LAMBERT_BTDF: b.diffTrans = 1.f; b.pDT = 1.f; break;
        default: b.alpha = p.params.x; b.activeLobes = 0xffu; b.pSR = 1.f; break;
    }
    return b;
}

__device__ uint32_t bin_of(const Probe& p, float3 wo) {
    const uint32_t cosBin = min(uint32_t(floor((double(wo.z) * 0.5 + 0.5) * double(p.cosBins))), p.cosBins - 1);
    float scaledPhi = fm::atan2(wo.y, wo.x) * kOneOver2Pi;
    if (scaledPhi < 0.f) scaledPhi += 1.f;
    const uint32_t phiBin = min(uint32_t(floorf(scaledPhi * float(p.phiBins))), p.phiBins - 1);
    return cosBin * p.phiBins + phiBin;
}

// tabulateHistogram / tabulateWeightAndPdfError: thread x draws
// threadSampleCount samples from UniformSampleGenerator((x, 0), 0).
template <bool HAS_T>
__global__ void probe_sampling(Probe p, uint32_t* hist, uint32_t* weightErr, uint32_t* pdfErr) {
    const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= p.threadCount) return;
    const float3 wi = normalize(p.wi);
    const StandardBSDF<HAS_T> bsdf = make_lobe<HAS_T>(p);
    UniformSG sg;
    sg.init(x, 0, 0);
    for (uint32_t i = 0; i < p.threadSampleCount; i++) {
        float3 wo, weight;
        float pdf;
        uint32_t lobe;
        if (!bsdf.sample(wi, wo, pdf, weight, lobe, sg)) continue;
        if (hist && !(wo.z < -1.f + kCosThetaMargin || wo.z > 1.f - kCosThetaMargin)) atomicAdd(hist + bin_of(p, wo), 1u);
        if (weightErr) {
            const float3 value = bsdf.eval(wi, wo);
            const float pdfRef = bsdf.eval_pdf(wi, wo);
            const float3 weightRef = pdfRef > 0.f ? value / pdfRef : make_float3(0.f, 0.f, 0.f);
            const float ex = fabsf(weight.x - weightRef.x) / (weightRef.x > 0.f ? weightRef.x : 1.f);
            const float ey = fabsf(weight.y - weightRef.y) / (weightRef.y > 0.f ? weightRef.y : 1.f);
            const float ez = fabsf(weight.z - weightRef.z) / (weightRef.z > 0.f ? weightRef.z : 1.f);
            const float we = fmaxf(fmaxf(ex, ey), ez);
            const float pe = fabsf(pdf - pdfRef) / (pdfRef > 0.f ? pdfRef : 1.f);
            const uint32_t b = bin_of(p, wo);
            atomicMax(weightErr + b, __float_as_uint(we));
            atomicMax(pdfErr + b, __float_as_uint(pe));
        }
    }
}

// tabulatePdf: midpoint integral of evalPdf over each bin, times sampleCount.
template <bool HAS_T>
__global__ void probe_pdf(Probe p, double* out) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= p.phiBins * p.cosBins) return;
    const uint32_t phiBin = t % p.phiBins, cosBin = t / p.phiBins;
    const float3 wi = normalize(p.wi);
    const StandardBSDF<HAS_T> bsdf = make_lobe<HAS_T>(p);
    const float phiStart = float(phiBin) * k2PiF / float(p.phiBins);
    const float phiEnd = float(phiBin + 1) * k2PiF / float(p.phiBins);
    float cosStart = -1.f + float(cosBin) * 2.f / float(p.cosBins);
    float cosEnd = -1.f + float(cosBin + 1) * 2.f / float(p.cosBins);
    cosStart = fmaxf(cosStart, -1.f + kCosThetaMargin);
    cosEnd = fminf(cosEnd, 1.f - kCosThetaMargin);
    float pdf = 0.f;
    for (uint32_t ix = 0; ix < p.binSamples; ix++)
        for (uint32_t iy = 0; iy < p.binSamples; iy++) {
            const float phi = phiStart + ((float(ix) + 0.5f) / float(p.binSamples)) * (phiEnd - phiStart);
            const float cosTheta = cosStart + ((float(iy) + 0.5f) / float(p.binSamples)) * (cosEnd - cosStart);
            const float sinTheta = sqrtf(1.f - cosTheta * cosTheta);
            float sp, cp;
            fm::sincos(phi, sp, cp);
            const float3 wo = normalize(make_float3(sinTheta * cp, sinTheta * sp, cosTheta));
            pdf += bsdf.eval_pdf(wi, wo);
        }
    pdf *= (cosEnd - cosStart) * (phiEnd - phiStart) / float(p.binSamples * p.binSamples);
    out[t] = double(pdf) * double(p.sampleCount);
}

template <bool HAS_T>
cudaError_t run(const Probe& p, uint32_t* hist, uint32_t* weightErr, uint32_t* pdfErr, double* pdfInt, cudaStream_t st) {
    const uint32_t block = 128;
    if (hist || weightErr) probe_sampling<HAS_T><<<(p.threadCount + block - 1) / block, block, 0, st>>>(p, hist, weightErr, pdfErr);
    if (pdfInt) probe_pdf<HAS_T><<<(p.phiBins * p.cosBins + block - 1) / block, block, 0, st>>>(p, pdfInt);
    return cudaGetLastError();
}

}  // namespace

extern "C" {

FPT_API fpt_status fpt_bsdf_probe_run(const fpt_bsdf_probe* probe, uint32_t* histogram, uint32_t* weight_error,
                                      uint32_t* pdf_error, double* pdf_integral, void* stream) {
    if (!probe) return fpt::set_error(FPT_ERR_INVALID_ARG, "fpt_bsdf_probe_run: null probe");
    if (probe->lobe > FPT_PROBE_MICROFACET_BRDF) return fpt::set_error(FPT_ERR_INVALID_ARG, "fpt_bsdf_probe_run: unknown lobe");
    if (!probe->thread_sample_count || !probe->sample_count || probe->sample_count % probe->thread_sample_count ||
        !probe->phi_bins || !probe->cos_bins || !probe->bin_sample_count)
        return fpt::set_error(FPT_ERR_INVALID_ARG, "fpt_bsdf_probe_run: invalid sample or bin counts");
    if ((weight_error == nullptr) != (pdf_error == nullptr))
        return fpt::set_error(FPT_ERR_INVALID_ARG, "fpt_bsdf_probe_run: weight_error and pdf_error go together");
    Probe p;
    p.lobe = probe->lobe;
    p.wi = make_float3(probe->wi[0], probe->wi[1], probe->wi[2]);
    p.params = make_float4(probe->params[0], probe->params[1], probe->params[2], probe->params[3]);
    p.sampleCount = probe->sample_count;
    p.threadSampleCount = probe->thread_sample_count;
    p.threadCount = probe->sample_count / probe->thread_sample_count;
    p.phiBins = probe->phi_bins;
    p.cosBins = probe->cos_bins;
    p.binSamples = probe->bin_sample_count;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const cudaError_t e = probe->lobe == FPT_PROBE_LAMBERT_BTDF ? run<true>(p, histogram, weight_error, pdf_error, pdf_integral, st)
                                                                : run<false>(p, histogram, weight_error, pdf_error, pdf_integral, st);
    if (e != cudaSuccess) return fpt::set_error(FPT_ERR_CUDA, std::string("fpt_bsdf_probe_run: ") + cudaGetErrorString(e));
    return FPT_OK;
}

}  // extern "C"
