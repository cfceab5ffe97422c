// Frame output after the pass: the ToneMapper pass's per-pixel chain and the 8-bit sRGB conversion
// the FrameDumper pass gets from its blit, as one kernel over the RGBA32F colour.
//
//   RenderPasses/ToneMapper/ToneMapping.ps.slang:45-173   operators, auto exposure, clamp
//   RenderPasses/ToneMapper/Luminance.ps.slang:35-44      log2 luminance for auto exposure
//   RenderPasses/ToneMapper/ToneMapper.cpp:538-550        exposure scale (compensation, manual EV)
//   RenderPasses/FrameDumper/FrameDumper.cpp:80-90,151-158 RGBA8UnormSrgb blit, .pam files
//
// The reference averages log luminance through the top mip of a log-luminance texture; here the
// average is the exact mean over all pixels, reduced in a fixed order (per-block partial sums, then
// one block over the partials), so the output does not depend on scheduling.  White balance
// (colour grading with a white point) is not implemented: the transform is the exposure scale.
// HBM-bound: 16 B read (twice with auto exposure) and 4 B written per pixel.
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/rs_b200.h"

namespace rs {
namespace {

constexpr int kReduceBlocks = 1024;
constexpr int kReduceThreads = 256;

__device__ __forceinline__ float tm_luminance(float r, float g, float b) { return r * 0.299f + g * 0.587f + b * 0.114f; }

// Mean of log2(max(1e-4, luminance)) in double: partial sums per block in a fixed order.
__global__ void __launch_bounds__(kReduceThreads) k_log_luminance(const float4* __restrict__ color, uint32_t n, double* __restrict__ partial)
{
    __shared__ double s[kReduceThreads];
    double acc = 0.0;
    for (uint32_t i = blockIdx.x * kReduceThreads + threadIdx.x; i < n; i += kReduceBlocks * kReduceThreads)
    {
        const float4 c = __ldg(&color[i]);
        acc += (double)log2f(fmaxf(0.0001f, tm_luminance(c.x, c.y, c.z)));
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kReduceThreads / 2; w > 0; w >>= 1)
    {
        if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

__global__ void __launch_bounds__(kReduceThreads) k_log_luminance_total(double* __restrict__ partial, uint32_t n)
{
    __shared__ double s[kReduceThreads];
    double acc = 0.0;
    for (int i = threadIdx.x; i < kReduceBlocks; i += kReduceThreads) acc += partial[i];
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int w = kReduceThreads / 2; w > 0; w >>= 1)
    {
        if ((int)threadIdx.x < w) s[threadIdx.x] += s[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[kReduceBlocks] = s[0] / (double)n;
}

__device__ __forceinline__ float uc2_curve(float x)
{
    const float A = 0.22f, B = 0.3f, C = 0.1f, D = 0.2f, E = 0.01f, F = 0.3f;
    return ((x * (A * x + C * B) + D * E) / (x * (A * x + B) + D * F)) - (E / F);
}

__device__ __forceinline__ void tone_map(uint32_t op, float& r, float& g, float& b, float whiteMaxLuminance, float whiteScale)
{
    switch (op)
    {
    case RS_TONEMAP_REINHARD:
    {
        const float l = tm_luminance(r, g, b);
        const float k = (l / (l + 1.f)) / l;
        r *= k; g *= k; b *= k;
        break;
    }
    case RS_TONEMAP_REINHARD_MODIFIED:
    {
        const float l = tm_luminance(r, g, b);
        const float k = (l * (1.f + l / (whiteMaxLuminance * whiteMaxLuminance)) * (1.f + l)) / l;
        r *= k; g *= k; b *= k;
        break;
    }
    case RS_TONEMAP_HEJI_HABLE_ALU:
    {
        float c[3] = {r, g, b};
        for (float& x : c)
        {
            x = fmaxf(0.f, x - 0.004f);
            x = (x * (6.2f * x + 0.5f)) / (x * (6.2f * x + 1.7f) + 0.06f);
            x = powf(x, 2.2f);
        }
        r = c[0]; g = c[1]; b = c[2];
        break;
    }
    case RS_TONEMAP_HABLE_UC2:
    {
        const float ws = 1.f / uc2_curve(whiteScale);
        r = uc2_curve(2.f * r) * ws; g = uc2_curve(2.f * g) * ws; b = uc2_curve(2.f * b) * ws;
        break;
    }
    case RS_TONEMAP_ACES:
    {
        float c[3] = {r * 0.6f, g * 0.6f, b * 0.6f};
        const float A = 2.51f, B = 0.03f, C = 2.43f, D = 0.59f, E = 0.14f;
        for (float& x : c) x = fminf(fmaxf((x * (A * x + B)) / (x * (C * x + D) + E), 0.f), 1.f);
        r = c[0]; g = c[1]; b = c[2];
        break;
    }
    default: break; // RS_TONEMAP_LINEAR
    }
}

// Linear [0, 1] -> sRGB-encoded 8-bit (the RGBA8UnormSrgb write); NaN and negatives give 0.
__device__ __forceinline__ uint32_t srgb8(float x)
{
    x = fminf(fmaxf(x, 0.f), 1.f);
    const float e = x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.f / 2.4f) - 0.055f;
    return (uint32_t)__float2int_rn(e * 255.f);
}
__device__ __forceinline__ uint32_t unorm8(float x) { return (uint32_t)__float2int_rn(fminf(fmaxf(x, 0.f), 1.f) * 255.f); }

__global__ void __launch_bounds__(256) k_tonemap(const float4* __restrict__ color, uint32_t n, rs_tonemap_options o, float scale,
                                                 const double* __restrict__ meanLog2, uint32_t* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 c = __ldg(&color[i]);
    float r = c.x, g = c.y, b = c.z;
    if (o.autoExposure)
    {
        const float k = 0.042f / exp2f((float)*meanLog2); // kExposureKey / average luminance
        r *= k; g *= k; b *= k;
    }
    r *= scale; g *= scale; b *= scale;
    tone_map(o.op, r, g, b, o.whiteMaxLuminance, o.whiteScale);
    if (o.clamp)
    {
        r = fminf(fmaxf(r, 0.f), 1.f); g = fminf(fmaxf(g, 0.f), 1.f); b = fminf(fmaxf(b, 0.f), 1.f);
    }
    out[i] = srgb8(r) | (srgb8(g) << 8) | (srgb8(b) << 16) | (unorm8(c.w) << 24);
}

} // namespace
} // namespace rs

using namespace rs;

extern "C" RS_API void rs_tonemap_default_options(rs_tonemap_options* o)
{
    if (!o) return;
    // ToneMapper.h:131-156 defaults
    o->op = RS_TONEMAP_ACES;
    o->exposureCompensation = 0.f;
    o->autoExposure = 0;
    o->filmSpeed = 100.f;
    o->fNumber = 1.f;
    o->shutter = 1.f;
    o->clamp = 1;
    o->whiteMaxLuminance = 1.f;
    o->whiteScale = 11.2f;
}

extern "C" RS_API size_t rs_tonemap_workspace_bytes(void) { return sizeof(double) * (kReduceBlocks + 1); }

extern "C" RS_API rs_status rs_tonemap(const void* colorDev, uint32_t width, uint32_t height, const rs_tonemap_options* opts, void* rgba8Dev,
                                       void* workspaceDev, void* stream)
{
    if (!colorDev || !opts || !rgba8Dev) return RS_INVALID_ARG;
    if (opts->op > RS_TONEMAP_ACES) return RS_INVALID_ARG;
    if (opts->autoExposure && !workspaceDev) return RS_INVALID_ARG;
    if (!(opts->fNumber > 0.f) || !(opts->shutter > 0.f) || !(opts->filmSpeed > 0.f)) return RS_INVALID_ARG;
    const uint64_t n64 = (uint64_t)width * height;
    if (n64 == 0) return RS_OK;
    if (n64 > 0xffffffffull) return RS_INVALID_ARG;
    const uint32_t n = (uint32_t)n64;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    // ToneMapper::updateColorTransform: 2^compensation, times the manual exposure without auto exposure
    float scale = exp2f(opts->exposureCompensation);
    if (!opts->autoExposure) scale *= (0.01f * opts->filmSpeed) / (opts->shutter * opts->fNumber * opts->fNumber);
    const float4* color = static_cast<const float4*>(colorDev);
    double* ws = static_cast<double*>(workspaceDev);
    if (opts->autoExposure)
    {
        k_log_luminance<<<kReduceBlocks, kReduceThreads, 0, s>>>(color, n, ws);
        k_log_luminance_total<<<1, kReduceThreads, 0, s>>>(ws, n);
    }
    k_tonemap<<<(n + 255) / 256, 256, 0, s>>>(color, n, *opts, scale, ws ? ws + kReduceBlocks : nullptr, static_cast<uint32_t*>(rgba8Dev));
    return cudaGetLastError() == cudaSuccess ? RS_OK : RS_CUDA_ERROR;
}
