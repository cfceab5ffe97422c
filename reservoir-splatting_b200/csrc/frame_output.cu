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
// one block over the partials), so the output does not depend on scheduling.  The colour grading
// transform is the exposure scale, times the white balance matrix when white balance is on
// (Utils/Color/ColorUtils.h:209-226: a von Kries scaling in CAT02 LMS space from the blackbody
// white of the white point, Kang et al. 2002, to that of 6500 K; computed on the host in double).
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

struct ColorTransform { float m[9]; };

__global__ void __launch_bounds__(256) k_tonemap(const float4* __restrict__ color, uint32_t n, rs_tonemap_options o, float scale,
                                                 ColorTransform T, const double* __restrict__ meanLog2, uint32_t* __restrict__ out)
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
    if (o.whiteBalance)
    {
        const float* m = T.m;
        const float r2 = m[0] * r + m[1] * g + m[2] * b, g2 = m[3] * r + m[4] * g + m[5] * b, b2 = m[6] * r + m[7] * g + m[8] * b;
        r = r2; g = g2; b = b2;
    }
    else { r *= scale; g *= scale; b *= scale; }
    tone_map(o.op, r, g, b, o.whiteMaxLuminance, o.whiteScale);
    if (o.clamp)
    {
        r = fminf(fmaxf(r, 0.f), 1.f); g = fminf(fmaxf(g, 0.f), 1.f); b = fminf(fmaxf(b, 0.f), 1.f);
    }
    out[i] = srgb8(r) | (srgb8(g) << 8) | (srgb8(b) << 16) | (unorm8(c.w) << 24);
}

// ColorUtils.h colour spaces: Rec.709 RGB <-> CIE XYZ (D65 primaries) and the CAT02 XYZ -> LMS
// matrix of CIECAM02; the inverses are computed.
const double kRgbToXyz[9] = {0.4123907992659595, 0.3575843393838780, 0.1804807884018343,
                             0.2126390058715104, 0.7151686787677559, 0.0721923153607337,
                             0.0193308187155918, 0.1191947797946259, 0.9505321522496608};
const double kXyzToLmsCat02[9] = {0.7328, 0.4296, -0.1624, -0.7036, 1.6975, 0.0061, 0.0030, 0.0136, 0.9834};

void mat3_mul_d(const double* a, const double* b, double* out)
{
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) out[3 * r + c] = a[3 * r] * b[c] + a[3 * r + 1] * b[3 + c] + a[3 * r + 2] * b[6 + c];
}
void mat3_inverse_d(const double* m, double* out)
{
    const double c00 = m[4] * m[8] - m[5] * m[7], c01 = m[5] * m[6] - m[3] * m[8], c02 = m[3] * m[7] - m[4] * m[6];
    const double inv = 1.0 / (m[0] * c00 + m[1] * c01 + m[2] * c02);
    out[0] = c00 * inv; out[1] = (m[2] * m[7] - m[1] * m[8]) * inv; out[2] = (m[1] * m[5] - m[2] * m[4]) * inv;
    out[3] = c01 * inv; out[4] = (m[0] * m[8] - m[2] * m[6]) * inv; out[5] = (m[2] * m[3] - m[0] * m[5]) * inv;
    out[6] = c02 * inv; out[7] = (m[1] * m[6] - m[0] * m[7]) * inv; out[8] = (m[0] * m[4] - m[1] * m[3]) * inv;
}

// Blackbody white of temperature T (K) in CIE XYZ with Y = 1: the chromaticity of Kang et al.,
// "Design of Advanced Color Temperature Control System for HDTV Applications" (2002), piecewise
// rational in T for x and cubic in x for y (ColorUtils.h:150-190).
void blackbody_xyz(double T, double xyz[3])
{
    const double t = T, t2 = t * t, t3 = t2 * t;
    const double x = T < 4000.0 ? -0.2661239e9 / t3 - 0.2343580e6 / t2 + 0.8776956e3 / t + 0.179910
                                : -3.0258469e9 / t3 + 2.1070379e6 / t2 + 0.2226347e3 / t + 0.240390;
    const double x2 = x * x, x3 = x2 * x;
    double y;
    if (T < 2222.0) y = -1.1063814 * x3 - 1.34811020 * x2 + 2.18555832 * x - 0.20219683;
    else if (T < 4000.0) y = -0.9549476 * x3 - 1.37418593 * x2 + 2.09137015 * x - 0.16748867;
    else y = 3.0817580 * x3 - 5.87338670 * x2 + 3.75112997 * x - 0.37001483;
    xyz[0] = x / y; xyz[1] = 1.0; xyz[2] = (1.0 - x - y) / y;
}

// calculateWhiteBalanceTransformRGB_Rec709 (ColorUtils.h:209-226) times the exposure scale.
void color_transform(const rs_tonemap_options& o, float scale, float out[9])
{
    double m[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    if (o.whiteBalance)
    {
        double ma[9], xyzToRgb[9], lmsToXyz[9], invMa[9];
        mat3_mul_d(kXyzToLmsCat02, kRgbToXyz, ma);
        mat3_inverse_d(kRgbToXyz, xyzToRgb);
        mat3_inverse_d(kXyzToLmsCat02, lmsToXyz);
        mat3_mul_d(xyzToRgb, lmsToXyz, invMa);
        double wdXyz[3], wsXyz[3], wd[3], ws[3];
        blackbody_xyz(6500.0, wdXyz);
        blackbody_xyz(o.whitePoint, wsXyz);
        for (int r = 0; r < 3; r++)
        {
            wd[r] = kXyzToLmsCat02[3 * r] * wdXyz[0] + kXyzToLmsCat02[3 * r + 1] * wdXyz[1] + kXyzToLmsCat02[3 * r + 2] * wdXyz[2];
            ws[r] = kXyzToLmsCat02[3 * r] * wsXyz[0] + kXyzToLmsCat02[3 * r + 1] * wsXyz[1] + kXyzToLmsCat02[3 * r + 2] * wsXyz[2];
        }
        double dma[9];
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++) dma[3 * r + c] = (wd[r] / ws[r]) * ma[3 * r + c];
        mat3_mul_d(invMa, dma, m);
    }
    for (int k = 0; k < 9; k++) out[k] = (float)(m[k] * scale);
}

float exposure_scale(const rs_tonemap_options& o)
{
    // ToneMapper::updateColorTransform: 2^compensation, times the manual exposure without auto exposure
    float scale = exp2f(o.exposureCompensation);
    if (!o.autoExposure) scale *= (0.01f * o.filmSpeed) / (o.shutter * o.fNumber * o.fNumber);
    return scale;
}

rs_status validate_tonemap(const rs_tonemap_options* o)
{
    if (o->op > RS_TONEMAP_ACES) return RS_INVALID_ARG;
    if (!(o->fNumber > 0.f) || !(o->shutter > 0.f) || !(o->filmSpeed > 0.f)) return RS_INVALID_ARG;
    if (o->whiteBalance && !(o->whitePoint >= 1905.f && o->whitePoint <= 25000.f)) return RS_INVALID_ARG; // ToneMapper.cpp:80-81
    return RS_OK;
}

} // namespace
} // namespace rs

using namespace rs;

extern "C" RS_API rs_status rs_tonemap_color_transform(const rs_tonemap_options* opts, float* out9)
{
    if (!opts || !out9) return RS_INVALID_ARG;
    if (validate_tonemap(opts) != RS_OK) return RS_INVALID_ARG;
    color_transform(*opts, exposure_scale(*opts), out9);
    return RS_OK;
}

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
    o->whiteBalance = 0;
    o->whitePoint = 6500.f;
}

extern "C" RS_API size_t rs_tonemap_workspace_bytes(void) { return sizeof(double) * (kReduceBlocks + 1); }

extern "C" RS_API rs_status rs_tonemap(const void* colorDev, uint32_t width, uint32_t height, const rs_tonemap_options* opts, void* rgba8Dev,
                                       void* workspaceDev, void* stream)
{
    if (!colorDev || !opts || !rgba8Dev) return RS_INVALID_ARG;
    if (validate_tonemap(opts) != RS_OK) return RS_INVALID_ARG;
    if (opts->autoExposure && !workspaceDev) return RS_INVALID_ARG;
    const uint64_t n64 = (uint64_t)width * height;
    if (n64 == 0) return RS_OK;
    if (n64 > 0xffffffffull) return RS_INVALID_ARG;
    const uint32_t n = (uint32_t)n64;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const float scale = exposure_scale(*opts);
    ColorTransform T;
    color_transform(*opts, scale, T.m);
    const float4* color = static_cast<const float4*>(colorDev);
    double* ws = static_cast<double*>(workspaceDev);
    if (opts->autoExposure)
    {
        k_log_luminance<<<kReduceBlocks, kReduceThreads, 0, s>>>(color, n, ws);
        k_log_luminance_total<<<1, kReduceThreads, 0, s>>>(ws, n);
    }
    k_tonemap<<<(n + 255) / 256, 256, 0, s>>>(color, n, *opts, scale, T, ws ? ws + kReduceBlocks : nullptr, static_cast<uint32_t*>(rgba8Dev));
    return cudaGetLastError() == cudaSuccess ? RS_OK : RS_CUDA_ERROR;
}
