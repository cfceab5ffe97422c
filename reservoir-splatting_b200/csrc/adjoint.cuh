// Path-replay adjoint of the resolved estimator (no reference counterpart).
//
// A pixel's colour is f(y) * W (ResolveReSTIR.cs.slang:45-63), y being the path its final
// reservoir selected.  k_backward holds y, W, the sampling densities and the MIS weights at their
// values for the current materials and differentiates f(y) with respect to each material's
// baseColor and roughness (the BSDF factors at x1 and x2) and its emitted radiance (the Le the
// path carries).  f(y) is the reconnection-shift evaluation of the pixel's record at its own
// primary hit (handleReconnectionHit / pathReconnectionShift, PathTracer.slang:1177-1397,
// ShiftMapping.slang:430-513) without the visibility ray, which no material changes.  A per-channel
// factor k = integrand / f(y), held fixed, makes the differentiated function equal the resolved
// colour exactly at the current materials.  E[d f(y)/d theta * W] is the derivative of the pixel
// integral because W is a contribution weight of y, so the gradient is unbiased.
//
// Only the final reservoirs are needed (the checkpoint); shading data, BSDF terms and the emitter
// behind x2 (one closest-hit ray) are recomputed.  Paths of more than three vertices carry suffix
// radiance from materials the record does not name: they are counted and skipped, and the host
// entry point accepts only maxSurfaceBounces <= 1, where none occur.
#pragma once
#include "core/material_grad.h"

namespace rs {

enum : uint32_t { kAdjReplayed = 0, kAdjTooLong = 1, kAdjNoEmitter = 2, kAdjValueMismatch = 3 };

// The emitter of a path is the triangle its last vertex lies on: the primary hit (length 1), the
// reconnection vertex x2 (length 2: the record's second hit is the light sample's or the BSDF
// hit's triangle) or the closest hit from x2 along the stored direction (length 3).  Its emissive
// material owns the Le the path carries.  The forward pass already decided that the triangle emits
// toward the path, so its facing is not tested again (a grazing light would flip the test by
// rounding and drop the path's Le gradient).
__device__ __forceinline__ uint32_t dev_emitter_of(const DevCtx& C, const ShadingData& sd)
{
    const MaterialData& m = C.materials[sd.materialID];
    return (m.emissive[0] > 0.f || m.emissive[1] > 0.f || m.emissive[2] > 0.f) ? sd.materialID : kInvalidIndex;
}

// Per-pixel terms are FP32; their sums are FP64, because the roughness terms of sharp GGX lobes are
// large and of both signs and an FP32 sum of them loses the result.
__device__ __forceinline__ void adj_add(double* acc, uint32_t idx, float v)
{
    if (v != 0.f) atomicAdd(acc + idx, (double)v);
}

__device__ inline void adj_pixel(const DevCtx& C, const ResPlanes& res, const RecPlanes& rec, const float4* gradColor, uint32_t i,
                                 double* acc, uint32_t* cnt)
{
    Res r = load_res(res, i);
    const float W = res_ucw(r);
    if (!(W > 0.f)) return;
    float4 gc = __ldg(gradColor + i);
    if (gc.x == 0.f && gc.y == 0.f && gc.z == 0.f) return;
    Recon rd = load_rec(rec, i);
    if (rd.pathLength == 0) return;
    if (rd.pathLength > 3) { atomicAdd(cnt + kAdjTooLong, 1u); return; }

    uint32_t nv = 0, emitter = kInvalidIndex;
    uint32_t mat[2] = {kInvalidIndex, kInvalidIndex};
    BsdfGrad V[2];
    float s = 1.f;
    ShadingData sd1 = dev_sd(C, rd.firstHit, -rd.firstWi);
    if (rd.pathLength == 1)
    {
        emitter = dev_emitter_of(C, sd1);
    }
    else
    {
        BsdfData d1 = dev_instance(C, sd1);
        f3 origin = sd_ray_origin(sd1, !rd.transmissionEvent);
        ShadingData sec = dev_sd(C, rd.secondHit, mk3(0.f));
        f3 off = sec.posW - sd1.posW;
        float jac = f_abs(dot(sec.faceN, -normalize(off))) / dot(off, off);
        f3 dir = normalize(sec.posW - origin);
        uint32_t mask1 = 1u << rd.firstComp;
        float lobePdf = mi_pdf(sd1, d1, mask1, dir), totalPdf = mi_pdf(sd1, d1, 0u, dir);
        mat[0] = sd1.materialID;
        if (rd.pathLength == 2)
        {
            float lightPdf = rd.lightPdf / jac;
            if (rd.lightIsNEE)
            {
                V[0] = mi_eval_grad(sd1, d1, 0u, dir);
                if (!any_gt0(V[0].value) || totalPdf == 0.f) return;
                s = dev_mis(C, lightPdf, totalPdf) / lightPdf;
            }
            else
            {
                V[0] = mi_eval_grad(sd1, d1, mask1, dir);
                if (!any_gt0(V[0].value) || lobePdf == 0.f) return;
                s = dev_mis(C, totalPdf, lightPdf) / lobePdf;
            }
            nv = 1;
            emitter = dev_emitter_of(C, dev_sd(C, rd.secondHit, dir));
        }
        else
        {
            V[0] = mi_eval_grad(sd1, d1, mask1, dir);
            if (!any_gt0(V[0].value) || lobePdf == 0.f) return;
            ShadingData sd2 = dev_sd(C, rd.secondHit, dir);
            BsdfData d2 = dev_instance(C, sd2);
            uint32_t mask2 = 1u << rd.secondComp;
            float lsp = mi_pdf(sd2, d2, mask2, rd.secondWo), tp = mi_pdf(sd2, d2, 0xFu, rd.secondWo);
            if (!any_gt0(mi_eval(sd2, d2, 0xFu, rd.secondWo))) return;
            if (rd.lightIsNEE)
            {
                V[1] = mi_eval_grad(sd2, d2, 0xFu, rd.secondWo);
                s = (1.f / lobePdf) * (dev_mis(C, rd.lightPdf, tp) / rd.lightPdf);
            }
            else
            {
                if (!(lsp > 0.f)) return;
                V[1] = mi_eval_grad(sd2, d2, mask2, rd.secondWo);
                s = (1.f / lobePdf) * (dev_mis(C, tp, rd.lightPdf) / lsp);
            }
            nv = 2;
            mat[1] = sd2.materialID;
            f3 o2 = computeRayOrigin(sd2.posW, dot(sd2.faceN, rd.secondWo) >= 0.f ? sd2.faceN : -sd2.faceN);
            HitInfo h; float t;
            if (trace_closest(C.bvh, mk_ray(o2, rd.secondWo, 0.f, kRayTMax), h, t, C.fault))
                emitter = dev_emitter_of(C, dev_sd(C, h, rd.secondWo));
            // a light sample whose ray slips through the seam between two triangles of the light
            if (emitter == kInvalidIndex && rd.lightIsNEE) emitter = emissive_material_with_radiance(C.lights, rd.irradiance);
        }
    }
    const f3 A = nv >= 1 ? V[0].value : mk3(1.f);
    const f3 B = nv == 2 ? V[1].value : mk3(1.f);
    const f3 Le = rd.irradiance;
    const f3 value = A * B * Le * s;
    const f3 k = mk3(value.x != 0.f ? r.integrand.x / value.x : 1.f, value.y != 0.f ? r.integrand.y / value.y : 1.f,
                     value.z != 0.f ? r.integrand.z / value.z : 1.f);
    atomicAdd(cnt + kAdjReplayed, 1u);
    if (emitter == kInvalidIndex) atomicAdd(cnt + kAdjNoEmitter, 1u);
    f3 diff = value - r.integrand;
    if (f_abs(diff.x) + f_abs(diff.y) + f_abs(diff.z) > 1e-3f * (f_abs(r.integrand.x) + f_abs(r.integrand.y) + f_abs(r.integrand.z)))
        atomicAdd(cnt + kAdjValueMismatch, 1u);

    const f3 g = mk3(gc.x, gc.y, gc.z) * W * k;
    if (emitter != kInvalidIndex)
    {
        f3 dLe = g * A * B * s;
        const uint32_t e = emitter * kGradStride + kGradEmissive;
        adj_add(acc, e + 0, dLe.x); adj_add(acc, e + 1, dLe.y); adj_add(acc, e + 2, dLe.z);
    }
    for (uint32_t v = 0; v < nv; v++)
    {
        f3 common = g * (v == 0 ? B : A) * Le * s;
        f3 dB = common * V[v].dBase;
        f3 dR = common * V[v].dRough;
        const uint32_t m = mat[v] * kGradStride;
        adj_add(acc, m + kGradBase + 0, dB.x); adj_add(acc, m + kGradBase + 1, dB.y); adj_add(acc, m + kGradBase + 2, dB.z);
        adj_add(acc, m + kGradRough, dR.x + dR.y + dR.z);
    }
}

// Adds d loss / d material parameters (numMaterials x 8: baseColor.xyz, roughness, emissive.xyz, 0)
// for d loss / d colour `gradColor`, over the reservoirs `res` / `rec` of one frame, into the FP64
// accumulator `acc`.  A grid of at most a few blocks per SM walks the pixels; each block stages its
// sums in shared memory (when they fit) and flushes them with one atomic per non-zero entry.
__global__ void __launch_bounds__(kAdjointThreads) k_backward(uint32_t slot, ResPlanes res, RecPlanes rec, const float4* __restrict__ gradColor,
                                                              double* __restrict__ acc, uint32_t numMaterials,
                                                              unsigned long long* __restrict__ stats)
{
    extern __shared__ double sGrad[];
    __shared__ uint32_t sCnt[4];
    const DevCtx& C = c_ctx[slot];
    const uint32_t M = numMaterials * kGradStride;
    const bool staged = M <= kAdjointSharedDoubles;
    if (staged)
        for (uint32_t k = threadIdx.x; k < M; k += blockDim.x) sGrad[k] = 0.0;
    if (threadIdx.x < 4) sCnt[threadIdx.x] = 0u;
    __syncthreads();
    double* dst = staged ? sGrad : acc;
    const uint32_t N = C.W * C.H;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < N; i += gridDim.x * blockDim.x)
        adj_pixel(C, res, rec, gradColor, i, dst, sCnt);
    __syncthreads();
    if (staged)
        for (uint32_t k = threadIdx.x; k < M; k += blockDim.x)
        {
            double v = sGrad[k];
            if (v != 0.0) atomicAdd(acc + k, v);
        }
    if (threadIdx.x < 4 && sCnt[threadIdx.x]) atomicAdd(stats + threadIdx.x, (unsigned long long)sCnt[threadIdx.x]);
}

// grad += acc (the caller's FP32 gradient accumulates across calls).
__global__ void __launch_bounds__(256) k_grad_flush(const double* __restrict__ acc, float* __restrict__ grad, uint32_t n)
{
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k < n) grad[k] += (float)acc[k];
}

} // namespace rs
