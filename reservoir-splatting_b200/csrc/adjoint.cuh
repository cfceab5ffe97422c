// Path-replay adjoint of the resolved estimator (no reference counterpart).
//
// A pixel's colour is f(y) * W (ResolveReSTIR.cs.slang:45-63), y being the path its final
// reservoir selected.  k_backward holds y, W, the sampling densities and the MIS weights at their
// values for the current materials and differentiates f(y) with respect to each material's
// baseColor, roughness and metallic (the BSDF factor of every vertex) and its emitted radiance (the
// Le the path carries).  f(y) is the reconnection-shift evaluation of the pixel's record at its own
// primary hit (handleReconnectionHit / pathReconnectionShift, PathTracer.slang:1177-1397,
// ShiftMapping.slang:430-513) without the visibility ray, which no material changes.  A per-channel
// factor k = integrand / f(y), held fixed, makes the differentiated function equal the resolved
// colour exactly at the current materials.  E[d f(y)/d theta * W] is the derivative of the pixel
// integral because W is a contribution weight of y, so the gradient is unbiased.
//
// Only the final reservoirs are needed (the checkpoint); shading data, BSDF terms and the emitter
// are recomputed.  A path of four or more vertices carries its suffix (x3 on) as radiance in the
// record; adj_replay_suffix re-runs the path tracer from x3 with the sample generator's state and
// the bounce counters and flags the record saved there, which gives the suffix's vertices and
// emitter bit for bit.
#pragma once
#include "core/material_grad.h"

namespace rs {

enum : uint32_t { kAdjReplayed = 0, kAdjSkipped = 1, kAdjNoEmitter = 2, kAdjValueMismatch = 3 };
constexpr uint32_t kAdjMaxFactors = 8; // BSDF factors on a replayed path (x1, x2 and the suffix)

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

__device__ __forceinline__ bool adj_finished(const DevCtx& C, uint32_t bounces) // finished_bounces
{
    uint32_t d = bounces & 0xffu, sp = (bounces >> 8) & 0xffu, t = (bounces >> 16) & 0xffu;
    return (d + sp + t) > C.maxSurfaceBounces || d > C.maxDiffuseBounces || sp > C.maxSpecularBounces || t > C.maxTransmissionBounces;
}

// The suffix of a path of four or more vertices: handle_hit re-run from x3 (the closest hit from x2
// along the stored direction) with the sample generator's state, bounce counters and flags the
// record saved there, taking every draw the path tracer takes (the candidate selections', Russian
// roulette's, the light and BSDF samples'), up to the light sample that ends the path.  Appends the
// BSDF factor of each suffix vertex (the sampled lobe's; at the last vertex all lobes' toward the
// light) and sets the emitter, its radiance and the replayed suffix radiance S, which equals the
// record's irradiance when the geometry has not moved since the record was made.  Emitted radiance
// beyond x2 that a BSDF sample reaches counts only after a delta lobe (handle_hit's computeEmissive),
// whose factor is no BSDF evaluation: such paths, delta lobes on the suffix and paths of more than
// kAdjMaxFactors factors are not replayed (adj_pixel then holds the suffix fixed).  A light
// sample of the environment map leaves emitter = kInvalidIndex: its radiance is no material's.
// The host accepts emissive triangles and an environment map here (no analytic lights).
__device__ __noinline__ bool adj_replay_suffix(const DevCtx& C, const Recon& rd, const ShadingData& sd2, uint32_t& nv, uint32_t* mat,
                                               BsdfGrad* V, uint32_t& emitter, f3& Le, f3& S)
{
    uint32_t bounces, flags;
    suffix_state_unpack(rd.suffixState, bounces, flags);
    SampleGen sg; sg.state = rd.suffixSeed; sg.kind = C.sgKind;
    f3 thp = mk3(1.f), dir = rd.secondWo;
    f3 origin = computeRayOrigin(sd2.posW, dot(sd2.faceN, dir) >= 0.f ? sd2.faceN : -sd2.faceN);
    const bool haveLights = C.lights.count > 0, haveEnv = C.env->present != 0;
    // handle_hit's light-type probabilities: with the emissive triangles alone p = {0, haveLights}
    // and the selection pdf is 1; without an env map pEnv = 0, so u - pEnv is u
    const float pEnv = haveEnv ? C.pEnvLight : 0.f;
    const float pEmissive = haveEnv ? C.pEmissiveLight : (haveLights ? 1.f : 0.f);
    for (uint32_t v = 3; v < rd.pathLength; v++)
    {
        HitInfo h; float t;
        if (!trace_closest(C.bvh, mk_ray(origin, dir, 0.f, kRayTMax), h, t, C.fault)) return false;
        ShadingData sd = dev_sd(C, h, dir);
        BsdfData d = dev_instance(C, sd);
        const bool lightSampled = (flags & (kPLightUpper | kPLightLower)) != 0;
        if (haveLights && (!lightSampled || (flags & kPDelta)) && any_gt0(d.emission))
            sampleNext1D(sg); // the emissive candidate's selection draw (cand_add_vertex)
        if (adj_finished(C, bounces)) return false;
        origin = sd_ray_origin(sd, true);
        const uint32_t lobeTypes = mi_lobe_types(d);
        flags &= ~(kPLightUpper | kPLightLower);
        if ((lobeTypes & kLobeNonDelta) != 0)
        {
            const bool sampleUpper = (lobeTypes & kLobeNonDeltaReflection) != 0;
            const bool sampleLower = (lobeTypes & kLobeNonDeltaTransmission) != 0;
            TriangleLightSample tls;
            f3 lsLi = mk3(0.f), lsOrigin = mk3(0.f), lsDir = mk3(0.f);
            float lsPdf = 0.f, lsDistance = 0.f, selectionPdf = 0.f;
            bool sampled = false, lsEnv = false;
            float u = sampleNext1D(sg); // the type-selection draw
            if (haveEnv && u < pEnv)
            {
                selectionPdf = pEnv;
                lsEnv = true;
                f2 r2; r2.x = sampleNext1D(sg); r2.y = sampleNext1D(sg);
                const EnvSample es = dev_env_sample(C.env, r2);
                lsDir = es.dir; lsPdf = es.pdf;
                lsLi = lsPdf > 0.f ? es.Le / lsPdf : mk3(0.f);
                lsOrigin = computeRayOrigin(sd.posW, dot(sd.faceN, lsDir) >= 0.f ? sd.faceN : -sd.faceN);
                lsDistance = kRayTMax;
                sampled = any_gt0(lsLi);
            }
            else if (u - pEnv < pEmissive)
            {
                selectionPdf = haveEnv ? pEmissive : 1.f;
                if (sample_emissive(C.lights, sd.posW, sg, tls))
                {
                    lsLi = tls.pdf > 0.f ? tls.Le / tls.pdf : mk3(0.f);
                    lsPdf = tls.pdf;
                    f3 lightPos = computeRayOrigin(tls.posW, tls.normalW);
                    f3 toL = lightPos - sd.posW;
                    lsOrigin = computeRayOrigin(sd.posW, dot(sd.faceN, toL) >= 0.f ? sd.faceN : -sd.faceN);
                    f3 toLight = lightPos - lsOrigin;
                    lsDistance = length(toLight);
                    lsDir = normalize(toLight);
                    sampled = any_gt0(lsLi);
                }
            }
            bool validSample = false;
            if (sampled)
            {
                float NdotL = dot(sd_oriented_face_normal(sd), lsDir);
                validSample = !((!sampleUpper && NdotL >= -kMinCosTheta) || (!sampleLower && NdotL <= kMinCosTheta));
                if (validSample) { lsPdf *= selectionPdf; lsLi /= selectionPdf; }
            }
            if (sampleUpper) flags |= kPLightUpper;
            if (sampleLower) flags |= kPLightLower;
            if (validSample)
            {
                const BsdfPair bp = mi_eval_pair(sd, d, 0u, lsDir);
                const float misWeight = dev_mis(C, lsPdf, bp.totalPdf);
                const f3 Lr = bp.totalBsdf * misWeight * lsLi;
                if (any_gt0(Lr) && dev_visible(C, mk_ray(lsOrigin, lsDir, 0.f, lsDistance)))
                {
                    sampleNext1D(sg); // the light candidate's selection draw
                    if (rd.lightIsNEE && v + 1 == rd.pathLength)
                    {
                        if (nv == kAdjMaxFactors) return false;
                        mat[nv] = sd.materialID;
                        V[nv++] = mi_eval_grad(sd, d, C.materials[sd.materialID], 0u, lsDir);
                        S = thp * Lr;
                        Le = lsLi * lsPdf;
                        emitter = lsEnv ? kInvalidIndex
                                        : dev_emitter_of(C, dev_sd(C, hit_tri(C.lights.tris[tls.triangleIndex].sceneTri, tls.uv.x, tls.uv.y), lsDir));
                        return true;
                    }
                }
            }
        }
        if (C.useRussianRoulette)
        {
            float ur = sampleNext1D(sg);
            const float prob = f_max(0.f, 1.f - luminance(thp));
            if (ur < prob) return false;
            thp /= 1.f - prob;
        }
        BSDFSample result;
        result.wo = mk3(0.f); result.pdf = 0.f; result.weight = mk3(0.f); result.lobeType = 0;
        float totalPdf;
        const bool valid = mi_sample_total_pdf(sd, d, 1u, sg, result, totalPdf);
        uint32_t comp = 0; // handle_hit's componentType
        const bool specOrDelta = (result.lobeType & kLobeSpecular) || (result.lobeType & kLobeDelta);
        if (result.lobeType & kLobeDiffuseReflection) { if (specOrDelta) comp = 3; }
        else if (result.lobeType & kLobeDiffuseTransmission) comp = 1;
        else if (specOrDelta) comp = 2;
        if (!valid || (result.lobeType & kLobeDelta) || (comp != 0 && comp != 2) || nv == kAdjMaxFactors) return false;
        mat[nv] = sd.materialID;
        V[nv++] = mi_eval_grad(sd, d, C.materials[sd.materialID], 1u << comp, result.wo);
        dir = result.wo;
        thp *= result.weight;
        flags &= ~(4u | kPSpecular | kPDelta);
        if (result.lobeType & kLobeReflection)
        {
            const bool isDiffuse = (result.lobeType & kLobeDiffuseReflection) || mi_roughness(d) > C.specularRoughnessThreshold;
            if (isDiffuse) bounces += 1u;
            else { bounces += (1u << 8); flags |= kPSpecular; }
        }
        if (adj_finished(C, bounces)) return false; // the path ends here: no later light sample
        if (C.disableCaustics && (bounces & 0xffu) > 0 && (flags & kPSpecular)) return false;
    }
    return false;
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
    // a primary miss sees the environment map: no material on the path
    if (rd.pathLength == 1 && rd.lightIsDistant) return;

    uint32_t nv = 0, emitter = kInvalidIndex;
    uint32_t mat[kAdjMaxFactors];
    BsdfGrad V[kAdjMaxFactors];
    float s = 1.f;
    f3 Le = rd.irradiance;
    bool suffixHeld = false;
    ShadingData sd1 = dev_sd(C, rd.firstHit, -rd.firstWi);
    if (rd.pathLength == 1)
    {
        emitter = dev_emitter_of(C, sd1);
    }
    else
    {
        BsdfData d1 = dev_instance(C, sd1);
        f3 origin = sd_ray_origin(sd1, !rd.transmissionEvent);
        // a length-2 path to the environment stores a direction as its second hit and has no
        // geometry term (handleReconnectionHit's secondHitIsDistant)
        const bool distant2 = rd.pathLength == 2 && rd.lightIsDistant;
        float jac = 1.f;
        f3 dir;
        if (distant2) dir = hit_as_direction(rd.secondHit);
        else
        {
            ShadingData sec = dev_sd(C, rd.secondHit, mk3(0.f));
            f3 off = sec.posW - sd1.posW;
            jac = f_abs(dot(sec.faceN, -normalize(off))) / dot(off, off);
            dir = normalize(sec.posW - origin);
        }
        uint32_t mask1 = 1u << rd.firstComp;
        float lobePdf = mi_pdf(sd1, d1, mask1, dir), totalPdf = mi_pdf(sd1, d1, 0u, dir);
        mat[0] = sd1.materialID;
        if (rd.pathLength == 2)
        {
            float lightPdf = rd.lightPdf / jac;
            if (rd.lightIsNEE)
            {
                V[0] = mi_eval_grad(sd1, d1, C.materials[sd1.materialID], 0u, dir);
                if (!any_gt0(V[0].value) || totalPdf == 0.f) return;
                s = dev_mis(C, lightPdf, totalPdf) / lightPdf;
            }
            else
            {
                V[0] = mi_eval_grad(sd1, d1, C.materials[sd1.materialID], mask1, dir);
                if (!any_gt0(V[0].value) || lobePdf == 0.f) return;
                s = dev_mis(C, totalPdf, lightPdf) / lobePdf;
            }
            nv = 1;
            if (!distant2) emitter = dev_emitter_of(C, dev_sd(C, rd.secondHit, dir));
        }
        else
        {
            V[0] = mi_eval_grad(sd1, d1, C.materials[sd1.materialID], mask1, dir);
            if (!any_gt0(V[0].value) || lobePdf == 0.f) return;
            ShadingData sd2 = dev_sd(C, rd.secondHit, dir);
            BsdfData d2 = dev_instance(C, sd2);
            uint32_t mask2 = 1u << rd.secondComp;
            float lsp = mi_pdf(sd2, d2, mask2, rd.secondWo), tp = mi_pdf(sd2, d2, 0xFu, rd.secondWo);
            if (!any_gt0(mi_eval(sd2, d2, 0xFu, rd.secondWo))) return;
            mat[1] = sd2.materialID;
            nv = 2;
            if (rd.pathLength > 3)
            {
                // pathReconnectionShift's lobe-specific x2 term; the suffix follows from x3
                if (!(lsp > 0.f)) return;
                V[1] = mi_eval_grad(sd2, d2, C.materials[sd2.materialID], mask2, rd.secondWo);
                s = (1.f / lobePdf) * (1.f / lsp);
                f3 S;
                const bool replayed = C.sgKind == kSgTinyUniform && adj_replay_suffix(C, rd, sd2, nv, mat, V, emitter, Le, S) &&
                                      S.x == rd.irradiance.x && S.y == rd.irradiance.y && S.z == rd.irradiance.z;
                if (!replayed)
                {
                    // the suffix is held fixed at the record's radiance and only x1 and x2 are
                    // differentiated: a delta lobe past x2, a PCG32 state, or a suffix traced in
                    // geometry that has moved since (a record reused from an earlier frame)
                    nv = 2;
                    emitter = kInvalidIndex;
                    Le = rd.irradiance;
                    suffixHeld = true;
                    atomicAdd(cnt + kAdjSkipped, 1u);
                }
            }
            else
            {
                if (rd.lightIsNEE)
                {
                    V[1] = mi_eval_grad(sd2, d2, C.materials[sd2.materialID], 0xFu, rd.secondWo);
                    s = (1.f / lobePdf) * (dev_mis(C, rd.lightPdf, tp) / rd.lightPdf);
                }
                else
                {
                    if (!(lsp > 0.f)) return;
                    V[1] = mi_eval_grad(sd2, d2, C.materials[sd2.materialID], mask2, rd.secondWo);
                    s = (1.f / lobePdf) * (dev_mis(C, tp, rd.lightPdf) / lsp);
                }
                if (!rd.lightIsDistant)
                {
                    f3 o2 = computeRayOrigin(sd2.posW, dot(sd2.faceN, rd.secondWo) >= 0.f ? sd2.faceN : -sd2.faceN);
                    HitInfo h; float t;
                    if (trace_closest(C.bvh, mk_ray(o2, rd.secondWo, 0.f, kRayTMax), h, t, C.fault))
                        emitter = dev_emitter_of(C, dev_sd(C, h, rd.secondWo));
                    // a light sample whose ray slips through the seam between two triangles of the light
                    if (emitter == kInvalidIndex && rd.lightIsNEE) emitter = emissive_material_with_radiance(C.lights, rd.irradiance);
                }
            }
        }
    }
    // before[v] = V[0] ... V[v-1]; the other factors of V[v] are before[v] * (V[v+1] ...)
    f3 before[kAdjMaxFactors];
    f3 prod = mk3(1.f);
    for (uint32_t v = 0; v < nv; v++) { before[v] = prod; prod = prod * V[v].value; }
    const f3 value = prod * Le * s;
    const f3 k = mk3(value.x != 0.f ? r.integrand.x / value.x : 1.f, value.y != 0.f ? r.integrand.y / value.y : 1.f,
                     value.z != 0.f ? r.integrand.z / value.z : 1.f);
    atomicAdd(cnt + kAdjReplayed, 1u);
    // a path that ends at the environment map carries its radiance, no material's
    if (emitter == kInvalidIndex && !rd.lightIsDistant && !suffixHeld) atomicAdd(cnt + kAdjNoEmitter, 1u);
    // a suffix path's value is checked through the record's irradiance (a replayed suffix radiance
    // equals it bit for bit); the suffix's densities and MIS weights fall into k
    const f3 check = rd.pathLength > 3 ? V[0].value * V[1].value * rd.irradiance * s : value;
    f3 diff = check - r.integrand;
    if (f_abs(diff.x) + f_abs(diff.y) + f_abs(diff.z) > 1e-3f * (f_abs(r.integrand.x) + f_abs(r.integrand.y) + f_abs(r.integrand.z)))
        atomicAdd(cnt + kAdjValueMismatch, 1u);

    const f3 g = mk3(gc.x, gc.y, gc.z) * W * k;
    if (emitter != kInvalidIndex)
    {
        f3 dLe = g * prod * s;
        const uint32_t e = emitter * kGradStride + kGradEmissive;
        adj_add(acc, e + 0, dLe.x); adj_add(acc, e + 1, dLe.y); adj_add(acc, e + 2, dLe.z);
    }
    f3 after = mk3(1.f);
    for (uint32_t v = nv; v-- > 0;)
    {
        f3 common = g * (before[v] * after) * Le * s;
        f3 dB = common * V[v].dBase;
        f3 dR = common * V[v].dRough;
        f3 dM = common * V[v].dMetal;
        const uint32_t m = mat[v] * kGradStride;
        adj_add(acc, m + kGradBase + 0, dB.x); adj_add(acc, m + kGradBase + 1, dB.y); adj_add(acc, m + kGradBase + 2, dB.z);
        adj_add(acc, m + kGradRough, dR.x + dR.y + dR.z);
        adj_add(acc, m + kGradMetal, dM.x + dM.y + dM.z);
        after = after * V[v].value;
    }
}

// Adds d loss / d material parameters (numMaterials x 8: baseColor.xyz, roughness, emissive.xyz, metallic)
// for d loss / d colour `gradColor`, over the reservoirs `res` / `rec` of one frame, into the FP64
// accumulator `acc`.  A grid of at most a few blocks per SM walks the pixels; each block stages its
// sums in shared memory (when they fit) and flushes them with one atomic per non-zero entry.
// 10 blocks of 128 per SM (the replay's per-path arrays live in the local frame either way), the
// grid sized to them: 0.194 ms per 512^2 frame at path length 4, against 0.233 at 8 blocks, 0.220 at
// 12 and 0.256 at 4 blocks of 128 registers.
__global__ void __launch_bounds__(kAdjointThreads, kAdjointBlocksPerSm) k_backward(uint32_t slot, ResPlanes res, RecPlanes rec, const float4* __restrict__ gradColor,
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
