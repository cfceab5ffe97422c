// Device-side per-pixel logic of the Reservoir Splatting pass: reservoirs,
// reconnection records, the candidate path tracer and the shift mappings.
//
// Each function names the reference lines it implements.  Device records are
// register-resident structs; the kernels (kernels.cu) move them to and from the
// structure-of-arrays planes in HBM.
#pragma once
#include "bvh.cuh"
#include "core/camera.h"
#include "core/lights.h"
#include "core/envmap.h"
#include "core/analytic_lights.h"

namespace rs {

constexpr uint32_t kNumRenderPasses = 8; // ReservoirSplatting.cpp:36
constexpr float kConfidenceCap = 20.f;   // Reservoir.slang:75

// Options and per-frame constants, passed by value to every kernel.
struct DevCtx
{
    BvhView bvh;
    const float4* prevTri; // the previous frame's triangles (scene order; bvh.tri when nothing moved)
    const MaterialData* materials;
    LightView lights;
    const EnvMapView* env;  // environment map (present = 0 without one), in device memory
    AnalyticLightView analytic; // the scene's analytic lights (count 0: none)
    float pEnvLight, pEmissiveLight, pAnalyticLight; // light-type selection probabilities (PathTracer.slang:606-622)
    CameraData camera;      // gScene.camera of this frame
    CameraData prevCamera;  // previous frame's camera (motion vectors)
    CameraManager cm;
    const CameraTable* camTable; // frame constants of orient_camera (k_camera_table)
    uint32_t W, H;
    uint32_t frameCount, seed;
    uint32_t useFixedSeed, fixedSeed;
    uint32_t sgKind;
    uint32_t spp;
    uint32_t maxSurfaceBounces, maxDiffuseBounces, maxSpecularBounces, maxTransmissionBounces;
    uint32_t useRussianRoulette, misHeuristic, disableCaustics;
    float misPowerExponent; // PowerExp heuristic (misHeuristic 2)
    float specularRoughnessThreshold;
    uint32_t useConfTemporal, useConfSpatial;
    uint32_t gatherOption, scatterBackupMIS, numTimePartitions;
    uint32_t neighborCount;
    float spatialGatherRadius;
    uint32_t* fault; // device status word: bit 0 traversal stack overflow
};

__device__ __forceinline__ uint32_t pass_seed(const DevCtx& C, uint32_t k)
{
    return C.useFixedSeed ? C.fixedSeed + k : kNumRenderPasses * (C.frameCount + C.seed) + k;
}
__device__ __forceinline__ bool valid_float(const DevCtx& C, f2 p) { return p.x >= 0.f && p.y >= 0.f && p.x < (float)C.W && p.y < (float)C.H; }
__device__ __forceinline__ bool valid_int(const DevCtx& C, int x, int y) { return x >= 0 && y >= 0 && x < (int)C.W && y < (int)C.H; }

// Pixel of this thread when each warp covers an 8 x 4 pixel tile and the warps of a block sit two
// tiles wide (a 128-thread block covers 16 x 8 pixels): a warp's primary rays leave from a compact
// patch, so their traversals share more nodes and cache lines than a 32 x 1 row.  Launch with
// tiled_blocks().  False for threads past the image edge.
__device__ __forceinline__ bool tiled_pixel(uint32_t W, uint32_t H, uint32_t& i)
{
    const uint32_t rowsPerBlock = (blockDim.x >> 5) * 2u;
    const uint32_t tilesX = (W + 15u) / 16u;
    const uint32_t bx = blockIdx.x % tilesX, by = blockIdx.x / tilesX;
    const uint32_t w = threadIdx.x >> 5, l = threadIdx.x & 31u;
    const uint32_t x = bx * 16u + (w & 1u) * 8u + (l & 7u);
    const uint32_t y = by * rowsPerBlock + (w >> 1) * 4u + (l >> 3);
    if (x >= W || y >= H) return false;
    i = y * W + x;
    return true;
}

// The work of one block of a stage kernel: its block index within the instance's grid and, for
// pixel kernels, the warp tile width tw (8, 16 or 32: a warp covers tw x 32/tw pixels, two warps
// side by side, the rest stacked).  The plain launch uses {blockIdx.x, 8}: tiled_pixel's mapping.
// Results do not depend on the mapping (every pixel's work is independent of which thread does it).
struct Blk { uint32_t b; uint32_t tw; };

__device__ __forceinline__ bool tiled_pixel_at(uint32_t W, uint32_t H, Blk blk, uint32_t& i)
{
    const uint32_t tw = blk.tw, th = 32u / tw;
    const uint32_t rowsPerBlock = (blockDim.x >> 6) * th;
    const uint32_t tilesX = (W + 2u * tw - 1u) / (2u * tw);
    const uint32_t bx = blk.b % tilesX, by = blk.b / tilesX;
    const uint32_t w = threadIdx.x >> 5, l = threadIdx.x & 31u;
    const uint32_t x = bx * 2u * tw + (w & 1u) * tw + (l % tw);
    const uint32_t y = by * rowsPerBlock + (w >> 1) * th + l / tw;
    if (x >= W || y >= H) return false;
    i = y * W + x;
    return true;
}
// Blocks of `threads` (a multiple of 64) that tiled_pixel_at needs for a W x H image at tile width tw.
RS_HD uint32_t tiled_blocks_tw(uint32_t W, uint32_t H, uint32_t threads, uint32_t tw)
{
    const uint32_t rows = (threads / 64u) * (32u / tw);
    return ((W + 2u * tw - 1u) / (2u * tw)) * ((H + rows - 1u) / rows);
}

// A flattened work queue over the instances of a batch: instance k owns the work items
// [start[k], start[k + 1]) (blocks of its own grid), runs with context slot[k] and warp tile width
// tile[k].  A persistent launch strides over all `total` items.
struct BatchQueue
{
    const uint32_t* start; // count + 1 entries
    const uint32_t* slot;
    const uint32_t* tile;
    uint32_t count, total;
};
__device__ __forceinline__ uint32_t batch_instance(const BatchQueue& q, uint32_t t)
{
    uint32_t lo = 0, hi = q.count; // start[lo] <= t < start[hi]
    while (hi - lo > 1u)
    {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(q.start + mid) <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}
__device__ __forceinline__ Blk batch_blk(const BatchQueue& q, uint32_t inst, uint32_t t)
{
    Blk b;
    b.b = t - __ldg(q.start + inst);
    b.tw = __ldg(q.tile + inst);
    return b;
}

__device__ __forceinline__ bool dev_visible(const DevCtx& C, const Ray& r) { return trace_visible(C.bvh, r, C.fault); }
// The environment light's evaluation, pdf and sampling as calls: the kernels reach them only on
// misses and env light samples, and inlined they would add their registers to every kernel's
// triangle work.
static __device__ __noinline__ f3 dev_env_eval(const EnvMapView* E, f3 dir) { return env_eval(*E, dir); }
static __device__ __noinline__ float dev_env_eval_pdf(const EnvMapView* E, f3 dir) { return env_eval_pdf(*E, dir); }
struct EnvSample { f3 dir; float pdf; f3 Le; };
static __device__ __noinline__ EnvSample dev_env_sample(const EnvMapView* E, f2 rnd)
{
    EnvSample r;
    env_sample(*E, rnd, r.dir, r.pdf, r.Le);
    return r;
}
__device__ __forceinline__ ShadingData dev_sd(const DevCtx& C, const HitInfo& h, f3 rayDir)
{
    return load_shading_data(reinterpret_cast<const f4*>(C.bvh.tri), C.materials, h, rayDir);
}
__device__ __forceinline__ BsdfData dev_instance(const DevCtx& C, const ShadingData& sd)
{
    return setup_material(C.materials[sd.materialID], sd.frontFacing);
}
__device__ __forceinline__ float dev_mis(const DevCtx& C, float p0, float p1) // PathTracer.slang:480-508
{
    if (C.misHeuristic == 1u)
    {
        float q0 = (1.f * p0) * (1.f * p0), q1 = (1.f * p1) * (1.f * p1);
        return q0 / (q0 + q1);
    }
    if (C.misHeuristic == 2u)
    {
        float q0 = f_pow_pos(1.f * p0, C.misPowerExponent), q1 = f_pow_pos(1.f * p1, C.misPowerExponent);
        return q0 / (q0 + q1);
    }
    float q0 = 1.f * p0, q1 = 1.f * p1;
    return q0 / (q0 + q1);
}
__device__ __forceinline__ void dev_orient(const DevCtx& C, CameraData& c, float t)
{
    // the memoised cameras of the table, for times with the same bits (orientation is a function of
    // the time alone within a frame)
    const CameraTable& T = *C.camTable;
    if (f2u(t) == f2u(T.time[0])) { c = T.at[0]; return; }
    if (f2u(t) == f2u(T.time[1])) { c = T.at[1]; return; }
    c = C.camera;
    orient_camera_table(C.cm, T, c, C.frameCount, t);
}

// ------------------------------------------------------------ records
struct Recon // ReconnectionData.slang:89-166 (earlyThroughput lives in the path state only)
{
    f2 subPixel;
    f2 lensSample;
    float time;
    uint32_t pathLength, firstComp, secondComp;
    bool transmissionEvent, lightIsNEE, lightIsDistant;
    float lightPdf;
    float subPixelJacobian, lensVertexJacobian, secondaryPathJacobian;
    HitInfo firstHit, secondHit;
    f3 firstWi, secondWo, irradiance;
    // Suffix replay state (no reference counterpart; word 27 and bits 15-26 of word 5, which the
    // reference's record leaves unused): the sample generator's state and the packed bounce
    // counters and path flags on entering the third vertex, so that the adjoint can re-run the
    // path tracer from x3 (suffix_state_pack).  Zero for paths that end before x3.
    uint32_t suffixSeed, suffixState;
};
__device__ __forceinline__ Recon recon_default()
{
    Recon r;
    r.subPixel = mk2(0.5f, 0.5f); r.lensSample = mk2(0.f, 0.f); r.time = 0.f;
    r.pathLength = 0; r.firstComp = 0; r.secondComp = 0;
    r.transmissionEvent = false; r.lightIsNEE = false; r.lightIsDistant = false;
    r.lightPdf = 0.f; r.subPixelJacobian = 1.f; r.lensVertexJacobian = 1.f; r.secondaryPathJacobian = 1.f;
    r.firstHit = hit_none(); r.secondHit = hit_none();
    r.firstWi = mk3(0.f); r.secondWo = mk3(0.f); r.irradiance = mk3(0.f);
    r.suffixSeed = 0u; r.suffixState = 0u;
    return r;
}

struct Shifted // ShiftedPathData (ReconnectionData.slang:35-82)
{
    HitInfo primaryHit;
    f2 fractionalPixel;
    f2 lensSample;
    f3 firstRayDir;
    float subPixelJacobian, lensVertexJacobian, secondaryPathJacobian;
    f3 radiance;
};
__device__ __forceinline__ Shifted shifted_default()
{
    Shifted s;
    s.primaryHit = hit_none(); s.fractionalPixel = mk2(-1.f, -1.f); s.lensSample = mk2(0.f, 0.f);
    s.firstRayDir = mk3(0.f); s.subPixelJacobian = 1.f; s.lensVertexJacobian = 1.f; s.secondaryPathJacobian = 1.f;
    s.radiance = mk3(0.f);
    return s;
}
__device__ __forceinline__ void recon_update(Recon& r, const Shifted& s) // ReconnectionData.slang:154-165
{
    r.firstHit = s.primaryHit;
    r.subPixel = s.fractionalPixel - floor2(s.fractionalPixel);
    r.lensSample = s.lensSample;
    r.firstWi = -s.firstRayDir;
    r.subPixelJacobian = s.subPixelJacobian;
    r.lensVertexJacobian = s.lensVertexJacobian;
    r.secondaryPathJacobian = s.secondaryPathJacobian;
}

struct Res // PathReservoir (Reservoir.slang:73-132)
{
    float confidence, totalWeight;
    f3 integrand;
    f2 subPixel;
};
__device__ __forceinline__ Res res_default() { Res r; r.confidence = 0.f; r.totalWeight = 0.f; r.integrand = mk3(0.f); r.subPixel = mk2(0.5f, 0.5f); return r; }
__device__ __forceinline__ float res_ucw(const Res& r)
{
    float pHat = luminance(r.integrand);
    return (pHat == 0.f) ? 0.f : r.totalWeight / pHat;
}
__device__ __forceinline__ bool res_add_sample(Res& d, SampleGen& sg, float mis, f3 integrand, float jacobian, const Res& other)
{
    float pHat = luminance(integrand);
    float w = mis * pHat * res_ucw(other) * jacobian;
    d.totalWeight = d.totalWeight + w;
    d.confidence = f_min(d.confidence + other.confidence, kConfidenceCap);
    float rng = sampleNext1D(sg);
    bool selected = (rng * d.totalWeight < w);
    d.integrand = selected ? integrand : d.integrand;
    d.subPixel = selected ? other.subPixel : d.subPixel;
    return selected;
}

// ------------------------------------------------------------ SoA storage
// Reservoir: two float4 planes: (integrand.xyz, totalWeight), (subPixel.xy, confidence, 0).
// Reconnection: seven uint4 planes (the canonical 28-word record split by 16 bytes).
struct ResPlanes { float4* a; float4* b; };
struct RecPlanes { uint4* p; size_t stride; }; // plane k at p + k * stride

__device__ __forceinline__ Res load_res(const ResPlanes& P, uint32_t i)
{
    float4 a = __ldg(P.a + i), b = __ldg(P.b + i);
    Res r; r.integrand = mk3(a.x, a.y, a.z); r.totalWeight = a.w; r.subPixel = mk2(b.x, b.y); r.confidence = b.z;
    return r;
}
__device__ __forceinline__ Res load_res_rw(const ResPlanes& P, uint32_t i)
{
    float4 a = P.a[i], b = P.b[i];
    Res r; r.integrand = mk3(a.x, a.y, a.z); r.totalWeight = a.w; r.subPixel = mk2(b.x, b.y); r.confidence = b.z;
    return r;
}
__device__ __forceinline__ void store_res(const ResPlanes& P, uint32_t i, const Res& r)
{
    P.a[i] = make_float4(r.integrand.x, r.integrand.y, r.integrand.z, r.totalWeight);
    P.b[i] = make_float4(r.subPixel.x, r.subPixel.y, r.confidence, 0.f);
}
__device__ __forceinline__ f3 load_integrand(const ResPlanes& P, uint32_t i) { float4 a = __ldg(P.a + i); return mk3(a.x, a.y, a.z); }
__device__ __forceinline__ float load_confidence(const ResPlanes& P, uint32_t i) { return __ldg(P.b + i).z; }

__device__ __forceinline__ uint32_t recon_flags(const Recon& r)
{
    return (r.pathLength & 0xffu) | ((r.firstComp & 3u) << 8) | ((r.secondComp & 3u) << 10) |
           ((r.transmissionEvent ? 1u : 0u) << 12) | ((r.lightIsNEE ? 1u : 0u) << 13) | ((r.lightIsDistant ? 1u : 0u) << 14) |
           ((r.suffixState & 0xfffu) << 15);
}
__device__ __forceinline__ void store_rec(const RecPlanes& P, uint32_t i, const Recon& r)
{
    uint4* p = P.p + i;
    const size_t s = P.stride;
    p[0 * s] = make_uint4(f2u(r.subPixel.x), f2u(r.subPixel.y), f2u(r.lensSample.x), f2u(r.lensSample.y));
    p[1 * s] = make_uint4(f2u(r.time), recon_flags(r), f2u(r.lightPdf), f2u(r.subPixelJacobian));
    p[2 * s] = make_uint4(r.firstHit.w[0], r.firstHit.w[1], r.firstHit.w[2], r.firstHit.w[3]);
    p[3 * s] = make_uint4(r.secondHit.w[0], r.secondHit.w[1], r.secondHit.w[2], r.secondHit.w[3]);
    p[4 * s] = make_uint4(f2u(r.firstWi.x), f2u(r.firstWi.y), f2u(r.firstWi.z), f2u(r.lensVertexJacobian));
    p[5 * s] = make_uint4(f2u(r.secondWo.x), f2u(r.secondWo.y), f2u(r.secondWo.z), f2u(r.secondaryPathJacobian));
    p[6 * s] = make_uint4(f2u(r.irradiance.x), f2u(r.irradiance.y), f2u(r.irradiance.z), r.suffixSeed);
}
template <bool RO>
__device__ __forceinline__ Recon load_rec_t(const RecPlanes& P, uint32_t i)
{
    const uint4* p = P.p + i;
    const size_t s = P.stride;
    uint4 q0, q1, q2, q3, q4, q5, q6;
    if (RO) { q0 = __ldg(p); q1 = __ldg(p + s); q2 = __ldg(p + 2 * s); q3 = __ldg(p + 3 * s); q4 = __ldg(p + 4 * s); q5 = __ldg(p + 5 * s); q6 = __ldg(p + 6 * s); }
    else { q0 = p[0]; q1 = p[s]; q2 = p[2 * s]; q3 = p[3 * s]; q4 = p[4 * s]; q5 = p[5 * s]; q6 = p[6 * s]; }
    Recon r;
    r.subPixel = mk2(u2f(q0.x), u2f(q0.y)); r.lensSample = mk2(u2f(q0.z), u2f(q0.w));
    r.time = u2f(q1.x);
    r.pathLength = q1.y & 0xffu; r.firstComp = (q1.y >> 8) & 3u; r.secondComp = (q1.y >> 10) & 3u;
    r.transmissionEvent = (q1.y >> 12) & 1u; r.lightIsNEE = (q1.y >> 13) & 1u; r.lightIsDistant = (q1.y >> 14) & 1u;
    r.suffixState = (q1.y >> 15) & 0xfffu;
    r.lightPdf = u2f(q1.z); r.subPixelJacobian = u2f(q1.w);
    r.firstHit.w[0] = q2.x; r.firstHit.w[1] = q2.y; r.firstHit.w[2] = q2.z; r.firstHit.w[3] = q2.w;
    r.secondHit.w[0] = q3.x; r.secondHit.w[1] = q3.y; r.secondHit.w[2] = q3.z; r.secondHit.w[3] = q3.w;
    r.firstWi = mk3(u2f(q4.x), u2f(q4.y), u2f(q4.z)); r.lensVertexJacobian = u2f(q4.w);
    r.secondWo = mk3(u2f(q5.x), u2f(q5.y), u2f(q5.z)); r.secondaryPathJacobian = u2f(q5.w);
    r.irradiance = mk3(u2f(q6.x), u2f(q6.y), u2f(q6.z));
    r.suffixSeed = q6.w;
    return r;
}
__device__ __forceinline__ Recon load_rec(const RecPlanes& P, uint32_t i) { return load_rec_t<true>(P, i); }
__device__ __forceinline__ Recon load_rec_rw(const RecPlanes& P, uint32_t i) { return load_rec_t<false>(P, i); }
__device__ __forceinline__ HitInfo load_first_hit(const RecPlanes& P, uint32_t i)
{
    uint4 q = __ldg(P.p + 2 * P.stride + i);
    HitInfo h; h.w[0] = q.x; h.w[1] = q.y; h.w[2] = q.z; h.w[3] = q.w; return h;
}

// ------------------------------------------------------------ reconnection (PathTracer.slang / ShiftMapping.slang)
// Path state subset used by the shifts: thp, origin, dir, hit, active flag.
struct ShiftPath
{
    f3 thp, origin, dir;
    HitInfo hit;
    bool active;
};

// handleReconnectionHit (PathTracer.slang:1177-1397).  The x1 -> x2 visibility test that ends it is
// not traced here: when the path is still active its ray is returned in `vis` (an occluded ray
// deactivates the path, ending the shift with 0), for the caller to trace once nothing else is left
// to compute.
__device__ inline void dev_reconnection_hit(const DevCtx& C, ShiftPath& path, const Recon& rd, float& dstJacobian, Ray& vis)
{
    ShadingData sd = dev_sd(C, path.hit, path.dir);
    BsdfData d = dev_instance(C, sd);
    path.origin = sd_ray_origin(sd, true);
    if (rd.transmissionEvent) path.origin = sd_ray_origin(sd, false);
    bool secondHitIsDistant = (rd.pathLength == 2) && rd.lightIsDistant;
    dstJacobian = 1.f;
    f3 nextDir = mk3(0.f);
    float rayLength = kRayTMax;
    if (!secondHitIsDistant)
    {
        ShadingData secondSd = hit_valid(rd.secondHit) ? dev_sd(C, rd.secondHit, mk3(0.f)) : sd_zero_vertex();
        f3 shiftedOffset = secondSd.posW - sd.posW;
        float shiftedDist2 = dot(shiftedOffset, shiftedOffset);
        float shiftedCosine = f_abs(dot(secondSd.faceN, -normalize(shiftedOffset)));
        dstJacobian = shiftedCosine / shiftedDist2;
        f3 adjustedOffset = secondSd.posW - path.origin;
        nextDir = normalize(adjustedOffset);
        rayLength = length(adjustedOffset) * 0.999f;
    }
    else nextDir = hit_as_direction(rd.secondHit);

    const BsdfPair bp = mi_eval_pair(sd, d, rd.firstComp, nextDir);
    const f3 lobeScatterBsdf = bp.lobeBsdf, totalScatterBsdf = bp.totalBsdf;
    const float lobeScatterPdf = bp.lobePdf, totalScatterPdf = bp.totalPdf;
    path.dir = nextDir;

    if (rd.pathLength == 2)
    {
        float lightPdf = rd.lightPdf / dstJacobian;
        float misWeight;
        if (rd.lightIsNEE)
        {
            if (!any_gt0(totalScatterBsdf) || totalScatterPdf == 0.f) { path.active = false; return; }
            dstJacobian *= lightPdf;
            misWeight = dev_mis(C, lightPdf, totalScatterPdf);
            path.thp *= totalScatterBsdf / lightPdf;
        }
        else
        {
            if (!any_gt0(lobeScatterBsdf) || lobeScatterPdf == 0.f) { path.active = false; return; }
            dstJacobian *= lobeScatterPdf;
            misWeight = dev_mis(C, totalScatterPdf, lightPdf);
            path.thp *= lobeScatterBsdf / lobeScatterPdf;
        }
        path.thp *= misWeight;
    }
    else
    {
        if (!any_gt0(lobeScatterBsdf) || lobeScatterPdf == 0.f) { path.active = false; return; }
        dstJacobian *= lobeScatterPdf;
        path.thp *= lobeScatterBsdf / lobeScatterPdf;
    }
    // disableCaustics: the shift paths carry no bounce counters or specular flag (a fresh
    // PathState), so the caustics test of :1378 never fires here.
    bool valid = any_gt0(path.thp);
    if (!valid) path.active = false;
    else vis = mk_ray(path.origin, path.dir, 0.f, rayLength);
}

// pathReconnectionShift (ShiftMapping.slang:430-513) with its visibility test deferred: returns the
// value for a visible reconnection; `needVis` tells whether the x1 -> x2 ray `vis` has to be traced,
// and if it is occluded the shift's value is 0 and dstJacobian is `jacobianIfOccluded` (the values
// the reference returns at its visibility test).
__device__ inline f3 dev_path_reconnection_shift_deferred(const DevCtx& C, const Recon& rd, ShiftPath& path, float& dstJacobian, Ray& vis,
                                                         bool& needVis, float& jacobianIfOccluded)
{
    dstJacobian = 1.f;
    needVis = false;
    dev_reconnection_hit(C, path, rd, dstJacobian, vis);
    if (!path.active) return mk3(0.f);
    needVis = true;
    jacobianIfOccluded = dstJacobian;
    if (rd.pathLength == 2) return 1.f * path.thp * rd.irradiance; // the x2 BSDF terms are not used for length 2
    ShadingData secondSd = dev_sd(C, rd.secondHit, path.dir);
    BsdfData d = dev_instance(C, secondSd);
    const BsdfPair bp = mi_eval_pair(secondSd, d, rd.secondComp, rd.secondWo);
    const f3 lobeSpecificBsdf = bp.lobeBsdf, totalBsdf = bp.totalBsdf;
    const float lobeSpecificPdf = bp.lobePdf, totalPdf = bp.totalPdf;
    if (rd.pathLength > 2 && !any_gt0(totalBsdf)) return mk3(0.f);
    float misWeight = 1.f;
    if (rd.pathLength == 3)
    {
        bool valid = rd.lightIsNEE ? true : (lobeSpecificPdf > 0.f);
        if (!valid) return mk3(0.f);
        misWeight = rd.lightIsNEE ? dev_mis(C, rd.lightPdf, totalPdf) : dev_mis(C, totalPdf, rd.lightPdf);
        f3 lightConnectionThp = rd.lightIsNEE ? totalBsdf / rd.lightPdf : lobeSpecificBsdf / lobeSpecificPdf;
        path.thp *= lightConnectionThp;
        dstJacobian *= rd.lightIsNEE ? 1.f : lobeSpecificPdf;
    }
    else if (rd.pathLength > 3)
    {
        if (!(lobeSpecificPdf > 0.f)) return mk3(0.f);
        path.thp *= lobeSpecificBsdf / lobeSpecificPdf;
        dstJacobian *= lobeSpecificPdf;
    }
    return misWeight * path.thp * rd.irradiance;
}

// pathReconnectionShift (ShiftMapping.slang:430-513), the visibility traced after the x2 terms.
__device__ inline f3 dev_path_reconnection_shift(const DevCtx& C, const Recon& rd, ShiftPath& path, float& dstJacobian)
{
    Ray vis;
    bool needVis;
    float jacobianIfOccluded;
    const f3 value = dev_path_reconnection_shift_deferred(C, rd, path, dstJacobian, vis, needVis, jacobianIfOccluded);
    if (needVis && !dev_visible(C, vis)) { dstJacobian = jacobianIfOccluded; return mk3(0.f); }
    return value;
}

__device__ __forceinline__ f3 dev_primary_light(const DevCtx& C, const ShiftPath& path) // PathTracer.slang:1399-1410
{
    ShadingData sd = dev_sd(C, path.hit, path.dir);
    return dev_instance(C, sd).emission;
}

// The shifts' environment branch (ShiftMapping.slang:151-166, 259-269, 383-393): the map seen along
// `dir` and the Jacobians of a primary vertex at infinity.
struct EnvPrimary { f3 radiance; float subPixelJacobian, lensVertexJacobian; };
static __device__ __noinline__ EnvPrimary dev_env_primary(const EnvMapView* E, f3 dir, f3 camDir, float lenW)
{
    EnvPrimary e;
    e.radiance = env_reconnection(*E, dir);
    const float cosSensor = dot(camDir, dir);
    e.subPixelJacobian = 1.f / f_abs(f_pow3(cosSensor));
    const float d0 = lenW / dot(camDir, dir);
    e.lensVertexJacobian = (d0 * d0) / f_abs(cosSensor);
    return e;
}

// gatherPrimaryHitReconnectionShift (ShiftMapping.slang:183-296) of an environment sample (a path
// of length 1 to a distant light): the film ray along the sample's direction, out of the lens.
static __device__ __noinline__ Shifted dev_gather_primary_reconnect_env(const DevCtx& C, SampleGen sg, f3 firstWi, float time, f2 fractionalPixel,
                                                                          HitInfo primaryHit)
{
    CameraData cam; dev_orient(C, cam, time);
    f2 p = mk2(fractionalPixel.x / (float)C.W, fractionalPixel.y / (float)C.H);
    f2 ndc = mk2(2.f * p.x + -1.f, -2.f * p.y + 1.f);
    f3 filmWorld = cam.posW + (cam.cameraU * ndc.x + cam.cameraV * ndc.y + cam.cameraW);
    const f3 dir = -firstWi;
    const f3 x1 = filmWorld + dir;
    const f3 camDir = cam.unitW;
    float camZ = dot(x1 - cam.posW, camDir);
    float rayT = camZ / dot(dir, camDir);
    const f3 origin = x1 - dir * rayT;
    f3 lensOffsetWorld = origin - cam.posW;
    f2 lensLocalNormalized = mk2(dot(lensOffsetWorld, cam.unitU) / cam.apertureRadius,
                                 dot(lensOffsetWorld, cam.unitV) / cam.apertureRadius);
    if (length(lensLocalNormalized) > 1.f) return shifted_default();
    if (!dev_visible(C, mk_ray(origin, dir, 0.001f, kRayTMax))) return shifted_default();
    Shifted sp = shifted_default();
    sp.firstRayDir = dir;
    sp.fractionalPixel = fractionalPixel;
    sp.lensSample = lensLocalNormalized;
    sp.primaryHit = primaryHit;
    (void)sampleNext1D(sg);
    const EnvPrimary e = dev_env_primary(C.env, dir, camDir, cam.lenW);
    sp.radiance = e.radiance; sp.subPixelJacobian = e.subPixelJacobian; sp.lensVertexJacobian = e.lensVertexJacobian;
    return sp;
}

// scatterReprojectionShift (ShiftMapping.slang:301-421) of an environment sample: the direction
// reprojected through the camera at `time`, the camera ray tested to infinity.
static __device__ __noinline__ Shifted dev_scatter_shift_env(const DevCtx& C, SampleGen sg, f3 firstWi, float time, HitInfo primaryHit, f2 lensSample,
                                                               bool skipVisibilityCheck)
{
    CameraData cam; dev_orient(C, cam, time);
    f2 lensLocal = mk2(cam.apertureRadius * lensSample.x, cam.apertureRadius * lensSample.y);
    const f3 origin = cam.posW + (cam.unitU * lensLocal.x + cam.unitV * lensLocal.y);
    const f3 dir = -firstWi;
    const f3 camDir = cam.unitW;
    f3 camRay = mk3(dot(cam.unitU, dir), dot(cam.unitV, dir), dot(camDir, dir));
    if (camRay.z <= 0.001f) return shifted_default();
    float lw = cam.lenW;
    f2 film = mk2(lensLocal.x + lw * (camRay.x / camRay.z), lensLocal.y + lw * (camRay.y / camRay.z));
    f2 ndc = mk2(film.x / cam.lenU, film.y / cam.lenV);
    f2 nfp = mk2((0.5f * ndc.x + 0.5f) * (float)C.W, (-0.5f * ndc.y + 0.5f) * (float)C.H);
    if (!valid_float(C, nfp)) return shifted_default();
    if (!skipVisibilityCheck && !dev_visible(C, mk_ray(origin, dir, 0.001f, kRayTMax))) return shifted_default();
    Shifted sp = shifted_default();
    sp.lensSample = lensSample;
    sp.firstRayDir = dir;
    sp.fractionalPixel = nfp;
    sp.primaryHit = primaryHit;
    (void)sampleNext1D(sg);
    const EnvPrimary e = dev_env_primary(C.env, dir, camDir, cam.lenW);
    sp.radiance = e.radiance; sp.subPixelJacobian = e.subPixelJacobian; sp.lensVertexJacobian = e.lensVertexJacobian;
    return sp;
}

// gatherLensVertexCopyShift (ShiftMapping.slang:90-180); `sg` is taken by value.
template <bool kEnv>
__device__ inline Shifted dev_gather_lens_copy(const DevCtx& C, SampleGen sg, const Recon& rd, float time, f2 fractionalPixel, f2 lensSample)
{
    if (!valid_float(C, fractionalPixel)) return shifted_default();
    const bool hitEnvMap = (rd.pathLength == 1 && rd.lightIsDistant);
    (void)sampleNext1D(sg); // seed of the shifted path's generator; the shift draws nothing from it
    CameraData cam; dev_orient(C, cam, time);
    Ray cr = camera_ray_thinlens(cam, C.W, C.H, fractionalPixel, lensSample);
    ShiftPath path;
    path.thp = mk3(1.f);
    path.dir = cr.dir;
    path.active = true;
    const TraceHit th = C.bvh.numTris ? trace_closest_call(C.bvh, mk_ray(cr.origin, cr.dir, 0.f, kRayTMax), C.fault) : TraceHit{kInvalidIndex, 0.f, 0.f, 0.f};
    const bool isHit = th.prim != kInvalidIndex;
    path.hit = isHit ? hit_tri(th.prim, th.u, th.v) : hit_none();
    path.origin = camera_lens_point_scaled(cam, lensSample);
    f3 camDir = cam.unitW;
    Shifted sp = shifted_default();
    sp.primaryHit = path.hit;
    sp.firstRayDir = path.dir;
    sp.fractionalPixel = fractionalPixel;
    sp.lensSample = lensSample;
    if (!kEnv && (!isHit || hitEnvMap)) return shifted_default();
    if (kEnv && isHit && hitEnvMap) return shifted_default(); // expected the environment, met geometry
    if (kEnv && !isHit)
    {
        if (!hitEnvMap) return shifted_default();      // expected geometry, saw the environment
        const EnvPrimary e = dev_env_primary(C.env, path.dir, camDir, cam.lenW);
        sp.radiance = e.radiance; sp.subPixelJacobian = e.subPixelJacobian; sp.lensVertexJacobian = e.lensVertexJacobian;
        return sp;
    }
    {
        ShadingData firstSd = dev_sd(C, path.hit, path.dir);
        f3 x1 = firstSd.posW;
        float dist = length(x1 - path.origin);
        float distSquared = dist * dist;
        float cosNormal = dot(-path.dir, firstSd.faceN);
        float cosSensor = dot(camDir, path.dir);
        sp.subPixelJacobian = f_abs(cosNormal / distSquared) / f_abs(f_pow3(cosSensor));
        float camZ = dot(x1 - cam.posW, camDir);
        float d0 = (cam.lenW / f_abs(camZ) * dist);
        float d1 = dist - d0;
        sp.lensVertexJacobian = (d0 * d0) / (d1 * d1) * f_abs(cosNormal) / f_abs(cosSensor);
    }
    if (rd.pathLength == 1) { sp.radiance = dev_primary_light(C, path); return sp; }
    sp.radiance = dev_path_reconnection_shift(C, rd, path, sp.secondaryPathJacobian);
    return sp;
}

// gatherPrimaryHitReconnectionShift (ShiftMapping.slang:183-296)
template <bool kEnv>
__device__ inline Shifted dev_gather_primary_reconnect(const DevCtx& C, SampleGen sg, const Recon& rd, float time, f2 fractionalPixel, const HitInfo& primaryHit)
{
    const bool hitEnvMap = (rd.pathLength == 1 && rd.lightIsDistant);
    if (kEnv && hitEnvMap) return dev_gather_primary_reconnect_env(C, sg, rd.firstWi, time, fractionalPixel, primaryHit);
    if (hitEnvMap || !hit_valid(primaryHit)) return shifted_default();
    CameraData cam; dev_orient(C, cam, time);
    f2 p = mk2(fractionalPixel.x / (float)C.W, fractionalPixel.y / (float)C.H);
    f2 ndc = mk2(2.f * p.x + -1.f, -2.f * p.y + 1.f);
    f3 filmWorld = cam.posW + (cam.cameraU * ndc.x + cam.cameraV * ndc.y + cam.cameraW);
    ShiftPath path;
    path.thp = mk3(1.f);
    path.active = true;
    ShadingData sd = dev_sd(C, primaryHit, mk3(0.f));
    f3 x1 = sd.posW, n = sd.faceN;
    path.dir = normalize(x1 - filmWorld);
    f3 camDir = cam.unitW;
    float camZ = dot(x1 - cam.posW, camDir);
    float rayT = camZ / dot(path.dir, camDir);
    path.origin = x1 - path.dir * rayT;
    path.dir = normalize(x1 - path.origin);
    f3 lensOffsetWorld = path.origin - cam.posW;
    f2 lensLocalNormalized = mk2(dot(lensOffsetWorld, cam.unitU) / cam.apertureRadius,
                                 dot(lensOffsetWorld, cam.unitV) / cam.apertureRadius);
    if (length(lensLocalNormalized) > 1.f) return shifted_default();
    float dist = length(x1 - path.origin);
    if (!dev_visible(C, mk_ray(path.origin, path.dir, 0.001f * dist, 0.999f * dist))) return shifted_default();
    Shifted sp = shifted_default();
    sp.firstRayDir = path.dir;
    sp.fractionalPixel = fractionalPixel;
    sp.lensSample = lensLocalNormalized;
    sp.primaryHit = primaryHit;
    (void)sampleNext1D(sg);
    path.hit = primaryHit;
    {
        float dist2 = length(x1 - path.origin);
        float distSquared = dist2 * dist2;
        float cosNormal = dot(path.dir, n);
        float cosSensor = dot(camDir, path.dir);
        sp.subPixelJacobian = f_abs(cosNormal / distSquared) / f_abs(f_pow3(cosSensor));
        float d0 = (cam.lenW / f_abs(camZ) * rayT);
        float d1 = rayT - d0;
        sp.lensVertexJacobian = (d0 * d0) / (d1 * d1) * (f_abs(cosNormal)) / (f_abs(cosSensor));
    }
    if (rd.pathLength == 1) { sp.radiance = dev_primary_light(C, path); return sp; }
    sp.radiance = dev_path_reconnection_shift(C, rd, path, sp.secondaryPathJacobian);
    return sp;
}

// scatterReprojectionShift (ShiftMapping.slang:301-421)
template <bool kEnv>
__device__ inline Shifted dev_scatter_shift(const DevCtx& C, SampleGen sg, const Recon& rd, float time, const HitInfo& primaryHit, f2 lensSample, bool skipVisibilityCheck)
{
    const bool hitEnvMap = (rd.pathLength == 1) && rd.lightIsDistant;
    if (kEnv && hitEnvMap) return dev_scatter_shift_env(C, sg, rd.firstWi, time, primaryHit, lensSample, skipVisibilityCheck);
    if (hitEnvMap || !hit_valid(primaryHit)) return shifted_default();
    CameraData cam; dev_orient(C, cam, time);
    f2 lensLocal = mk2(cam.apertureRadius * lensSample.x, cam.apertureRadius * lensSample.y);
    f3 camU = cam.unitU;
    f3 camV = cam.unitV;
    ShiftPath path;
    path.thp = mk3(1.f);
    path.active = true;
    path.origin = cam.posW + (camU * lensLocal.x + camV * lensLocal.y);
    ShadingData firstSd = dev_sd(C, primaryHit, mk3(0.f));
    f3 x1 = firstSd.posW, n = firstSd.faceN;
    path.dir = normalize(x1 - path.origin);
    f3 camDir = cam.unitW;
    f3 camRay = mk3(dot(camU, path.dir), dot(camV, path.dir), dot(camDir, path.dir));
    if (camRay.z <= 0.001f) return shifted_default();
    float lw = cam.lenW;
    f2 film = mk2(lensLocal.x + lw * (camRay.x / camRay.z), lensLocal.y + lw * (camRay.y / camRay.z));
    f2 ndc = mk2(film.x / cam.lenU, film.y / cam.lenV);
    f2 nfp = mk2((0.5f * ndc.x + 0.5f) * (float)C.W, (-0.5f * ndc.y + 0.5f) * (float)C.H);
    if (!valid_float(C, nfp)) return shifted_default();
    float dist = length(x1 - path.origin);
    // the camera -> x1 test (occluded: the shift fails) and the reconnection's x1 -> x2 test are
    // traced in that order after the rest of the shift, when only their outcomes are left to apply
    const Ray camVis = mk_ray(path.origin, path.dir, 0.001f, 0.999f * dist);
    Shifted sp = shifted_default();
    sp.lensSample = lensSample;
    sp.firstRayDir = path.dir;
    sp.fractionalPixel = nfp;
    sp.primaryHit = primaryHit;
    (void)sampleNext1D(sg);
    path.hit = primaryHit;
    {
        float distSquared = dist * dist;
        float cosNormal = dot(-path.dir, n);
        float cosSensor = dot(cam.unitW, path.dir);
        sp.subPixelJacobian = f_abs(cosNormal / distSquared) / f_abs(f_pow3(cosSensor));
        float camZ = dot(x1 - cam.posW, camDir);
        float d0 = (cam.lenW / f_abs(camZ) * dist);
        float d1 = dist - d0;
        sp.lensVertexJacobian = (d0 * d0) / (d1 * d1) * f_abs(cosNormal) / f_abs(cosSensor);
    }
    Ray vis;
    bool needVis = false;
    float jacobianIfOccluded = 0.f;
    if (rd.pathLength == 1) sp.radiance = dev_primary_light(C, path);
    else sp.radiance = dev_path_reconnection_shift_deferred(C, rd, path, sp.secondaryPathJacobian, vis, needVis, jacobianIfOccluded);
    if (!skipVisibilityCheck && !dev_visible(C, camVis)) return shifted_default();
    if (needVis && !dev_visible(C, vis)) { sp.radiance = mk3(0.f); sp.secondaryPathJacobian = jacobianIfOccluded; }
    return sp;
}

__device__ __forceinline__ float jac_scatter(const Shifted& s, const Recon& r)
{
    return (s.subPixelJacobian * s.secondaryPathJacobian) / (r.subPixelJacobian * r.secondaryPathJacobian);
}

// Depth-of-field shift probabilities of a pixel (ShiftMapping.slang:43-80; GatherTemporalResampling.rt.slang:75-96)
__device__ __forceinline__ f2 pixel_dof_probs(const DevCtx& C, const uint4* vbuffer, uint32_t i)
{
    if (!(C.camera.apertureRadius > 0.f)) return mk2(1.f, 0.f);
    uint4 q = __ldg(&vbuffer[i]);
    HitInfo h; h.w[0] = q.x; h.w[1] = q.y; h.w[2] = q.z; h.w[3] = q.w;
    const CameraData& cam = C.camera;
    float normalizedFilm = length(cam.cameraU / (float)C.W + cam.cameraV / (float)C.H);
    float coc;
    if (hit_valid(h))
    {
        f3 x1 = dev_sd(C, h, mk3(0.f)).posW;
        f3 camDir = cam.unitW;
        float camZ = dot(x1 - cam.posW, camDir);
        float filmZ = camZ - cam.lenW;
        float filmRadius = f_abs(cam.apertureRadius / camZ * filmZ);
        coc = filmRadius / normalizedFilm;
    }
    else coc = cam.apertureRadius / normalizedFilm;
    float gamma = 0.2f + 6.2f / (coc - 5.6f);
    gamma = (coc <= 0.2f) ? 1.f : f_clamp(gamma, 0.2f, 1.f);
    return mk2(gamma, 1.f - gamma);
}

} // namespace rs
