// CPU oracle of the Reservoir Splatting per-frame path.  TEST INFRASTRUCTURE:
// only the tests, the smoke check and the bench's CPU-baseline leg load it; the
// CUDA pass never links it.
//
// This file restates, one scalar pixel at a time and in the reference's own
// array-of-structs form, the pass logic of
//   Source/RenderPasses/ReservoirSplatting/*.slang  and  ReservoirSplatting.cpp
// (each function below cites the lines it follows).  It shares with the CUDA
// pass only the Falcor-library layer (RNG, camera basis, BSDF, light sampling,
// triangle intersection, light-collection build: the headers in
// reservoir-splatting_b200/csrc/core), and has its own BVH (a CPU median-split
// tree, a different topology from the pass's LBVH: closest-hit results agree
// because the hit is the (t, triangle index) minimum, which no topology changes).
//
// Parity: the reference's GPU path cannot run here (Slang/DXR), so the oracle is
// pinned only by the reference's RNG known-answer tests (LCG/TEA) and by the
// properties its tests and the path define; see the parity section of the docs.
//
// Deliberate, documented deviations from the reference:
//  * splats inside one cell are ordered by ascending source pixel (the reference's
//    order is atomic arrival order and not reproducible, SortReprojectedReservoirs.cs.slang:68,94);
//  * pow(x, n) is x*...*x, acos clamps its argument to [-1, 1];
//  * environment maps, analytic lights, transmission and nested dielectrics are absent
//    (kUseEnvLight = kUseAnalyticLights = false, all materials opaque).
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <algorithm>
#include <vector>
#include <memory>
#include <array>
#include <omp.h>

#include "../include/rs_b200.h"
#include "../reservoir-splatting_b200/csrc/core/camera.h"
#include "../reservoir-splatting_b200/csrc/core/envmap.h"
#include "../reservoir-splatting_b200/csrc/core/analytic_lights.h"
#include "../reservoir-splatting_b200/csrc/core/scene_prep.h"
#include "../reservoir-splatting_b200/csrc/core/material_grad.h"
#include <cmath>

using namespace rs;

namespace oracle {

static const uint32_t kNumRenderPasses = 8;      // ReservoirSplatting.cpp:36
static const float kConfidenceCap = 20.f;        // Reservoir.slang:75

// ------------------------------------------------------------------ BVH (CPU)
struct Node
{
    float lo[3], hi[3];
    uint32_t left, right;   // internal: child node indices; leaf: first/count
    uint32_t leaf;
};

struct Bvh
{
    std::vector<Node> nodes;
    std::vector<uint32_t> prims;
    const f4* tri = nullptr;

    void build(const std::vector<f4>& t, uint32_t n)
    {
        tri = t.data();
        prims.resize(n);
        for (uint32_t i = 0; i < n; i++) prims[i] = i;
        nodes.clear();
        nodes.reserve(2 * (size_t)n + 1);
        std::vector<float> cen(3 * (size_t)n);
        for (uint32_t i = 0; i < n; i++)
            for (int k = 0; k < 3; k++)
            {
                float a = (&tri[3 * i].x)[k], b = (&tri[3 * i + 1].x)[k], c = (&tri[3 * i + 2].x)[k];
                cen[3 * i + k] = (a + b + c) * (1.f / 3.f);
            }
        if (n == 0) return;
        buildRec(0, n, cen);
    }

    uint32_t buildRec(uint32_t b, uint32_t e, const std::vector<float>& cen)
    {
        uint32_t idx = (uint32_t)nodes.size();
        nodes.push_back(Node());
        Node nd;
        for (int k = 0; k < 3; k++) { nd.lo[k] = 3e38f; nd.hi[k] = -3e38f; }
        float clo[3] = {3e38f, 3e38f, 3e38f}, chi[3] = {-3e38f, -3e38f, -3e38f};
        for (uint32_t i = b; i < e; i++)
        {
            uint32_t p = prims[i];
            for (int v = 0; v < 3; v++)
                for (int k = 0; k < 3; k++)
                {
                    float x = (&tri[3 * p + v].x)[k];
                    nd.lo[k] = std::min(nd.lo[k], x);
                    nd.hi[k] = std::max(nd.hi[k], x);
                }
            for (int k = 0; k < 3; k++) { clo[k] = std::min(clo[k], cen[3 * p + k]); chi[k] = std::max(chi[k], cen[3 * p + k]); }
        }
        // Conservative padding: a box test may only prune, never reject a true hit.
        for (int k = 0; k < 3; k++)
        {
            float pad = (std::fabs(nd.lo[k]) + std::fabs(nd.hi[k]) + (nd.hi[k] - nd.lo[k])) * 1e-6f + 1e-30f;
            nd.lo[k] -= pad; nd.hi[k] += pad;
        }
        if (e - b <= 4)
        {
            nd.leaf = 1; nd.left = b; nd.right = e - b;
            nodes[idx] = nd;
            return idx;
        }
        int axis = 0;
        float ext = chi[0] - clo[0];
        for (int k = 1; k < 3; k++) if (chi[k] - clo[k] > ext) { ext = chi[k] - clo[k]; axis = k; }
        uint32_t mid = (b + e) / 2;
        std::nth_element(prims.begin() + b, prims.begin() + mid, prims.begin() + e, [&](uint32_t x, uint32_t y) {
            float cx = cen[3 * x + axis], cy = cen[3 * y + axis];
            return cx < cy || (cx == cy && x < y);
        });
        nd.leaf = 0;
        nodes[idx] = nd;
        uint32_t l = buildRec(b, mid, cen);
        uint32_t r = buildRec(mid, e, cen);
        nodes[idx].left = l; nodes[idx].right = r;
        return idx;
    }

    static bool boxHit(const Node& n, f3 o, f3 invd, float tmax)
    {
        float t0 = 0.f, t1 = tmax;
        const float* oo = &o.x; const float* id = &invd.x;
        for (int k = 0; k < 3; k++)
        {
            float a = (n.lo[k] - oo[k]) * id[k], b = (n.hi[k] - oo[k]) * id[k];
            if (a != a) a = -3e38f; // 0 * inf
            if (b != b) b = 3e38f;
            float lo = std::min(a, b), hi = std::max(a, b);
            t0 = std::max(t0, lo); t1 = std::min(t1, hi);
        }
        return t0 <= t1 + 2e-6f * std::fabs(t1);
    }

    // Closest hit on (tMin, tMax); ties on t go to the lower triangle index.
    bool closest(const Ray& r, HitInfo& hit, float& tHit) const
    {
        if (nodes.empty() || ray_has_nan(r)) return false;
        f3 invd = mk3(1.f / r.dir.x, 1.f / r.dir.y, 1.f / r.dir.z);
        float best = r.tMax; uint32_t bestPrim = kInvalidIndex; float bu = 0, bv = 0;
        uint32_t stack[128]; int sp = 0; stack[sp++] = 0;
        while (sp)
        {
            const Node& n = nodes[stack[--sp]];
            if (!boxHit(n, r.origin, invd, best)) continue;
            if (n.leaf)
            {
                for (uint32_t i = 0; i < n.right; i++)
                {
                    uint32_t p = prims[n.left + i];
                    float t, u, v;
                    if (intersect_triangle(r.origin, r.dir, f4xyz(tri[3 * p]), f4xyz(tri[3 * p + 1]), f4xyz(tri[3 * p + 2]), r.tMin, r.tMax, t, u, v))
                    {
                        if (t < best || (t == best && p < bestPrim)) { best = t; bestPrim = p; bu = u; bv = v; }
                    }
                }
            }
            else { stack[sp++] = n.left; stack[sp++] = n.right; }
        }
        if (bestPrim == kInvalidIndex) return false;
        hit = hit_tri(bestPrim, bu, bv);
        tHit = best;
        return true;
    }

    // True when nothing is hit on (tMin, tMax).
    bool visible(const Ray& r) const
    {
        if (nodes.empty() || ray_has_nan(r)) return true;
        f3 invd = mk3(1.f / r.dir.x, 1.f / r.dir.y, 1.f / r.dir.z);
        uint32_t stack[128]; int sp = 0; stack[sp++] = 0;
        while (sp)
        {
            const Node& n = nodes[stack[--sp]];
            if (!boxHit(n, r.origin, invd, r.tMax)) continue;
            if (n.leaf)
            {
                for (uint32_t i = 0; i < n.right; i++)
                {
                    uint32_t p = prims[n.left + i];
                    float t, u, v;
                    if (intersect_triangle(r.origin, r.dir, f4xyz(tri[3 * p]), f4xyz(tri[3 * p + 1]), f4xyz(tri[3 * p + 2]), r.tMin, r.tMax, t, u, v))
                        return false;
                }
            }
            else { stack[sp++] = n.left; stack[sp++] = n.right; }
        }
        return true;
    }
};

// ------------------------------------------------------------------ reservoirs
// ReconnectionData.slang:89-166
struct ReconnectionData
{
    f2 subPixel = mk2(0.5f, 0.5f);
    f2 lensSample = mk2(0.f, 0.f);
    float time = 0.f;
    uint32_t pathLength = 0;
    HitInfo firstHit = hit_none();
    uint32_t firstBSDFComponentType = 0;
    f3 firstWi = mk3(0.f);
    HitInfo secondHit = hit_none();
    uint32_t secondBSDFComponentType = 0;
    f3 secondWo = mk3(0.f);
    bool transmissionEvent = false;
    bool lightIsNEE = false;
    bool lightIsDistant = false;
    float lightPdf = 0.f;
    float subPixelJacobian = 1.f;
    float lensVertexJacobian = 1.f;
    float secondaryPathJacobian = 1.f;
    f3 irradiance = mk3(0.f);
    f3 earlyThroughput = mk3(1.f);
    // suffix replay state of the adjoint (no reference counterpart): the sample generator's state
    // and the packed bounce counters and path flags on entering the third vertex
    uint32_t suffixSeed = 0, suffixState = 0;
};

// ReconnectionData.slang:35-82
struct ShiftedPathData
{
    HitInfo primaryHit = hit_none();
    f2 fractionalPixel = mk2(-1.f, -1.f);
    f2 lensSample = mk2(0.f, 0.f);
    f3 firstRayDir = mk3(0.f);
    float subPixelJacobian = 1.f;
    float lensVertexJacobian = 1.f;
    float secondaryPathJacobian = 1.f;
    f3 radiance = mk3(0.f);
};

// ReconnectionData::update (ReconnectionData.slang:154-165)
static void recon_update(ReconnectionData& r, const ShiftedPathData& s)
{
    r.firstHit = s.primaryHit;
    r.subPixel = s.fractionalPixel - floor2(s.fractionalPixel);
    r.lensSample = s.lensSample;
    r.firstWi = -s.firstRayDir;
    r.subPixelJacobian = s.subPixelJacobian;
    r.lensVertexJacobian = s.lensVertexJacobian;
    r.secondaryPathJacobian = s.secondaryPathJacobian;
}

// CandidateReservoir (Reservoir.slang:35-71)
struct CandidateReservoir
{
    float totalWeight = 0.f;
    f3 integrand = mk3(0.f);
    ReconnectionData selectedReconnection;

    bool addVertex(SampleGen& sg, float sampleMIS, f3 sampleIntegrand)
    {
        float samplePHat = luminance(sampleIntegrand);
        float sampleWeight = sampleMIS * samplePHat;
        sampleWeight = f_isnan(sampleWeight) ? 0.f : sampleWeight;
        totalWeight += sampleWeight;
        float rng = sampleNext1D(sg);
        bool selected = (rng * totalWeight < sampleWeight);
        integrand = selected ? sampleIntegrand : integrand;
        return selected;
    }
};

// PathReservoir (Reservoir.slang:73-132)
struct PathReservoir
{
    float confidence = 0.f;
    float totalWeight = 0.f;
    f3 integrand = mk3(0.f);
    f2 subPixel = mk2(0.5f, 0.5f);

    float computeUCW() const
    {
        float pHat = luminance(integrand);
        return (pHat == 0.f) ? 0.f : totalWeight / pHat;
    }
    bool addSampleFromReservoir(SampleGen& sg, float mis, f3 otherIntegrand, float jacobian, const PathReservoir& other)
    {
        float pHat = luminance(otherIntegrand);
        float w = mis * pHat * other.computeUCW() * jacobian;
        totalWeight = totalWeight + w;
        confidence = f_min(confidence + other.confidence, kConfidenceCap);
        float rng = sampleNext1D(sg);
        bool selected = (rng * totalWeight < w);
        integrand = selected ? otherIntegrand : integrand;
        subPixel = selected ? other.subPixel : subPixel;
        return selected;
    }
    bool add(SampleGen& sg, float mis, const CandidateReservoir& c)
    {
        float weight = mis * c.totalWeight;
        totalWeight = totalWeight + weight;
        confidence = f_min(confidence + 1.f, kConfidenceCap);
        float rng = sampleNext1D(sg);
        bool selected = (rng * totalWeight < weight);
        integrand = selected ? c.integrand : integrand;
        return selected;
    }
};

// ------------------------------------------------------------------ path state
// PathStates.slang:51-80, 85-219 (flags, bounce counters, vertex index)
enum PathFlags : uint32_t
{
    kActive = 0x0001, kHit = 0x0002, kTransmission = 0x0004, kSpecular = 0x0008, kDelta = 0x0010,
    kInsideDielectric = 0x0020, kLightSampledUpper = 0x0040, kLightSampledLower = 0x0080,
};
static const uint32_t kVertexIndexBits = 10u;

// The bounce counters (two bits each: on entering x3 each is at most 2) and the path flags 4..128
// on entering the third vertex, in the 12 bits of ReconnectionData::suffixState.
static uint32_t suffix_state_pack(uint32_t bounces, uint32_t flags)
{
    return (bounces & 3u) | (((bounces >> 8) & 3u) << 2) | (((bounces >> 16) & 3u) << 4) | (((flags >> 2) & 0x3fu) << 6);
}
static void suffix_state_unpack(uint32_t st, uint32_t& bounces, uint32_t& flags)
{
    bounces = (st & 3u) | (((st >> 2) & 3u) << 8) | (((st >> 4) & 3u) << 16);
    flags = ((st >> 6) & 0x3fu) << 2;
}

struct PathState
{
    uint32_t id = 0;
    uint32_t flagsAndVertexIndex = 0;
    uint32_t bounceCounters = 0;
    float time = 0.f;
    f3 origin = mk3(0.f), dir = mk3(0.f);
    float pdf = 0.f, totalPdf = 0.f;
    f3 normal = mk3(0.f);
    HitInfo hit = hit_none();
    f3 prevHitPos = mk3(0.f);
    f3 thp = mk3(0.f);
    SampleGen sg = {0, 0};
    ReconnectionData reconnection;
    CandidateReservoir reservoir;

    bool hasFlag(uint32_t f) const { return (flagsAndVertexIndex & (f << kVertexIndexBits)) != 0; }
    void setFlag(uint32_t f, bool v = true)
    {
        if (v) flagsAndVertexIndex |= (f << kVertexIndexBits);
        else flagsAndVertexIndex &= ~(f << kVertexIndexBits);
    }
    bool isActive() const { return hasFlag(kActive); }
    bool isHit() const { return hasFlag(kHit); }
    bool isDelta() const { return hasFlag(kDelta); }
    bool isSpecular() const { return hasFlag(kSpecular); }
    bool isLightSampled() const { return (flagsAndVertexIndex & ((kLightSampledUpper | kLightSampledLower) << kVertexIndexBits)) != 0; }
    bool isLightSamplable() const { return !isDelta(); }
    void terminate() { setFlag(kActive, false); }
    uint32_t getVertexIndex() const { return flagsAndVertexIndex & ((1u << kVertexIndexBits) - 1u); }
    void incrementVertexIndex() { flagsAndVertexIndex += 1; }
    uint32_t getBounces(uint32_t type) const { return (bounceCounters >> (type << 3)) & 0xffu; }
    void incrementBounces(uint32_t type) { bounceCounters += (1u << (type << 3)); }
    uint32_t pixelX() const { return id & 0xfffu; }
    uint32_t pixelY() const { return (id >> 12) & 0xfffu; }
    uint32_t sampleIdx() const { return id >> 24; }
    void clearEventFlags() { flagsAndVertexIndex &= ~((kTransmission | kSpecular | kDelta) << kVertexIndexBits); }
};

// ------------------------------------------------------------------ the pass
struct Pass
{
    rs_options opt;
    PreparedScene scene;
    Bvh bvh;
    bool hasScene = false;
    LightView lv;
    // environment map (PathTracer.slang kUseEnvLight = env.present): texels and importance mips
    EnvMapView env = {};
    std::vector<float> envTexels, envImportance;
    std::vector<AnalyticLight> analytic; // the scene's analytic lights (ro_set_analytic_lights)

    uint32_t W = 0, H = 0;
    uint32_t frameCount = 0, seed = 0;
    bool frozen = false;
    bool swapped = false;   // the last frame ended with the curr/prev swap
    uint32_t K = 2;             // camera keyframes
    uint32_t prevK = 0;
    CameraManager cm;
    CameraData camera;           // gScene.camera of this frame
    CameraData prevFrameCamera;  // the previous frame's camera (VBuffer motion vectors)
    bool havePrevFrameCamera = false;

    std::vector<PathReservoir> curr, prev, intermediate, temp, candidates;
    std::vector<ReconnectionData> currR, prevR, intermediateR, tempR, candidatesR;
    std::vector<f2> mvec, floatingCoords;
    std::vector<HitInfo> vbuffer;
    std::vector<uint32_t> cellCounters, cellOffsets, sorted, splatTargets;
    std::vector<std::vector<uint32_t>> mCellCounters, mCellOffsets, mSorted;
    std::vector<ShiftedPathData> shiftedPaths;
    std::vector<f2> neighborOffsets;  // RG8Snorm decoded
    std::vector<f4> prevTri;          // the previous frame's triangles, after a geometry update
    bool geometryMoved = false;       // positions changed since the last frame

    // ---- options
    uint32_t maxSurface() const { return opt.maxSurfaceBounces; }
    uint32_t passSeed(uint32_t k) const { return opt.useFixedSeed ? opt.fixedSeed + k : kNumRenderPasses * (frameCount + seed) + k; }
    SampleGen makeSg(uint32_t px, uint32_t py, uint32_t s) const { return sg_create(px, py, s, opt.sampleGenerator); }
    bool validFloat(f2 p) const { return p.x >= 0.f && p.y >= 0.f && p.x < (float)W && p.y < (float)H; }
    bool validInt(int x, int y) const { return x >= 0 && y >= 0 && x < (int)W && y < (int)H; }
    uint32_t lin(uint32_t x, uint32_t y) const { return y * W + x; }

    // ---- ray queries (replace SceneRayQuery, RaytracingInline.slang:86-362)
    bool traceVisibilityRay(const Ray& r) const { return bvh.visible(r); }
    ShadingData loadSD(const HitInfo& h, f3 rayDir) const { return load_shading_data(scene.tri.data(), scene.materials.data(), h, rayDir); }
    BsdfData instance(const ShadingData& sd) const { return setup_material(scene.materials[sd.materialID], sd.frontFacing); }

    static float evalMIS(uint32_t heuristic, float exponent, float p0, float p1)
    {
        // PathTracer.slang:480-508 with n0 = n1 = 1
        if (heuristic == RS_MIS_HEURISTIC_POWER_TWO)
        {
            float q0 = (1.f * p0) * (1.f * p0), q1 = (1.f * p1) * (1.f * p1);
            return q0 / (q0 + q1);
        }
        if (heuristic == RS_MIS_HEURISTIC_POWER_EXP) // :498-503, pow(n * p, kMISPowerExponent)
        {
            float q0 = f_pow_pos(1.f * p0, exponent), q1 = f_pow_pos(1.f * p1, exponent);
            return q0 / (q0 + q1);
        }
        float q0 = 1.f * p0, q1 = 1.f * p1;
        return q0 / (q0 + q1);
    }
    float mis(float p0, float p1) const { return evalMIS(opt.misHeuristic, opt.misPowerExponent, p0, p1); }

    void orient(CameraData& c, float t) const { c = camera; orient_camera(cm, c, frameCount, t); }

    // ================================================= PathTracer.slang
    bool hasFinishedSurfaceBounces(const PathState& p) const // :161-172
    {
        uint32_t d = p.getBounces(0), s = p.getBounces(1), t = p.getBounces(2);
        uint32_t surf = d + s + t;
        return surf > opt.maxSurfaceBounces || d > opt.maxDiffuseBounces || s > opt.maxSpecularBounces || t > opt.maxTransmissionBounces;
    }

    void generatePath(PathState& path, uint32_t sd, uint32_t pathID) const // :194-221
    {
        path = PathState();
        path.setFlag(kActive);
        path.id = pathID;
        path.thp = mk3(1.f);
        path.sg = makeSg(path.pixelX(), path.pixelY(), sd);
        CameraData cam = camera;
        path.reconnection.time = sampleNext1D(path.sg) * cam.shutterSpeed;
        path.reconnection.subPixel.x = sampleNext1D(path.sg);
        path.reconnection.subPixel.y = sampleNext1D(path.sg);
        if (cam.apertureRadius > 0.f)
        {
            f2 u; u.x = sampleNext1D(path.sg); u.y = sampleNext1D(path.sg);
            path.reconnection.lensSample = sample_disk(u);
        }
        else path.reconnection.lensSample = mk2(0.f, 0.f);
        orient_camera(cm, cam, frameCount, path.reconnection.time);
        Ray r = camera_ray_thinlens(cam, W, H, mk2((float)path.pixelX() + path.reconnection.subPixel.x, (float)path.pixelY() + path.reconnection.subPixel.y), path.reconnection.lensSample);
        path.origin = r.origin;
        path.dir = r.dir;
        path.prevHitPos = camera_lens_point(cam, path.reconnection.lensSample);
    }

    void generatePathWithParameters(PathState& path, uint32_t sd, float time, f2 fractionalPixel, f2 lensSample) const // :230-255
    {
        path = PathState();
        path.setFlag(kActive);
        path.thp = mk3(1.f);
        path.sg = makeSg((uint32_t)fractionalPixel.x, (uint32_t)fractionalPixel.y, sd);
        CameraData cam = camera;
        orient_camera(cm, cam, frameCount, time);
        path.time = time;
        Ray r = camera_ray_thinlens(cam, W, H, fractionalPixel, lensSample);
        path.origin = r.origin;
        path.dir = r.dir;
        path.prevHitPos = camera_lens_point(cam, path.reconnection.lensSample);
    }

    void nextHit(PathState& path) const // :278-299
    {
        path.incrementVertexIndex();
        Ray r = mk_ray(path.origin, path.dir, 0.f, kRayTMax);
        HitInfo h; float t;
        if (bvh.closest(r, h, t)) { path.hit = h; path.setFlag(kHit); }
        else path.setFlag(kHit, false);
    }

    // generateScatterRay(bs, ...) (:391-471), reflection-only materials
    bool generateScatterRayBS(const BSDFSample& bs, const ShadingData& sd, const BsdfData& d, PathState& path) const
    {
        path.dir = bs.wo;
        path.thp *= bs.weight;
        path.clearEventFlags();
        if (bs.lobeType & kLobeReflection)
        {
            float roughness = mi_roughness(d);
            bool isDiffuse = (bs.lobeType & kLobeDiffuseReflection) || roughness > opt.specularRoughnessThreshold;
            if (isDiffuse) path.incrementBounces(0);
            else { path.incrementBounces(1); path.setFlag(kSpecular); }
        }
        if (bs.lobeType & kLobeDelta) path.setFlag(kDelta);
        path.normal = sd_oriented_face_normal(sd);
        return any_gt0(path.thp);
    }

    // generateScatterRay(sd, mi, path) (:331-382)
    // componentOut (the adjoint's suffix replay): the sampled lobe's BSDF component type
    bool generateScatterRay(const ShadingData& sd, const BsdfData& d, PathState& path, uint32_t* componentOut = nullptr) const
    {
        BSDFSample result;
        result.wo = mk3(0.f); result.pdf = 0.f; result.weight = mk3(0.f); result.lobeType = 0;
        bool valid = mi_sample(sd, d, 1u, path.sg, result);
        path.pdf = result.pdf;
        uint32_t componentType = 0;
        if (result.lobeType & kLobeDiffuseReflection)
        {
            if ((result.lobeType & kLobeSpecular) || (result.lobeType & kLobeDelta)) { componentType = 3; result.lobeType &= ~kLobeDiffuseReflection; }
        }
        else
        {
            if (result.lobeType & kLobeDiffuseTransmission) componentType = 1;
            else if ((result.lobeType & kLobeSpecular) || (result.lobeType & kLobeDelta)) componentType = 2;
        }
        if (path.getVertexIndex() == 1) path.reconnection.firstBSDFComponentType = componentType;
        else if (path.getVertexIndex() == 2)
        {
            path.reconnection.secondBSDFComponentType = componentType;
            path.reconnection.secondWo = result.wo;
        }
        path.totalPdf = mi_pdf(sd, d, 0xFu, result.wo);
        if (componentOut) *componentOut = componentType;
        if (valid) generateScatterRayBS(result, sd, d, path);
        if (path.getVertexIndex() == 1 || path.getVertexIndex() == 2)
        {
            path.reconnection.earlyThroughput *= result.weight;
            path.thp = mk3(1.f);
        }
        return valid;
    }

    struct LightSample
    {
        f3 Li; float pdf; f3 origin; float distance; f3 dir; uint32_t triangleId; f2 barycentrics; float geometryTerm;
        uint32_t lightType; // 0 env map, 1 emissive, 2 analytic (LightType)
    };

    // getLightTypeSelectionProbabilities (:606-622): p = {env, emissive, analytic} normalised
    void lightTypeProbabilities(float& pEnv, float& pEmissive, float& pAnalytic) const
    {
        light_type_probabilities(env.present != 0, lv.count > 0, !analytic.empty(), pEnv, pEmissive, pAnalytic);
    }

    // generateLightSample (:668-701); the type-selection draw is always taken.
    bool generateLightSample(f3 vpos, f3 vfaceN, bool vfront, bool sampleUpper, bool sampleLower, SampleGen& sg, LightSample& ls) const
    {
        ls = LightSample();
        float p[3];
        lightTypeProbabilities(p[0], p[1], p[2]);
        float u = sampleNext1D(sg);
        // selectLightType (:634-656)
        uint32_t lightType = 3;
        for (uint32_t t = 0; t < 3; t++)
        {
            if (u < p[t]) { lightType = t; break; }
            u -= p[t];
        }
        if (lightType == 3) return false;
        float selectionPdf = p[lightType];
        ls.lightType = lightType;
        if (lightType == 0)
        {
            // generateEnvMapSample (:516-534)
            f2 r; r.x = sampleNext1D(sg); r.y = sampleNext1D(sg);
            f3 Le;
            env_sample(env, r, ls.dir, ls.pdf, Le);
            ls.Li = ls.pdf > 0.f ? Le / ls.pdf : mk3(0.f);
            ls.origin = computeRayOrigin(vpos, dot(vfaceN, ls.dir) >= 0.f ? vfaceN : -vfaceN);
            ls.distance = kRayTMax;
        }
        else if (lightType == 2)
        {
            // generateAnalyticLightSample (:573-599)
            AnalyticLightView av;
            av.lights = analytic.data();
            av.count = (uint32_t)analytic.size();
            AnalyticSample as;
            if (!analytic_light_sample(av, vpos, sg, as)) return false;
            ls.Li = as.Li;
            ls.pdf = as.pdf;
            ls.dir = as.dir;
            ls.distance = as.distance;
            ls.origin = computeRayOrigin(vpos, dot(vfaceN, ls.dir) >= 0.f ? vfaceN : -vfaceN);
        }
        else
        {
            // generateEmissiveSample (:543-565)
            TriangleLightSample tls;
            if (!sample_emissive(lv, vpos, sg, tls)) return false;
            ls.Li = tls.pdf > 0.f ? tls.Le / tls.pdf : mk3(0.f);
            ls.pdf = tls.pdf;
            f3 lightPos = computeRayOrigin(tls.posW, tls.normalW);
            f3 toL = lightPos - vpos;
            ls.origin = computeRayOrigin(vpos, dot(vfaceN, toL) >= 0.f ? vfaceN : -vfaceN);
            f3 toLight = lightPos - ls.origin;
            ls.distance = length(toLight);
            ls.dir = normalize(toLight);
            ls.barycentrics = tls.uv;
            ls.triangleId = tls.triangleIndex;
            ls.geometryTerm = tls.geometryTerm;
        }
        if (!any_gt0(ls.Li)) return false;
        float NdotL = dot(vfront ? vfaceN : -vfaceN, ls.dir);
        if ((!sampleUpper && NdotL >= -kMinCosTheta) || (!sampleLower && NdotL <= kMinCosTheta)) return false;
        ls.pdf *= selectionPdf;
        ls.Li /= selectionPdf;
        return true;
    }

    // handleHit (:783-1168)
    void handleHit(PathState& path) const
    {
        const bool isPrimaryHit = path.getVertexIndex() == 1;
        ShadingData sd = loadSD(path.hit, path.dir);
        float distanceToPrevVertex = length(sd.posW - path.prevHitPos);
        float geometryFactor = f_abs(dot(sd.faceN, sd.V)) / (distanceToPrevVertex * distanceToPrevVertex);
        float prevScatterPdf = path.pdf;
        path.prevHitPos = sd.posW;

        if (path.getVertexIndex() == 1)
        {
            path.reconnection.firstHit = path.hit;
            path.reconnection.firstWi = -path.dir;
            CameraData cam; orient(cam, path.time);
            f3 x0 = camera_lens_point(cam, path.reconnection.lensSample);
            float dist = length(sd.posW - x0);
            float distSquared = dist * dist;
            float cosNormal = dot(-path.dir, sd.faceN);
            float cosSensor = dot(normalize(cam.cameraW), path.dir);
            path.reconnection.subPixelJacobian = f_abs(cosNormal / distSquared) / f_abs(f_pow3(cosSensor));
            f3 camDir = normalize(cam.cameraW);
            float camZ = dot(sd.posW - cam.posW, camDir);
            float d0 = (length(cam.cameraW) / f_abs(camZ) * dist);
            float d1 = dist - d0;
            path.reconnection.lensVertexJacobian = (d0 * d0) / (d1 * d1) * (f_abs(dot(-path.dir, sd.faceN))) / (f_abs(dot(-path.dir, camDir)));
        }
        else if (path.getVertexIndex() == 2)
        {
            path.reconnection.secondHit = path.hit;
            path.reconnection.secondaryPathJacobian = prevScatterPdf * geometryFactor;
        }
        else if (path.getVertexIndex() == 3)
        {
            path.reconnection.secondaryPathJacobian *= prevScatterPdf;
            path.reconnection.suffixSeed = (uint32_t)path.sg.state;
            path.reconnection.suffixState = suffix_state_pack(path.bounceCounters, path.flagsAndVertexIndex >> kVertexIndexBits);
        }

        BsdfData d = instance(sd);
        const bool isLightSamplable = path.isLightSamplable();
        bool computeEmissive = isPrimaryHit || (lv.count > 0 && (!path.isLightSampled() || !isLightSamplable));
        if (computeEmissive && any_gt0(d.emission))
        {
            float misWeight = 1.f;
            float lightPdf = 0.f;
            if (lv.count > 0 && !isPrimaryHit && path.isLightSampled() && isLightSamplable)
            {
                // upperHemisphere is ignored by the power sampler
                float pEnv, pEmissive, pAnalytic;
                lightTypeProbabilities(pEnv, pEmissive, pAnalytic);
                lightPdf = pEmissive * eval_emissive_pdf(lv, path.origin, sd.lightIndex, sd.posW, sd_oriented_face_normal(sd));
                misWeight = mis(path.totalPdf, lightPdf);
            }
            bool selected = path.reservoir.addVertex(path.sg, 1.f, path.reconnection.earlyThroughput * path.thp * d.emission * misWeight);
            if (selected)
            {
                path.reservoir.selectedReconnection = path.reconnection;
                ReconnectionData& s = path.reservoir.selectedReconnection;
                s.pathLength = path.getVertexIndex();
                s.lightIsNEE = false;
                s.lightIsDistant = false;
                s.lightPdf = lightPdf;
                if (path.getVertexIndex() == 2) s.lightPdf *= geometryFactor;
                if (path.getVertexIndex() == 2 || path.getVertexIndex() == 3) s.irradiance = d.emission;
                else s.irradiance = path.thp * d.emission * misWeight;
            }
        }

        if (hasFinishedSurfaceBounces(path)) { path.terminate(); return; }

        path.origin = sd_ray_origin(sd, true);

        const uint32_t lobeTypes = mi_lobe_types(d);
        const bool hasNonDeltaLobes = (lobeTypes & kLobeNonDelta) != 0;
        path.setFlag(kLightSampledUpper, false); path.setFlag(kLightSampledLower, false);
        if (hasNonDeltaLobes)
        {
            bool sampleUpper = (lobeTypes & kLobeNonDeltaReflection) != 0;
            bool sampleLower = (lobeTypes & kLobeNonDeltaTransmission) != 0;
            LightSample ls;
            bool validSample = generateLightSample(sd.posW, sd.faceN, sd.frontFacing, sampleUpper, sampleLower, path.sg, ls);
            path.setFlag(kLightSampledUpper, sampleUpper); path.setFlag(kLightSampledLower, sampleLower);
            if (validSample)
            {
                f3 Le = ls.Li * ls.pdf;
                // analytic lights: no scatter pdf, MIS weight 1 (:1025-1031)
                float scatterPdf = ls.lightType == 2 ? 0.f : mi_pdf(sd, d, 0u, ls.dir);
                float misWeight = ls.lightType == 2 ? 1.f : mis(ls.pdf, scatterPdf);
                f3 weight = mi_eval(sd, d, 0u, ls.dir);
                f3 Lr = weight * misWeight * ls.Li;
                if (any_gt0(Lr))
                {
                    Ray ray = mk_ray(ls.origin, ls.dir, 0.f, ls.distance);
                    if (traceVisibilityRay(ray))
                    {
                        bool selected = path.reservoir.addVertex(path.sg, 1.f, path.reconnection.earlyThroughput * path.thp * weight * ls.Li * misWeight);
                        if (selected)
                        {
                            path.reservoir.selectedReconnection = path.reconnection;
                            ReconnectionData& s = path.reservoir.selectedReconnection;
                            s.pathLength = path.getVertexIndex() + 1;
                            s.lightIsNEE = true;
                            s.irradiance = Le;
                            if (path.getVertexIndex() == 1) s.transmissionEvent = dot(sd.faceN, sd.V) * dot(sd.faceN, ls.dir) < 0.f;
                            s.lightIsDistant = ls.lightType == 0;
                            if (path.getVertexIndex() == 1)
                            {
                                if (ls.lightType == 0)
                                {
                                    s.secondHit = hit_direction(ls.dir);
                                    s.secondaryPathJacobian = ls.pdf;
                                    s.lightPdf = ls.pdf; // a distant light: no area measure
                                }
                                else if (ls.lightType == 1) // an analytic light leaves the light vertex unset
                                {
                                    s.secondHit = hit_tri(lv.tris[ls.triangleId].sceneTri, ls.barycentrics.x, ls.barycentrics.y);
                                    s.secondaryPathJacobian = ls.pdf * ls.geometryTerm;
                                    s.lightPdf = ls.pdf * ls.geometryTerm;
                                }
                            }
                            else if (path.getVertexIndex() == 2)
                            {
                                s.secondWo = ls.dir;
                                s.lightPdf = ls.pdf;
                            }
                            else
                            {
                                s.irradiance = path.thp * Lr;
                            }
                        }
                    }
                }
            }
        }

        if (opt.useRussianRoulette)
        {
            float u = sampleNext1D(path.sg);
            // terminatePathByRussianRoulette (:743-754)
            const float rrVal = luminance(path.thp);
            const float prob = f_max(0.f, 1.f - rrVal);
            if (u < prob) { path.terminate(); return; }
            path.thp /= 1.f - prob;
        }

        bool valid = generateScatterRay(sd, d, path);
        const bool isLastVertex = hasFinishedSurfaceBounces(path);
        if (isLastVertex && path.isLightSamplable()) valid = false;
        if (opt.disableCaustics && path.getBounces(0) > 0 && path.isSpecular()) valid = false;
        if (!valid) path.terminate();
    }

    // handleMiss (:1433-1524)
    void handleMiss(PathState& path) const
    {
        float prevScatterPdf = path.pdf;
        float geometryFactor = 1.f;
        if (path.getVertexIndex() == 2) path.reconnection.secondaryPathJacobian = prevScatterPdf * geometryFactor;
        else if (path.getVertexIndex() == 3) path.reconnection.secondaryPathJacobian *= prevScatterPdf;
        const bool isLightSamplable = path.isLightSamplable();
        bool computeEnv = env.present && (!path.isLightSampled() || !isLightSamplable);
        if (computeEnv)
        {
            float misWeight = 1.f;
            float lightPdf = 0.f;
            if (path.isLightSampled() && isLightSamplable)
            {
                float pEnv, pEmissive, pAnalytic;
                lightTypeProbabilities(pEnv, pEmissive, pAnalytic);
                lightPdf = pEnv * env_eval_pdf(env, path.dir);
                misWeight = mis(path.totalPdf, lightPdf);
            }
            f3 Le = env_eval(env, path.dir);
            f3 emitterRadiance = misWeight * Le;
            bool selected = path.reservoir.addVertex(path.sg, 1.f, path.reconnection.earlyThroughput * path.thp * Le * misWeight);
            if (selected)
            {
                path.reservoir.selectedReconnection = path.reconnection;
                ReconnectionData& s = path.reservoir.selectedReconnection;
                s.pathLength = path.getVertexIndex();
                s.lightIsNEE = false;
                s.lightIsDistant = true;
                s.lightPdf = lightPdf;
                if (path.getVertexIndex() == 2) s.secondHit = hit_direction(path.dir);
                if (path.getVertexIndex() == 2 || path.getVertexIndex() == 3) s.irradiance = Le;
                else s.irradiance = path.thp * emitterRadiance;
            }
        }
        path.terminate();
    }

    // handlePrimaryMiss (:1529-1569)
    void handlePrimaryMiss(PathState& path) const
    {
        if (env.present)
        {
            f3 Le = env_eval(env, path.dir);
            bool selected = path.reservoir.addVertex(path.sg, 1.f, Le);
            if (selected)
            {
                path.reservoir.selectedReconnection = path.reconnection;
                ReconnectionData& s = path.reservoir.selectedReconnection;
                s.lightIsDistant = true;
                CameraData cam; orient(cam, path.time);
                f3 camDir = normalize(cam.cameraW);
                float cosSensor = dot(camDir, path.dir);
                s.subPixelJacobian = 1.f / f_abs(f_pow3(cosSensor));
                float focalPlaneZ = length(cam.cameraW);
                float d0 = focalPlaneZ / dot(camDir, path.dir);
                s.lensVertexJacobian = (d0 * d0) / f_abs(cosSensor);
                s.firstWi = -path.dir;
                s.pathLength = 1;
                s.irradiance = Le;
            }
        }
        path.terminate();
    }

    // handleReconnectionHit (:1177-1397)
    f3 handleReconnectionHit(PathState& path, const ReconnectionData& rd, float& dstJacobian) const
    {
        ShadingData sd = loadSD(path.hit, path.dir);
        BsdfData d = instance(sd);
        path.origin = sd_ray_origin(sd, true);
        if (rd.transmissionEvent) path.origin = sd_ray_origin(sd, false);
        bool secondHitIsDistant = (rd.pathLength == 2) && rd.lightIsDistant;
        dstJacobian = 1.f;
        f3 nextDir = mk3(0.f);
        float rayLength = kRayTMax;
        if (!secondHitIsDistant)
        {
            ShadingData secondSd = hit_valid(rd.secondHit) ? loadSD(rd.secondHit, mk3(0.f)) : sd_zero_vertex(); // LoadShadingData.slang:69-74
            f3 shiftedOffset = secondSd.posW - sd.posW;
            float shiftedDist2 = dot(shiftedOffset, shiftedOffset);
            float shiftedCosine = f_abs(dot(secondSd.faceN, -normalize(shiftedOffset)));
            dstJacobian = shiftedCosine / shiftedDist2;
            f3 adjustedOffset = secondSd.posW - path.origin;
            nextDir = normalize(adjustedOffset);
            rayLength = length(adjustedOffset) * 0.999f;
        }
        else nextDir = hit_as_direction(rd.secondHit);

        uint32_t lobeMask = 1u << rd.firstBSDFComponentType;
        f3 lobeScatterBsdf = mi_eval(sd, d, lobeMask, nextDir);
        float lobeScatterPdf = mi_pdf(sd, d, lobeMask, nextDir);
        f3 totalScatterBsdf = mi_eval(sd, d, 0u, nextDir);
        float totalScatterPdf = mi_pdf(sd, d, 0u, nextDir);
        path.dir = nextDir;
        path.pdf = lobeScatterPdf;

        if (rd.pathLength == 2)
        {
            float lightPdf = rd.lightPdf / dstJacobian;
            float misWeight = 1.f;
            if (rd.lightIsNEE)
            {
                if (!any_gt0(totalScatterBsdf) || totalScatterPdf == 0.f) { path.terminate(); return sd.posW; }
                dstJacobian *= lightPdf;
                misWeight = mis(lightPdf, totalScatterPdf);
                path.thp *= totalScatterBsdf / lightPdf;
            }
            else
            {
                if (!any_gt0(lobeScatterBsdf) || lobeScatterPdf == 0.f) { path.terminate(); return sd.posW; }
                dstJacobian *= lobeScatterPdf;
                misWeight = mis(totalScatterPdf, lightPdf);
                path.thp *= lobeScatterBsdf / lobeScatterPdf;
            }
            path.thp *= misWeight;
        }
        else
        {
            if (!any_gt0(lobeScatterBsdf) || lobeScatterPdf == 0.f) { path.terminate(); return sd.posW; }
            dstJacobian *= lobeScatterPdf;
            path.thp *= lobeScatterBsdf / lobeScatterPdf;
        }
        bool valid = any_gt0(path.thp);
        if (opt.disableCaustics && path.getBounces(0) > 0 && path.isSpecular()) valid = false;
        if (!valid) path.terminate();
        else
        {
            Ray reconnectionRay = mk_ray(path.origin, path.dir, 0.f, rayLength);
            if (!traceVisibilityRay(reconnectionRay)) path.terminate();
        }
        return sd.posW;
    }

    // handleReconnectionPrimaryLight (:1399-1410)
    // handleReconnectionEnvMap (:1412-1416)
    f3 handleReconnectionEnvMap(const PathState& path) const { return env_reconnection(env, path.dir); }

    f3 handleReconnectionPrimaryLight(const PathState& path) const
    {
        ShadingData sd = loadSD(path.hit, path.dir);
        return instance(sd).emission;
    }

    // ================================================= ShiftMapping.slang
    // pathReconnectionShift (:430-513)
    f3 pathReconnectionShift(const ReconnectionData& rd, PathState& path, float& dstJacobian) const
    {
        dstJacobian = 1.f;
        handleReconnectionHit(path, rd, dstJacobian);
        if (!path.isActive()) return mk3(0.f);
        // Length 2 uses none of the x2 terms (misWeight stays 1); the reference still loads x2's
        // shading data, which for an environment vertex is a direction, not a hit, so skip it.
        if (rd.pathLength == 2) return 1.f * path.thp * rd.irradiance;
        ShadingData secondSd = loadSD(rd.secondHit, path.dir);
        BsdfData d = instance(secondSd);
        uint32_t lobeMask = 1u << rd.secondBSDFComponentType;
        f3 lobeSpecificBsdf = mi_eval(secondSd, d, lobeMask, rd.secondWo);
        float lobeSpecificPdf = mi_pdf(secondSd, d, lobeMask, rd.secondWo);
        f3 totalBsdf = mi_eval(secondSd, d, 0xFu, rd.secondWo);
        float totalPdf = mi_pdf(secondSd, d, 0xFu, rd.secondWo);
        if (rd.pathLength > 2 && !any_gt0(totalBsdf)) return mk3(0.f);
        float misWeight = 1.f;
        if (rd.pathLength == 3)
        {
            bool valid = rd.lightIsNEE ? true : (lobeSpecificPdf > 0.f);
            if (!valid) return mk3(0.f);
            misWeight = rd.lightIsNEE ? mis(rd.lightPdf, totalPdf) : mis(totalPdf, rd.lightPdf);
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

    // gatherLensVertexCopyShift (:90-180); sg is a copy (by value)
    ShiftedPathData gatherLensVertexCopyShift(SampleGen sg, const ReconnectionData& rd, float time, f2 fractionalPixel, f2 lensSample) const
    {
        ShiftedPathData sp;
        if (!validFloat(fractionalPixel)) return ShiftedPathData();
        const bool hitEnvMap = (rd.pathLength == 1 && rd.lightIsDistant);
        PathState path;
        uint32_t s = f2u(sampleNext1D(sg));
        generatePathWithParameters(path, s, time, fractionalPixel, lensSample);
        nextHit(path);
        CameraData cam; orient(cam, time);
        path.time = time;
        path.origin = camera_lens_point_scaled(cam, lensSample);
        f3 camDir = normalize(cam.cameraW);
        sp.primaryHit = path.hit;
        sp.firstRayDir = path.dir;
        sp.fractionalPixel = fractionalPixel;
        sp.lensSample = lensSample;
        if (path.isHit())
        {
            if (hitEnvMap) return ShiftedPathData();
            ShadingData firstSd = loadSD(path.hit, path.dir);
            f3 x1 = firstSd.posW;
            float dist = length(x1 - path.origin);
            float distSquared = dist * dist;
            float cosNormal = dot(-path.dir, firstSd.faceN);
            float cosSensor = dot(camDir, path.dir);
            sp.subPixelJacobian = f_abs(cosNormal / distSquared) / f_abs(f_pow3(cosSensor));
            float camZ = dot(x1 - cam.posW, camDir);
            float d0 = (length(cam.cameraW) / f_abs(camZ) * dist);
            float d1 = dist - d0;
            sp.lensVertexJacobian = (d0 * d0) / (d1 * d1) * f_abs(cosNormal) / f_abs(cosSensor);
        }
        else
        {
            if (!hitEnvMap) return ShiftedPathData(); // an expected hit that misses fails
            sp.radiance = handleReconnectionEnvMap(path);
            float cosSensor = dot(camDir, path.dir);
            sp.subPixelJacobian = 1.f / f_abs(f_pow3(cosSensor));
            float focalPlaneZ = length(cam.cameraW);
            float d0 = focalPlaneZ / dot(camDir, path.dir);
            sp.lensVertexJacobian = (d0 * d0) / f_abs(cosSensor);
            return sp;
        }
        if (rd.pathLength == 1)
        {
            sp.radiance = handleReconnectionPrimaryLight(path);
            return sp;
        }
        sp.radiance = pathReconnectionShift(rd, path, sp.secondaryPathJacobian);
        return sp;
    }

    // gatherPrimaryHitReconnectionShift (:183-296)
    ShiftedPathData gatherPrimaryHitReconnectionShift(SampleGen sg, const ReconnectionData& rd, float time, f2 fractionalPixel, const HitInfo& primaryHit) const
    {
        ShiftedPathData sp;
        const bool hitEnvMap = (rd.pathLength == 1 && rd.lightIsDistant);
        PathState path;
        path.setFlag(kActive);
        path.thp = mk3(1.f);
        CameraData cam; orient(cam, time);
        path.time = time;
        f2 p = mk2(fractionalPixel.x / (float)W, fractionalPixel.y / (float)H);
        f2 ndc = mk2(2.f * p.x + -1.f, -2.f * p.y + 1.f);
        f3 filmWorld = cam.posW + (cam.cameraU * ndc.x + cam.cameraV * ndc.y + cam.cameraW);
        f3 x1, n;
        if (hitEnvMap)
        {
            path.dir = -rd.firstWi;
            x1 = filmWorld + path.dir;
            n = mk3(0.f);
        }
        else
        {
            if (!hit_valid(primaryHit)) return ShiftedPathData();
            ShadingData sd = loadSD(primaryHit, mk3(0.f));
            x1 = sd.posW;
            path.dir = normalize(x1 - filmWorld);
            n = sd.faceN;
        }
        f3 camDir = normalize(cam.cameraW);
        float camZ = dot(x1 - cam.posW, camDir);
        float rayT = camZ / dot(path.dir, camDir);
        path.origin = x1 - path.dir * rayT;
        path.dir = hitEnvMap ? path.dir : normalize(x1 - path.origin);
        f3 lensOffsetWorld = path.origin - cam.posW;
        f2 lensLocalNormalized = mk2(dot(lensOffsetWorld, normalize(cam.cameraU)) / cam.apertureRadius,
                                     dot(lensOffsetWorld, normalize(cam.cameraV)) / cam.apertureRadius);
        if (length(lensLocalNormalized) > 1.f) return ShiftedPathData();
        float dist = length(x1 - path.origin);
        float rayMin = hitEnvMap ? 0.001f : 0.001f * dist;
        float rayMax = hitEnvMap ? kRayTMax : 0.999f * dist;
        if (!traceVisibilityRay(mk_ray(path.origin, path.dir, rayMin, rayMax))) return ShiftedPathData();
        sp.firstRayDir = path.dir;
        sp.fractionalPixel = fractionalPixel;
        sp.lensSample = lensLocalNormalized;
        sp.primaryHit = primaryHit;
        path.sg = makeSg((uint32_t)fractionalPixel.x, (uint32_t)fractionalPixel.y, f2u(sampleNext1D(sg)));
        path.incrementVertexIndex();
        path.hit = primaryHit; path.setFlag(kHit);
        if (hitEnvMap)
        {
            sp.radiance = handleReconnectionEnvMap(path);
            float cosSensor = dot(camDir, path.dir);
            sp.subPixelJacobian = 1.f / f_abs(f_pow3(cosSensor));
            float focalPlaneZ = length(cam.cameraW);
            float d0 = focalPlaneZ / dot(camDir, path.dir);
            sp.lensVertexJacobian = (d0 * d0) / f_abs(dot(camDir, path.dir));
            return sp;
        }
        {
            float dist2 = length(x1 - path.origin);
            float distSquared = dist2 * dist2;
            float cosNormal = dot(path.dir, n);
            float cosSensor = dot(camDir, path.dir);
            sp.subPixelJacobian = f_abs(cosNormal / distSquared) / f_abs(f_pow3(cosSensor));
            float d0 = (length(cam.cameraW) / f_abs(camZ) * rayT);
            float d1 = rayT - d0;
            sp.lensVertexJacobian = (d0 * d0) / (d1 * d1) * (f_abs(cosNormal)) / (f_abs(cosSensor));
        }
        if (rd.pathLength == 1)
        {
            sp.radiance = handleReconnectionPrimaryLight(path);
            return sp;
        }
        sp.radiance = pathReconnectionShift(rd, path, sp.secondaryPathJacobian);
        return sp;
    }

    // scatterReprojectionShift (:301-421)
    ShiftedPathData scatterReprojectionShift(SampleGen sg, const ReconnectionData& rd, float time, const HitInfo& primaryHit, f2 lensSample, bool skipVisibilityCheck) const
    {
        ShiftedPathData sp;
        const bool hitEnvMap = (rd.pathLength == 1) && rd.lightIsDistant;
        PathState path;
        path.setFlag(kActive);
        path.thp = mk3(1.f);
        CameraData cam; orient(cam, time);
        path.time = time;
        f2 lensLocal = mk2(cam.apertureRadius * lensSample.x, cam.apertureRadius * lensSample.y);
        f3 camU = normalize(cam.cameraU);
        f3 camV = normalize(cam.cameraV);
        f3 lensWorld = camU * lensLocal.x + camV * lensLocal.y;
        path.origin = cam.posW + lensWorld;
        f3 x1 = mk3(0.f), n = mk3(0.f);
        if (hitEnvMap) path.dir = -rd.firstWi;
        else
        {
            if (!hit_valid(primaryHit)) return ShiftedPathData();
            ShadingData firstSd = loadSD(primaryHit, mk3(0.f));
            x1 = firstSd.posW;
            n = firstSd.faceN;
            path.dir = normalize(x1 - path.origin);
        }
        f3 camDir = normalize(cam.cameraW);
        f3 camRay = mk3(dot(camU, path.dir), dot(camV, path.dir), dot(camDir, path.dir));
        if (camRay.z <= 0.001f) return ShiftedPathData();
        float lw = length(cam.cameraW);
        f2 film = mk2(lensLocal.x + lw * (camRay.x / camRay.z), lensLocal.y + lw * (camRay.y / camRay.z));
        f2 ndc = mk2(film.x / length(cam.cameraU), film.y / length(cam.cameraV));
        f2 nfp = mk2((0.5f * ndc.x + 0.5f) * (float)W, (-0.5f * ndc.y + 0.5f) * (float)H);
        if (!validFloat(nfp)) return ShiftedPathData();
        float dist = length(x1 - path.origin);
        float rayMax = hitEnvMap ? kRayTMax : 0.999f * dist;
        if (!skipVisibilityCheck && !traceVisibilityRay(mk_ray(path.origin, path.dir, 0.001f, rayMax))) return ShiftedPathData();
        sp.lensSample = lensSample;
        sp.firstRayDir = path.dir;
        sp.fractionalPixel = nfp;
        sp.primaryHit = primaryHit;
        path.sg = makeSg((uint32_t)nfp.x, (uint32_t)nfp.y, f2u(sampleNext1D(sg)));
        path.incrementVertexIndex();
        path.hit = primaryHit; path.setFlag(kHit);
        if (hitEnvMap)
        {
            sp.radiance = handleReconnectionEnvMap(path);
            float cosSensor = dot(camDir, path.dir);
            sp.subPixelJacobian = 1.f / f_abs(f_pow3(cosSensor));
            float focalPlaneZ = length(cam.cameraW);
            float d0 = focalPlaneZ / dot(camDir, path.dir);
            sp.lensVertexJacobian = (d0 * d0) / f_abs(cosSensor);
            return sp;
        }
        {
            float distSquared = dist * dist;
            float cosNormal = dot(-path.dir, n);
            float cosSensor = dot(normalize(cam.cameraW), path.dir);
            sp.subPixelJacobian = f_abs(cosNormal / distSquared) / f_abs(f_pow3(cosSensor));
            float camZ = dot(x1 - cam.posW, camDir);
            float d0 = (length(cam.cameraW) / f_abs(camZ) * dist);
            float d1 = dist - d0;
            sp.lensVertexJacobian = (d0 * d0) / (d1 * d1) * f_abs(cosNormal) / f_abs(cosSensor);
        }
        if (rd.pathLength == 1)
        {
            sp.radiance = handleReconnectionPrimaryLight(path);
            return sp;
        }
        sp.radiance = pathReconnectionShift(rd, path, sp.secondaryPathJacobian);
        return sp;
    }

    // ShiftMapping.slang:43-80 (circle of confusion uses the scene camera, not the oriented one)
    float primaryHitCoC(f3 x1) const
    {
        float lensRadius = camera.apertureRadius;
        f3 camDir = normalize(camera.cameraW);
        float camZ = dot(x1 - camera.posW, camDir);
        float filmZ = camZ - length(camera.cameraW);
        float filmRadius = f_abs(lensRadius / camZ * filmZ);
        float normalizedFilm = length(camera.cameraU / (float)W + camera.cameraV / (float)H);
        return filmRadius / normalizedFilm;
    }
    float envCoC() const
    {
        float normalizedFilm = length(camera.cameraU / (float)W + camera.cameraV / (float)H);
        return camera.apertureRadius / normalizedFilm;
    }
    static f2 dofProbs(float r)
    {
        float gamma = 0.2f + 6.2f / (r - 5.6f);
        gamma = (r <= 0.2f) ? 1.f : f_clamp(gamma, 0.2f, 1.f);
        return mk2(gamma, 1.f - gamma);
    }
    f2 pixelDofProbs(uint32_t x, uint32_t y) const
    {
        if (!(camera.apertureRadius > 0.f)) return mk2(1.f, 0.f);
        const HitInfo& h = vbuffer[lin(x, y)];
        float coc = hit_valid(h) ? primaryHitCoC(loadSD(h, mk3(0.f)).posW) : envCoC();
        return dofProbs(coc);
    }

    // ================================================= passes
    // InitialCandidates.cs.slang:52-141
    void initialCandidates()
    {
        const uint32_t spp = opt.samplesPerPixel;
        #pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < (int)H; y++)
            for (uint32_t x = 0; x < W; x++)
                for (uint32_t sIdx = 0; sIdx < spp; sIdx++)
                {
                    uint32_t pathID = x | ((uint32_t)y << 12) | (spp == 1 ? 0u : (sIdx << 24));
                    PathState path;
                    generatePath(path, opt.useFixedSeed ? opt.fixedSeed + 0 : kNumRenderPasses * (frameCount + seed) + 0, pathID);
                    nextHit(path);
                    if (path.isHit())
                    {
                        handleHit(path);
                        while (path.isActive())
                        {
                            nextHit(path);
                            if (path.isHit()) handleHit(path);
                            else handleMiss(path);
                        }
                    }
                    else
                    {
                        handlePrimaryMiss(path);
                    }
                    // addCandidateReservoir (:52-75)
                    const bool isFirstSample = (path.sampleIdx() == (spp - 1));
                    uint32_t idx = lin(x, (uint32_t)y);
                    PathReservoir ex = isFirstSample ? PathReservoir() : curr[idx];
                    bool selected = ex.add(path.sg, 1.f / (float)spp, path.reservoir);
                    ex.subPixel = selected ? path.reconnection.subPixel : ex.subPixel;
                    ex.confidence = 1.f;
                    curr[idx] = ex;
                    ReconnectionData exr = isFirstSample ? ReconnectionData() : currR[idx];
                    currR[idx] = selected ? path.reservoir.selectedReconnection : exr;
                }
    }

    // VBufferRT.slang:71-150 with samplePattern "Center" and no depth of field: primary hit and
    // motion vector mvec = prevScreenPos - (pixel + 0.5) / dim.  The previous-frame projection is the
    // film projection of the previous frame's camera (the same projection the splat uses).
    void vbufferPass()
    {
        const CameraData& pc = havePrevFrameCamera ? prevFrameCamera : camera;
        #pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < (int)H; y++)
            for (uint32_t x = 0; x < W; x++)
            {
                f2 p = mk2(((float)x + 0.5f) / (float)W, ((float)y + 0.5f) / (float)H);
                f2 ndc = mk2(2.f * p.x + -1.f, -2.f * p.y + 1.f);
                f3 dir = normalize(camera.cameraU * ndc.x + camera.cameraV * ndc.y + camera.cameraW);
                HitInfo h; float t;
                uint32_t idx = lin(x, (uint32_t)y);
                if (bvh.closest(mk_ray(camera.posW, dir, 0.f, kRayTMax), h, t))
                {
                    vbuffer[idx] = h;
                    // Scene::getPrevPosW (VBufferRT.slang:84): the hit on the previous frame's geometry
                    f3 prevPosW = hit_position(geometryMoved ? prevTri.data() : scene.tri.data(), h);
                    f3 d = prevPosW - pc.posW;
                    f3 camRay = mk3(dot(normalize(pc.cameraU), d), dot(normalize(pc.cameraV), d), dot(normalize(pc.cameraW), d));
                    float lw = length(pc.cameraW);
                    f2 film = mk2(lw * (camRay.x / camRay.z), lw * (camRay.y / camRay.z));
                    f2 pndc = mk2(film.x / length(pc.cameraU), film.y / length(pc.cameraV));
                    f2 prevCrd = mk2(0.5f * pndc.x + 0.5f, -0.5f * pndc.y + 0.5f);
                    mvec[idx] = mk2(prevCrd.x - p.x, prevCrd.y - p.y);
                }
                else
                {
                    vbuffer[idx] = hit_none();
                    // writeMiss (VBufferRT.slang:128-149)
                    mvec[idx] = env.present ? env_miss_motion_vector(camera, pc, dir, p) : mk2(0.f, 0.f);
                }
            }
    }

    f2 prevPixelFromMvec(uint32_t x, uint32_t y) const // GatherHelper.slang:197-204
    {
        f2 mv = mvec[lin(x, y)];
        mv = (length(mv) < 1e-06f) ? mk2(0.f, 0.f) : mv;
        return mk2((float)x + mv.x * (float)W, (float)y + mv.y * (float)H);
    }

    // ReprojectTemporalSamples.rt.slang:64-175 (destination per source; counting done in sortCells)
    void reproject()
    {
        std::fill(splatTargets.begin(), splatTargets.end(), kInvalidIndex);
        #pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < (int)H; y++)
            for (uint32_t x = 0; x < W; x++)
            {
                uint32_t ci = lin(x, (uint32_t)y);
                const PathReservoir& pr = prev[ci];
                if (all_eq0(pr.integrand)) continue;
                const ReconnectionData& rd = prevR[ci];
                // The reference also orients a camera at artificialFrameTime + time, used only as the
                // (ignored) ray origin of loadShadingData.
                CameraData currCam; orient(currCam, rd.time);
                f2 lensLocal = mk2(currCam.apertureRadius * rd.lensSample.x, currCam.apertureRadius * rd.lensSample.y);
                f3 lensWorld = normalize(currCam.cameraU) * lensLocal.x + normalize(currCam.cameraV) * lensLocal.y;
                Ray nr;
                nr.origin = currCam.posW + lensWorld;
                if (hit_valid(rd.firstHit))
                {
                    f3 x1 = loadSD(rd.firstHit, mk3(0.f)).posW;
                    nr.dir = normalize(x1 - nr.origin);
                    nr.tMin = 0.001f * length(x1 - nr.origin);
                    nr.tMax = 0.999f * length(x1 - nr.origin);
                }
                else if (rd.lightIsDistant)
                {
                    // an environment sample reprojects by its direction (:110-118)
                    nr.dir = -rd.firstWi;
                    nr.tMin = 0.001f;
                    nr.tMax = kRayTMax;
                }
                else continue; // an invalid first hit cannot be reprojected
                f3 camDir = mk3(dot(normalize(currCam.cameraU), nr.dir), dot(normalize(currCam.cameraV), nr.dir), dot(normalize(currCam.cameraW), nr.dir));
                if (camDir.z <= 0.001f) continue;
                if (!traceVisibilityRay(nr)) continue;
                float lw = length(currCam.cameraW);
                f2 film = mk2(lensLocal.x + lw * (camDir.x / camDir.z), lensLocal.y + lw * (camDir.y / camDir.z));
                f2 ndc = mk2(film.x / length(currCam.cameraU), film.y / length(currCam.cameraV));
                f2 nfp = mk2((0.5f * ndc.x + 0.5f) * (float)W, (-0.5f * ndc.y + 0.5f) * (float)H);
                if (!validFloat(nfp)) continue;
                splatTargets[ci] = lin((uint32_t)f_floor(nfp.x), (uint32_t)f_floor(nfp.y));
            }
    }

    // SortReprojectedReservoirs.cs.slang:56-95 with the canonical in-cell order (ascending source):
    // cellOffsets is the exclusive prefix sum of the cell counts.
    void sortCells(const std::vector<uint32_t>& targets, std::vector<uint32_t>& counts, std::vector<uint32_t>& offsets, std::vector<uint32_t>& out)
    {
        const uint32_t N = W * H;
        std::fill(counts.begin(), counts.end(), 0u);
        for (uint32_t s = 0; s < N; s++) if (targets[s] != kInvalidIndex) counts[targets[s]]++;
        uint32_t acc = 0;
        for (uint32_t c = 0; c < N; c++) { offsets[c] = acc; acc += counts[c]; }
        out.assign(acc, 0u);
        std::vector<uint32_t> cursor(offsets);
        for (uint32_t s = 0; s < N; s++) if (targets[s] != kInvalidIndex) out[cursor[targets[s]]++] = s;
    }

    // RobustReuseOptimization.rt.slang:63-89
    void robustReuse()
    {
        static const int kOff[8][2] = {{-1, -1}, {0, -1}, {1, -1}, {-1, 0}, {1, 0}, {-1, 1}, {0, 1}, {1, 1}};
        shiftedPaths.assign(8 * (size_t)W * H, ShiftedPathData());
        #pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < (int)H; y++)
            for (uint32_t x = 0; x < W; x++)
            {
                SampleGen sg = makeSg(x, (uint32_t)y, passSeed(1));
                uint32_t idx = lin(x, (uint32_t)y);
                const PathReservoir& pr = prev[idx];
                const ReconnectionData& rd = prevR[idx];
                for (int k = 0; k < 8; k++)
                {
                    int nx = (int)x + kOff[k][0], ny = y + kOff[k][1];
                    bool neighborIsValid = validFloat(mk2((float)nx, (float)ny));
                    bool canShift = any_gt0(pr.integrand);
                    shiftedPaths[8 * (size_t)idx + k] = (neighborIsValid && canShift)
                        ? gatherLensVertexCopyShift(sg, rd, rd.time + cm.artificialFrameTime, mk2((float)nx + pr.subPixel.x, (float)ny + pr.subPixel.y), rd.lensSample)
                        : ShiftedPathData();
                }
            }
    }

    // CollectTemporalSamples.cs.slang:70-257
    void collect()
    {
        const bool useConf = opt.useConfidenceWeightsTemporally != 0;
        #pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < (int)H; y++)
            for (uint32_t x = 0; x < W; x++)
            {
                SampleGen sg = makeSg(x, (uint32_t)y, passSeed(2));
                uint32_t ci = lin(x, (uint32_t)y);
                f2 prevPixel = prevPixelFromMvec(x, (uint32_t)y);
                PathReservoir dst;
                ReconnectionData dstR;
                f2 dstFC = mk2(-1.f, -1.f);
                if (!validFloat(prevPixel))
                {
                    intermediate[ci] = dst; intermediateR[ci] = dstR; floatingCoords[ci] = dstFC;
                    continue;
                }
                int tlx = (int)f_floor(prevPixel.x), tly = (int)f_floor(prevPixel.y);
                f2 frac = mk2(f_saturate(prevPixel.x - (float)tlx), f_saturate(prevPixel.y - (float)tly));
                if (opt.gatherOption == RS_GATHER_FAST)
                {
                    dstFC = prevPixel;
                    float totalConfidence = 0.f;
                    for (int ox = 0; ox < 2; ox++)
                        for (int oy = 0; oy < 2; oy++)
                        {
                            int nx = tlx + ox, ny = tly + oy;
                            if (!validInt(nx, ny)) continue;
                            uint32_t ni = lin((uint32_t)nx, (uint32_t)ny);
                            PathReservoir nr = prev[ni];
                            f2 rel = mk2((float)ox + nr.subPixel.x - frac.x, (float)oy + nr.subPixel.y - frac.y);
                            float bw = f_lerp((float)(1 - ox), (float)ox, frac.x) * f_lerp((float)(1 - oy), (float)oy, frac.y);
                            totalConfidence += bw * (useConf ? nr.confidence : 1.f);
                            if (rel.x >= 0.f && rel.x < 1.f && rel.y >= 0.f && rel.y < 1.f)
                            {
                                nr.subPixel = rel;
                                bool sel = dst.addSampleFromReservoir(sg, 1.f, nr.integrand, 1.f, nr);
                                dstR = sel ? prevR[ni] : dstR;
                            }
                        }
                    dst.confidence = totalConfidence;
                }
                else if (opt.gatherOption == RS_GATHER_CLAMPED)
                {
                    float rx = f_round(prevPixel.x), ry = f_round(prevPixel.y);
                    dstFC = mk2(rx, ry);
                    if (validInt((int)rx, (int)ry))
                    {
                        uint32_t pi = lin((uint32_t)rx, (uint32_t)ry);
                        dst = prev[pi];
                        dstR = prevR[pi];
                    }
                }
                else
                {
                    dstFC = prevPixel;
                    float totalConfidence = 0.f;
                    for (int ox = 0; ox < 2; ox++)
                        for (int oy = 0; oy < 2; oy++)
                        {
                            int nx = tlx + ox, ny = tly + oy;
                            if (!validInt(nx, ny)) continue;
                            uint32_t ni = lin((uint32_t)nx, (uint32_t)ny);
                            PathReservoir nr = prev[ni];
                            ReconnectionData nrd = prevR[ni];
                            f2 rel = mk2((float)ox + nr.subPixel.x - frac.x, (float)oy + nr.subPixel.y - frac.y);
                            float bw = f_lerp((float)(1 - ox), (float)ox, frac.x) * f_lerp((float)(1 - oy), (float)oy, frac.y);
                            totalConfidence += bw * (useConf ? nr.confidence : 1.f);
                            int rox = 0, roy = 0;
                            if (rel.x < 0.f) rox += 1;
                            if (rel.x >= 1.f) rox -= 1;
                            if (rel.y < 0.f) roy += 1;
                            if (rel.y >= 1.f) roy -= 1;
                            rel = mk2(rel.x + (float)rox, rel.y + (float)roy);
                            rox += 1; roy += 1;
                            uint32_t offsetIndex = (uint32_t)(rox + 3 * roy);
                            bool noShiftNeeded = (offsetIndex == 4);
                            offsetIndex = (offsetIndex > 4) ? offsetIndex - 1 : offsetIndex;
                            ShiftedPathData sp;
                            if (noShiftNeeded)
                            {
                                sp.primaryHit = nrd.firstHit;
                                sp.fractionalPixel = mk2((float)nx + nr.subPixel.x, (float)ny + nr.subPixel.y);
                                sp.lensSample = nrd.lensSample;
                                sp.firstRayDir = -nrd.firstWi;
                                sp.subPixelJacobian = nrd.subPixelJacobian;
                                sp.lensVertexJacobian = nrd.lensVertexJacobian;
                                sp.secondaryPathJacobian = nrd.secondaryPathJacobian;
                                sp.radiance = nr.integrand;
                            }
                            else sp = shiftedPaths[8 * (size_t)ni + offsetIndex];
                            float shiftedJacobian = noShiftNeeded ? 1.f : sp.secondaryPathJacobian / nrd.secondaryPathJacobian;
                            float pHatSource = luminance(nr.integrand);
                            float sourceWeight = bw * pHatSource * (useConf ? nr.confidence : 1.f);
                            float totalPHat = sourceWeight;
                            for (int tx = 0; tx < 2; ++tx)
                                for (int ty = 0; ty < 2; ++ty)
                                {
                                    int px = tlx + tx, py = tly + ty;
                                    if (!validInt(px, py)) continue;
                                    int dx = tx - ox, dy = ty - oy;
                                    if (dx == 0 && dy == 0) continue;
                                    float tbw = f_lerp((float)(1 - tx), (float)tx, frac.x) * f_lerp((float)(1 - ty), (float)ty, frac.y);
                                    uint32_t tIdx = (uint32_t)((dx + 1) + 3 * (dy + 1));
                                    tIdx = (tIdx > 4) ? tIdx - 1 : tIdx;
                                    const ShiftedPathData& tp = shiftedPaths[8 * (size_t)ni + tIdx];
                                    float tPHat = luminance(tp.radiance);
                                    float tJac = tp.secondaryPathJacobian / nrd.secondaryPathJacobian;
                                    float tConf = useConf ? prev[lin((uint32_t)px, (uint32_t)py)].confidence : 1.f;
                                    totalPHat += tbw * tPHat * tJac * tConf;
                                }
                            float misWeight = (totalPHat > 0.f) ? sourceWeight / totalPHat : 0.f;
                            nr.subPixel = rel;
                            recon_update(nrd, sp);
                            nrd.subPixel = rel;
                            float lum = luminance(sp.radiance);
                            bool sel = dst.addSampleFromReservoir(sg, misWeight, mk3(lum), shiftedJacobian, nr);
                            dstR = sel ? nrd : dstR;
                        }
                    dst.confidence = totalConfidence;
                }
                if (f_isnan(dst.totalWeight))
                {
                    dst.integrand = mk3(0.f);
                    dst.totalWeight = 0.f;
                    dstR.subPixelJacobian = 1.f;
                    dstR.lensVertexJacobian = 1.f;
                    dstR.secondaryPathJacobian = 1.f;
                    dstR.pathLength = 0;
                }
                intermediate[ci] = dst; intermediateR[ci] = dstR; floatingCoords[ci] = dstFC;
            }
    }

    // bilinear confidence update shared by the scatter passes (e.g. ScatterTemporalResampling.rt.slang:150-170)
    float bilinearConfidence(uint32_t x, uint32_t y, float newConfidence, bool useConf) const
    {
        f2 prevPixel = prevPixelFromMvec(x, y);
        int tlx = (int)f_floor(prevPixel.x), tly = (int)f_floor(prevPixel.y);
        f2 frac = mk2(f_saturate(prevPixel.x - (float)tlx), f_saturate(prevPixel.y - (float)tly));
        for (int ox = 0; ox < 2; ox++)
            for (int oy = 0; oy < 2; oy++)
            {
                int nx = tlx + ox, ny = tly + oy;
                if (!validInt(nx, ny)) continue;
                const PathReservoir& nr = prev[lin((uint32_t)nx, (uint32_t)ny)];
                float bw = f_lerp((float)(1 - ox), (float)ox, frac.x) * f_lerp((float)(1 - oy), (float)oy, frac.y);
                newConfidence += bw * (useConf ? nr.confidence : 1.f);
            }
        return f_min(kConfidenceCap, newConfidence);
    }

    static float shiftJacobianSP(const ShiftedPathData& s, const ReconnectionData& r)
    {
        return (s.subPixelJacobian * s.secondaryPathJacobian) / (r.subPixelJacobian * r.secondaryPathJacobian);
    }

    // ScatterTemporalResampling.rt.slang:65-174
    void scatterResample()
    {
        const bool useConf = opt.useConfidenceWeightsTemporally != 0;
        #pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < (int)H; y++)
            for (uint32_t x = 0; x < W; x++)
            {
                SampleGen sg = makeSg(x, (uint32_t)y, passSeed(5));
                PathReservoir dst; ReconnectionData dstR;
                uint32_t ri = lin(x, (uint32_t)y);
                PathReservoir cr = curr[ri]; ReconnectionData crd = currR[ri];
                float currSampleMIS = 1.f;
                if (any_gt0(cr.integrand))
                {
                    float m1 = luminance(cr.integrand) * (useConf ? cr.confidence : 1.f);
                    ShiftedPathData sc = scatterReprojectionShift(sg, crd, crd.time + cm.artificialFrameTime, crd.firstHit, crd.lensSample, false);
                    float sj = shiftJacobianSP(sc, crd);
                    float m2 = luminance(sc.radiance) * sj;
                    m2 = f_isnan(m2) ? 0.f : m2;
                    int spx = (int)f_floor(sc.fractionalPixel.x), spy = (int)f_floor(sc.fractionalPixel.y);
                    if (validInt(spx, spy)) m2 *= useConf ? prev[lin((uint32_t)spx, (uint32_t)spy)].confidence : 1.f;
                    else m2 = 0.f;
                    currSampleMIS = (m1 + m2 == 0.f) ? 0.f : m1 / (m1 + m2);
                }
                bool cs = dst.addSampleFromReservoir(sg, currSampleMIS, cr.integrand, 1.f, cr);
                dstR = cs ? crd : dstR;
                float newConfidence = dst.confidence;
                uint32_t n = cellCounters[ri], off = cellOffsets[ri];
                for (uint32_t i = 0; i < n; i++)
                {
                    uint32_t si = sorted[off + i];
                    PathReservoir pr = prev[si]; ReconnectionData prd = prevR[si];
                    float prevSampleMIS = 0.f;
                    f3 prevPHat = mk3(0.f);
                    float sj = 1.f;
                    if (any_gt0(pr.integrand))
                    {
                        ShiftedPathData sp = scatterReprojectionShift(sg, prd, prd.time, prd.firstHit, prd.lensSample, false);
                        sj = shiftJacobianSP(sp, prd);
                        float m1 = luminance(sp.radiance) * sj * (useConf ? cr.confidence : 1.f);
                        prevPHat = f_isnan(m1) ? mk3(0.f) : sp.radiance;
                        sj = f_isnan(m1) ? 1.f : sj;
                        recon_update(prd, sp);
                        pr.subPixel = prd.subPixel;
                        float m2 = luminance(pr.integrand) * (useConf ? pr.confidence : 1.f);
                        prevSampleMIS = ((m1 + m2) == 0.f) ? 0.f : m2 / (m1 + m2);
                    }
                    bool ps = dst.addSampleFromReservoir(sg, prevSampleMIS, prevPHat, sj, pr);
                    dstR = ps ? prd : dstR;
                }
                dst.confidence = bilinearConfidence(x, (uint32_t)y, newConfidence, useConf);
                curr[ri] = dst; currR[ri] = dstR;
            }
    }

    // ScatterBackupTemporalResampling.rt.slang:69-283
    void scatterBackupResample()
    {
        const bool useConf = opt.useConfidenceWeightsTemporally != 0;
        const bool balance = opt.scatterBackupMISOption == RS_MIS_BALANCE;
        #pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < (int)H; y++)
            for (uint32_t x = 0; x < W; x++)
            {
                SampleGen sg = makeSg(x, (uint32_t)y, passSeed(6));
                PathReservoir dst; ReconnectionData dstR;
                uint32_t ri = lin(x, (uint32_t)y);
                PathReservoir cr = curr[ri]; ReconnectionData crd = currR[ri];
                PathReservoir br = intermediate[ri]; ReconnectionData brd = intermediateR[ri];
                float misScale = balance ? 1.f : 0.5f;
                f2 floatingCoord = floatingCoords[ri];
                {
                    float currSampleMIS = 1.f;
                    if (any_gt0(cr.integrand))
                    {
                        float m1 = luminance(cr.integrand) * (useConf ? cr.confidence : 1.f);
                        ShiftedPathData sc = scatterReprojectionShift(sg, crd, crd.time + cm.artificialFrameTime, crd.firstHit, crd.lensSample, false);
                        float scj = shiftJacobianSP(sc, crd);
                        float m2 = luminance(sc.radiance) * scj;
                        m2 = f_isnan(m2) ? 0.f : m2;
                        int spx = (int)f_floor(sc.fractionalPixel.x), spy = (int)f_floor(sc.fractionalPixel.y);
                        if (validInt(spx, spy)) m2 *= 0.5f * (useConf ? prev[lin((uint32_t)spx, (uint32_t)spy)].confidence : 1.f);
                        else m2 = 0.f;
                        float m3 = 0.f;
                        f2 rel = cr.subPixel;
                        if (validFloat(floatingCoord))
                        {
                            ShiftedPathData gc = gatherLensVertexCopyShift(sg, crd, crd.time + cm.artificialFrameTime, floatingCoord + rel, crd.lensSample);
                            float gj = gc.secondaryPathJacobian / crd.secondaryPathJacobian;
                            m3 = luminance(gc.radiance) * gj * 0.5f * (useConf ? br.confidence : 1.f);
                        }
                        m3 = f_isnan(m3) ? 0.f : m3;
                        if (balance) currSampleMIS = (m1 + m2 + m3 == 0.f) ? 0.f : m1 / (m1 + m2 + m3);
                        else currSampleMIS = 0.5f * (((m1 + m2 == 0.f) ? 0.f : 0.5f * m1 / (0.5f * m1 + m2)) +
                                                     ((m1 + m3 == 0.f) ? 0.f : 0.5f * m1 / (0.5f * m1 + m3)));
                    }
                    bool cs = dst.addSampleFromReservoir(sg, currSampleMIS, cr.integrand, 1.f, cr);
                    dstR = cs ? crd : dstR;
                }
                {
                    float backupSampleMIS = 0.f;
                    f3 backupPHat = mk3(0.f);
                    float sj = 1.f;
                    if (any_gt0(br.integrand))
                    {
                        ShiftedPathData sb = gatherLensVertexCopyShift(sg, brd, brd.time, mk2((float)x + br.subPixel.x, (float)y + br.subPixel.y), brd.lensSample);
                        sj = sb.secondaryPathJacobian / brd.secondaryPathJacobian;
                        float m1 = luminance(sb.radiance) * sj * (useConf ? cr.confidence : 1.f);
                        backupPHat = f_isnan(m1) ? mk3(0.f) : sb.radiance;
                        sj = f_isnan(m1) ? 1.f : sj;
                        m1 = f_isnan(m1) ? 0.f : m1;
                        recon_update(brd, sb);
                        float m2 = 0.f;
                        if (balance)
                        {
                            ShiftedPathData ss = scatterReprojectionShift(sg, brd, brd.time + cm.artificialFrameTime, brd.firstHit, brd.lensSample, false);
                            float scj = shiftJacobianSP(ss, brd);
                            m2 = luminance(ss.radiance) * scj * sj;
                            m2 = f_isnan(m2) ? 0.f : m2;
                            int spx = (int)f_floor(ss.fractionalPixel.x), spy = (int)f_floor(ss.fractionalPixel.y);
                            if (validInt(spx, spy)) m2 *= 0.5f * (useConf ? prev[lin((uint32_t)spx, (uint32_t)spy)].confidence : 1.f);
                            else m2 = 0.f;
                        }
                        float m3 = luminance(br.integrand) * 0.5f * (useConf ? br.confidence : 1.f);
                        backupSampleMIS = misScale * ((m1 + m2 + m3 == 0.f) ? 0.f : m3 / (misScale * m1 + m2 + m3));
                    }
                    bool bs = dst.addSampleFromReservoir(sg, backupSampleMIS, backupPHat, sj, br);
                    dstR = bs ? brd : dstR;
                }
                float newConfidence = dst.confidence;
                uint32_t n = cellCounters[ri], off = cellOffsets[ri];
                for (uint32_t i = 0; i < n; i++)
                {
                    uint32_t si = sorted[off + i];
                    PathReservoir pr = prev[si]; ReconnectionData prd = prevR[si];
                    float prevSampleMIS = 0.f;
                    f3 prevPHat = mk3(0.f);
                    float scj = 1.f;
                    if (any_gt0(pr.integrand))
                    {
                        ShiftedPathData sp = scatterReprojectionShift(sg, prd, prd.time, prd.firstHit, prd.lensSample, true);
                        scj = shiftJacobianSP(sp, prd);
                        float m1 = luminance(sp.radiance) * scj * (useConf ? cr.confidence : 1.f);
                        m1 = f_isnan(m1) ? 0.f : m1;
                        prevPHat = f_isnan(m1) ? mk3(0.f) : sp.radiance;
                        scj = f_isnan(m1) ? 1.f : scj;
                        recon_update(prd, sp);
                        pr.subPixel = prd.subPixel;
                        float m2 = luminance(pr.integrand) * 0.5f * (useConf ? pr.confidence : 1.f);
                        float m3 = 0.f;
                        if (balance)
                        {
                            f2 rel = pr.subPixel;
                            if (validFloat(floatingCoord + rel))
                            {
                                ShiftedPathData gp = gatherLensVertexCopyShift(sg, prd, prd.time + cm.artificialFrameTime, floatingCoord + rel, prd.lensSample);
                                float gj = gp.secondaryPathJacobian / prd.secondaryPathJacobian;
                                m3 = luminance(gp.radiance) * gj * scj * 0.5f * (useConf ? br.confidence : 1.f);
                            }
                            m3 = f_isnan(m3) ? 0.f : m3;
                        }
                        prevSampleMIS = misScale * ((m1 + m2 + m3 == 0.f) ? 0.f : m2 / (misScale * m1 + m2 + m3));
                    }
                    bool ps = dst.addSampleFromReservoir(sg, prevSampleMIS, prevPHat, scj, pr);
                    dstR = ps ? prd : dstR;
                }
                dst.confidence = bilinearConfidence(x, (uint32_t)y, newConfidence, useConf);
                curr[ri] = dst; currR[ri] = dstR;
            }
    }

    // GatherTemporalResampling.rt.slang:68-235
    void gatherResample()
    {
        const bool useConf = opt.useConfidenceWeightsTemporally != 0;
        #pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < (int)H; y++)
            for (uint32_t x = 0; x < W; x++)
            {
                SampleGen sg = makeSg(x, (uint32_t)y, passSeed(3));
                uint32_t ri = lin(x, (uint32_t)y);
                const bool hasDoF = camera.apertureRadius > 0.f;
                f2 probs = pixelDofProbs(x, (uint32_t)y);
                const bool doLensCopy = probs.x > 0.f;
                const bool doPrimaryReconnect = probs.y > 0.f;
                PathReservoir dst; ReconnectionData dstR;
                f2 floatingCoord = floatingCoords[ri];
                for (int stage = 0; stage < 2; stage++)
                {
                    bool lens = stage == 0;
                    if (lens && !doLensCopy) continue;
                    if (!lens && !(hasDoF && doPrimaryReconnect)) continue;
                    float prob = lens ? probs.x : probs.y;
                    PathReservoir pr = intermediate[ri];
                    PathReservoir cr = (lens || !doLensCopy) ? curr[ri] : dst;
                    ReconnectionData prd = intermediateR[ri];
                    ReconnectionData crd = (lens || !doLensCopy) ? currR[ri] : dstR;
                    if (!lens) { dst = PathReservoir(); dstR = ReconnectionData(); }
                    float currSampleMIS = 0.f;
                    f3 currPHat = mk3(0.f);
                    if (any_gt0(cr.integrand))
                    {
                        float m1 = luminance(cr.integrand) * (useConf ? cr.confidence : 1.f);
                        currPHat = cr.integrand;
                        f2 rel = cr.subPixel;
                        ShiftedPathData sc = lens
                            ? gatherLensVertexCopyShift(sg, crd, crd.time + cm.artificialFrameTime, floatingCoord + rel, crd.lensSample)
                            : gatherPrimaryHitReconnectionShift(sg, crd, crd.time + cm.artificialFrameTime, floatingCoord + rel, crd.firstHit);
                        float sj = lens ? sc.secondaryPathJacobian / crd.secondaryPathJacobian
                                        : (sc.lensVertexJacobian * sc.secondaryPathJacobian) / (crd.lensVertexJacobian * crd.secondaryPathJacobian);
                        float m2 = luminance(sc.radiance) * sj * (useConf ? pr.confidence : 1.f) * prob;
                        m2 = f_isnan(m2) ? 0.f : m2;
                        currSampleMIS = (m1 + m2 == 0.f) ? 0.f : m1 / (m1 + m2);
                    }
                    bool cs = dst.addSampleFromReservoir(sg, currSampleMIS, currPHat, 1.f, cr);
                    dstR = cs ? crd : dstR;
                    float prevSampleMIS = 0.f;
                    f3 prevPHat = mk3(0.f);
                    float sj = 1.f;
                    if (any_gt0(pr.integrand))
                    {
                        f2 fp = mk2((float)x + pr.subPixel.x, (float)y + pr.subPixel.y);
                        ShiftedPathData sp = lens
                            ? gatherLensVertexCopyShift(sg, prd, prd.time, fp, prd.lensSample)
                            : gatherPrimaryHitReconnectionShift(sg, prd, prd.time, fp, prd.firstHit);
                        sj = lens ? sp.secondaryPathJacobian / prd.secondaryPathJacobian
                                  : (sp.lensVertexJacobian * sp.secondaryPathJacobian) / (prd.lensVertexJacobian * prd.secondaryPathJacobian);
                        float m1 = luminance(sp.radiance) * sj * (useConf ? cr.confidence : 1.f);
                        prevPHat = f_isnan(m1) ? mk3(0.f) : sp.radiance;
                        sj = f_isnan(m1) ? 1.f : sj;
                        m1 = f_isnan(m1) ? 0.f : m1;
                        recon_update(prd, sp);
                        float m2 = luminance(pr.integrand) * (useConf ? pr.confidence : 1.f) * prob;
                        prevSampleMIS = ((m1 + m2) == 0.f) ? 0.f : m2 / (m1 + m2);
                    }
                    bool ps = dst.addSampleFromReservoir(sg, prevSampleMIS, prevPHat, sj, pr);
                    dstR = ps ? prd : dstR;
                }
                curr[ri] = dst; currR[ri] = dstR;
            }
    }

    // MultiReprojectTemporalSamples.rt.slang:65-168: destination cell per (partition, source)
    void multiReproject(std::vector<std::vector<uint32_t>>& targets)
    {
        const uint32_t P = opt.numTimePartitions;
        for (uint32_t i = 0; i < P; i++) std::fill(targets[i].begin(), targets[i].end(), kInvalidIndex);
        #pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < (int)H; y++)
            for (uint32_t x = 0; x < W; x++)
            {
                uint32_t ci = lin(x, (uint32_t)y);
                const PathReservoir& pr = prev[ci];
                if (all_eq0(pr.integrand)) continue;
                const ReconnectionData& rd = prevR[ci];
                float fractionalTime = rd.time / camera.shutterSpeed;
                float timePartitions = camera.shutterSpeed / (float)P;
                CameraData oldCam; orient(oldCam, cm.artificialFrameTime + rd.time);
                for (uint32_t i = 0; i < P; i++)
                {
                    float newTime = (fractionalTime + (float)i) * timePartitions;
                    CameraData cc; orient(cc, newTime);
                    f3 rayDir; float rayLength;
                    if (hit_valid(rd.firstHit))
                    {
                        f3 x1 = loadSD(rd.firstHit, mk3(0.f)).posW;
                        rayDir = x1 - cc.posW;
                        rayLength = 0.999f;
                    }
                    else if (rd.lightIsDistant)
                    {
                        rayDir = -rd.firstWi;
                        rayLength = kRayTMax;
                    }
                    else continue;
                    f3 nd = normalize(rayDir);
                    float d = dot(nd, normalize(cc.cameraW));
                    if (d <= 0.001f) continue;
                    if (!traceVisibilityRay(mk_ray(cc.posW, rayDir, 0.001f, rayLength))) continue;
                    float tanFovY = cc.focalLength == 0.f ? 0.f : cc.frameHeight / cc.focalLength;
                    d *= tanFovY;
                    f2 offset = mk2(dot(nd, normalize(cc.cameraU)), -dot(nd, normalize(cc.cameraV)));
                    f2 ndc = mk2(0.5f + offset.x / (d * cc.aspectRatio), 0.5f + offset.y / d);
                    f2 nfp = mk2(ndc.x * (float)W, ndc.y * (float)H);
                    if (!validFloat(nfp)) continue;
                    targets[i][ci] = lin((uint32_t)f_floor(nfp.x), (uint32_t)f_floor(nfp.y));
                }
            }
    }

    // MultiScatterTemporalResampling.rt.slang:65-186
    void multiScatterResample()
    {
        const bool useConf = opt.useConfidenceWeightsTemporally != 0;
        const uint32_t P = opt.numTimePartitions;
        #pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < (int)H; y++)
            for (uint32_t x = 0; x < W; x++)
            {
                SampleGen sg = makeSg(x, (uint32_t)y, passSeed(5));
                PathReservoir dst; ReconnectionData dstR;
                float timePartitions = camera.shutterSpeed / (float)P;
                float jacobianScale = 1.f / (float)P;
                uint32_t ri = lin(x, (uint32_t)y);
                PathReservoir cr = curr[ri]; ReconnectionData crd = currR[ri];
                float currSampleMIS = 1.f;
                if (any_gt0(cr.integrand))
                {
                    float m1 = luminance(cr.integrand) * (useConf ? cr.confidence : 1.f);
                    float fractionalTime = (crd.time - f_floor(crd.time / timePartitions) * timePartitions) / timePartitions;
                    float shiftedTime = fractionalTime * camera.shutterSpeed;
                    ShiftedPathData sc = scatterReprojectionShift(sg, crd, shiftedTime + cm.artificialFrameTime, crd.firstHit, crd.lensSample, false);
                    float sj = shiftJacobianSP(sc, crd);
                    float m2 = luminance(sc.radiance) * sj;
                    m2 = f_isnan(m2) ? 0.f : m2;
                    int spx = (int)f_floor(sc.fractionalPixel.x), spy = (int)f_floor(sc.fractionalPixel.y);
                    if (validInt(spx, spy)) m2 *= useConf ? prev[lin((uint32_t)spx, (uint32_t)spy)].confidence : 1.f;
                    else m2 = 0.f;
                    currSampleMIS = (m1 + m2 == 0.f) ? 0.f : m1 / (m1 + m2);
                }
                bool cs = dst.addSampleFromReservoir(sg, currSampleMIS, cr.integrand, 1.f, cr);
                dstR = cs ? crd : dstR;
                float newConfidence = dst.confidence;
                for (uint32_t j = 0; j < P; j++)
                {
                    uint32_t n = mCellCounters[j][ri], off = mCellOffsets[j][ri];
                    for (uint32_t i = 0; i < n; i++)
                    {
                        uint32_t si = mSorted[j][off + i];
                        PathReservoir pr = prev[si]; ReconnectionData prd = prevR[si];
                        f3 prevPHat = mk3(0.f);
                        float sj = 1.f;
                        float prevMIS = 0.f;
                        if (any_gt0(pr.integrand))
                        {
                            float fractionalTime = prd.time / camera.shutterSpeed;
                            float newTime = (fractionalTime + (float)j) * timePartitions;
                            ShiftedPathData sp = scatterReprojectionShift(sg, prd, newTime, prd.firstHit, prd.lensSample, false);
                            sj = shiftJacobianSP(sp, prd);
                            float m1 = luminance(sp.radiance) * sj * (useConf ? cr.confidence : 1.f);
                            prevPHat = f_isnan(m1) ? mk3(0.f) : sp.radiance;
                            sj = f_isnan(m1) ? 1.f : sj;
                            recon_update(prd, sp);
                            prd.time = newTime;
                            pr.subPixel = prd.subPixel;
                            float m2 = luminance(pr.integrand) * (useConf ? pr.confidence : 1.f);
                            prevMIS = ((m1 + m2) == 0.f) ? 0.f : m2 / (m1 + m2);
                        }
                        bool ps = dst.addSampleFromReservoir(sg, prevMIS, prevPHat, sj * jacobianScale, pr);
                        dstR = ps ? prd : dstR;
                    }
                }
                dst.confidence = bilinearConfidence(x, (uint32_t)y, newConfidence, useConf);
                curr[ri] = dst; currR[ri] = dstR;
            }
    }

    // SpatialResampling.rt.slang:67-185 for one iteration: reads (srcRes, srcRec), writes (dstRes, dstRec)
    void spatialIteration(uint32_t iteration, const std::vector<PathReservoir>& srcRes, const std::vector<ReconnectionData>& srcRec,
                          std::vector<PathReservoir>& dstRes, std::vector<ReconnectionData>& dstRec)
    {
        const bool useConf = opt.useConfidenceWeightsSpatially != 0;
        const uint32_t neighborCount = opt.neighborCount;
        const uint32_t kSpatialNeighborSamples = 8192;
        #pragma omp parallel for schedule(dynamic, 4)
        for (int y = 0; y < (int)H; y++)
            for (uint32_t x = 0; x < W; x++)
            {
                SampleGen sg = makeSg(x, (uint32_t)y, opt.useFixedSeed ? opt.fixedSeed + 7 : kNumRenderPasses * (frameCount + seed) + 1337u * iteration + 7u);
                uint32_t ri = lin(x, (uint32_t)y);
                f2 probs = pixelDofProbs(x, (uint32_t)y);
                const uint32_t numLensCopy = (uint32_t)f_round(probs.x * (float)neighborCount);
                PathReservoir cent = srcRes[ri]; ReconnectionData centR = srcRec[ri];
                float centralSampleMIS = 1.f;
                float centralWeight = luminance(cent.integrand) / (float)neighborCount * (useConf ? cent.confidence : 1.f);
                PathReservoir dst; ReconnectionData dstR;
                int validNeighbors = 0;
                uint32_t startIdx = (uint32_t)(sampleNext1D(sg) * (float)kSpatialNeighborSamples);
                for (uint32_t i = 0; i < neighborCount; i++)
                {
                    bool lensCopy = (i < numLensCopy);
                    uint32_t oi = (startIdx + i) % kSpatialNeighborSamples;
                    f2 off = neighborOffsets[oi];
                    int nx = (int)f_round((float)x + opt.spatialGatherRadius * off.x);
                    int ny = (int)f_round((float)y + opt.spatialGatherRadius * off.y);
                    if (!validInt(nx, ny)) continue;
                    validNeighbors += 1;
                    uint32_t ni = lin((uint32_t)nx, (uint32_t)ny);
                    PathReservoir nr = srcRes[ni]; ReconnectionData nrd = srcRec[ni];
                    float m1 = 0.f;
                    if (any_gt0(cent.integrand))
                    {
                        f2 fp = mk2((float)nx + cent.subPixel.x, (float)ny + cent.subPixel.y);
                        ShiftedPathData sc = lensCopy ? gatherLensVertexCopyShift(sg, centR, centR.time, fp, centR.lensSample)
                                                      : gatherPrimaryHitReconnectionShift(sg, centR, centR.time, fp, centR.firstHit);
                        float sj = (lensCopy ? 1.f : (sc.lensVertexJacobian / centR.lensVertexJacobian)) * (sc.secondaryPathJacobian / centR.secondaryPathJacobian);
                        m1 = luminance(sc.radiance) * sj * (useConf ? nr.confidence : 1.f);
                        m1 = f_isnan(m1) ? 0.f : m1;
                    }
                    centralSampleMIS += 1.f;
                    centralSampleMIS -= (m1 + centralWeight > 0.f) ? m1 / (m1 + centralWeight) : 0.f;
                    float neighborSampleMIS = 0.f;
                    f3 neighborPHat = mk3(0.f);
                    float sj = 1.f;
                    if (any_gt0(nr.integrand))
                    {
                        f2 fp = mk2((float)x + nr.subPixel.x, (float)y + nr.subPixel.y);
                        ShiftedPathData sn = lensCopy ? gatherLensVertexCopyShift(sg, nrd, nrd.time, fp, nrd.lensSample)
                                                      : gatherPrimaryHitReconnectionShift(sg, nrd, nrd.time, fp, nrd.firstHit);
                        sj = (lensCopy ? 1.f : (sn.lensVertexJacobian / nrd.lensVertexJacobian)) * (sn.secondaryPathJacobian / nrd.secondaryPathJacobian);
                        float nw = luminance(sn.radiance) * sj * (useConf ? cent.confidence : 1.f);
                        neighborPHat = f_isnan(nw) ? mk3(0.f) : sn.radiance;
                        sj = f_isnan(nw) ? 1.f : sj;
                        nw = f_isnan(nw) ? 0.f : nw / (float)neighborCount;
                        recon_update(nrd, sn);
                        float m2 = luminance(nr.integrand) * (useConf ? nr.confidence : 1.f);
                        neighborSampleMIS = (m2 + nw > 0.f) ? m2 / (nw + m2) : 0.f;
                    }
                    bool ns = dst.addSampleFromReservoir(sg, neighborSampleMIS, neighborPHat, sj, nr);
                    dstR = ns ? nrd : dstR;
                }
                bool cs = dst.addSampleFromReservoir(sg, centralSampleMIS, cent.integrand, 1.f, cent);
                dstR = cs ? centR : dstR;
                dst.totalWeight /= (float)(validNeighbors + 1);
                dstRes[ri] = dst; dstRec[ri] = dstR;
            }
    }

    // createNeighborOffsetTexture (ReservoirSplatting.cpp:1072-1097) decoded as RG8Snorm (c / 127, clamped at -1)
    void buildNeighborOffsets()
    {
        const uint32_t sampleCount = 8192;
        std::vector<int8_t> offsets(sampleCount * 2);
        const int R = 254;
        const float phi2 = 1.f / 1.3247179572447f;
        float u = 0.5f, v = 0.5f;
        for (uint32_t index = 0; index < sampleCount * 2;)
        {
            u += phi2;
            v += phi2 * phi2;
            if (u >= 1.f) u -= 1.f;
            if (v >= 1.f) v -= 1.f;
            float rSq = (u - 0.5f) * (u - 0.5f) + (v - 0.5f) * (v - 0.5f);
            if (rSq > 0.25f) continue;
            offsets[index++] = (int8_t)((u - 0.5f) * (float)R);
            offsets[index++] = (int8_t)((v - 0.5f) * (float)R);
        }
        neighborOffsets.resize(sampleCount);
        for (uint32_t i = 0; i < sampleCount; i++)
        {
            float a = (float)offsets[2 * i] / 127.f, b = (float)offsets[2 * i + 1] / 127.f;
            neighborOffsets[i] = mk2(a < -1.f ? -1.f : a, b < -1.f ? -1.f : b);
        }
    }

    // ================================================= host orchestration
    void resize(uint32_t w, uint32_t h)
    {
        W = w; H = h;
        size_t N = (size_t)w * h;
        curr.assign(N, PathReservoir()); prev.assign(N, PathReservoir()); intermediate.assign(N, PathReservoir()); temp.assign(N, PathReservoir());
        currR.assign(N, ReconnectionData()); prevR.assign(N, ReconnectionData()); intermediateR.assign(N, ReconnectionData()); tempR.assign(N, ReconnectionData());
        candidates.assign(N, PathReservoir()); candidatesR.assign(N, ReconnectionData());
        mvec.assign(N, mk2(0.f, 0.f)); floatingCoords.assign(N, mk2(-1.f, -1.f));
        vbuffer.assign(N, hit_none());
        cellCounters.assign(N, 0); cellOffsets.assign(N, 0); sorted.clear(); splatTargets.assign(N, kInvalidIndex);
        mCellCounters.assign(8, std::vector<uint32_t>(N, 0)); mCellOffsets.assign(8, std::vector<uint32_t>(N, 0)); mSorted.assign(8, std::vector<uint32_t>());
    }

    static CameraData toCamera(const rs_camera& c)
    {
        CameraData d;
        d.posW = mk3(c.position[0], c.position[1], c.position[2]);
        d.target = mk3(c.target[0], c.target[1], c.target[2]);
        d.up = mk3(c.up[0], c.up[1], c.up[2]);
        d.focalLength = c.focalLength; d.frameHeight = c.frameHeight; d.aspectRatio = c.aspectRatio;
        d.focalDistance = c.focalDistance; d.apertureRadius = c.apertureRadius; d.shutterSpeed = c.shutterSpeed;
        d.nearZ = c.nearZ; d.farZ = c.farZ;
        camera_update_basis(d);
        return d;
    }

    // ReservoirSplatting::execute (ReservoirSplatting.cpp:399-509), beginFrame (:1550-1646),
    // prepareCameraManager (:1359-1388), spatialResampling (:1994-2020), endFrame (:1648-1680)
    int execute(const rs_frame_desc* f, const float* mvecIn, float* colorOut)
    {
        if (!hasScene) return RS_NOT_READY;
        // beginFrame
        seed = opt.useFixedSeed ? opt.fixedSeed : seed + 1;
        camera = toCamera(f->camera);
        K = 1u + (uint32_t)ceilf(camera.shutterSpeed / opt.artificialFrameTime) + 1u;
        if (K > kMaxCameraKeyframes) K = kMaxCameraKeyframes;
        bool keyframesChanged = (K != prevK);
        prevK = K;
        bool shouldReset = f->sceneShouldReset != 0;
        // prepareCameraManager
        cm.artificialFrameTime = opt.artificialFrameTime;
        cm.keyframes = K;
        if (frameCount == 0 || shouldReset || keyframesChanged)
            for (uint32_t i = 0; i < K; i++) { cm.positions[i] = camera.posW; cm.targets[i] = camera.target; }
        else { cm.positions[frameCount % K] = camera.posW; cm.targets[frameCount % K] = camera.target; }

        // producer side (VBufferRT): primary hits + motion vectors
        vbufferPass();
        if (mvecIn) for (size_t i = 0; i < mvec.size(); i++) mvec[i] = mk2(mvecIn[2 * i], mvecIn[2 * i + 1]);

        initialCandidates();
        candidates = curr; candidatesR = currR;

        shouldReset = shouldReset || (frameCount == 0);
        std::fill(cellCounters.begin(), cellCounters.end(), 0u);
        if (opt.enableTemporalResampling && !shouldReset)
        {
            switch (opt.temporalReuse)
            {
            case RS_GATHER_ONLY:
                if (opt.gatherOption == RS_GATHER_ROBUST) robustReuse();
                collect();
                gatherResample();
                break;
            case RS_SCATTER_ONLY:
                reproject();
                sortCells(splatTargets, cellCounters, cellOffsets, sorted);
                scatterResample();
                break;
            case RS_SCATTER_BACKUP:
                if (opt.gatherOption == RS_GATHER_ROBUST) robustReuse();
                collect();
                reproject();
                sortCells(splatTargets, cellCounters, cellOffsets, sorted);
                scatterBackupResample();
                break;
            case RS_MULTI_SCATTER:
            {
                std::vector<std::vector<uint32_t>> targets(opt.numTimePartitions, std::vector<uint32_t>((size_t)W * H));
                multiReproject(targets);
                for (uint32_t i = 0; i < opt.numTimePartitions; i++) sortCells(targets[i], mCellCounters[i], mCellOffsets[i], mSorted[i]);
                multiScatterResample();
                break;
            }
            }
        }
        if (opt.enableSpatialResampling)
        {
            std::vector<PathReservoir>& swapRes = frozen ? temp : prev;
            std::vector<ReconnectionData>& swapRec = frozen ? tempR : prevR;
            for (uint32_t i = 0; i < opt.numSpatialIterations; i++)
            {
                std::swap(currR, swapRec);
                std::swap(curr, swapRes);
                spatialIteration(i, swapRes, swapRec, curr, currR);
            }
        }
        // ResolveReSTIR.cs.slang:45-63
        if (colorOut)
            for (size_t i = 0; i < curr.size(); i++)
            {
                f3 c = curr[i].integrand * curr[i].computeUCW();
                colorOut[4 * i + 0] = c.x; colorOut[4 * i + 1] = c.y; colorOut[4 * i + 2] = c.z; colorOut[4 * i + 3] = 1.f;
            }
        // endFrame
        swapped = !frozen;
        if (!frozen)
        {
            frameCount++;
            std::swap(curr, prev);
            std::swap(currR, prevR);
        }
        prevFrameCamera = camera;
        havePrevFrameCamera = true;
        geometryMoved = false;
        return RS_OK;
    }
};

// canonical export layouts (shared with the CUDA pass's rs_get_buffer)
static void export_reservoir(const PathReservoir& r, float* o)
{
    o[0] = r.integrand.x; o[1] = r.integrand.y; o[2] = r.integrand.z; o[3] = r.totalWeight;
    o[4] = r.subPixel.x; o[5] = r.subPixel.y; o[6] = r.confidence; o[7] = 0.f;
}
static void import_reservoir(PathReservoir& r, const float* o)
{
    r.integrand = mk3(o[0], o[1], o[2]); r.totalWeight = o[3]; r.subPixel = mk2(o[4], o[5]); r.confidence = o[6];
}
static void export_recon(const ReconnectionData& r, uint32_t* o)
{
    o[0] = f2u(r.subPixel.x); o[1] = f2u(r.subPixel.y); o[2] = f2u(r.lensSample.x); o[3] = f2u(r.lensSample.y);
    o[4] = f2u(r.time);
    o[5] = (r.pathLength & 0xffu) | ((r.firstBSDFComponentType & 3u) << 8) | ((r.secondBSDFComponentType & 3u) << 10) |
           ((r.transmissionEvent ? 1u : 0u) << 12) | ((r.lightIsNEE ? 1u : 0u) << 13) | ((r.lightIsDistant ? 1u : 0u) << 14) |
           ((r.suffixState & 0xfffu) << 15);
    o[6] = f2u(r.lightPdf); o[7] = f2u(r.subPixelJacobian);
    for (int k = 0; k < 4; k++) { o[8 + k] = r.firstHit.w[k]; o[12 + k] = r.secondHit.w[k]; }
    o[16] = f2u(r.firstWi.x); o[17] = f2u(r.firstWi.y); o[18] = f2u(r.firstWi.z); o[19] = f2u(r.lensVertexJacobian);
    o[20] = f2u(r.secondWo.x); o[21] = f2u(r.secondWo.y); o[22] = f2u(r.secondWo.z); o[23] = f2u(r.secondaryPathJacobian);
    o[24] = f2u(r.irradiance.x); o[25] = f2u(r.irradiance.y); o[26] = f2u(r.irradiance.z); o[27] = r.suffixSeed;
}
static void import_recon(ReconnectionData& r, const uint32_t* o)
{
    r.subPixel = mk2(u2f(o[0]), u2f(o[1])); r.lensSample = mk2(u2f(o[2]), u2f(o[3])); r.time = u2f(o[4]);
    r.pathLength = o[5] & 0xffu; r.firstBSDFComponentType = (o[5] >> 8) & 3u; r.secondBSDFComponentType = (o[5] >> 10) & 3u;
    r.transmissionEvent = (o[5] >> 12) & 1u; r.lightIsNEE = (o[5] >> 13) & 1u; r.lightIsDistant = (o[5] >> 14) & 1u;
    r.suffixState = (o[5] >> 15) & 0xfffu;
    r.lightPdf = u2f(o[6]); r.subPixelJacobian = u2f(o[7]);
    for (int k = 0; k < 4; k++) { r.firstHit.w[k] = o[8 + k]; r.secondHit.w[k] = o[12 + k]; }
    r.firstWi = mk3(u2f(o[16]), u2f(o[17]), u2f(o[18])); r.lensVertexJacobian = u2f(o[19]);
    r.secondWo = mk3(u2f(o[20]), u2f(o[21]), u2f(o[22])); r.secondaryPathJacobian = u2f(o[23]);
    r.irradiance = mk3(u2f(o[24]), u2f(o[25]), u2f(o[26]));
    r.suffixSeed = o[27];
}

// ================================================= path-replay adjoint (no reference counterpart)
// The resolved colour of a pixel is f(y) * W (ResolveReSTIR.cs.slang:45-63).  The adjoint holds the
// frame's selected path y, its contribution weight W, the sampling densities and the MIS weights at
// their values for the pass's materials, and differentiates f(y) with respect to each material's
// baseColor and roughness (the BSDF factor of every vertex) and emitted radiance (the Le the path
// carries).  f(y) is the reconnection-shift evaluation of the record at its own primary hit
// (handleReconnectionHit / pathReconnectionShift above) without the visibility ray, which does not
// depend on materials.  A path of four or more vertices carries the radiance of its suffix (x3 on)
// in the record; the suffix is re-run from x3 by the path tracer's own steps (handleHit below) from
// the sample generator's state and the bounce counters and flags the record saved on entering x3,
// which gives its vertices, their BSDF factors and the emitter.
static const uint32_t kReplayMaxVertices = 8; // BSDF factors on a replayed path (x1, x2 and the suffix)

struct ReplayVertex
{
    uint32_t material = kInvalidIndex;
    f3 wi = mk3(0.f), wo = mk3(0.f); // local frame
    bool valid = false;               // hemisphere test and minimum cosine
    bool diffuseOn = false, specularOn = false;
    BsdfGrad g;                       // value and derivatives at the pass's materials
};
struct Replay
{
    uint32_t L = 0;
    float W = 0.f;                    // contribution weight of the pixel's reservoir
    float s = 0.f;                    // detached factor: MIS weight over the sampling densities
    f3 Le = mk3(0.f);                 // emitted radiance the path carries
    uint32_t emitter = kInvalidIndex; // material that emits Le, when the replay finds it
    uint32_t nv = 0;                  // BSDF vertices on the path
    ReplayVertex v[kReplayMaxVertices];
    f3 value = mk3(0.f);              // prod factors * Le * s
    f3 k = mk3(1.f);                  // integrand / value per channel (detached; 1 where value is 0)
};
enum { kStatReplayed = 0, kStatSkipped = 1, kStatNoEmitter = 2, kStatValueMismatch = 3 };

static ReplayVertex replay_vertex(const Pass& p, const ShadingData& sd, uint32_t lobeMask, f3 wo)
{
    ReplayVertex v;
    BsdfData d = p.instance(sd);
    v.material = sd.materialID;
    v.wi = sd_to_local(sd, sd.V);
    v.wo = sd_to_local(sd, wo);
    v.valid = valid_hemisphere(sd, v.wi, v.wo, wo) && f_min(v.wi.z, v.wo.z) >= kMinCosTheta;
    StandardBSDF b = make_bsdf(v.wi, d, lobeMask);
    uint32_t mask = lobeMask == 0 ? 0xfu : lobeMask;
    v.diffuseOn = b.pDiffuseReflection > 0.f && (mask & 0x1u);
    v.specularOn = b.pSpecularReflection > 0.f && (mask & 0x4u) && b.alpha != 0.f;
    v.g = mi_eval_grad(sd, d, p.scene.materials[sd.materialID], lobeMask, wo);
    return v;
}

// The emissive material of the triangle the path ends on (the primary hit, the record's second hit,
// or the closest hit from x2 along the stored direction); its facing was decided by the forward pass.
static uint32_t emitter_of(const Pass& p, const ShadingData& sd)
{
    return material_is_emissive(p.scene.materials[sd.materialID]) ? sd.materialID : kInvalidIndex;
}

// The suffix of a path of four or more vertices: handleHit re-run from x3 (the closest hit from x2
// along the stored direction) with the sample generator's state, bounce counters and flags the
// record saved there, taking every draw the path tracer takes (the candidate selections', Russian
// roulette's, the light and BSDF samples'), up to the light sample that ends the path.  Appends the
// BSDF factor of each suffix vertex (the sampled lobe's; at the last vertex all lobes' toward the
// light) and sets the emitter, its radiance and the replayed suffix radiance S, which equals the
// record's irradiance.  Emitted radiance beyond x2 that a BSDF sample reaches counts only after a
// delta lobe (handleHit's computeEmissive), whose factor is no BSDF evaluation: such paths, delta
// lobes on the suffix and paths of more than kReplayMaxVertices factors are not replayed, and in
// geometry that has moved since the record was made the replay differs from the record's radiance:
// replay_pixel then holds the suffix fixed.
static bool replay_suffix(const Pass& p, const ReconnectionData& rd, const ShadingData& sd2, Replay& out, f3& S)
{
    PathState path;
    uint32_t bounces, flags;
    suffix_state_unpack(rd.suffixState, bounces, flags);
    path.bounceCounters = bounces;
    path.flagsAndVertexIndex = ((flags | kActive) << kVertexIndexBits) | 2u;
    path.sg.state = rd.suffixSeed;
    path.sg.kind = p.opt.sampleGenerator;
    path.thp = mk3(1.f);
    path.dir = rd.secondWo;
    path.origin = computeRayOrigin(sd2.posW, dot(sd2.faceN, rd.secondWo) >= 0.f ? sd2.faceN : -sd2.faceN);
    while (true)
    {
        path.incrementVertexIndex();
        const uint32_t v = path.getVertexIndex();
        HitInfo h; float t;
        if (v >= rd.pathLength || !p.bvh.closest(mk_ray(path.origin, path.dir, 0.f, kRayTMax), h, t)) return false;
        ShadingData sd = p.loadSD(h, path.dir);
        BsdfData d = p.instance(sd);
        if (p.lv.count > 0 && (!path.isLightSampled() || !path.isLightSamplable()) && any_gt0(d.emission))
            sampleNext1D(path.sg); // the emissive candidate's selection draw (addVertex)
        if (p.hasFinishedSurfaceBounces(path)) return false;
        path.origin = sd_ray_origin(sd, true);
        const uint32_t lobeTypes = mi_lobe_types(d);
        path.setFlag(kLightSampledUpper, false); path.setFlag(kLightSampledLower, false);
        if ((lobeTypes & kLobeNonDelta) != 0)
        {
            bool sampleUpper = (lobeTypes & kLobeNonDeltaReflection) != 0;
            bool sampleLower = (lobeTypes & kLobeNonDeltaTransmission) != 0;
            Pass::LightSample ls;
            bool validSample = p.generateLightSample(sd.posW, sd.faceN, sd.frontFacing, sampleUpper, sampleLower, path.sg, ls);
            path.setFlag(kLightSampledUpper, sampleUpper); path.setFlag(kLightSampledLower, sampleLower);
            if (validSample)
            {
                float misWeight = p.mis(ls.pdf, mi_pdf(sd, d, 0u, ls.dir));
                f3 Lr = mi_eval(sd, d, 0u, ls.dir) * misWeight * ls.Li;
                if (any_gt0(Lr) && p.traceVisibilityRay(mk_ray(ls.origin, ls.dir, 0.f, ls.distance)))
                {
                    sampleNext1D(path.sg); // the light candidate's selection draw (addVertex)
                    if (rd.lightIsNEE && v + 1 == rd.pathLength)
                    {
                        if (out.nv == kReplayMaxVertices) return false;
                        out.v[out.nv++] = replay_vertex(p, sd, 0u, ls.dir);
                        S = path.thp * Lr;
                        out.Le = ls.Li * ls.pdf;
                        if (ls.lightType == 1) // an environment-map sample's radiance is no material's
                        {
                            const HitInfo lh = hit_tri(p.lv.tris[ls.triangleId].sceneTri, ls.barycentrics.x, ls.barycentrics.y);
                            out.emitter = emitter_of(p, p.loadSD(lh, ls.dir));
                        }
                        return true;
                    }
                }
            }
        }
        if (p.opt.useRussianRoulette)
        {
            float u = sampleNext1D(path.sg);
            const float prob = f_max(0.f, 1.f - luminance(path.thp));
            if (u < prob) return false;
            path.thp /= 1.f - prob;
        }
        uint32_t comp = 0;
        bool valid = p.generateScatterRay(sd, d, path, &comp);
        if (!valid || path.isDelta() || (comp != 0 && comp != 2) || out.nv == kReplayMaxVertices) return false;
        out.v[out.nv++] = replay_vertex(p, sd, 1u << comp, path.dir);
        if (p.hasFinishedSurfaceBounces(path)) return false; // the path ends here: no later light sample
        if (p.opt.disableCaustics && path.getBounces(0) > 0 && path.isSpecular()) return false;
    }
}

static bool replay_pixel(const Pass& p, const PathReservoir& r, const ReconnectionData& rd, Replay& out, uint64_t* stats)
{
    out = Replay();
    out.W = r.computeUCW();
    if (!(out.W > 0.f) || rd.pathLength == 0) return false;
    // a primary miss sees the environment map: no material on the path
    if (rd.pathLength == 1 && rd.lightIsDistant) return false;
    out.L = rd.pathLength;
    out.Le = rd.irradiance;
    bool suffixHeld = false;
    ShadingData sd1 = p.loadSD(rd.firstHit, -rd.firstWi);
    if (rd.pathLength == 1)
    {
        out.s = 1.f;
        out.emitter = emitter_of(p, sd1);
    }
    else
    {
        BsdfData d1 = p.instance(sd1);
        f3 origin = sd_ray_origin(sd1, !rd.transmissionEvent);
        // a length-2 path to the environment stores a direction as its second hit and has no
        // geometry term (handleReconnectionHit's secondHitIsDistant)
        const bool distant2 = rd.pathLength == 2 && rd.lightIsDistant;
        float jac = 1.f;
        f3 dir;
        if (distant2) dir = hit_as_direction(rd.secondHit);
        else
        {
            ShadingData sec = p.loadSD(rd.secondHit, mk3(0.f));
            f3 off = sec.posW - sd1.posW;
            jac = f_abs(dot(sec.faceN, -normalize(off))) / dot(off, off);
            dir = normalize(sec.posW - origin);
        }
        uint32_t mask1 = 1u << rd.firstBSDFComponentType;
        float lobePdf = mi_pdf(sd1, d1, mask1, dir), totalPdf = mi_pdf(sd1, d1, 0u, dir);
        if (rd.pathLength == 2)
        {
            float lightPdf = rd.lightPdf / jac;
            if (rd.lightIsNEE)
            {
                out.v[0] = replay_vertex(p, sd1, 0u, dir);
                if (!any_gt0(out.v[0].g.value) || totalPdf == 0.f) return false;
                out.s = p.mis(lightPdf, totalPdf) / lightPdf;
            }
            else
            {
                out.v[0] = replay_vertex(p, sd1, mask1, dir);
                if (!any_gt0(out.v[0].g.value) || lobePdf == 0.f) return false;
                out.s = p.mis(totalPdf, lightPdf) / lobePdf;
            }
            out.nv = 1;
            if (!distant2) out.emitter = emitter_of(p, p.loadSD(rd.secondHit, dir));
        }
        else
        {
            out.v[0] = replay_vertex(p, sd1, mask1, dir);
            if (!any_gt0(out.v[0].g.value) || lobePdf == 0.f) return false;
            ShadingData sd2 = p.loadSD(rd.secondHit, dir);
            BsdfData d2 = p.instance(sd2);
            uint32_t mask2 = 1u << rd.secondBSDFComponentType;
            float lsp = mi_pdf(sd2, d2, mask2, rd.secondWo), tp = mi_pdf(sd2, d2, 0xFu, rd.secondWo);
            if (!any_gt0(mi_eval(sd2, d2, 0xFu, rd.secondWo))) return false;
            if (rd.pathLength > 3)
            {
                // pathReconnectionShift's lobe-specific x2 term; the suffix follows from x3
                if (!(lsp > 0.f)) return false;
                out.v[1] = replay_vertex(p, sd2, mask2, rd.secondWo);
                out.s = (1.f / lobePdf) * (1.f / lsp);
                out.nv = 2;
                f3 S;
                const bool replayed = p.opt.sampleGenerator == kSgTinyUniform && replay_suffix(p, rd, sd2, out, S) &&
                                      S.x == rd.irradiance.x && S.y == rd.irradiance.y && S.z == rd.irradiance.z;
                if (!replayed)
                {
                    // the suffix is held fixed at the record's radiance and only x1 and x2 are
                    // differentiated: a delta lobe past x2, a PCG32 state, or a suffix traced in
                    // geometry that has moved since (a record reused from an earlier frame)
                    out.nv = 2;
                    out.emitter = kInvalidIndex;
                    out.Le = rd.irradiance;
                    suffixHeld = true;
                    stats[kStatSkipped]++;
                }
            }
            else
            {
                if (rd.lightIsNEE)
                {
                    out.v[1] = replay_vertex(p, sd2, 0xFu, rd.secondWo);
                    out.s = (1.f / lobePdf) * (p.mis(rd.lightPdf, tp) / rd.lightPdf);
                }
                else
                {
                    if (!(lsp > 0.f)) return false;
                    out.v[1] = replay_vertex(p, sd2, mask2, rd.secondWo);
                    out.s = (1.f / lobePdf) * (p.mis(tp, rd.lightPdf) / lsp);
                }
                out.nv = 2;
                if (!rd.lightIsDistant)
                {
                    f3 o2 = computeRayOrigin(sd2.posW, dot(sd2.faceN, rd.secondWo) >= 0.f ? sd2.faceN : -sd2.faceN);
                    HitInfo h; float t;
                    if (p.bvh.closest(mk_ray(o2, rd.secondWo, 0.f, kRayTMax), h, t))
                        out.emitter = emitter_of(p, p.loadSD(h, rd.secondWo));
                    // a light sample whose ray slips through the seam between two triangles of the light
                    if (out.emitter == kInvalidIndex && rd.lightIsNEE) out.emitter = emissive_material_with_radiance(p.lv, rd.irradiance);
                }
            }
        }
    }
    f3 prod = mk3(1.f);
    for (uint32_t k = 0; k < out.nv; k++) prod = prod * out.v[k].g.value;
    out.value = prod * out.Le * out.s;
    // a suffix path's value is checked through the record's irradiance (the replayed suffix
    // radiance equals it bit for bit); the suffix's densities and MIS weights fall into k
    const f3 check = out.L > 3 ? out.v[0].g.value * out.v[1].g.value * rd.irradiance * out.s : out.value;
    // The differentiated function is k * W * s * prod_k F_k(theta) * Le(theta) with k fixed, so that
    // at the pass's materials it equals the resolved colour integrand * W exactly (the replay and the
    // path tracer place ray origins slightly differently, which moves f(y) by ~1e-5 relative).
    out.k = mk3(out.value.x != 0.f ? r.integrand.x / out.value.x : 1.f, out.value.y != 0.f ? r.integrand.y / out.value.y : 1.f,
                out.value.z != 0.f ? r.integrand.z / out.value.z : 1.f);
    stats[kStatReplayed]++;
    // a path that ends at the environment map carries its radiance, no material's
    if (out.emitter == kInvalidIndex && !rd.lightIsDistant && !suffixHeld) stats[kStatNoEmitter]++;
    f3 diff = check - r.integrand;
    if (f_abs(diff.x) + f_abs(diff.y) + f_abs(diff.z) > 1e-3f * (f_abs(r.integrand.x) + f_abs(r.integrand.y) + f_abs(r.integrand.z)))
        stats[kStatValueMismatch]++;
    return true;
}

// d loss / d parameters of one pixel, given d loss / d colour (analytic, FP32 per pixel).
static void replay_accumulate(const Replay& q, f3 gradColor, double* grad)
{
    f3 g = gradColor * q.W * q.k;
    // before[k] = F_0 ... F_{k-1}, after = F_{k+1} ... (products of the other factors, no division)
    f3 before[kReplayMaxVertices];
    f3 run = mk3(1.f);
    for (uint32_t k = 0; k < q.nv; k++) { before[k] = run; run = run * q.v[k].g.value; }
    if (q.emitter != kInvalidIndex)
    {
        f3 dLe = g * run * q.s;
        double* e = grad + (size_t)q.emitter * kGradStride + kGradEmissive;
        e[0] += dLe.x; e[1] += dLe.y; e[2] += dLe.z;
    }
    f3 after = mk3(1.f);
    for (uint32_t k = q.nv; k-- > 0;)
    {
        const ReplayVertex& v = q.v[k];
        f3 common = g * (before[k] * after) * q.Le * q.s;
        f3 dB = common * v.g.dBase;
        f3 dR = common * v.g.dRough;
        f3 dM = common * v.g.dMetal;
        double* m = grad + (size_t)v.material * kGradStride;
        m[kGradBase + 0] += dB.x; m[kGradBase + 1] += dB.y; m[kGradBase + 2] += dB.z;
        m[kGradRough] += (double)dR.x + (double)dR.y + (double)dR.z;
        m[kGradMetal] += (double)dM.x + (double)dM.y + (double)dM.z;
        after = after * v.g.value;
    }
}

// FP64 value of one BSDF factor of the replay at material parameters `m` (the gates and the
// local directions stay those of the pass's materials).
// FP64 material parameters of the replay: baseColor.xyz, roughness, emissive.xyz, metallic.
struct ParamsFp64 { double v[kGradStride]; };

// Spec-gloss materials (kMtlSpecGloss): the diffuse albedo is baseColor, the specular colour the
// material's own, and the roughness 1 - the stored glossiness (setup_material).
static void replay_vertex_fp64(const ReplayVertex& v, const ParamsFp64& q, const MaterialData& mat, double out[3])
{
    const bool specGloss = (mat.flags & kMtlSpecGloss) != 0;
    const float ior = mat.ior;
    out[0] = out[1] = out[2] = 0.0;
    if (!v.valid) return;
    const double wi[3] = {v.wi.x, v.wi.y, v.wi.z}, wo[3] = {v.wo.x, v.wo.y, v.wo.z};
    double h[3] = {wi[0] + wo[0], wi[1] + wo[1], wi[2] + wo[2]};
    double hl = std::sqrt(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
    for (double& x : h) x /= hl;
    const double r = specGloss ? 1.0 - q.v[kGradRough] : q.v[kGradRough], metal = q.v[7];
    const double kPiD = 3.14159265358979323846;
    if (v.diffuseOn)
    {
        double woDotH = wo[0] * h[0] + wo[1] * h[1] + wo[2] * h[2];
        double E = 1.0 + r * (1.0 / 1.51 - 1.0);
        double fd90 = 0.5 * r + 2.0 * woDotH * woDotH * r;
        double Pi = std::pow(std::max(1.0 - wi[2], 0.0), 5.0), Po = std::pow(std::max(1.0 - wo[2], 0.0), 5.0);
        double S = (1.0 + (fd90 - 1.0) * Pi) * (1.0 + (fd90 - 1.0) * Po) * E / kPiD * wo[2];
        for (int c = 0; c < 3; c++) out[c] += q.v[kGradBase + c] * (specGloss ? 1.0 : 1.0 - metal) * S;
    }
    if (v.specularOn)
    {
        double alpha = std::max(r * r, (double)kMinGGXAlpha), a2 = alpha * alpha;
        double c = h[2];
        double dd = c * c * (a2 - 1.0) + 1.0;
        double D = a2 / (dd * dd * kPiD);
        auto lambda = [&](double cs) { double t2 = std::max(1.0 - cs * cs, 0.0) / (cs * cs); return 0.5 * (std::sqrt(1.0 + a2 * t2) - 1.0); };
        double G = 1.0 / (1.0 + lambda(wi[2]) + lambda(wo[2]));
        double wiDotH = wi[0] * h[0] + wi[1] * h[1] + wi[2] * h[2];
        double P = std::pow(std::max(1.0 - wiDotH, 0.0), 5.0);
        double f = (double)((ior - 1.f) / (ior + 1.f));
        double F0 = f * f;
        for (int k = 0; k < 3; k++)
        {
            double spec = specGloss ? (double)mat.specular[k] : F0 + (q.v[kGradBase + k] - F0) * metal;
            out[k] += (spec + (1.0 - spec) * P) * D * G * 0.25 / wi[2];
        }
    }
}

static ParamsFp64 params_of(const MaterialData& m)
{
    ParamsFp64 q;
    for (int c = 0; c < 3; c++) { q.v[kGradBase + c] = m.baseColor[c]; q.v[kGradEmissive + c] = m.emissive[c]; }
    q.v[kGradRough] = m.roughness;
    q.v[7] = m.metallic;
    return q;
}

// The FP64 replay: f(theta) = integrand * W * prod_k factor_k(theta) / factor_k(theta0), so that
// it equals the resolved colour at the pass's materials theta0 and moves with the FP64 factors.
static void replay_fp64(const Replay& q, const ParamsFp64* params, const MaterialData* mats, const f3& integrand, double out[3])
{
    double F[3] = {1.0, 1.0, 1.0}, F0[3] = {1.0, 1.0, 1.0};
    for (uint32_t k = 0; k < q.nv; k++)
    {
        const uint32_t m = q.v[k].material;
        double a[3], a0[3];
        replay_vertex_fp64(q.v[k], params[m], mats[m], a);
        replay_vertex_fp64(q.v[k], params_of(mats[m]), mats[m], a0);
        for (int c = 0; c < 3; c++) { F[c] *= a[c]; F0[c] *= a0[c]; }
    }
    double Le[3] = {q.Le.x, q.Le.y, q.Le.z}, Le0[3] = {q.Le.x, q.Le.y, q.Le.z};
    if (q.emitter != kInvalidIndex)
        for (int c = 0; c < 3; c++) { Le[c] = params[q.emitter].v[kGradEmissive + c]; Le0[c] = mats[q.emitter].emissive[c]; }
    const double I[3] = {integrand.x, integrand.y, integrand.z};
    for (int c = 0; c < 3; c++)
    {
        double den = F0[c] * Le0[c];
        out[c] = den != 0.0 ? I[c] * (double)q.W * (F[c] * Le[c] / den) : 0.0;
    }
}

static double replay_loss_fp64(const Replay& q, const ParamsFp64* params, const MaterialData* mats, const f3& integrand,
                               const float* target)
{
    double v[3];
    replay_fp64(q, params, mats, integrand, v);
    double loss = 0.0;
    for (int c = 0; c < 3; c++)
    {
        double e = v[c] - (double)target[c];
        loss += e * e;
    }
    return loss;
}

} // namespace oracle

// ------------------------------------------------------------------ C API (ctypes)
extern "C" {

struct ro_pass
{
    oracle::Pass p;
    std::vector<float> positions;      // the scene's triangle soup, kept for material updates
    std::vector<uint32_t> materialIds;
};

__attribute__((visibility("default"))) ro_pass* ro_create(const rs_options* opt)
{
    ro_pass* r = new ro_pass();
    r->p.opt = *opt;
    r->p.resize(opt->frameWidth, opt->frameHeight);
    r->p.buildNeighborOffsets();
    return r;
}
__attribute__((visibility("default"))) void ro_destroy(ro_pass* r) { delete r; }
__attribute__((visibility("default"))) int ro_set_threads(int n) { if (n > 0) omp_set_num_threads(n); return omp_get_max_threads(); }

// The scene's analytic lights, prepared as the pass prepares them (prepare_analytic_light).
__attribute__((visibility("default"))) int ro_set_analytic_lights(ro_pass* r, const rs_analytic_light* lights, uint32_t count)
{
    if (count > 0 && !lights) return RS_INVALID_ARG;
    std::vector<AnalyticLight> out(count);
    for (uint32_t i = 0; i < count; i++)
    {
        AnalyticLightDesc d;
        memcpy(&d, &lights[i], sizeof(d));
        if (!prepare_analytic_light(d, out[i])) return RS_INVALID_ARG;
    }
    r->p.analytic.swap(out);
    return RS_OK;
}

// Scene envMap + EnvMapSampler::createImportanceMap (EnvMap.cpp:60-137, EnvMapSampler.cpp:80-113):
// the texels, the transform, and the importance mips built on the host with the device's
// per-texel and reduction functions.
__attribute__((visibility("default"))) int ro_set_env_map(ro_pass* r, const rs_env_map* m)
{
    oracle::Pass& p = r->p;
    EnvMapView v = {};
    if (m && m->width > 0)
    {
        if (!m->texels || m->height == 0) return RS_INVALID_ARG;
        p.envTexels.assign(m->texels, m->texels + 4 * (size_t)m->width * m->height);
        p.envImportance.assign(kEnvImportanceTexels, 0.f);
        v.texels = p.envTexels.data();
        v.importance = p.envImportance.data();
        v.w = m->width; v.h = m->height;
        v.present = m->intensity > 0.f ? 1u : 0u;
        env_transform(m->rotation, v.toWorld, v.toLocal);
        for (int k = 0; k < 3; k++) v.scale[k] = m->intensity * m->tint[k];
        float* imp = p.envImportance.data();
        #pragma omp parallel for schedule(dynamic, 8)
        for (int y = 0; y < (int)kEnvImportanceDim; y++)
            for (uint32_t x = 0; x < kEnvImportanceDim; x++) imp[(size_t)y * kEnvImportanceDim + x] = env_importance_texel(v, x, (uint32_t)y);
        for (uint32_t mip = 1; mip < kEnvImportanceMips; mip++)
        {
            const uint32_t d = kEnvImportanceDim >> mip;
            for (uint32_t y = 0; y < d; y++)
                for (uint32_t x = 0; x < d; x++) imp[env_mip_offset(mip) + y * d + x] = env_importance_reduce(imp, mip, x, y);
        }
    }
    p.env = v;
    return RS_OK;
}

// Sampler checks: for each of n pairs of uniform numbers, env_sample's direction, pdf and radiance,
// then env_eval_pdf and env_eval of that direction (9 + 2 floats per sample).
__attribute__((visibility("default"))) int ro_env_debug(ro_pass* r, const float* rnd, uint32_t n, float* out)
{
    const EnvMapView& e = r->p.env;
    if (!e.importance) return RS_NOT_READY;
    for (uint32_t i = 0; i < n; i++)
    {
        f3 dir, Le; float pdf;
        env_sample(e, mk2(rnd[2 * i], rnd[2 * i + 1]), dir, pdf, Le);
        const f3 ev = env_eval(e, dir);
        const float o[11] = {dir.x, dir.y, dir.z, pdf, Le.x, Le.y, Le.z, env_eval_pdf(e, dir), ev.x, ev.y, ev.z};
        memcpy(out + 11 * (size_t)i, o, sizeof(o));
    }
    return RS_OK;
}

__attribute__((visibility("default"))) int ro_get_env_importance(ro_pass* r, float* out)
{
    if (r->p.envImportance.size() != kEnvImportanceTexels) return RS_NOT_READY;
    memcpy(out, r->p.envImportance.data(), kEnvImportanceTexels * sizeof(float));
    return RS_OK;
}

__attribute__((visibility("default"))) int ro_set_scene(ro_pass* r, const rs_scene_desc* s)
{
    oracle::Pass& p = r->p;
    if (!prepare_scene(s->numTriangles, s->positions, s->materialIds, s->numMaterials, reinterpret_cast<const MaterialData*>(s->materials), p.scene))
        return RS_INVALID_ARG;
    r->positions.assign(s->positions, s->positions + 9 * (size_t)s->numTriangles);
    r->materialIds.assign(s->materialIds, s->materialIds + s->numTriangles);
    p.bvh.build(p.scene.tri, s->numTriangles);
    p.lv.tris = p.scene.lights.data();
    p.lv.aliasTable = p.scene.alias.data();
    p.lv.count = (uint32_t)p.scene.lights.size();
    p.lv.invWeightsSum = p.scene.invWeightsSum;
    p.lv.sampler = p.opt.emissiveSampler;
    p.hasScene = true;
    p.frameCount = 0;
    return RS_OK;
}

__attribute__((visibility("default"))) int ro_execute(ro_pass* r, const rs_frame_desc* f, const float* mvecHost, float* colorHost)
{
    r->p.lv.sampler = r->p.opt.emissiveSampler;
    return r->p.execute(f, mvecHost, colorHost);
}

__attribute__((visibility("default"))) int ro_freeze(ro_pass* r, int frozen) { r->p.frozen = frozen != 0; return RS_OK; }
// ReservoirSplatting::reset (ReservoirSplatting.cpp:813-820)
__attribute__((visibility("default"))) int ro_reset(ro_pass* r)
{
    if (!r->p.frozen) { r->p.frameCount = 0; r->p.seed = 0; }
    return RS_OK;
}

// Same buffer ids and canonical layouts as rs_get_buffer.
__attribute__((visibility("default"))) long ro_get_buffer(ro_pass* r, int id, void* dst, size_t cap)
{
    oracle::Pass& p = r->p;
    size_t N = (size_t)p.W * p.H;
    auto resv = [&](const std::vector<oracle::PathReservoir>& v) -> long {
        size_t need = N * 32; if (!dst) return (long)need; if (cap < need) return -1;
        for (size_t i = 0; i < N; i++) oracle::export_reservoir(v[i], (float*)dst + 8 * i);
        return (long)need;
    };
    auto recn = [&](const std::vector<oracle::ReconnectionData>& v) -> long {
        size_t need = N * 112; if (!dst) return (long)need; if (cap < need) return -1;
        for (size_t i = 0; i < N; i++) oracle::export_recon(v[i], (uint32_t*)dst + 28 * i);
        return (long)need;
    };
    auto u32 = [&](const std::vector<uint32_t>& v) -> long {
        size_t need = v.size() * 4; if (!dst) return (long)need; if (cap < need) return -1;
        memcpy(dst, v.data(), need); return (long)need;
    };
    switch (id)
    {
    // After endFrame's swap the frame's result sits in `prev`.
    case RS_BUF_CURR_RESERVOIRS: return resv(p.swapped ? p.prev : p.curr);
    case RS_BUF_CURR_RECONNECTION: return recn(p.swapped ? p.prevR : p.currR);
    case RS_BUF_PREV_RESERVOIRS: return resv(p.swapped ? p.curr : p.prev);
    case RS_BUF_PREV_RECONNECTION: return recn(p.swapped ? p.currR : p.prevR);
    case RS_BUF_CANDIDATE_RESERVOIRS: return resv(p.candidates);
    case RS_BUF_CANDIDATE_RECONNECTION: return recn(p.candidatesR);
    case RS_BUF_BACKUP_RESERVOIRS: return resv(p.intermediate);
    case RS_BUF_BACKUP_RECONNECTION: return recn(p.intermediateR);
    case RS_BUF_CELL_COUNTERS: return u32(p.cellCounters);
    case RS_BUF_CELL_OFFSETS: return u32(p.cellOffsets);
    case RS_BUF_SORTED_SPLATS: return u32(p.sorted);
    case RS_BUF_SPLAT_TARGETS: return u32(p.splatTargets);
    case RS_BUF_FLOATING_COORDS: { size_t need = N * 8; if (!dst) return (long)need; if (cap < need) return -1; memcpy(dst, p.floatingCoords.data(), need); return (long)need; }
    case RS_BUF_MVEC: { size_t need = N * 8; if (!dst) return (long)need; if (cap < need) return -1; memcpy(dst, p.mvec.data(), need); return (long)need; }
    case RS_BUF_VBUFFER: { size_t need = N * 16; if (!dst) return (long)need; if (cap < need) return -1; memcpy(dst, p.vbuffer.data(), need); return (long)need; }
    default: return -2;
    }
}

__attribute__((visibility("default"))) int ro_set_buffer(ro_pass* r, int id, const void* src, size_t bytes)
{
    oracle::Pass& p = r->p;
    size_t N = (size_t)p.W * p.H;
    if (id == RS_BUF_PREV_RESERVOIRS || id == RS_BUF_CURR_RESERVOIRS)
    {
        if (bytes != N * 32) return RS_INVALID_ARG;
        bool toPrev = (id == RS_BUF_CURR_RESERVOIRS) == p.swapped;
        auto& v = toPrev ? p.prev : p.curr;
        for (size_t i = 0; i < N; i++) oracle::import_reservoir(v[i], (const float*)src + 8 * i);
        return RS_OK;
    }
    if (id == RS_BUF_PREV_RECONNECTION || id == RS_BUF_CURR_RECONNECTION)
    {
        if (bytes != N * 112) return RS_INVALID_ARG;
        bool toPrev = (id == RS_BUF_CURR_RECONNECTION) == p.swapped;
        auto& v = toPrev ? p.prevR : p.currR;
        for (size_t i = 0; i < N; i++) oracle::import_recon(v[i], (const uint32_t*)src + 28 * i);
        return RS_OK;
    }
    return RS_INVALID_ARG;
}

__attribute__((visibility("default"))) uint32_t ro_frame_count(ro_pass* r) { return r->p.frameCount; }

// Moves the scene's triangles (same count; materials stay) for the next frame: the previous
// positions are kept for that frame's motion vectors, the BVH is rebuilt and the light records
// take their triangles' new vertices (their flux, and the power sampler, stay).
__attribute__((visibility("default"))) int ro_update_geometry(ro_pass* r, const float* positions, uint32_t numTriangles)
{
    oracle::Pass& p = r->p;
    if (!p.hasScene || numTriangles != r->materialIds.size()) return RS_INVALID_ARG;
    p.prevTri = p.scene.tri;
    for (size_t t = 0; t < numTriangles; t++)
        for (int v = 0; v < 3; v++)
        {
            f4& q = p.scene.tri[3 * t + v];
            q.x = positions[9 * t + 3 * v + 0]; q.y = positions[9 * t + 3 * v + 1]; q.z = positions[9 * t + 3 * v + 2];
        }
    r->positions.assign(positions, positions + 9 * (size_t)numTriangles);
    for (LightTriangle& L : p.scene.lights)
    {
        const f4* q = &p.scene.tri[3 * (size_t)L.sceneTri];
        light_set_vertices(L, f4xyz(q[0]), f4xyz(q[1]), f4xyz(q[2]));
    }
    p.bvh.build(p.scene.tri, numTriangles);
    p.geometryMoved = true;
    return RS_OK;
}

// Replaces the material parameters (same count) and rebuilds the light collection; the geometry
// and its BVH stay.
__attribute__((visibility("default"))) int ro_set_materials(ro_pass* r, const rs_material* mats, uint32_t count)
{
    oracle::Pass& p = r->p;
    if (!p.hasScene || count != p.scene.materials.size()) return RS_INVALID_ARG;
    if (!prepare_scene((uint32_t)r->materialIds.size(), r->positions.data(), r->materialIds.data(), count,
                       reinterpret_cast<const MaterialData*>(mats), p.scene))
        return RS_INVALID_ARG;
    p.lv.tris = p.scene.lights.data();
    p.lv.aliasTable = p.scene.alias.data();
    p.lv.count = (uint32_t)p.scene.lights.size();
    p.lv.invWeightsSum = p.scene.invWeightsSum;
    p.lv.sampler = p.opt.emissiveSampler;
    return RS_OK;
}

// Analytic path-replay gradient of the last frame: adds d loss / d material parameters (count x 8
// doubles: baseColor.xyz, roughness, emissive.xyz, 0) given d loss / d colour (float4 per pixel).
// stats: replayed paths, paths whose suffix is held fixed (a delta lobe or an emissive hit past x2,
// more than kReplayMaxVertices factors, a PCG32 sample generator, geometry that moved since the
// record was made), paths without an identified emitter, replays whose value differs from the
// reservoir's integrand by more than 1e-3.
__attribute__((visibility("default"))) int ro_backward(ro_pass* r, const float* gradColor, double* gradOut, uint64_t* stats)
{
    oracle::Pass& p = r->p;
    if (!p.hasScene) return RS_NOT_READY;
    const auto& res = p.swapped ? p.prev : p.curr;
    const auto& rec = p.swapped ? p.prevR : p.currR;
    const size_t N = (size_t)p.W * p.H, M = p.scene.materials.size() * kGradStride;
    int T = omp_get_max_threads();
    std::vector<std::vector<double>> part(T, std::vector<double>(M, 0.0));
    std::vector<std::array<uint64_t, 4>> st(T, std::array<uint64_t, 4>{0, 0, 0, 0});
#pragma omp parallel for schedule(dynamic, 256)
    for (long i = 0; i < (long)N; i++)
    {
        int t = omp_get_thread_num();
        oracle::Replay q;
        if (!oracle::replay_pixel(p, res[i], rec[i], q, st[t].data())) continue;
        oracle::replay_accumulate(q, mk3(gradColor[4 * i], gradColor[4 * i + 1], gradColor[4 * i + 2]), part[t].data());
    }
    for (int t = 0; t < T; t++)
    {
        for (size_t k = 0; k < M; k++) gradOut[k] += part[t][k];
        if (stats) for (int k = 0; k < 4; k++) stats[k] += st[t][k];
    }
    return RS_OK;
}

// FP64 replay loss of the last frame, sum over pixels and channels of (f(y) W - target)^2, with the
// differentiated parameters taken from `params` (count x 8 doubles: baseColor.xyz, roughness,
// emissive.xyz, metallic) and everything detached taken from the pass's materials.
__attribute__((visibility("default"))) double ro_replay_loss(ro_pass* r, const float* target, const double* params, uint32_t count)
{
    oracle::Pass& p = r->p;
    if (!p.hasScene || count != p.scene.materials.size()) return -1.0;
    const auto& res = p.swapped ? p.prev : p.curr;
    const auto& rec = p.swapped ? p.prevR : p.currR;
    const oracle::ParamsFp64* q64 = reinterpret_cast<const oracle::ParamsFp64*>(params);
    const MaterialData* m = p.scene.materials.data();
    const size_t N = (size_t)p.W * p.H;
    double loss = 0.0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : loss)
    for (long i = 0; i < (long)N; i++)
    {
        uint64_t st[4] = {0, 0, 0, 0};
        oracle::Replay q;
        const float* t = target + 4 * i;
        if (!oracle::replay_pixel(p, res[i], rec[i], q, st))
        {
            loss += (double)t[0] * t[0] + (double)t[1] * t[1] + (double)t[2] * t[2];
            continue;
        }
        loss += oracle::replay_loss_fp64(q, q64, m, res[i].integrand, t);
    }
    return loss;
}

} // extern "C"

// ------------------------------------------------------------------ test hooks (known-answer tests)
extern "C" {

// First n 32-bit outputs of the per-pixel stream of `kind` (0 TinyUniform, 2 PCG32).
__attribute__((visibility("default"))) void ro_test_rng(uint32_t kind, uint32_t px, uint32_t py, uint32_t seed, uint32_t n, uint32_t* out)
{
    SampleGen sg = sg_create(px, py, seed, kind);
    for (uint32_t i = 0; i < n; i++) out[i] = sg_next(sg);
}
__attribute__((visibility("default"))) void ro_test_tea(uint32_t v0, uint32_t v1, uint32_t* out)
{
    tea16(v0, v1);
    out[0] = v0; out[1] = v1;
}
__attribute__((visibility("default"))) uint32_t ro_test_interleave(uint32_t x, uint32_t y) { return interleave_32bit(x, y); }

// kind: 0 sin, 1 cos, 2 tan, 3 atan, 4 acos
__attribute__((visibility("default"))) void ro_test_fmath(int kind, const float* x, float* y, uint32_t n)
{
    for (uint32_t i = 0; i < n; i++)
    {
        float v = x[i];
        switch (kind)
        {
        case 0: y[i] = f_sin(v); break;
        case 1: y[i] = f_cos(v); break;
        case 2: y[i] = f_tan(v); break;
        case 3: y[i] = f_atan(v); break;
        default: y[i] = f_acos(v); break;
        }
    }
}
// f_pow_pos(x[i], e[i]) (the PowerExp MIS heuristic's power).
// One analytic light prepared from its description and sampled at a shading point with the given
// two uniform numbers: out = {ok, posW.xyz, normalW.xyz, dir.xyz, distance, Li.xyz, pdf} and the
// prepared record (out[15..]: cosOpeningAngle, penumbraAngle, cosSubtendedAngle, surfaceArea,
// transMat[12], transMatIT[9]).  Returns 0 when the description is rejected.
__attribute__((visibility("default"))) int ro_test_analytic(const rs_analytic_light* desc, const float* pos3, const float* u2, float* out)
{
    AnalyticLightDesc d;
    memcpy(&d, desc, sizeof(d));
    AnalyticLight L;
    if (!prepare_analytic_light(d, L)) return 0;
    AnalyticSample ls;
    ls.posW = mk3(0.f); ls.normalW = mk3(0.f); ls.dir = mk3(0.f); ls.Li = mk3(0.f); ls.distance = 0.f; ls.pdf = 0.f;
    const f3 x = mk3(pos3[0], pos3[1], pos3[2]);
    const f2 u = mk2(u2[0], u2[1]);
    bool ok;
    if (L.type == kLightPoint) ok = al_sample_point(x, L, ls);
    else if (L.type == kLightDirectional) ok = al_sample_directional(L, ls);
    else if (L.type == kLightDistant) ok = al_sample_distant(L, u, ls);
    else ok = al_sample_area(x, L, u, ls);
    const float v[15] = {ok ? 1.f : 0.f, ls.posW.x, ls.posW.y, ls.posW.z, ls.normalW.x, ls.normalW.y, ls.normalW.z,
                         ls.dir.x, ls.dir.y, ls.dir.z, ls.distance, ls.Li.x, ls.Li.y, ls.Li.z, ls.pdf};
    for (int k = 0; k < 15; k++) out[k] = v[k];
    out[15] = L.cosOpeningAngle; out[16] = L.penumbraAngle; out[17] = L.cosSubtendedAngle; out[18] = L.surfaceArea;
    for (int k = 0; k < 12; k++) out[19 + k] = L.transMat[k];
    for (int k = 0; k < 9; k++) out[31 + k] = L.transMatIT[k];
    return 1;
}

__attribute__((visibility("default"))) void ro_test_pow(const float* x, const float* e, float* y, uint32_t n)
{
    for (uint32_t i = 0; i < n; i++) y[i] = f_pow_pos(x[i], e[i]);
}
__attribute__((visibility("default"))) void ro_test_f16(const float* x, uint16_t* h, float* back, uint32_t n)
{
    for (uint32_t i = 0; i < n; i++) { h[i] = f32_to_f16(x[i]); back[i] = f16_to_f32(h[i]); }
}
// Alias table of `weights`; writes the packed table (2 words per entry) and returns the weight sum.
__attribute__((visibility("default"))) double ro_test_alias(const float* w, uint32_t n, uint32_t* table)
{
    std::vector<float> weights(w, w + n);
    std::vector<u2> t;
    double sum;
    build_alias_table(weights, t, sum);
    for (uint32_t i = 0; i < n; i++) { table[2 * i] = t[i].x; table[2 * i + 1] = t[i].y; }
    return sum;
}
// BSDF derivative check: material = (baseColor.xyz, roughness, metallic, ior, spec-gloss flag,
// specular.xyz), directions in the local frame (normal +z).  out = value.xyz, dBase.xyz, dRough.xyz,
// dMetal.xyz (FP32 analytic); valueFp64 = the FP64 value at the same parameters (for central
// differences).
__attribute__((visibility("default"))) void ro_test_bsdf_grad(const float* mat, const float* wi, const float* wo, uint32_t lobeMask,
                                                             float* out, double* valueFp64)
{
    MaterialData m;
    memset(&m, 0, sizeof(m));
    m.baseColor[0] = mat[0]; m.baseColor[1] = mat[1]; m.baseColor[2] = mat[2];
    m.roughness = mat[3]; m.metallic = mat[4]; m.ior = mat[5];
    if (mat[6] != 0.f) // spec-gloss: mat[3] is the glossiness, mat[7..9] the specular colour
    {
        m.flags = kMtlSpecGloss;
        m.specular[0] = mat[7]; m.specular[1] = mat[8]; m.specular[2] = mat[9];
    }
    ShadingData sd;
    memset(&sd, 0, sizeof(sd));
    sd.N = mk3(0.f, 0.f, 1.f); sd.T = mk3(1.f, 0.f, 0.f); sd.B = mk3(0.f, 1.f, 0.f); sd.faceN = sd.N;
    sd.V = mk3(wi[0], wi[1], wi[2]);
    sd.frontFacing = true;
    f3 w = mk3(wo[0], wo[1], wo[2]);
    BsdfData d = setup_material(m, true);
    BsdfGrad g = mi_eval_grad(sd, d, m, lobeMask, w);
    const f3 v[4] = {g.value, g.dBase, g.dRough, g.dMetal};
    for (int k = 0; k < 4; k++) { out[3 * k] = v[k].x; out[3 * k + 1] = v[k].y; out[3 * k + 2] = v[k].z; }
    oracle::ParamsFp64 q64;
    for (int k = 0; k < 8; k++) q64.v[k] = 0.0;
    for (int k = 0; k < 3; k++) q64.v[kGradBase + k] = mat[k];
    q64.v[kGradRough] = mat[3];
    q64.v[7] = mat[4];
    oracle::ReplayVertex rv;
    f3 wil = sd_to_local(sd, sd.V), wol = sd_to_local(sd, w);
    rv.wi = wil; rv.wo = wol;
    rv.valid = valid_hemisphere(sd, wil, wol, w) && f_min(wil.z, wol.z) >= kMinCosTheta;
    StandardBSDF b = make_bsdf(wil, d, lobeMask);
    uint32_t mask = lobeMask == 0 ? 0xfu : lobeMask;
    rv.diffuseOn = b.pDiffuseReflection > 0.f && (mask & 0x1u);
    rv.specularOn = b.pSpecularReflection > 0.f && (mask & 0x4u) && b.alpha != 0.f;
    oracle::replay_vertex_fp64(rv, q64, m, valueFp64);
}

// ---- BSDF property hooks (the sampling test of Tests/Scene/Material/BSDFTests.cpp restated on the
// shared BSDF; the checks themselves live in tests/test_core_properties_cpu.py).
//
// kind 0: FrostbiteDiffuseBRDF alone, albedo 1, roughness params[0]
// kind 1: SpecularMicrofacetBRDF alone, albedo 1, GGX alpha params[0]
// kind 2: StandardBSDF of the opaque metal-rough material baseColor params[0] (grey), roughness
//         params[1], metallic params[2], ior params[3], all lobes (lobe mask 0)
static StandardBSDF test_bsdf(uint32_t kind, const float* params, f3 wi)
{
    StandardBSDF b;
    memset(&b, 0, sizeof(b));
    if (kind == 0)
    {
        b.diffAlbedo = mk3(1.f); b.diffRoughness = params[0];
        b.pDiffuseReflection = 1.f;
    }
    else if (kind == 1)
    {
        b.specAlbedo = mk3(1.f); b.alpha = params[0];
        b.pSpecularReflection = 1.f;
    }
    else
    {
        MaterialData m;
        memset(&m, 0, sizeof(m));
        m.baseColor[0] = m.baseColor[1] = m.baseColor[2] = params[0];
        m.roughness = params[1]; m.metallic = params[2]; m.ior = params[3];
        b = make_bsdf(wi, setup_material(m, true), 0u);
    }
    return b;
}

// n samples of the BSDF for incident direction wi (local frame, normal +z), drawn from the PCG32
// streams of pixels (0, seed) .. : wo[3n], pdf[n], weight[3n], valid[n], lobe[n].
__attribute__((visibility("default"))) void ro_test_bsdf_sample(uint32_t kind, const float* params, const float* wi3, uint32_t n, uint32_t seed,
                                                               float* wo, float* pdf, float* weight, uint32_t* valid, uint32_t* lobe)
{
    const f3 wi = normalize(mk3(wi3[0], wi3[1], wi3[2]));
    const StandardBSDF b = test_bsdf(kind, params, wi);
    const uint32_t chunk = 4096;
    #pragma omp parallel for schedule(dynamic, 1)
    for (int64_t c = 0; c < (int64_t)((n + chunk - 1) / chunk); c++)
    {
        SampleGen sg = sg_create((uint32_t)c, seed, 12345u, kSgPCG32);
        for (uint32_t i = (uint32_t)c * chunk; i < n && i < (uint32_t)(c + 1) * chunk; i++)
        {
            f3 w, wt; float p; uint32_t lt;
            valid[i] = bsdf_sample_local(b, wi, w, p, wt, lt, sg) ? 1u : 0u;
            wo[3 * i] = w.x; wo[3 * i + 1] = w.y; wo[3 * i + 2] = w.z;
            weight[3 * i] = wt.x; weight[3 * i + 1] = wt.y; weight[3 * i + 2] = wt.z;
            pdf[i] = p; lobe[i] = lt;
        }
    }
}

// eval (value * cos, as the BSDF returns it) and evalPdf of n direction pairs: value[3n], pdf[n].
__attribute__((visibility("default"))) void ro_test_bsdf_eval(uint32_t kind, const float* params, const float* wi3, const float* wo3, uint32_t n,
                                                             float* value, float* pdf)
{
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++)
    {
        const f3 wi = mk3(wi3[3 * i], wi3[3 * i + 1], wi3[3 * i + 2]);
        const f3 wo = mk3(wo3[3 * i], wo3[3 * i + 1], wo3[3 * i + 2]);
        const StandardBSDF b = test_bsdf(kind, params, wi);
        const f3 v = bsdf_eval_local(b, wi, wo);
        value[3 * i] = v.x; value[3 * i + 1] = v.y; value[3 * i + 2] = v.z;
        pdf[i] = bsdf_pdf_local(b, wi, wo);
    }
}

// The sampling histograms of BSDFTests.cs.slang: sampled directions binned by (cos theta, phi)
// (hist[cosBins * phiBins], samples within 1e-3 of the poles skipped), the pdf integrated over each
// bin with binSamples^2 midpoint samples times the sample count (expected[...]), and the largest
// relative error of the sample weight against eval / evalPdf and of the sample pdf against evalPdf
// (maxErr[0], maxErr[1]).
__attribute__((visibility("default"))) void ro_test_bsdf_histogram(uint32_t kind, const float* params, const float* wi3, uint32_t sampleCount,
                                                                  uint32_t phiBins, uint32_t cosBins, uint32_t binSamples, uint32_t seed,
                                                                  double* hist, double* expected, double* maxErr)
{
    const f3 wi = normalize(mk3(wi3[0], wi3[1], wi3[2]));
    const StandardBSDF b = test_bsdf(kind, params, wi);
    const double kCosThetaMargin = 1e-3;
    const uint32_t bins = phiBins * cosBins;
    const uint32_t chunk = 1u << 16;
    const int64_t chunks = (sampleCount + chunk - 1) / chunk;
    std::vector<std::vector<double>> part(omp_get_max_threads(), std::vector<double>(bins, 0.0));
    std::vector<double> wErr(omp_get_max_threads(), 0.0), pErr(omp_get_max_threads(), 0.0);
    #pragma omp parallel for schedule(dynamic, 1)
    for (int64_t c = 0; c < chunks; c++)
    {
        const int t = omp_get_thread_num();
        SampleGen sg = sg_create((uint32_t)c, seed, 777u, kSgPCG32);
        for (uint32_t i = (uint32_t)c * chunk; i < sampleCount && i < (uint32_t)(c + 1) * chunk; i++)
        {
            f3 wo, wt; float p; uint32_t lt;
            if (!bsdf_sample_local(b, wi, wo, p, wt, lt, sg)) continue;
            const f3 value = bsdf_eval_local(b, wi, wo);
            const float pdfRef = bsdf_pdf_local(b, wi, wo);
            const f3 wRef = pdfRef > 0.f ? value / pdfRef : mk3(0.f);
            const double e = std::max({std::fabs(wt.x - wRef.x) / (wRef.x > 0.f ? wRef.x : 1.f),
                                       std::fabs(wt.y - wRef.y) / (wRef.y > 0.f ? wRef.y : 1.f),
                                       std::fabs(wt.z - wRef.z) / (wRef.z > 0.f ? wRef.z : 1.f)});
            wErr[t] = std::max(wErr[t], e);
            pErr[t] = std::max(pErr[t], (double)std::fabs(p - pdfRef) / (pdfRef > 0.f ? pdfRef : 1.0));
            if (wo.z < -1.0 + kCosThetaMargin || wo.z > 1.0 - kCosThetaMargin) continue;
            const uint32_t cb = std::min(cosBins - 1, (uint32_t)std::floor(((double)wo.z * 0.5 + 0.5) * cosBins));
            double sp = std::atan2((double)wo.y, (double)wo.x) / (2.0 * M_PI);
            if (sp < 0.0) sp += 1.0;
            const uint32_t pb = std::min(phiBins - 1, (uint32_t)std::floor(sp * phiBins));
            part[t][cb * phiBins + pb] += 1.0;
        }
    }
    for (uint32_t k = 0; k < bins; k++)
    {
        double s = 0.0;
        for (auto& v : part) s += v[k];
        hist[k] = s;
    }
    maxErr[0] = *std::max_element(wErr.begin(), wErr.end());
    maxErr[1] = *std::max_element(pErr.begin(), pErr.end());
    #pragma omp parallel for schedule(dynamic, 4)
    for (int64_t k = 0; k < (int64_t)bins; k++)
    {
        const uint32_t cb = (uint32_t)k / phiBins, pb = (uint32_t)k % phiBins;
        const double phi0 = pb * 2.0 * M_PI / phiBins, phi1 = (pb + 1) * 2.0 * M_PI / phiBins;
        const double c0 = std::max(-1.0 + cb * 2.0 / cosBins, -1.0 + kCosThetaMargin);
        const double c1 = std::min(-1.0 + (cb + 1) * 2.0 / cosBins, 1.0 - kCosThetaMargin);
        double acc = 0.0;
        for (uint32_t ix = 0; ix < binSamples; ix++)
            for (uint32_t iy = 0; iy < binSamples; iy++)
            {
                const double phi = phi0 + (phi1 - phi0) * (ix + 0.5) / binSamples;
                const double ct = c0 + (c1 - c0) * (iy + 0.5) / binSamples;
                const double st = std::sqrt(std::max(0.0, 1.0 - ct * ct));
                const f3 wo = normalize(mk3((float)(st * std::cos(phi)), (float)(st * std::sin(phi)), (float)ct));
                acc += bsdf_pdf_local(b, wi, wo);
            }
        expected[k] = acc * (c1 - c0) * (phi1 - phi0) / ((double)binSamples * binSamples) * sampleCount;
    }
}

// Emissive NEE at shading point posW of the pass's light collection: n draws of
// sample_emissive_power from PCG32 streams, each with the triangle picked, the sample's pdf, the
// eval_emissive_pdf of the sampled point and the sampled position (tri[n], pdf[n], evalPdf[n],
// pos[3n]; pdf = 0 for a sample rejected because the triangle faces away).
__attribute__((visibility("default"))) int ro_test_emissive(ro_pass* r, const float* posW3, uint32_t n, uint32_t seed, uint32_t* tri, float* pdf,
                                                           float* evalPdf, float* pos)
{
    const LightView& L = r->p.lv;
    if (!L.count) return RS_NOT_READY;
    const f3 x = mk3(posW3[0], posW3[1], posW3[2]);
    #pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; i++)
    {
        // one stream per sample; pixel coordinates carry 16 bits each (interleave_32bit)
        SampleGen sg = sg_create((uint32_t)i & 0xffffu, ((uint32_t)i >> 16) + (seed << 8), 99u, kSgPCG32);
        TriangleLightSample ls;
        ls.triangleIndex = kInvalidIndex;
        const bool ok = sample_emissive(L, x, sg, ls);
        tri[i] = ls.triangleIndex;
        if (ok)
        {
            pdf[i] = ls.pdf;
            evalPdf[i] = eval_emissive_pdf(L, x, ls.triangleIndex, ls.posW, ls.normalW);
            pos[3 * i] = ls.posW.x; pos[3 * i + 1] = ls.posW.y; pos[3 * i + 2] = ls.posW.z;
        }
        else
        {
            pdf[i] = 0.f; evalPdf[i] = 0.f;
            pos[3 * i] = pos[3 * i + 1] = pos[3 * i + 2] = 0.f;
        }
    }
    return RS_OK;
}
// The light collection's records: per light 20 floats (p0, sceneTri bits, p1, area, p2, flux,
// normal, materialID bits, Le, 0); returns the count.
__attribute__((visibility("default"))) uint32_t ro_test_lights(ro_pass* r, float* out)
{
    const auto& v = r->p.scene.lights;
    if (out) memcpy(out, v.data(), v.size() * sizeof(LightTriangle));
    return (uint32_t)v.size();
}

// Camera basis (Camera.cpp:179-185) of cam: out = cameraU, cameraV, cameraW (9 floats).
__attribute__((visibility("default"))) void ro_test_camera_basis(const rs_camera* cam, float* out)
{
    CameraData d;
    memset(&d, 0, sizeof(d));
    d.posW = mk3(cam->position[0], cam->position[1], cam->position[2]);
    d.target = mk3(cam->target[0], cam->target[1], cam->target[2]);
    d.up = mk3(cam->up[0], cam->up[1], cam->up[2]);
    d.focalLength = cam->focalLength; d.frameHeight = cam->frameHeight; d.aspectRatio = cam->aspectRatio;
    d.focalDistance = cam->focalDistance;
    camera_update_basis(d);
    const f3 v[3] = {d.cameraU, d.cameraV, d.cameraW};
    for (int k = 0; k < 3; k++) { out[3 * k] = v[k].x; out[3 * k + 1] = v[k].y; out[3 * k + 2] = v[k].z; }
}

// orientCamera (CameraManager.slang:90-113) of cam over K keyframes (positions[3K], targets[3K]) at
// frameCount and time: out = posW, cameraU, cameraV, cameraW (12 floats).
__attribute__((visibility("default"))) void ro_test_orient_camera(const rs_camera* cam, uint32_t K, const float* positions, const float* targets,
                                                                 float artificialFrameTime, uint32_t frameCount, float time, float* out)
{
    CameraData d;
    memset(&d, 0, sizeof(d));
    d.posW = mk3(cam->position[0], cam->position[1], cam->position[2]);
    d.target = mk3(cam->target[0], cam->target[1], cam->target[2]);
    d.up = mk3(cam->up[0], cam->up[1], cam->up[2]);
    d.focalLength = cam->focalLength; d.frameHeight = cam->frameHeight; d.aspectRatio = cam->aspectRatio;
    d.focalDistance = cam->focalDistance;
    camera_update_basis(d);
    CameraManager cm;
    memset(&cm, 0, sizeof(cm));
    cm.artificialFrameTime = artificialFrameTime;
    cm.keyframes = K;
    for (uint32_t i = 0; i < K; i++)
    {
        cm.positions[i] = mk3(positions[3 * i], positions[3 * i + 1], positions[3 * i + 2]);
        cm.targets[i] = mk3(targets[3 * i], targets[3 * i + 1], targets[3 * i + 2]);
    }
    orient_camera(cm, d, frameCount, time);
    const f3 v[4] = {d.posW, d.cameraU, d.cameraV, d.cameraW};
    for (int k = 0; k < 4; k++) { out[3 * k] = v[k].x; out[3 * k + 1] = v[k].y; out[3 * k + 2] = v[k].z; }
}

// Closest hit of one ray against the oracle's BVH of a triangle soup (prim = -1 on a miss).
__attribute__((visibility("default"))) int ro_test_closest(ro_pass* r, const float* ray, float* tuv)
{
    Ray q = mk_ray(mk3(ray[0], ray[1], ray[2]), mk3(ray[3], ray[4], ray[5]), ray[6], ray[7]);
    HitInfo h; float t;
    if (!r->p.bvh.closest(q, h, t)) return -1;
    tuv[0] = t; f2 b = hit_bary(h); tuv[1] = b.x; tuv[2] = b.y;
    return (int)hit_prim(h);
}

} // extern "C"
