// Host side of the B200 Reservoir Splatting pass behind the C ABI of
// include/rs_b200.h: option parsing and validation, scene upload and LBVH build,
// per-frame orchestration (ReservoirSplatting::execute, ReservoirSplatting.cpp:399-509),
// buffer ping-pong (endFrame, :1648-1680) and the parity/checkpoint views.
//
// All device work of rs_execute is issued on the caller's stream with no host
// synchronisation and no allocation once the frame size and options are stable,
// so a frame can be captured into a CUDA graph after the first call.
#include <algorithm>
#include <cstdio>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>
#include <memory>
#include <mutex>
#include <functional>
#include "../../include/rs_b200.h"
#include "kernels.h"
#include "bvh_build.h"
#include "radix_sort.h"
#include "core/scene_prep.h"

using namespace rs;

static thread_local std::string g_lastError;

static rs_status fail(rs_status s, const std::string& msg)
{
    g_lastError = msg;
    return s;
}

// Lets entry points defined in other files report through rs_last_error_string().
namespace rs { void set_last_error(const std::string& msg) { g_lastError = msg; } }

#define RS_CUDA_STATUS(call)                                                                        \
    do {                                                                                            \
        rs_status s_ = (call);                                                                      \
        if (s_ != RS_OK) return s_;                                                                 \
    } while (0)

#define RS_CUDA(call)                                                                               \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return fail(e_ == cudaErrorMemoryAllocation ? RS_OOM : RS_CUDA_ERROR,                   \
                        std::string(#call) + ": " + cudaGetErrorString(e_));                      \
    } while (0)

namespace {

template <typename T>
struct DevBuf
{
    T* p = nullptr;
    size_t n = 0;
    ~DevBuf() { release(); }
    void release() { if (p) cudaFree(p); p = nullptr; n = 0; }
    cudaError_t ensure(size_t count)
    {
        if (count <= n && p) return cudaSuccess;
        release();
        if (count == 0) return cudaSuccess;
        cudaError_t e = cudaMalloc(&p, count * sizeof(T));
        if (e == cudaSuccess) n = count;
        return e;
    }
};

struct ReservoirSet
{
    DevBuf<float4> a, b;     // reservoir planes
    DevBuf<uint4> rec;       // 7 reconnection planes
    size_t N = 0;
    cudaError_t ensure(size_t n)
    {
        N = n;
        cudaError_t e;
        if ((e = a.ensure(n)) != cudaSuccess) return e;
        if ((e = b.ensure(n)) != cudaSuccess) return e;
        return rec.ensure(7 * n);
    }
    ResPlanes res() const { return ResPlanes{a.p, b.p}; }
    RecPlanes recp() const { return RecPlanes{rec.p, N}; }
};

} // namespace

static std::mutex g_slotMutex;
static bool g_slotUsed[kMaxPassSlots] = {};

static uint32_t acquire_slot()
{
    std::lock_guard<std::mutex> lock(g_slotMutex);
    for (uint32_t i = 0; i < kMaxPassSlots; i++)
        if (!g_slotUsed[i]) { g_slotUsed[i] = true; return i; }
    return kMaxPassSlots;
}
static void release_slot(uint32_t s)
{
    std::lock_guard<std::mutex> lock(g_slotMutex);
    if (s < kMaxPassSlots) g_slotUsed[s] = false;
}

struct rs_pass
{
    rs_options opt;
    // scene
    PreparedScene scene;
    DevBuf<float4> dTri;
    WideBvh bvh;
    DevBuf<float4> dPrevTri;    // triangles of the previous frame after rs_update_geometry
    DevBuf<float> dPosStage;    // host positions staged for rs_update_geometry
    bool geometryMoved = false; // rs_update_geometry since the last frame
    BvhBuilder bvhBuilder = kBvhPloc;
    bool hostTriStale = false;  // scene.tri positions behind the device copy
    DevBuf<MaterialData> dMaterials;
    DevBuf<LightTriangle> dLights;
    DevBuf<u2> dAlias;
    bool hasScene = false;
    // environment map: texels, importance mips and the view the kernels read (present = 0 without one)
    DevBuf<float> envTexels, envImportance;
    DevBuf<EnvMapView> envView;
    EnvMapView envHost = {};
    // analytic lights (rs_set_analytic_lights): device records and their count
    DevBuf<AnalyticLight> dAnalytic;
    uint32_t numAnalytic = 0;
    // frame state
    uint32_t W = 0, H = 0;
    uint32_t frameCount = 0, seed = 0;
    bool frozen = false, swapped = false;
    uint32_t K = 2, prevK = 0;
    CameraManager cm;
    CameraData camera, prevCamera;
    bool havePrevCamera = false;
    // buffers
    ReservoirSet sets[3];
    int currIdx = 0, prevIdx = 1, tempIdx = 2;
    ReservoirSet inter, cand;
    DevBuf<float2> mvec, floatingCoords, neighborOffsets;
    DevBuf<uint4> vbuffer;
    DevBuf<uint32_t> targets, counts, offsets, unsortedSplats, sortedSplats, tileSums, total, radixScratch;
    DevBuf<Shifted> shiftedPaths;
    DevBuf<float4> scratchColor;
    // wavefront ScatterBackup / spatial buffers
    DevBuf<uint32_t> sortedCell;
    DevBuf<float> m2curr, m3curr, spM1, spNw;
    DevBuf<uint4> backupShift, splatShift, spShift;
    DevBuf<float4> backupTerms, splatTerms, splatM, spTerms;
    DevBuf<float2> backupM;
    DevBuf<float> msCurr;                 // wavefront MultiSplatting buffers
    DevBuf<uint4> msShift;
    DevBuf<float4> msTerms, msMisSub;
    DevBuf<uint32_t> fault;
    uint32_t* hostFault = nullptr; // two words: frames alternate between them when host output is pipelined
    uint32_t faultSlot = 0;        // the word this frame's status is copied to
    // pipelined host output (rs_set_host_output_latency 1): frame k's colour is copied to the host on
    // copyStream from one of two device images while frame k + 1 renders on the caller's stream
    uint32_t hostLatency = 0;
    DevBuf<float4> pipeColor[2];
    int pipeIdx = 0;
    cudaStream_t copyStream = nullptr;
    cudaEvent_t frameDoneEv = nullptr, copyDoneEv = nullptr;
    bool copyPending = false;       // a host copy is in flight (copyDoneEv marks it)
    uint32_t pendingFaultSlot = 0;  // the status word of the frame whose copy is in flight
    DevBuf<CameraTable> camTable;
    // side streams for independent kernels of a frame (fork/join through events on the frame's
    // stream, so the frame stays one ordered unit for the caller and for graph capture)
    static constexpr int kSide = 3;
    cudaStream_t side[kSide] = {};
    cudaEvent_t forkEv = nullptr;
    cudaEvent_t joinEv[kSide] = {};
    DevBuf<unsigned long long> adjStats; // rs_backward counters (replayed, too long, no emitter, value mismatch)
    DevBuf<double> adjAcc;               // rs_backward FP64 sums, numMaterials x 8
    bool haveFrameCtx = false;           // hostCtx holds a frame's context (set by begin_frame)
    uint32_t slot = kMaxPassSlots;  // this pass's entry of the constant context table
    DevCtx* hostCtx = nullptr;      // staging copy of the frame's context (begin_frame)
    static constexpr int kRing = 8;
    DevCtx* ringCtx = nullptr;      // pinned upload sources for rs_execute, reused round-robin
    cudaEvent_t ringEv[kRing] = {};
    int ringNext = 0;
    DevCtx* graphCtx = nullptr;     // pinned upload source read by a replayed batch graph
    bool frameShouldReset = false;
    bool keepCandidates = false;
    bool lastFusedCollect = false;
    cudaStream_t lastStream = 0;
    uint32_t launches = 0;
    // Bumped by every call that can reallocate a buffer or change which kernels a frame launches
    // (options, scene, env map, candidate snapshots, geometry updates): a batch graph captured
    // under an older generation holds stale pointers, grids or kernel choices and is not replayed.
    uint64_t generation = 0;
    // stage timing
    bool timing = false;
    std::vector<std::string> stageNames;
    std::vector<cudaEvent_t> events;
    std::vector<float> stageMs;
#ifdef RS_RAY_STATS
    std::vector<unsigned long long> stageRays; // closest, visibility per stage (RS_RAY_STATS builds)
#endif

    ~rs_pass()
    {
        for (auto e : events) cudaEventDestroy(e);
        for (auto e : ringEv) if (e) cudaEventDestroy(e);
        for (auto e : joinEv) if (e) cudaEventDestroy(e);
        for (auto q : side) if (q) cudaStreamDestroy(q);
        if (forkEv) cudaEventDestroy(forkEv);
        if (copyStream) cudaStreamDestroy(copyStream);
        if (frameDoneEv) cudaEventDestroy(frameDoneEv);
        if (copyDoneEv) cudaEventDestroy(copyDoneEv);
        if (hostFault) cudaFreeHost(hostFault);
        if (hostCtx) cudaFreeHost(hostCtx);
        if (ringCtx) cudaFreeHost(ringCtx);
        if (graphCtx) cudaFreeHost(graphCtx);
        free_wide_bvh(&bvh);
        release_slot(slot);
    }
};

// ------------------------------------------------------------------ options
extern "C" RS_API void rs_default_options(rs_options* o)
{
    // ReservoirSplatting.h:124-184 defaults
    memset(o, 0, sizeof(*o));
    o->samplesPerPixel = 1;
    o->maxSurfaceBounces = 9; o->maxDiffuseBounces = 9; o->maxSpecularBounces = 9; o->maxTransmissionBounces = 9;
    o->sampleGenerator = RS_SG_TINY_UNIFORM;
    o->useFixedSeed = 0; o->fixedSeed = 1;
    o->useRussianRoulette = 1;
    o->misHeuristic = RS_MIS_HEURISTIC_BALANCE;
    o->misPowerExponent = 2.f;
    o->disableCaustics = 0;
    o->specularRoughnessThreshold = 0.25f;
    o->enableTemporalResampling = 1;
    o->enableSpatialResampling = 1;
    o->temporalReuse = RS_GATHER_ONLY;
    o->scatterBackupMISOption = RS_MIS_BALANCE;
    o->gatherOption = RS_GATHER_FAST;
    o->numTimePartitions = 2;
    o->useConfidenceWeightsTemporally = 1;
    o->numSpatialIterations = 1;
    o->spatialGatherRadius = 30.f;
    o->neighborCount = 1;
    o->useConfidenceWeightsSpatially = 1;
    o->artificialFrameTime = 1.f / 60.f;
    o->frameWidth = 1920; o->frameHeight = 1080;
    o->emissiveSampler = RS_EMISSIVE_POWER;
}

// validateOptions (ReservoirSplatting.cpp:263-301): out-of-range values are rejected here
// (the reference clamps with a warning; a C caller gets RS_INVALID_ARG and the reason).
static rs_status validate(const rs_options* o)
{
    if (!o) return fail(RS_INVALID_ARG, "options is NULL");
    if (o->samplesPerPixel < 1 || o->samplesPerPixel > 16) return fail(RS_INVALID_ARG, "samplesPerPixel must be in [1, 16]");
    if (o->maxSurfaceBounces > 254 || o->maxDiffuseBounces > 254 || o->maxSpecularBounces > 254 || o->maxTransmissionBounces > 254)
        return fail(RS_INVALID_ARG, "bounce limits must be <= 254");
    if (o->frameWidth == 0 || o->frameHeight == 0 || o->frameWidth > 4096 || o->frameHeight > 4096)
        return fail(RS_INVALID_ARG, "Frame dimensions up to 4096 pixels width/height are supported");
    if (o->sampleGenerator != RS_SG_TINY_UNIFORM && o->sampleGenerator != RS_SG_PCG32) return fail(RS_INVALID_ARG, "unknown sampleGenerator");
    if (o->misHeuristic > 2) return fail(RS_INVALID_ARG, "misHeuristic must be Balance, PowerTwo or PowerExp");
    if (o->emissiveSampler != RS_EMISSIVE_UNIFORM && o->emissiveSampler != RS_EMISSIVE_POWER)
        return fail(RS_INVALID_ARG, "emissiveSampler must be Uniform or Power (the LightBVH sampler is not built)");
    if (o->misHeuristic == RS_MIS_HEURISTIC_POWER_EXP && !(o->misPowerExponent >= 0.01f && o->misPowerExponent <= 10.f))
        return fail(RS_INVALID_ARG, "misPowerExponent must be in [0.01, 10]");
    if (o->temporalReuse > 3) return fail(RS_INVALID_ARG, "unknown temporalReuse");
    if (o->gatherOption > 2) return fail(RS_INVALID_ARG, "unknown gatherOption");
    if (o->scatterBackupMISOption > 1) return fail(RS_INVALID_ARG, "unknown scatterBackupMISOption");
    if (o->numTimePartitions < 1 || o->numTimePartitions > 8) return fail(RS_INVALID_ARG, "numTimePartitions must be in [1, 8]");
    if (o->enableSpatialResampling && (o->neighborCount < 1 || o->numSpatialIterations < 1)) return fail(RS_INVALID_ARG, "spatial reuse needs neighborCount and numSpatialIterations >= 1");
    if (!(o->artificialFrameTime > 0.f)) return fail(RS_INVALID_ARG, "artificialFrameTime must be > 0");
    if (o->specularRoughnessThreshold < 0.f || o->specularRoughnessThreshold > 1.f) return fail(RS_INVALID_ARG, "specularRoughnessThreshold must be in [0, 1]");
    return RS_OK;
}

static rs_status allocate(rs_pass* p)
{
    const size_t N = (size_t)p->opt.frameWidth * p->opt.frameHeight;
    const size_t P = p->opt.temporalReuse == RS_MULTI_SCATTER ? p->opt.numTimePartitions : 1;
    p->W = p->opt.frameWidth; p->H = p->opt.frameHeight;
    for (auto& s : p->sets) RS_CUDA(s.ensure(N));
    const bool needInter = p->opt.temporalReuse == RS_GATHER_ONLY || p->opt.temporalReuse == RS_SCATTER_BACKUP;
    if (needInter) RS_CUDA(p->inter.ensure(N));
    RS_CUDA(p->mvec.ensure(N));
    RS_CUDA(p->floatingCoords.ensure(N));
    RS_CUDA(p->vbuffer.ensure(N));
    RS_CUDA(p->targets.ensure(P * N));
    RS_CUDA(p->counts.ensure(P * N));
    RS_CUDA(p->offsets.ensure(P * N));
    RS_CUDA(p->unsortedSplats.ensure(P * N));
    RS_CUDA(p->sortedSplats.ensure(P * N));
    RS_CUDA(p->sortedCell.ensure(P * N));
    if (p->opt.temporalReuse == RS_SCATTER_ONLY)
    {
        RS_CUDA(p->m2curr.ensure(N));
        RS_CUDA(p->splatShift.ensure(5 * N)); RS_CUDA(p->splatTerms.ensure(N)); RS_CUDA(p->splatM.ensure(N));
    }
    if (p->opt.temporalReuse == RS_GATHER_ONLY)
    {
        RS_CUDA(p->m2curr.ensure(N));
        RS_CUDA(p->backupShift.ensure(5 * N)); RS_CUDA(p->backupTerms.ensure(N)); RS_CUDA(p->backupM.ensure(N));
    }
    if (p->opt.temporalReuse == RS_SCATTER_BACKUP)
    {
        RS_CUDA(p->m2curr.ensure(N)); RS_CUDA(p->m3curr.ensure(N));
        RS_CUDA(p->backupShift.ensure(5 * N)); RS_CUDA(p->backupTerms.ensure(N)); RS_CUDA(p->backupM.ensure(N));
        RS_CUDA(p->splatShift.ensure(5 * N)); RS_CUDA(p->splatTerms.ensure(N)); RS_CUDA(p->splatM.ensure(N));
    }
    if (p->opt.temporalReuse == RS_MULTI_SCATTER)
    {
        RS_CUDA(p->msCurr.ensure(N));
        RS_CUDA(p->msShift.ensure(5 * P * N)); RS_CUDA(p->msTerms.ensure(P * N)); RS_CUDA(p->msMisSub.ensure(P * N));
    }
    if (p->opt.enableSpatialResampling)
    {
        const size_t M = (size_t)p->opt.neighborCount * N;
        RS_CUDA(p->spM1.ensure(M)); RS_CUDA(p->spNw.ensure(M)); RS_CUDA(p->spShift.ensure(5 * M)); RS_CUDA(p->spTerms.ensure(M));
    }
    RS_CUDA(p->tileSums.ensure((N + kScanTileElems - 1) / kScanTileElems + 1));
    RS_CUDA(p->radixScratch.ensure(radix_scratch_words((uint32_t)N, bit_length(N))));
    RS_CUDA(p->total.ensure(8));
    if (p->opt.gatherOption == RS_GATHER_ROBUST && needInter) RS_CUDA(p->shiftedPaths.ensure(8 * N));
    RS_CUDA(p->fault.ensure(1));
    RS_CUDA(p->camTable.ensure(1));
    if (!p->forkEv)
    {
        RS_CUDA(cudaEventCreateWithFlags(&p->forkEv, cudaEventDisableTiming));
        for (int i = 0; i < rs_pass::kSide; i++)
        {
            RS_CUDA(cudaStreamCreateWithFlags(&p->side[i], cudaStreamNonBlocking));
            RS_CUDA(cudaEventCreateWithFlags(&p->joinEv[i], cudaEventDisableTiming));
        }
    }
    if (!p->hostFault)
    {
        RS_CUDA(cudaMallocHost(&p->hostFault, 2 * sizeof(uint32_t)));
        p->hostFault[0] = p->hostFault[1] = 0u;
    }
    if (!p->hostCtx) RS_CUDA(cudaMallocHost(&p->hostCtx, sizeof(DevCtx)));
    if (!p->ringCtx)
    {
        RS_CUDA(cudaMallocHost(&p->ringCtx, sizeof(DevCtx) * rs_pass::kRing));
        for (auto& e : p->ringEv) RS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    if (!p->graphCtx) RS_CUDA(cudaMallocHost(&p->graphCtx, sizeof(DevCtx)));
    if (!p->neighborOffsets.p)
    {
        // createNeighborOffsetTexture (ReservoirSplatting.cpp:1072-1097), decoded as RG8Snorm
        const uint32_t sampleCount = 8192;
        std::vector<int8_t> off(sampleCount * 2);
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
            off[index++] = (int8_t)((u - 0.5f) * (float)R);
            off[index++] = (int8_t)((v - 0.5f) * (float)R);
        }
        std::vector<float2> dec(sampleCount);
        for (uint32_t i = 0; i < sampleCount; i++)
        {
            float a = (float)off[2 * i] / 127.f, b = (float)off[2 * i + 1] / 127.f;
            dec[i] = make_float2(a < -1.f ? -1.f : a, b < -1.f ? -1.f : b);
        }
        RS_CUDA(p->neighborOffsets.ensure(sampleCount));
        RS_CUDA(cudaMemcpy(p->neighborOffsets.p, dec.data(), sampleCount * sizeof(float2), cudaMemcpyHostToDevice));
    }
    return RS_OK;
}

extern "C" RS_API rs_status rs_create(const rs_options* opts, rs_pass** out)
{
    if (!out) return fail(RS_INVALID_ARG, "out is NULL");
    rs_status s = validate(opts);
    if (s != RS_OK) return s;
    std::unique_ptr<rs_pass> p(new rs_pass());
    p->slot = acquire_slot();
    if (p->slot >= kMaxPassSlots) return fail(RS_INVALID_ARG, "at most 64 passes can exist at once");
    p->opt = *opts;
    s = allocate(p.get());
    if (s != RS_OK) return s;
    RS_CUDA(p->envView.ensure(1));
    RS_CUDA(cudaMemcpy(p->envView.p, &p->envHost, sizeof(EnvMapView), cudaMemcpyHostToDevice));
    *out = p.release();
    return RS_OK;
}

extern "C" RS_API rs_status rs_destroy(rs_pass* p)
{
    if (!p) return fail(RS_INVALID_ARG, "pass is NULL");
    cudaDeviceSynchronize();
    delete p;
    return RS_OK;
}

extern "C" RS_API rs_status rs_set_options(rs_pass* p, const rs_options* opts)
{
    if (!p) return fail(RS_INVALID_ARG, "pass is NULL");
    rs_status s = validate(opts);
    if (s != RS_OK) return s;
    bool resized = opts->frameWidth != p->opt.frameWidth || opts->frameHeight != p->opt.frameHeight;
    p->opt = *opts;
    s = allocate(p);
    if (s != RS_OK) return s;
    if (resized) p->frameCount = 0;
    p->generation++;
    return RS_OK;
}

extern "C" RS_API rs_status rs_set_scene(rs_pass* p, const rs_scene_desc* sd)
{
    if (!p || !sd) return fail(RS_INVALID_ARG, "pass or scene is NULL");
    if (sd->numTriangles > 0 && (!sd->positions || !sd->materialIds)) return fail(RS_INVALID_ARG, "scene arrays are NULL");
    if (sd->numMaterials == 0 || !sd->materials) return fail(RS_INVALID_ARG, "scene has no materials");
    if (sd->numTriangles >= kMaxBvhTriangles) return fail(RS_INVALID_ARG, "too many triangles (limit 2^29)");
    static_assert(sizeof(rs_material) == sizeof(MaterialData), "material layout");
    if (!prepare_scene(sd->numTriangles, sd->positions, sd->materialIds, sd->numMaterials,
                       reinterpret_cast<const MaterialData*>(sd->materials), p->scene))
        return fail(RS_INVALID_ARG, "material id out of range");
    const uint32_t n = sd->numTriangles;
    RS_CUDA(cudaDeviceSynchronize());
    RS_CUDA(p->dTri.ensure(3ull * (n ? n : 1)));
    RS_CUDA(p->dMaterials.ensure(sd->numMaterials));
    RS_CUDA(p->dLights.ensure(p->scene.lights.size() ? p->scene.lights.size() : 1));
    RS_CUDA(p->dAlias.ensure(p->scene.alias.size() ? p->scene.alias.size() : 1));
    if (n) RS_CUDA(cudaMemcpy(p->dTri.p, p->scene.tri.data(), 48ull * n, cudaMemcpyHostToDevice));
    RS_CUDA(cudaMemcpy(p->dMaterials.p, p->scene.materials.data(), sizeof(MaterialData) * sd->numMaterials, cudaMemcpyHostToDevice));
    if (!p->scene.lights.empty())
    {
        RS_CUDA(cudaMemcpy(p->dLights.p, p->scene.lights.data(), sizeof(LightTriangle) * p->scene.lights.size(), cudaMemcpyHostToDevice));
        RS_CUDA(cudaMemcpy(p->dAlias.p, p->scene.alias.data(), sizeof(u2) * p->scene.alias.size(), cudaMemcpyHostToDevice));
    }
    cudaStream_t s;
    RS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaError_t e = build_wide_bvh(p->dTri.p, n, &p->bvh, s, p->bvhBuilder);
    cudaStreamDestroy(s);
    if (e != cudaSuccess) return fail(RS_CUDA_ERROR, std::string("BVH build: ") + cudaGetErrorString(e));
    p->hasScene = true;
    p->hostTriStale = false;
    p->geometryMoved = false;
    p->frameCount = 0; // setScene resets the frame count (ReservoirSplatting.cpp:380)
    p->generation++;
    return RS_OK;
}

static_assert(sizeof(rs_analytic_light) == sizeof(AnalyticLightDesc), "rs_analytic_light mirrors AnalyticLightDesc");

// The scene's analytic lights (Scene::getLight, used when Scene::useAnalyticLights): each is
// prepared on the host as Falcor's light classes derive LightData, then copied to the device.
extern "C" RS_API rs_status rs_set_analytic_lights(rs_pass* p, const rs_analytic_light* lights, uint32_t count)
{
    if (!p) return fail(RS_INVALID_ARG, "pass is NULL");
    if (count > 0 && !lights) return fail(RS_INVALID_ARG, "lights is NULL");
    std::vector<AnalyticLight> dev(count);
    for (uint32_t i = 0; i < count; i++)
    {
        AnalyticLightDesc d;
        memcpy(&d, &lights[i], sizeof(d));
        if (d.type > kLightSphere) return fail(RS_INVALID_ARG, "analytic light " + std::to_string(i) + ": unknown type");
        if (!prepare_analytic_light(d, dev[i]))
            return fail(RS_INVALID_ARG, "analytic light " + std::to_string(i) + ": zero direction or singular transform");
    }
    if (count > 0)
    {
        RS_CUDA(cudaDeviceSynchronize()); // frames in flight may still read the previous list
        RS_CUDA(p->dAnalytic.ensure(count));
        RS_CUDA(cudaMemcpy(p->dAnalytic.p, dev.data(), sizeof(AnalyticLight) * count, cudaMemcpyHostToDevice));
    }
    p->numAnalytic = count;
    p->generation++;
    return RS_OK;
}

extern "C" RS_API rs_status rs_set_env_map(rs_pass* p, const rs_env_map* m)
{
    if (!p) return fail(RS_INVALID_ARG, "pass is NULL");
    EnvMapView v = {};
    if (m && m->width > 0)
    {
        if (!m->texels || m->height == 0) return fail(RS_INVALID_ARG, "env map texels are NULL or its height is 0");
        if (m->width > 16384 || m->height > 16384) return fail(RS_INVALID_ARG, "env map larger than 16384 x 16384");
        if (!(m->intensity >= 0.f) || !std::isfinite(m->intensity)) return fail(RS_INVALID_ARG, "env map intensity must be finite and >= 0");
        for (int k = 0; k < 3; k++)
            if (!std::isfinite(m->tint[k]) || !std::isfinite(m->rotation[k])) return fail(RS_INVALID_ARG, "env map tint and rotation must be finite");
        const size_t texels = (size_t)m->width * m->height;
        RS_CUDA(cudaDeviceSynchronize());
        RS_CUDA(p->envTexels.ensure(4 * texels));
        RS_CUDA(p->envImportance.ensure(kEnvImportanceTexels));
        RS_CUDA(cudaMemcpy(p->envTexels.p, m->texels, 16 * texels, cudaMemcpyHostToDevice));
        v.texels = p->envTexels.p;
        v.importance = p->envImportance.p;
        v.w = m->width; v.h = m->height;
        v.present = m->intensity > 0.f ? 1u : 0u;
        env_transform(m->rotation, v.toWorld, v.toLocal);
        for (int k = 0; k < 3; k++) v.scale[k] = m->intensity * m->tint[k];
        // the importance map (EnvMapSampler::createImportanceMap), then its mips
        k_env_importance<<<kEnvImportanceDim * kEnvImportanceDim / 256, 256>>>(v, p->envImportance.p);
        for (uint32_t mip = 1; mip < kEnvImportanceMips; mip++)
        {
            const uint32_t d = kEnvImportanceDim >> mip;
            k_env_reduce<<<(d * d + 255) / 256, 256>>>(p->envImportance.p, mip);
        }
        RS_CUDA(cudaGetLastError());
        RS_CUDA(cudaDeviceSynchronize());
    }
    else RS_CUDA(cudaDeviceSynchronize());
    p->envHost = v;
    p->generation++;
    RS_CUDA(cudaMemcpy(p->envView.p, &p->envHost, sizeof(EnvMapView), cudaMemcpyHostToDevice));
    return RS_OK;
}

static CameraData to_camera(const rs_camera& c)
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

// Streams for n independent launch chains after the work queued on s: s itself and n - 1 side
// streams that wait for it.  With stage timing on, every chain runs on s in order.
static void fork_streams(rs_pass* p, cudaStream_t s, int n, cudaStream_t* out)
{
    out[0] = s;
    for (int i = 1; i < n; i++) out[i] = p->timing ? s : p->side[i - 1];
    if (p->timing || n < 2) return;
    cudaEventRecord(p->forkEv, s);
    for (int i = 1; i < n; i++) cudaStreamWaitEvent(p->side[i - 1], p->forkEv, 0);
}
// s waits for the side streams of fork_streams(p, s, n, ...).
static void join_streams(rs_pass* p, cudaStream_t s, int n)
{
    if (p->timing) return;
    for (int i = 1; i < n; i++)
    {
        cudaEventRecord(p->joinEv[i - 1], p->side[i - 1]);
        cudaStreamWaitEvent(s, p->joinEv[i - 1], 0);
    }
}

static void stage(rs_pass* p, const char* name, cudaStream_t s)
{
    if (!p->timing) return;
    size_t k = p->stageNames.size();
#ifdef RS_RAY_STATS
    // rays of the stage that ends here (stage timing runs every launch on s in order)
    unsigned long long r[2] = {0ull, 0ull};
    ray_stats_take(r, s);
    if (k > 0) { p->stageRays.push_back(r[0]); p->stageRays.push_back(r[1]); }
#endif
    p->stageNames.push_back(name);
    if (p->events.size() < k + 2)
    {
        while (p->events.size() < k + 2)
        {
            cudaEvent_t e;
            cudaEventCreate(&e);
            p->events.push_back(e);
        }
    }
    cudaEventRecord(p->events[k], s);
}

// beginFrame (ReservoirSplatting.cpp:1550-1646) and prepareCameraManager (:1359-1388): host-side
// frame state and the device context of the frame (written to p->hostCtx).
static void begin_frame(rs_pass* p, const rs_frame_desc* f)
{
    const rs_options& o = p->opt;
    p->seed = o.useFixedSeed ? o.fixedSeed : p->seed + 1;
    p->camera = to_camera(f->camera);
    uint32_t K = 1u + (uint32_t)ceilf(p->camera.shutterSpeed / o.artificialFrameTime) + 1u;
    if (K > kMaxCameraKeyframes) K = kMaxCameraKeyframes;
    bool keyframesChanged = K != p->prevK;
    p->prevK = K;
    p->K = K;
    p->frameShouldReset = f->sceneShouldReset != 0;
    p->cm.artificialFrameTime = o.artificialFrameTime;
    p->cm.keyframes = K;
    if (p->frameCount == 0 || p->frameShouldReset || keyframesChanged)
        for (uint32_t i = 0; i < K; i++) { p->cm.positions[i] = p->camera.posW; p->cm.targets[i] = p->camera.target; }
    else { p->cm.positions[p->frameCount % K] = p->camera.posW; p->cm.targets[p->frameCount % K] = p->camera.target; }

    DevCtx& C = *p->hostCtx;
    memset(&C, 0, sizeof(C));
    C.bvh.binNodes = p->bvh.binNodes;
    C.bvh.binRoot = p->bvh.binRoot;
    C.bvh.nodes = p->bvh.nodes;
    C.bvh.leafTri = p->bvh.leafTri;
    C.bvh.tri = p->dTri.p;
    C.prevTri = p->geometryMoved ? p->dPrevTri.p : p->dTri.p;
    C.bvh.numTris = (uint32_t)(p->scene.tri.size() / 3);
    C.materials = p->dMaterials.p;
    C.lights.tris = p->dLights.p;
    C.lights.aliasTable = p->dAlias.p;
    C.lights.count = (uint32_t)p->scene.lights.size();
    C.lights.invWeightsSum = p->scene.invWeightsSum;
    C.lights.sampler = p->opt.emissiveSampler;
    C.env = p->envView.p;
    C.analytic.lights = p->dAnalytic.p;
    C.analytic.count = p->numAnalytic;
    light_type_probabilities(p->envHost.present != 0, C.lights.count > 0, p->numAnalytic > 0, C.pEnvLight, C.pEmissiveLight, C.pAnalyticLight);
    C.camera = p->camera;
    C.prevCamera = p->havePrevCamera ? p->prevCamera : p->camera;
    C.cm = p->cm;
    C.camTable = p->camTable.p;
    C.W = p->W; C.H = p->H;
    C.frameCount = p->frameCount; C.seed = p->seed;
    C.useFixedSeed = o.useFixedSeed; C.fixedSeed = o.fixedSeed;
    C.sgKind = o.sampleGenerator;
    C.spp = o.samplesPerPixel;
    C.maxSurfaceBounces = o.maxSurfaceBounces; C.maxDiffuseBounces = o.maxDiffuseBounces;
    C.maxSpecularBounces = o.maxSpecularBounces; C.maxTransmissionBounces = o.maxTransmissionBounces;
    C.useRussianRoulette = o.useRussianRoulette; C.misHeuristic = o.misHeuristic; C.disableCaustics = o.disableCaustics;
    C.misPowerExponent = o.misPowerExponent;
    C.specularRoughnessThreshold = o.specularRoughnessThreshold;
    C.useConfTemporal = o.useConfidenceWeightsTemporally; C.useConfSpatial = o.useConfidenceWeightsSpatially;
    C.gatherOption = o.gatherOption; C.scatterBackupMIS = o.scatterBackupMISOption; C.numTimePartitions = o.numTimePartitions;
    C.neighborCount = o.neighborCount; C.spatialGatherRadius = o.spatialGatherRadius;
    C.fault = p->fault.p;
    p->haveFrameCtx = true;
}

// The spatial ping-pong of spatialResampling (ReservoirSplatting.cpp:2002-2018) on the host-side indices.
static void apply_spatial_swaps(rs_pass* p)
{
    if (!p->opt.enableSpatialResampling) return;
    int& swapIdx = p->frozen ? p->tempIdx : p->prevIdx;
    for (uint32_t i = 0; i < p->opt.numSpatialIterations; i++) std::swap(p->currIdx, swapIdx);
}

// endFrame (ReservoirSplatting.cpp:1648-1680)
static void end_frame(rs_pass* p)
{
    apply_spatial_swaps(p);
    p->swapped = !p->frozen;
    if (!p->frozen)
    {
        p->frameCount++;
        std::swap(p->currIdx, p->prevIdx);
    }
    p->prevCamera = p->camera;
    p->havePrevCamera = true;
    p->geometryMoved = false;
}

// Launches the variant of an env-dependent kernel for a pass with (env) or without an environment
// light; the one without carries no env branches.
#define RS_ENV_LAUNCH(env, kernel, grid, block, stream, ...) launch_##kernel(env, grid, block, stream, __VA_ARGS__)

// Issues the frame's device work on `s`.  The frame context goes to the pass's constant-memory
// slot by a stream-ordered copy from pinned memory: in graph mode from p->graphCtx (a replayed graph
// reads the context current at replay time), otherwise from a ring entry that is not reused until
// its copy has run.
static rs_status enqueue_frame(rs_pass* p, cudaStream_t s, float4* colorDev, const float2* mvecIn, const uint4* vbufIn, bool graphMode)
{
    const bool env = p->envHost.present != 0; // which variant of the env-dependent kernels runs
    const uint32_t W = p->W, H = p->H;
    const uint32_t N = W * H;
    const rs_options& o = p->opt;
    if (graphMode)
    {
        RS_CUDA(upload_ctx(p->slot, p->graphCtx, s));
    }
    else
    {
        const int k = p->ringNext;
        p->ringNext = (k + 1) % rs_pass::kRing;
        RS_CUDA(cudaEventSynchronize(p->ringEv[k])); // the copy issued kRing frames ago has run
        p->ringCtx[k] = *p->hostCtx;
        RS_CUDA(upload_ctx(p->slot, &p->ringCtx[k], s));
        RS_CUDA(cudaEventRecord(p->ringEv[k], s));
    }
    const uint32_t C = p->slot;
    bool shouldReset = p->frameShouldReset;
    ReservoirSet& curr = p->sets[p->currIdx];
    ReservoirSet& prev = p->sets[p->prevIdx];
    auto grid = [](uint32_t n, uint32_t b) { return dim3((n + b - 1) / b); };
    RS_CUDA(cudaMemsetAsync(p->fault.p, 0, sizeof(uint32_t), s));
    k_camera_table<<<1, kMaxCameraKeyframes, 0, s>>>(C, p->camTable.p); p->launches++;

    // the caller's motion vectors and primary hits (the pass's mvec / vbuffer inputs) replace the
    // pass's own; k_vbuffer computes whichever of the two is missing
    const float2* mvec = mvecIn ? mvecIn : p->mvec.p;
    const uint4* vbuf = vbufIn ? vbufIn : p->vbuffer.p;
    if (p->keepCandidates) RS_CUDA(p->cand.ensure(N));
    shouldReset = shouldReset || p->frameCount == 0;
    const bool temporal = o.enableTemporalResampling && !shouldReset;
    const bool spatial = o.enableSpatialResampling != 0;
    bool colorWritten = false;
    p->lastFusedCollect = false;
    const uint32_t numTiles = (N + kScanTileElems - 1) / kScanTileElems;

    // Cell lists of one partition: offsets = exclusive scan of the counts; the splats in (cell,
    // source) order = a stable radix sort of the source indices by target (an invalid target sorts
    // last), so the work per splat is bounded however many splats share a cell.
    auto buildCells = [&](cudaStream_t q, const uint32_t* tg, uint32_t* cn, uint32_t* of, uint32_t* un, uint32_t* so, uint32_t* sc,
                          uint32_t* tot) -> cudaError_t {
        k_scan_tiles<<<numTiles, 1024, 0, q>>>(cn, of, p->tileSums.p, N);
        k_scan_tile_sums<<<1, 1024, 0, q>>>(p->tileSums.p, numTiles, tot);
        k_scan_add<<<grid(N, 256), 256, 0, q>>>(of, p->tileSums.p, N);
        cudaError_t e = radix_sort_indices_u32(tg, N, N, bit_length(N), so, un, p->radixScratch.p, q);
        k_sorted_cells<<<grid(N, 256), 256, 0, q>>>(tg, so, sc, N);
        p->launches += 4 + radix_sort_launches(N, bit_length(N));
        return e;
    };

    // Three independent chains: the primary hits and motion vectors (VBufferRT); the candidate path
    // tracer (current reservoirs); and the temporal work that reads only the previous frame (robust
    // neighbour shifts, reprojection of the previous samples and their cell lists).  They join
    // before the first kernel that reads two of them.
    cudaStream_t q[3];
    fork_streams(p, s, 3, q);
    if (!(mvecIn && vbufIn))
    {
        stage(p, "vbuffer", q[0]);
        k_vbuffer<<<tiled_blocks(W, H, 256), 256, 0, q[0]>>>(C, p->vbuffer.p, p->mvec.p); p->launches++;
    }
    stage(p, "initialCandidates", q[1]);
    // the path tracer's light configuration: env map, analytic lights, uniform emissive sampler
    const uint32_t lights = (env ? 1u : 0u) | (p->numAnalytic > 0 ? 2u : 0u) | (o.emissiveSampler == RS_EMISSIVE_UNIFORM ? 4u : 0u);
    if (o.samplesPerPixel == 1) launch_k_candidates_direct(lights, tiled_blocks(W, H, 128), 128, q[1], C, curr.res(), curr.recp());
    else launch_k_candidates(lights, grid(N, 128), 128, q[1], C, curr.res(), curr.recp());
    p->launches++;
    if (p->keepCandidates)
    {
        RS_CUDA(cudaMemcpyAsync(p->cand.a.p, curr.a.p, N * 16ull, cudaMemcpyDeviceToDevice, q[1]));
        RS_CUDA(cudaMemcpyAsync(p->cand.b.p, curr.b.p, N * 16ull, cudaMemcpyDeviceToDevice, q[1]));
        RS_CUDA(cudaMemcpyAsync(p->cand.rec.p, curr.rec.p, 7ull * N * 16ull, cudaMemcpyDeviceToDevice, q[1]));
    }
    if (temporal)
    {
        const bool robust = o.gatherOption == RS_GATHER_ROBUST && (o.temporalReuse == RS_GATHER_ONLY || o.temporalReuse == RS_SCATTER_BACKUP);
        if (robust)
        {
            stage(p, "robustReuse", q[2]);
            RS_ENV_LAUNCH(env, k_robust, dim3(tiled_blocks(W, H, 128), 8), 128, q[2], C, prev.res(), prev.recp(), p->shiftedPaths.p); p->launches++;
        }
        if (o.temporalReuse == RS_SCATTER_ONLY || o.temporalReuse == RS_SCATTER_BACKUP)
        {
            stage(p, "reproject", q[2]);
            RS_CUDA(cudaMemsetAsync(p->counts.p, 0, N * 4ull, q[2]));
            k_reproject<<<tiled_blocks(W, H, 256), 256, 0, q[2]>>>(C, prev.res(), prev.recp(), p->targets.p, p->counts.p); p->launches++;
            stage(p, "sortCells", q[2]);
            RS_CUDA(buildCells(q[2], p->targets.p, p->counts.p, p->offsets.p, p->unsortedSplats.p, p->sortedSplats.p,
                               p->sortedCell.p, p->total.p));
        }
        else if (o.temporalReuse == RS_MULTI_SCATTER)
        {
            const uint32_t P = o.numTimePartitions;
            stage(p, "multiReproject", q[2]);
            RS_CUDA(cudaMemsetAsync(p->counts.p, 0, (size_t)P * N * 4ull, q[2]));
            k_multi_reproject<<<tiled_blocks(W, H, 256), 256, 0, q[2]>>>(C, prev.res(), prev.recp(), p->targets.p, p->counts.p); p->launches++;
            stage(p, "multiSortCells", q[2]);
            for (uint32_t j = 0; j < P; j++)
            {
                size_t b = (size_t)j * N;
                RS_CUDA(buildCells(q[2], p->targets.p + b, p->counts.p + b, p->offsets.p + b, p->unsortedSplats.p + b,
                                   p->sortedSplats.p + b, p->sortedCell.p + b, p->total.p + j));
            }
        }
    }
    join_streams(p, s, 3);

    float4* temporalColor = spatial ? nullptr : colorDev;
    if (temporal)
    {
        switch (o.temporalReuse)
        {
        case RS_GATHER_ONLY:
            stage(p, "collect", s);
            k_collect<<<tiled_blocks(W, H, 128), 128, 0, s>>>(C, mvec, prev.res(), prev.recp(), p->inter.res(), p->inter.recp(), p->floatingCoords.p, p->shiftedPaths.p); p->launches++;
            if (!(p->camera.apertureRadius > 0.f))
            {
                // without depth of field only the lens-copy stage runs: two shift kernels on two
                // streams, then the combine (k_go_*)
                WaveCtx K = {};
                K.curr = curr.res(); K.currRec = curr.recp();
                K.inter = p->inter.res(); K.interRec = p->inter.recp();
                K.floatingCoords = p->floatingCoords.p;
                K.m2curr = p->m2curr.p;
                K.backupShift = ShiftPlanes{p->backupShift.p, (size_t)N}; K.backupTerms = p->backupTerms.p; K.backupM = p->backupM.p;
                cudaStream_t q[2];
                fork_streams(p, s, 2, q);
                stage(p, "gatherCurrShift", q[0]);
                RS_ENV_LAUNCH(env, k_go_curr, tiled_blocks(W, H, 128), 128, q[0], C, K);
                stage(p, "gatherPrevShift", q[1]);
                RS_ENV_LAUNCH(env, k_go_prev, tiled_blocks(W, H, 128), 128, q[1], C, K);
                join_streams(p, s, 2);
                stage(p, "gatherResample", s);
                k_go_combine<<<tiled_blocks(W, H, 128), 128, 0, s>>>(C, K, temporalColor);
                p->launches += 3;
                break;
            }
            stage(p, "gatherResample", s);
            RS_ENV_LAUNCH(env, k_gather_resample, tiled_blocks(W, H, 128), 128, s, C, vbuf, curr.res(), curr.recp(), p->inter.res(), p->inter.recp(), p->floatingCoords.p, temporalColor); p->launches++;
            break;
        case RS_SCATTER_ONLY:
        {
            // the current sample's shift and the splats' shifts on two streams, then the combine
            WaveCtx K = {};
            K.mvec = mvec;
            K.curr = curr.res(); K.currRec = curr.recp();
            K.prev = prev.res(); K.prevRec = prev.recp();
            K.counts = p->counts.p; K.offsets = p->offsets.p; K.sorted = p->sortedSplats.p; K.sortedCell = p->sortedCell.p;
            K.totalSplats = p->total.p;
            K.m2curr = p->m2curr.p;
            K.splatShift = ShiftPlanes{p->splatShift.p, (size_t)N}; K.splatTerms = p->splatTerms.p; K.splatM = p->splatM.p;
            cudaStream_t q[2];
            fork_streams(p, s, 2, q);
            stage(p, "scatterCurrShift", q[0]);
            RS_ENV_LAUNCH(env, k_so_curr, tiled_blocks(W, H, 128), 128, q[0], C, K);
            stage(p, "scatterSplatShift", q[1]);
            RS_ENV_LAUNCH(env, k_so_splat, grid(N, 128), 128, q[1], C, K);
            join_streams(p, s, 2);
            stage(p, "scatterResample", s);
            k_so_combine<<<tiled_blocks(W, H, 128), 128, 0, s>>>(C, K, temporalColor);
            p->launches += 3;
            break;
        }
        case RS_SCATTER_BACKUP:
        {
            const bool fused = o.gatherOption == RS_GATHER_CLAMPED;
            p->lastFusedCollect = fused;
            if (!fused)
            {
                stage(p, "collect", s);
                k_collect<<<tiled_blocks(W, H, 128), 128, 0, s>>>(C, mvec, prev.res(), prev.recp(), p->inter.res(), p->inter.recp(), p->floatingCoords.p, p->shiftedPaths.p); p->launches++;
            }
            WaveCtx K;
            K.fused = fused;
            K.mvec = mvec;
            K.curr = curr.res(); K.currRec = curr.recp();
            K.prev = prev.res(); K.prevRec = prev.recp();
            K.inter = fused ? prev.res() : p->inter.res(); K.interRec = fused ? prev.recp() : p->inter.recp();
            K.floatingCoords = p->floatingCoords.p;
            K.counts = p->counts.p; K.offsets = p->offsets.p; K.sorted = p->sortedSplats.p; K.sortedCell = p->sortedCell.p;
            K.totalSplats = p->total.p;
            K.m2curr = p->m2curr.p; K.m3curr = p->m3curr.p;
            K.backupShift = ShiftPlanes{p->backupShift.p, (size_t)N}; K.backupTerms = p->backupTerms.p; K.backupM = p->backupM.p;
            K.splatShift = ShiftPlanes{p->splatShift.p, (size_t)N}; K.splatTerms = p->splatTerms.p; K.splatM = p->splatM.p;
            const bool balance = o.scatterBackupMISOption == RS_MIS_BALANCE;
            // four independent chains: current -> previous by scatter and by gather, backup
            // gather (-> scatter), splat scatter (-> gather); the combine reads all of them
            cudaStream_t q[4];
            fork_streams(p, s, 4, q);
            stage(p, "sbCurrScatter", q[0]);
            RS_ENV_LAUNCH(env, k_sb_curr_scatter, tiled_blocks(W, H, 128), 128, q[0], C, K);
            stage(p, "sbCurrGather", q[1]);
            RS_ENV_LAUNCH(env, k_sb_curr_gather, tiled_blocks(W, H, 128), 128, q[1], C, K);
            stage(p, "sbBackupGather", q[2]);
            RS_ENV_LAUNCH(env, k_sb_backup_gather, tiled_blocks(W, H, 128), 128, q[2], C, K);
            stage(p, "sbSplatScatter", q[3]);
            RS_ENV_LAUNCH(env, k_sb_splat_scatter, grid(N, 128), 128, q[3], C, K);
            p->launches += 4;
            if (balance)
            {
                stage(p, "sbBackupScatter", q[2]);
                RS_ENV_LAUNCH(env, k_sb_backup_scatter, tiled_blocks(W, H, 128), 128, q[2], C, K);
                stage(p, "sbSplatGather", q[3]);
                RS_ENV_LAUNCH(env, k_sb_splat_gather, grid(N, 128), 128, q[3], C, K);
                p->launches += 2;
            }
            join_streams(p, s, 4);
            stage(p, "sbCombine", s);
            k_sb_combine<<<tiled_blocks(W, H, 128), 128, 0, s>>>(C, K, temporalColor);
            p->launches++;
            break;
        }
        case RS_MULTI_SCATTER:
        {
            const uint32_t P = o.numTimePartitions;
            MultiCtx M;
            M.mvec = mvec; M.curr = curr.res(); M.currRec = curr.recp(); M.prev = prev.res(); M.prevRec = prev.recp();
            M.counts = p->counts.p; M.offsets = p->offsets.p; M.sorted = p->sortedSplats.p; M.sortedCell = p->sortedCell.p;
            M.totals = p->total.p; M.currMIS = p->msCurr.p;
            M.shift = ShiftPlanes{p->msShift.p, (size_t)P * N}; M.terms = p->msTerms.p; M.misSub = p->msMisSub.p;
            // the current sample's shifts and the splats' shifts on two streams, then the combine
            cudaStream_t q[2];
            fork_streams(p, s, 2, q);
            stage(p, "multiCurrShift", q[0]);
            RS_ENV_LAUNCH(env, k_ms_curr, tiled_blocks(W, H, 128), 128, q[0], C, M);
            stage(p, "multiSplatShift", q[1]);
            RS_ENV_LAUNCH(env, k_ms_splat, grid(P * N, 128), 128, q[1], C, M);
            join_streams(p, s, 2);
            stage(p, "multiScatterResample", s);
            k_ms_combine<<<tiled_blocks(W, H, 128), 128, 0, s>>>(C, M, temporalColor);
            p->launches += 3;
            break;
        }
        }
        colorWritten = !spatial;
    }
    if (spatial)
    {
        // spatialResampling (ReservoirSplatting.cpp:1994-2020): ping-pong with the prev (or, when
        // frozen, the temp) buffer
        // (on local indices: the host-side transition is apply_spatial_swaps, run for every frame
        // whether this function issued the work or a replayed graph did)
        int cur = p->currIdx, prv = p->prevIdx, tmp = p->tempIdx;
        int& swapIdx = p->frozen ? tmp : prv;
        for (uint32_t i = 0; i < o.numSpatialIterations; i++)
        {
            std::swap(cur, swapIdx);
            ReservoirSet& src = p->sets[swapIdx];
            ReservoirSet& dst = p->sets[cur];
            SpatialCtx S;
            S.iteration = i;
            S.vbuffer = vbuf;
            S.neighborOffsets = p->neighborOffsets.p;
            S.src = src.res(); S.srcRec = src.recp();
            S.dst = dst.res(); S.dstRec = dst.recp();
            S.m1 = p->spM1.p; S.nw = p->spNw.p; S.terms = p->spTerms.p;
            S.shift = ShiftPlanes{p->spShift.p, (size_t)N * o.neighborCount};
            const uint32_t M = N * o.neighborCount;
            cudaStream_t q[2];
            fork_streams(p, s, 2, q); // the two shift directions are independent
            stage(p, "spatialCentral", q[0]);
            RS_ENV_LAUNCH(env, k_sp_central, dim3(tiled_blocks(W, H, 128), o.neighborCount), 128, q[0], C, S);
            stage(p, "spatialNeighbor", q[1]);
            RS_ENV_LAUNCH(env, k_sp_neighbor, dim3(tiled_blocks(W, H, 128), o.neighborCount), 128, q[1], C, S);
            join_streams(p, s, 2);
            stage(p, "spatialCombine", s);
            k_sp_combine<<<tiled_blocks(W, H, 128), 128, 0, s>>>(C, S, i + 1 == o.numSpatialIterations ? colorDev : nullptr);
            p->launches += 2;
            p->launches++;
        }
        colorWritten = true;
    }
    if (!colorWritten)
    {
        stage(p, "resolve", s);
        k_resolve<<<grid(N, 256), 256, 0, s>>>(N, p->sets[p->currIdx].res(), colorDev); p->launches++;
    }
    stage(p, "end", s);
    RS_CUDA(cudaGetLastError());
    RS_CUDA(cudaMemcpyAsync(p->hostFault + p->faultSlot, p->fault.p, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    return RS_OK;
}

// Waits for the host copy in flight (pipelined host output), orders `s` after it, and reports the
// device status word of the frame it belongs to.
static rs_status wait_host_copy(rs_pass* p, cudaStream_t s)
{
    if (!p->copyPending) return RS_OK;
    p->copyPending = false;
    RS_CUDA(cudaEventSynchronize(p->copyDoneEv));
    RS_CUDA(cudaStreamWaitEvent(s, p->copyDoneEv, 0));
    if (p->hostFault[p->pendingFaultSlot]) return fail(RS_DEVICE_FAULT, "device status word set: BVH traversal stack overflow");
    return RS_OK;
}

// rs_execute with a host colour output and one frame of latency: the frame renders into one of two
// device images, an event on `s` lets copyStream copy that image to f->colorHost, and the call
// returns once the previous frame's copy has finished (so that copy overlapped this frame's
// kernels), reporting that frame's device status.  f->color, when given too, gets a device copy.
static rs_status execute_pipelined(rs_pass* p, const rs_frame_desc* f, cudaStream_t s, size_t N)
{
    if (!p->copyStream)
    {
        RS_CUDA(cudaStreamCreateWithFlags(&p->copyStream, cudaStreamNonBlocking));
        RS_CUDA(cudaEventCreateWithFlags(&p->frameDoneEv, cudaEventDisableTiming));
        RS_CUDA(cudaEventCreateWithFlags(&p->copyDoneEv, cudaEventDisableTiming));
    }
    if (p->pipeColor[0].n < N || p->pipeColor[1].n < N)
    {
        rs_status w = wait_host_copy(p, s); // the images are about to be reallocated
        if (w != RS_OK) return w;
        RS_CUDA(p->pipeColor[0].ensure(N));
        RS_CUDA(p->pipeColor[1].ensure(N));
    }
    // the image written two frames ago was copied before the previous call returned
    p->pipeIdx ^= 1;
    float4* colorDev = p->pipeColor[p->pipeIdx].p;
    p->faultSlot ^= 1u;
    begin_frame(p, f);
    rs_status st = enqueue_frame(p, s, colorDev, reinterpret_cast<const float2*>(f->mvec), reinterpret_cast<const uint4*>(f->vbuffer), false);
    if (st != RS_OK) return st;
    if (f->color) RS_CUDA(cudaMemcpyAsync(f->color, colorDev, N * 16ull, cudaMemcpyDeviceToDevice, s));
    RS_CUDA(cudaEventRecord(p->frameDoneEv, s));
    RS_CUDA(cudaStreamWaitEvent(p->copyStream, p->frameDoneEv, 0));
    RS_CUDA(cudaMemcpyAsync(f->colorHost, colorDev, N * 16ull, cudaMemcpyDeviceToHost, p->copyStream));
    end_frame(p);
    rs_status w = wait_host_copy(p, s); // the previous frame's copy
    RS_CUDA(cudaEventRecord(p->copyDoneEv, p->copyStream));
    p->copyPending = true;
    p->pendingFaultSlot = p->faultSlot;
    return w;
}

extern "C" RS_API rs_status rs_execute(rs_pass* p, const rs_frame_desc* f, void* streamPtr)
{
    if (!p || !f) return fail(RS_INVALID_ARG, "pass or frame is NULL");
    if (!p->hasScene) return fail(RS_NOT_READY, "no scene set");
    if (!f->color && !f->colorHost) return fail(RS_INVALID_ARG, "no colour output");
    cudaStream_t s = (cudaStream_t)streamPtr;
    p->lastStream = s;
    p->launches = 0;
    p->stageNames.clear();
#ifdef RS_RAY_STATS
    p->stageRays.clear();
#endif
    const size_t N = (size_t)p->W * p->H;
    if (f->colorHost && p->hostLatency == 1) return execute_pipelined(p, f, s, N);
    p->faultSlot = 0;
    float4* colorDev = reinterpret_cast<float4*>(f->color);
    if (!colorDev)
    {
        RS_CUDA(p->scratchColor.ensure(N)); // allocated on the first host-output frame only
        colorDev = p->scratchColor.p;
    }
    if (p->copyPending) { rs_status w = wait_host_copy(p, s); if (w != RS_OK) return w; }
    begin_frame(p, f);
    rs_status st = enqueue_frame(p, s, colorDev, reinterpret_cast<const float2*>(f->mvec), reinterpret_cast<const uint4*>(f->vbuffer), false);
    if (st != RS_OK) return st;
    if (f->colorHost)
    {
        RS_CUDA(cudaMemcpyAsync(f->colorHost, colorDev, N * 16ull, cudaMemcpyDeviceToHost, s));
        RS_CUDA(cudaStreamSynchronize(s));
    }
    end_frame(p);
    if (f->colorHost && *p->hostFault) return fail(RS_DEVICE_FAULT, "device status word set: BVH traversal stack overflow");
    return RS_OK;
}

// Host colour outputs with 0 (default: rs_execute returns with the image on the host) or 1 frame of
// latency (the copy overlaps the next frame; rs_wait_host_output completes the last one).
extern "C" RS_API rs_status rs_set_host_output_latency(rs_pass* p, uint32_t frames)
{
    if (!p) return fail(RS_INVALID_ARG, "pass is NULL");
    if (frames > 1) return fail(RS_INVALID_ARG, "host output latency must be 0 or 1 frames");
    if (frames == 0 && p->copyPending) { rs_status w = wait_host_copy(p, p->lastStream); if (w != RS_OK) return w; }
    p->hostLatency = frames;
    return RS_OK;
}

extern "C" RS_API rs_status rs_wait_host_output(rs_pass* p)
{
    if (!p) return fail(RS_INVALID_ARG, "pass is NULL");
    return wait_host_copy(p, p->lastStream);
}

// reset() (ReservoirSplatting.cpp:813-820): frame count and seed restart unless the scene is frozen.
extern "C" RS_API rs_status rs_reset(rs_pass* p)
{
    if (!p) return fail(RS_INVALID_ARG, "pass is NULL");
    if (!p->frozen)
    {
        p->frameCount = 0;
        p->seed = 0;
    }
    return RS_OK;
}

extern "C" RS_API rs_status rs_set_seed(rs_pass* p, uint32_t useFixedSeed, uint32_t fixedSeed)
{
    if (!p) return fail(RS_INVALID_ARG, "pass is NULL");
    p->opt.useFixedSeed = useFixedSeed ? 1u : 0u;
    p->opt.fixedSeed = fixedSeed;
    return RS_OK;
}

extern "C" RS_API rs_status rs_freeze(rs_pass* p, uint32_t frozen)
{
    if (!p) return fail(RS_INVALID_ARG, "pass is NULL");
    p->frozen = frozen != 0;
    return RS_OK;
}

// ------------------------------------------------------------------ buffer views
static rs_status copy_out(rs_pass* p, const void* src, size_t need, void* dst, size_t* bytes)
{
    if (!dst) { *bytes = need; return RS_OK; }
    if (*bytes < need) { *bytes = need; return fail(RS_INVALID_ARG, "destination too small"); }
    RS_CUDA(cudaStreamSynchronize(p->lastStream));
    RS_CUDA(cudaMemcpy(dst, src, need, cudaMemcpyDeviceToHost));
    *bytes = need;
    return RS_OK;
}

static rs_status export_res(rs_pass* p, const ReservoirSet& s, void* dst, size_t* bytes)
{
    const size_t N = (size_t)p->W * p->H;
    if (!dst) { *bytes = N * 32; return RS_OK; }
    if (*bytes < N * 32) { *bytes = N * 32; return fail(RS_INVALID_ARG, "destination too small"); }
    std::vector<float4> a(N), b(N);
    RS_CUDA(cudaStreamSynchronize(p->lastStream));
    RS_CUDA(cudaMemcpy(a.data(), s.a.p, N * 16, cudaMemcpyDeviceToHost));
    RS_CUDA(cudaMemcpy(b.data(), s.b.p, N * 16, cudaMemcpyDeviceToHost));
    float* o = (float*)dst;
    for (size_t i = 0; i < N; i++)
    {
        o[8 * i + 0] = a[i].x; o[8 * i + 1] = a[i].y; o[8 * i + 2] = a[i].z; o[8 * i + 3] = a[i].w;
        o[8 * i + 4] = b[i].x; o[8 * i + 5] = b[i].y; o[8 * i + 6] = b[i].z; o[8 * i + 7] = 0.f;
    }
    *bytes = N * 32;
    return RS_OK;
}

static rs_status export_rec(rs_pass* p, const ReservoirSet& s, void* dst, size_t* bytes)
{
    const size_t N = (size_t)p->W * p->H;
    if (!dst) { *bytes = N * 112; return RS_OK; }
    if (*bytes < N * 112) { *bytes = N * 112; return fail(RS_INVALID_ARG, "destination too small"); }
    std::vector<uint4> planes(7 * N);
    RS_CUDA(cudaStreamSynchronize(p->lastStream));
    RS_CUDA(cudaMemcpy(planes.data(), s.rec.p, 7 * N * 16, cudaMemcpyDeviceToHost));
    uint32_t* o = (uint32_t*)dst;
    for (size_t i = 0; i < N; i++)
        for (int k = 0; k < 7; k++)
        {
            const uint4& q = planes[k * N + i];
            o[28 * i + 4 * k + 0] = q.x; o[28 * i + 4 * k + 1] = q.y; o[28 * i + 4 * k + 2] = q.z; o[28 * i + 4 * k + 3] = q.w;
        }
    *bytes = N * 112;
    return RS_OK;
}

extern "C" RS_API rs_status rs_get_buffer(rs_pass* p, rs_buffer_id id, void* dst, size_t* bytes)
{
    if (!p || !bytes) return fail(RS_INVALID_ARG, "pass or bytes is NULL");
    const size_t N = (size_t)p->W * p->H;
    const ReservoirSet& last = p->sets[p->swapped ? p->prevIdx : p->currIdx];
    const ReservoirSet& other = p->sets[p->swapped ? p->currIdx : p->prevIdx];
    switch (id)
    {
    case RS_BUF_CURR_RESERVOIRS: return export_res(p, last, dst, bytes);
    case RS_BUF_CURR_RECONNECTION: return export_rec(p, last, dst, bytes);
    case RS_BUF_PREV_RESERVOIRS: return export_res(p, other, dst, bytes);
    case RS_BUF_PREV_RECONNECTION: return export_rec(p, other, dst, bytes);
    case RS_BUF_CANDIDATE_RESERVOIRS:
        if (!p->cand.a.p) return fail(RS_INVALID_ARG, "candidate snapshots are off (keep-candidates option)");
        return export_res(p, p->cand, dst, bytes);
    case RS_BUF_CANDIDATE_RECONNECTION:
        if (!p->cand.a.p) return fail(RS_INVALID_ARG, "candidate snapshots are off (keep-candidates option)");
        return export_rec(p, p->cand, dst, bytes);
    case RS_BUF_BACKUP_RESERVOIRS:
        if (!p->inter.a.p || p->lastFusedCollect) return fail(RS_INVALID_ARG, "no backup buffer in this mode");
        return export_res(p, p->inter, dst, bytes);
    case RS_BUF_BACKUP_RECONNECTION:
        if (!p->inter.a.p || p->lastFusedCollect) return fail(RS_INVALID_ARG, "no backup buffer in this mode");
        return export_rec(p, p->inter, dst, bytes);
    case RS_BUF_CELL_COUNTERS: return copy_out(p, p->counts.p, N * 4, dst, bytes);
    case RS_BUF_CELL_OFFSETS: return copy_out(p, p->offsets.p, N * 4, dst, bytes);
    case RS_BUF_SPLAT_TARGETS: return copy_out(p, p->targets.p, N * 4, dst, bytes);
    case RS_BUF_SORTED_SPLATS:
    {
        uint32_t total = 0;
        RS_CUDA(cudaStreamSynchronize(p->lastStream));
        // the number of splats is the sum of the counts
        std::vector<uint32_t> c(N);
        RS_CUDA(cudaMemcpy(c.data(), p->counts.p, N * 4, cudaMemcpyDeviceToHost));
        for (uint32_t v : c) total += v;
        return copy_out(p, p->sortedSplats.p, (size_t)total * 4, dst, bytes);
    }
    case RS_BUF_FLOATING_COORDS: return copy_out(p, p->floatingCoords.p, N * 8, dst, bytes);
    case RS_BUF_MVEC: return copy_out(p, p->mvec.p, N * 8, dst, bytes);
    case RS_BUF_VBUFFER: return copy_out(p, p->vbuffer.p, N * 16, dst, bytes);
    case RS_BUF_ENV_IMPORTANCE:
        if (!p->envHost.importance) return fail(RS_NOT_READY, "no env map set");
        return copy_out(p, p->envImportance.p, kEnvImportanceTexels * 4ull, dst, bytes);
    default: return fail(RS_INVALID_ARG, "unknown buffer id");
    }
}

extern "C" RS_API rs_status rs_set_buffer(rs_pass* p, rs_buffer_id id, const void* src, size_t bytes)
{
    if (!p || !src) return fail(RS_INVALID_ARG, "pass or src is NULL");
    const size_t N = (size_t)p->W * p->H;
    bool curr = id == RS_BUF_CURR_RESERVOIRS || id == RS_BUF_CURR_RECONNECTION;
    ReservoirSet& s = p->sets[(curr == p->swapped) ? p->prevIdx : p->currIdx];
    RS_CUDA(cudaDeviceSynchronize());
    if (id == RS_BUF_CURR_RESERVOIRS || id == RS_BUF_PREV_RESERVOIRS)
    {
        if (bytes != N * 32) return fail(RS_INVALID_ARG, "reservoir buffer size mismatch");
        const float* in = (const float*)src;
        std::vector<float4> a(N), b(N);
        for (size_t i = 0; i < N; i++)
        {
            a[i] = make_float4(in[8 * i], in[8 * i + 1], in[8 * i + 2], in[8 * i + 3]);
            b[i] = make_float4(in[8 * i + 4], in[8 * i + 5], in[8 * i + 6], 0.f);
        }
        RS_CUDA(cudaMemcpy(s.a.p, a.data(), N * 16, cudaMemcpyHostToDevice));
        RS_CUDA(cudaMemcpy(s.b.p, b.data(), N * 16, cudaMemcpyHostToDevice));
        return RS_OK;
    }
    if (id == RS_BUF_CURR_RECONNECTION || id == RS_BUF_PREV_RECONNECTION)
    {
        if (bytes != N * 112) return fail(RS_INVALID_ARG, "reconnection buffer size mismatch");
        const uint32_t* in = (const uint32_t*)src;
        std::vector<uint4> planes(7 * N);
        for (size_t i = 0; i < N; i++)
            for (int k = 0; k < 7; k++)
                planes[k * N + i] = make_uint4(in[28 * i + 4 * k], in[28 * i + 4 * k + 1], in[28 * i + 4 * k + 2], in[28 * i + 4 * k + 3]);
        RS_CUDA(cudaMemcpy(s.rec.p, planes.data(), 7 * N * 16, cudaMemcpyHostToDevice));
        return RS_OK;
    }
    return fail(RS_INVALID_ARG, "buffer cannot be restored");
}

// ------------------------------------------------------------------ moving geometry
// Moves every triangle to `positions` (x, y, z of p0, p1, p2 per triangle; host memory, or device
// memory of the current device when onDevice is set) for the next frame (Falcor's animated scene
// update).  The previous positions serve that frame's motion vectors (Scene::getPrevPosW,
// VBufferRT.slang:84); reprojection and shifts read the new positions through the hit records
// (ReprojectTemporalSamples.rt.slang:104).  Both trees are refitted in place (same topology), and
// the light records take their triangles' new vertices with the flux of the last scene or material
// update.  Stream-ordered on `cudaStream`.
__global__ void k_set_positions(float4* __restrict__ tri, const float* __restrict__ pos, uint32_t n)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 3u * n) return;
    float4 q = tri[i];
    q.x = pos[3 * (size_t)i]; q.y = pos[3 * (size_t)i + 1]; q.z = pos[3 * (size_t)i + 2];
    tri[i] = q;
}

__global__ void k_update_lights(LightTriangle* __restrict__ lights, uint32_t count, const float4* __restrict__ tri)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    LightTriangle L = lights[i];
    const float4* q = tri + 3 * (size_t)L.sceneTri;
    light_set_vertices(L, mk3(q[0].x, q[0].y, q[0].z), mk3(q[1].x, q[1].y, q[1].z), mk3(q[2].x, q[2].y, q[2].z));
    lights[i] = L;
}

extern "C" RS_API rs_status rs_update_geometry(rs_pass* p, const float* positions, uint32_t numTriangles, uint32_t onDevice, void* streamPtr)
{
    if (!p || !positions) return fail(RS_INVALID_ARG, "pass or positions is NULL");
    if (!p->hasScene) return fail(RS_NOT_READY, "rs_update_geometry needs a scene");
    const uint32_t n = (uint32_t)(p->scene.tri.size() / 3);
    if (numTriangles != n) return fail(RS_INVALID_ARG, "triangle count differs from the scene's");
    if (n == 0) return RS_OK;
    cudaStream_t s = static_cast<cudaStream_t>(streamPtr);
    RS_CUDA(p->dPrevTri.ensure(3ull * n));
    const float* src = positions;
    if (!onDevice)
    {
        RS_CUDA(p->dPosStage.ensure(9ull * n));
        RS_CUDA(cudaMemcpyAsync(p->dPosStage.p, positions, 36ull * n, cudaMemcpyHostToDevice, s));
        src = p->dPosStage.p;
    }
    RS_CUDA(cudaMemcpyAsync(p->dPrevTri.p, p->dTri.p, 48ull * n, cudaMemcpyDeviceToDevice, s));
    k_set_positions<<<(3 * n + 255) / 256, 256, 0, s>>>(p->dTri.p, src, n);
    const uint32_t nl = (uint32_t)p->scene.lights.size();
    if (nl) k_update_lights<<<(nl + 127) / 128, 128, 0, s>>>(p->dLights.p, nl, p->dTri.p);
    RS_CUDA(cudaGetLastError());
    cudaError_t e = refit_wide_bvh(p->dTri.p, &p->bvh, s);
    if (e != cudaSuccess) return fail(RS_CUDA_ERROR, std::string("BVH refit: ") + cudaGetErrorString(e));
    p->hostTriStale = true; // rs_set_materials reads the positions back before it rebuilds the lights
    p->geometryMoved = true;
    p->lastStream = s;
    return RS_OK;
}

// ------------------------------------------------------------------ path-replay adjoint
// (no reference counterpart; the kernel and its estimator are described in adjoint.cuh)

// Replaces the material parameters in place.  The triangle records keep their positions, so the
// BVH stays; the light collection and its alias table are rebuilt for the new emission.
extern "C" RS_API rs_status rs_set_materials(rs_pass* p, const rs_material* materials, uint32_t count)
{
    if (!p || !materials) return fail(RS_INVALID_ARG, "pass or materials is NULL");
    if (!p->hasScene) return fail(RS_NOT_READY, "rs_set_materials needs a scene");
    if (count != p->scene.materials.size()) return fail(RS_INVALID_ARG, "material count differs from the scene's");
    const size_t n = p->scene.tri.size() / 3;
    if (p->hostTriStale && n)
    {
        RS_CUDA(cudaDeviceSynchronize());
        RS_CUDA(cudaMemcpy(p->scene.tri.data(), p->dTri.p, 48ull * n, cudaMemcpyDeviceToHost));
        p->hostTriStale = false;
    }
    std::vector<float> pos(9 * n);
    std::vector<uint32_t> ids(n);
    for (size_t t = 0; t < n; t++)
    {
        for (int v = 0; v < 3; v++)
        {
            const f4& q = p->scene.tri[3 * t + v];
            pos[9 * t + 3 * v + 0] = q.x; pos[9 * t + 3 * v + 1] = q.y; pos[9 * t + 3 * v + 2] = q.z;
        }
        ids[t] = f2u(p->scene.tri[3 * t].w);
    }
    PreparedScene ps;
    if (!prepare_scene((uint32_t)n, pos.data(), ids.data(), count, reinterpret_cast<const MaterialData*>(materials), ps))
        return fail(RS_INVALID_ARG, "material id out of range");
    RS_CUDA(cudaDeviceSynchronize());
    RS_CUDA(p->dLights.ensure(ps.lights.size() ? ps.lights.size() : 1));
    RS_CUDA(p->dAlias.ensure(ps.alias.size() ? ps.alias.size() : 1));
    if (n) RS_CUDA(cudaMemcpy(p->dTri.p, ps.tri.data(), 48ull * n, cudaMemcpyHostToDevice));
    RS_CUDA(cudaMemcpy(p->dMaterials.p, ps.materials.data(), sizeof(MaterialData) * count, cudaMemcpyHostToDevice));
    if (!ps.lights.empty())
    {
        RS_CUDA(cudaMemcpy(p->dLights.p, ps.lights.data(), sizeof(LightTriangle) * ps.lights.size(), cudaMemcpyHostToDevice));
        RS_CUDA(cudaMemcpy(p->dAlias.p, ps.alias.data(), sizeof(u2) * ps.alias.size(), cudaMemcpyHostToDevice));
    }
    p->scene = std::move(ps);
    return RS_OK;
}

extern "C" RS_API rs_status rs_checkpoint_bytes(rs_pass* p, size_t* bytes)
{
    if (!p || !bytes) return fail(RS_INVALID_ARG, "pass or bytes is NULL");
    *bytes = (size_t)p->W * p->H * 144ull;
    return RS_OK;
}

// Copies the last frame's final reservoirs into `dst` (device memory, rs_checkpoint_bytes):
// reservoir plane a, plane b, then the seven reconnection planes, N entries of 16 bytes each.
extern "C" RS_API rs_status rs_checkpoint(rs_pass* p, void* dst, void* streamPtr)
{
    if (!p || !dst) return fail(RS_INVALID_ARG, "pass or destination is NULL");
    if (!p->haveFrameCtx) return fail(RS_NOT_READY, "no frame has been rendered");
    cudaStream_t s = static_cast<cudaStream_t>(streamPtr);
    const size_t N = (size_t)p->W * p->H;
    const ReservoirSet& last = p->sets[p->swapped ? p->prevIdx : p->currIdx];
    char* d = static_cast<char*>(dst);
    RS_CUDA(cudaMemcpyAsync(d, last.a.p, N * 16, cudaMemcpyDeviceToDevice, s));
    RS_CUDA(cudaMemcpyAsync(d + N * 16, last.b.p, N * 16, cudaMemcpyDeviceToDevice, s));
    RS_CUDA(cudaMemcpyAsync(d + N * 32, last.rec.p, N * 112, cudaMemcpyDeviceToDevice, s));
    return RS_OK;
}

// Adds d loss / d material parameters to gradMaterials (device, numMaterials x 8 floats in the
// order baseColor.xyz, roughness, emissive.xyz, metallic; the metallic slot is not differentiated)
// for d loss / d colour `gradColor` (device float4 per pixel) of the frame whose reservoirs are in
// `checkpoint` (rs_checkpoint layout), or of the last frame when checkpoint is NULL.  The
// materials must be those the frame was rendered with.
extern "C" RS_API rs_status rs_backward(rs_pass* p, const void* checkpoint, const float* gradColor, float* gradMaterials, void* streamPtr)
{
    if (!p || !gradColor || !gradMaterials) return fail(RS_INVALID_ARG, "pass, gradColor or gradMaterials is NULL");
    if (!p->hasScene || !p->haveFrameCtx) return fail(RS_NOT_READY, "rs_backward needs a rendered frame");
    if (p->numAnalytic)
        return fail(RS_INVALID_ARG, "rs_backward differentiates scenes lit by emissive triangles and an env map; the pass has analytic lights");
    cudaStream_t s = static_cast<cudaStream_t>(streamPtr);
    const size_t N = (size_t)p->W * p->H;
    if (!p->adjStats.p)
    {
        RS_CUDA(p->adjStats.ensure(4));
        RS_CUDA(cudaMemset(p->adjStats.p, 0, 4 * sizeof(unsigned long long)));
    }
    ResPlanes res;
    RecPlanes rec;
    if (checkpoint)
    {
        char* c = const_cast<char*>(static_cast<const char*>(checkpoint));
        res = ResPlanes{reinterpret_cast<float4*>(c), reinterpret_cast<float4*>(c + N * 16)};
        rec = RecPlanes{reinterpret_cast<uint4*>(c + N * 32), N};
    }
    else
    {
        const ReservoirSet& last = p->sets[p->swapped ? p->prevIdx : p->currIdx];
        res = last.res();
        rec = last.recp();
    }
    const int k = p->ringNext;
    p->ringNext = (k + 1) % rs_pass::kRing;
    RS_CUDA(cudaEventSynchronize(p->ringEv[k]));
    p->ringCtx[k] = *p->hostCtx;
    RS_CUDA(upload_ctx(p->slot, &p->ringCtx[k], s));
    RS_CUDA(cudaEventRecord(p->ringEv[k], s));
    const uint32_t numMaterials = (uint32_t)p->scene.materials.size();
    const uint32_t M = numMaterials * kGradStride;
    RS_CUDA(p->adjAcc.ensure(M));
    RS_CUDA(cudaMemsetAsync(p->adjAcc.p, 0, M * sizeof(double), s));
    const size_t smem = M <= kAdjointSharedDoubles ? M * sizeof(double) : 0;
    const uint32_t blocks = (uint32_t)std::min<size_t>((N + kAdjointThreads - 1) / kAdjointThreads, 148ull * kAdjointBlocksPerSm);
    k_backward<<<blocks, kAdjointThreads, smem, s>>>(p->slot, res, rec, reinterpret_cast<const float4*>(gradColor), p->adjAcc.p,
                                                     numMaterials, p->adjStats.p);
    k_grad_flush<<<(M + 255) / 256, 256, 0, s>>>(p->adjAcc.p, gradMaterials, M);
    RS_CUDA(cudaGetLastError());
    p->lastStream = s;
    p->launches = 2;
    return RS_OK;
}

// Reads and clears the counters of rs_backward since the last read: paths replayed, paths longer
// than three vertices (skipped), paths whose emitter the replay could not identify (no emission
// gradient), replays that differ from the stored integrand by more than 1e-3 relative.
extern "C" RS_API rs_status rs_backward_stats(rs_pass* p, uint64_t* out)
{
    if (!p || !out) return fail(RS_INVALID_ARG, "pass or out is NULL");
    for (int i = 0; i < 4; i++) out[i] = 0;
    if (!p->adjStats.p) return RS_OK;
    unsigned long long h[4];
    RS_CUDA(cudaStreamSynchronize(p->lastStream));
    RS_CUDA(cudaMemcpy(h, p->adjStats.p, sizeof(h), cudaMemcpyDeviceToHost));
    RS_CUDA(cudaMemset(p->adjStats.p, 0, sizeof(h)));
    for (int i = 0; i < 4; i++) out[i] = h[i];
    return RS_OK;
}

// ------------------------------------------------------------------ ray-query diagnostics
// Closest hits of n host rays (8 floats each: origin, direction, tMin, tMax) against the pass's
// tree: prim (-1 on a miss), t/u/v, and per ray the nodes visited and triangles tested.
extern "C" RS_API rs_status rs_debug_trace_rays(rs_pass* p, const float* rays, uint32_t n, int32_t* prim, float* tuv, uint32_t* counts)
{
    if (!p || !rays || !prim || !tuv || !counts) return fail(RS_INVALID_ARG, "NULL argument");
    if (!p->hasScene) return fail(RS_NOT_READY, "no scene");
    if (n == 0) return RS_OK;
    DevBuf<float> dr;
    DevBuf<int32_t> dp;
    DevBuf<float> dt;
    DevBuf<uint32_t> dc, dof;
    RS_CUDA(dr.ensure(8ull * n)); RS_CUDA(dp.ensure(n)); RS_CUDA(dt.ensure(3ull * n)); RS_CUDA(dc.ensure(2ull * n)); RS_CUDA(dof.ensure(1));
    RS_CUDA(cudaMemcpy(dr.p, rays, 32ull * n, cudaMemcpyHostToDevice));
    RS_CUDA(cudaMemset(dof.p, 0, 4));
    BvhView bv;
    bv.binNodes = p->bvh.binNodes; bv.binRoot = p->bvh.binRoot; bv.nodes = p->bvh.nodes; bv.leafTri = p->bvh.leafTri;
    bv.tri = p->dTri.p; bv.numTris = (uint32_t)(p->scene.tri.size() / 3);
    k_debug_trace<<<(n + 127) / 128, 128>>>(bv, dr.p, n, dp.p, dt.p, dc.p, dof.p);
    RS_CUDA(cudaGetLastError());
    RS_CUDA(cudaDeviceSynchronize());
    uint32_t of = 0;
    RS_CUDA(cudaMemcpy(&of, dof.p, 4, cudaMemcpyDeviceToHost));
    if (of) return fail(RS_DEVICE_FAULT, "traversal stack overflow");
    RS_CUDA(cudaMemcpy(prim, dp.p, 4ull * n, cudaMemcpyDeviceToHost));
    RS_CUDA(cudaMemcpy(tuv, dt.p, 12ull * n, cudaMemcpyDeviceToHost));
    RS_CUDA(cudaMemcpy(counts, dc.p, 8ull * n, cudaMemcpyDeviceToHost));
    return RS_OK;
}

// The binary-tree builder of the next rs_set_scene: 0 = PLOC (default), 1 = LBVH (Karras radix tree).
extern "C" RS_API rs_status rs_set_bvh_builder(rs_pass* p, uint32_t builder)
{
    if (!p) return fail(RS_INVALID_ARG, "pass is NULL");
    if (builder > kBvhLbvh) return fail(RS_INVALID_ARG, "builder must be 0 (PLOC) or 1 (LBVH)");
    p->bvhBuilder = static_cast<BvhBuilder>(builder);
    return RS_OK;
}

// Shape of the pass's tree: {nodes, depth, internal children, leaf children, leaf triangles,
// surface-area cost per root-box ray (node visits + triangle tests)}.
extern "C" RS_API rs_status rs_debug_bvh_shape(rs_pass* p, double* out6)
{
    if (!p || !out6) return fail(RS_INVALID_ARG, "NULL argument");
    wide_bvh_shape(p->bvh, out6);
    return RS_OK;
}

extern "C" RS_API rs_status rs_enable_stage_timing(rs_pass* p, uint32_t enable)
{
    if (!p) return fail(RS_INVALID_ARG, "pass is NULL");
    p->timing = enable != 0;
    return RS_OK;
}

extern "C" RS_API rs_status rs_get_stage_times(rs_pass* p, float* ms, uint32_t* count, char* names, size_t namesBytes)
{
    if (!p || !count) return fail(RS_INVALID_ARG, "pass or count is NULL");
    if (!p->timing || p->stageNames.size() < 2) { *count = 0; return RS_OK; }
    RS_CUDA(cudaStreamSynchronize(p->lastStream));
    uint32_t n = (uint32_t)p->stageNames.size() - 1;
    if (ms)
        for (uint32_t i = 0; i < n && i < *count; i++) cudaEventElapsedTime(&ms[i], p->events[i], p->events[i + 1]);
    if (names)
    {
        size_t off = 0;
        for (uint32_t i = 0; i < n; i++)
        {
            size_t l = p->stageNames[i].size() + 1;
            if (off + l > namesBytes) break;
            memcpy(names + off, p->stageNames[i].c_str(), l);
            off += l;
        }
    }
    *count = n;
    return RS_OK;
}

extern "C" RS_API rs_status rs_debug_stage_rays(rs_pass* p, uint64_t* rays, uint32_t* count)
{
    if (!p || !count) return fail(RS_INVALID_ARG, "pass or count is NULL");
#ifdef RS_RAY_STATS
    if (!p->timing || p->stageNames.size() < 2) { *count = 0; return RS_OK; }
    RS_CUDA(cudaStreamSynchronize(p->lastStream));
    const uint32_t n = (uint32_t)std::min(p->stageNames.size() - 1, p->stageRays.size() / 2);
    if (rays)
        for (uint32_t i = 0; i < n && i < *count; i++) { rays[2 * i] = p->stageRays[2 * i]; rays[2 * i + 1] = p->stageRays[2 * i + 1]; }
    *count = n;
#else
    *count = 0;
#endif
    return RS_OK;
}

extern "C" RS_API uint32_t rs_last_launch_count(rs_pass* p) { return p ? p->launches : 0u; }
extern "C" RS_API const char* rs_last_error_string(void) { return g_lastError.c_str(); }

// Test hook (not part of the public header): keep a copy of the candidate reservoirs each frame.
extern "C" RS_API rs_status rs_debug_keep_candidates(rs_pass* p, uint32_t keep)
{
    if (!p) return fail(RS_INVALID_ARG, "pass is NULL");
    p->keepCandidates = keep != 0;
    p->generation++;
    return RS_OK;
}

// ------------------------------------------------------------------ batched instances
// A batch renders one frame of every member pass with a single CUDA graph launch.  Two forms:
//
// * Flattened (members in the same temporal mode: ScatterBackup with the Clamped gather, one sample
//   per pixel, matching spatial settings and environment light, past their first frame): every stage
//   is ONE launch for all members over a flattened work queue (instance k owns work items
//   [start[k], start[k+1]), each a block of its own grid); the kb_* kernels are persistent by
//   default (a grid of SMs x resident blocks striding over the queue) and read each instance's
//   context slot, warp tile width and buffers from device tables built at capture.  The cell lists
//   (scan and radix sort per member) run as member chains on a side stream.  Stage tile widths
//   (per stage and resolution) and grid forms (per stage) come from the batch's tuning
//   (rs_batch_tune times the candidates on a real frame; rs_batch_get/set_tuning carry it).
// * Per member (any other mix): each member's stage chain is a graph branch.
// Kernels read each instance's context from device memory, copied from the pinned host context by a
// node of the graph, so one graph is replayed every frame; a graph is captured per buffer-parity
// pattern of the members and set of colour buffers.
namespace {

constexpr uint32_t kBatchTileChoices[3] = {8u, 16u, 32u};
enum : uint32_t { kGridPersistent = 0, kGridFull = 1 };

// The pixel stages take a warp tile width; the per-splat ones do not.
bool stage_is_pixel(BatchStage st) { return st != kBatchSbSplatScatter && st != kBatchSbSplatGather; }
// Stages whose kernels are pure functions of their inputs (a repeated launch writes the same
// values), so rs_batch_tune may run each candidate configuration in place; the reprojection's
// counters are cleared before each trial.
bool stage_tunable(BatchStage st) { return st != kBatchSbCombine; }

struct DeviceBlob
{
    void* p = nullptr;
    ~DeviceBlob() { if (p) cudaFree(p); }
};

// Host image of the device tables of one flattened frame; every array starts on 256 bytes.
struct TableBuilder
{
    std::vector<uint8_t> bytes;
    template <typename T> size_t add(const std::vector<T>& v)
    {
        size_t off = (bytes.size() + 255) & ~(size_t)255;
        bytes.resize(off + std::max<size_t>(v.size() * sizeof(T), 1));
        if (!v.empty()) memcpy(bytes.data() + off, v.data(), v.size() * sizeof(T));
        return off;
    }
};

} // namespace

struct rs_batch_tuning_store
{
    // tile width per (stage, width, height); grid form per stage
    std::vector<rs_batch_tuning_entry> tiles;
    uint32_t grid[kBatchStageCount];
    rs_batch_tuning_store() { for (auto& g : grid) g = kGridPersistent; }
    uint32_t tile(BatchStage st, uint32_t w, uint32_t h) const
    {
        for (const auto& e : tiles)
            if (e.stage == (uint32_t)st && e.width == w && e.height == h) return e.tile;
        return 8u;
    }
    void set_tile(BatchStage st, uint32_t w, uint32_t h, uint32_t tw, float ms)
    {
        for (auto& e : tiles)
            if (e.stage == (uint32_t)st && e.width == w && e.height == h) { e.tile = tw; e.ms = ms; return; }
        rs_batch_tuning_entry e = {};
        e.stage = st; e.width = w; e.height = h; e.tile = tw; e.grid = kGridPersistent; e.ms = ms;
        tiles.push_back(e);
    }
};

struct rs_batch
{
    std::vector<rs_pass*> passes;
    std::vector<cudaStream_t> branch;
    std::vector<cudaEvent_t> joins;
    cudaEvent_t fork = nullptr, done = nullptr;
    cudaStream_t capture = nullptr;
    static constexpr int kChains = 4; // chains of one group's flattened pipeline: its stream + 3
    // Stream sets of the flattened groups (one group per resolution): group g uses
    // groupStream[g * kChains + c], c = 0 its main stream; events likewise.
    std::vector<cudaStream_t> groupStream;
    std::vector<cudaEvent_t> groupFork, groupJoin; // per group: fork of its chains; per chain: join
    bool inFlight = false;
    bool flatten = true;
    uint32_t numSMs = 0;
    rs_batch_tuning_store tuning;
    uint64_t tuningVersion = 0; // bumped by rs_batch_tune / rs_batch_set_tuning: cached graphs go stale
    struct Cached
    {
        std::vector<uint64_t> key;
        std::vector<void*> colors;
        cudaGraphExec_t exec;
        std::shared_ptr<DeviceBlob> tables; // device tables of a flattened graph (kept alive with it)
    };
    std::vector<Cached> graphs;
    std::vector<uint64_t> generations; // the members' generations when the cached graphs were captured
    uint32_t lastLaunches = 0;
    bool lastFlattened = false;
    ~rs_batch()
    {
        if (done) cudaEventSynchronize(done);
        for (auto& g : graphs) cudaGraphExecDestroy(g.exec);
        for (auto e : joins) cudaEventDestroy(e);
        for (auto s : branch) cudaStreamDestroy(s);
        for (auto s : groupStream) cudaStreamDestroy(s);
        for (auto e : groupFork) cudaEventDestroy(e);
        for (auto e : groupJoin) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (done) cudaEventDestroy(done);
        if (capture) cudaStreamDestroy(capture);
    }
};

extern "C" RS_API rs_status rs_batch_create(rs_pass* const* passes, uint32_t count, rs_batch** out)
{
    if (!passes || !out || count == 0 || count > 64) return fail(RS_INVALID_ARG, "a batch holds 1 to 64 passes");
    std::unique_ptr<rs_batch> b(new rs_batch());
    for (uint32_t i = 0; i < count; i++)
    {
        if (!passes[i] || !passes[i]->hasScene) return fail(RS_INVALID_ARG, "every batch member needs a scene");
        b->passes.push_back(passes[i]);
        cudaStream_t s;
        cudaEvent_t e;
        RS_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        RS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        b->branch.push_back(s);
        b->joins.push_back(e);
    }
    RS_CUDA(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming));
    RS_CUDA(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming));
    RS_CUDA(cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking));
    int dev = 0, sms = 0;
    RS_CUDA(cudaGetDevice(&dev));
    RS_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    b->numSMs = (uint32_t)sms;
    *out = b.release();
    return RS_OK;
}

extern "C" RS_API rs_status rs_batch_destroy(rs_batch* b)
{
    if (!b) return fail(RS_INVALID_ARG, "batch is NULL");
    delete b;
    return RS_OK;
}

extern "C" RS_API rs_status rs_batch_set_flatten(rs_batch* b, uint32_t enable)
{
    if (!b) return fail(RS_INVALID_ARG, "batch is NULL");
    b->flatten = enable != 0;
    return RS_OK;
}

// The flattened form applies when every member renders the same stage sequence this frame.
static bool batch_flattenable(const rs_batch* b, const rs_frame_desc* frames)
{
    if (!b->flatten) return false;
    const rs_options& o0 = b->passes[0]->opt;
    const bool env0 = b->passes[0]->envHost.present != 0;
    for (size_t i = 0; i < b->passes.size(); i++)
    {
        const rs_pass* p = b->passes[i];
        const rs_options& o = p->opt;
        if (o.temporalReuse != RS_SCATTER_BACKUP || o.gatherOption != RS_GATHER_CLAMPED || o.samplesPerPixel != 1 || !o.enableTemporalResampling)
            return false;
        if (o.enableSpatialResampling != o0.enableSpatialResampling || o.numSpatialIterations != o0.numSpatialIterations ||
            o.neighborCount != o0.neighborCount || o.scatterBackupMISOption != o0.scatterBackupMISOption)
            return false;
        if ((p->envHost.present != 0) != env0 || p->numAnalytic || o.emissiveSampler != RS_EMISSIVE_POWER || p->keepCandidates || p->frozen ||
            p->timing)
            return false;
        if (p->frameCount == 0 || frames[i].sceneShouldReset || frames[i].mvec || frames[i].vbuffer) return false;
    }
    return true;
}

namespace {

// Everything a flattened frame launches with: per stage its queue (starts, tiles) and grid, and the
// per-instance argument arrays, as offsets into one device table blob.
struct FlatPlan
{
    std::vector<uint32_t> members; // indices into the batch's passes
    uint32_t n = 0;
    bool env = false, spatial = false, balance = true;
    uint32_t iterations = 0, neighborCount = 1;
    uint32_t items[kBatchStageCount] = {};
    size_t offStart[kBatchStageCount] = {}, offTile[kBatchStageCount] = {};
    size_t offSlots = 0, offTables = 0, offVbuf = 0, offCand = 0, offReproj = 0, offWave = 0, offWaveColor = 0;
    std::vector<size_t> offSpatial, offSpatialColor; // per spatial iteration
    uint32_t grid[kBatchStageCount] = {};
    TableBuilder tb;
};

uint32_t stage_items(BatchStage st, uint32_t W, uint32_t H, uint32_t tw)
{
    if (!stage_is_pixel(st)) return (W * H + 127u) / 128u;
    return tiled_blocks_tw(W, H, batched_threads(st), tw);
}

} // namespace

// Builds the tables of a flattened frame of the batch members `members` from their state after
// begin_frame.
static void build_flat_plan(rs_batch* b, const rs_frame_desc* frames, const std::vector<uint32_t>& members, FlatPlan& P)
{
    const size_t n = members.size();
    P.members = members;
    P.n = (uint32_t)n;
    const rs_options& o0 = b->passes[members[0]]->opt;
    P.env = b->passes[members[0]]->envHost.present != 0;
    P.spatial = o0.enableSpatialResampling != 0;
    P.balance = o0.scatterBackupMISOption == RS_MIS_BALANCE;
    P.iterations = P.spatial ? o0.numSpatialIterations : 0u;
    P.neighborCount = o0.neighborCount;
    std::vector<uint32_t> slots(n);
    std::vector<CameraTable*> tables(n);
    std::vector<VbufArgs> vbuf(n);
    std::vector<CandArgs> cand(n);
    std::vector<ReprojArgs> reproj(n);
    std::vector<WaveCtx> wave(n);
    std::vector<WaveColorArgs> waveColor(n);
    std::vector<std::vector<SpatialCtx>> sp(P.iterations, std::vector<SpatialCtx>(n));
    std::vector<std::vector<SpatialColorArgs>> spColor(P.iterations, std::vector<SpatialColorArgs>(n));
    for (size_t i = 0; i < n; i++)
    {
        rs_pass* p = b->passes[members[i]];
        const rs_frame_desc& fr = frames[members[i]];
        const uint32_t N = p->W * p->H;
        ReservoirSet& curr = p->sets[p->currIdx];
        ReservoirSet& prev = p->sets[p->prevIdx];
        slots[i] = p->slot;
        tables[i] = p->camTable.p;
        vbuf[i] = VbufArgs{p->vbuffer.p, p->mvec.p};
        cand[i] = CandArgs{curr.res(), curr.recp()};
        reproj[i] = ReprojArgs{prev.res(), prev.recp(), p->targets.p, p->counts.p};
        WaveCtx K;
        K.fused = true;
        K.mvec = p->mvec.p;
        K.curr = curr.res(); K.currRec = curr.recp();
        K.prev = prev.res(); K.prevRec = prev.recp();
        K.inter = prev.res(); K.interRec = prev.recp();
        K.floatingCoords = p->floatingCoords.p;
        K.counts = p->counts.p; K.offsets = p->offsets.p; K.sorted = p->sortedSplats.p; K.sortedCell = p->sortedCell.p;
        K.totalSplats = p->total.p;
        K.m2curr = p->m2curr.p; K.m3curr = p->m3curr.p;
        K.backupShift = ShiftPlanes{p->backupShift.p, (size_t)N}; K.backupTerms = p->backupTerms.p; K.backupM = p->backupM.p;
        K.splatShift = ShiftPlanes{p->splatShift.p, (size_t)N}; K.splatTerms = p->splatTerms.p; K.splatM = p->splatM.p;
        wave[i] = K;
        float4* color = reinterpret_cast<float4*>(fr.color);
        waveColor[i] = WaveColorArgs{K, P.spatial ? nullptr : color};
        // the spatial ping-pong of enqueue_frame on local indices (members are not frozen)
        int cur = p->currIdx, prv = p->prevIdx;
        for (uint32_t it = 0; it < P.iterations; it++)
        {
            std::swap(cur, prv);
            ReservoirSet& src = p->sets[prv];
            ReservoirSet& dst = p->sets[cur];
            SpatialCtx S;
            S.iteration = it;
            S.vbuffer = p->vbuffer.p;
            S.neighborOffsets = p->neighborOffsets.p;
            S.src = src.res(); S.srcRec = src.recp();
            S.dst = dst.res(); S.dstRec = dst.recp();
            S.m1 = p->spM1.p; S.nw = p->spNw.p; S.terms = p->spTerms.p;
            S.shift = ShiftPlanes{p->spShift.p, (size_t)N * p->opt.neighborCount};
            sp[it][i] = S;
            spColor[it][i] = SpatialColorArgs{S, it + 1 == P.iterations ? color : nullptr};
        }
    }
    for (uint32_t st = 0; st < kBatchStageCount; st++)
    {
        const BatchStage S = (BatchStage)st;
        std::vector<uint32_t> start(n + 1), tile(n);
        uint32_t total = 0;
        for (size_t i = 0; i < n; i++)
        {
            const rs_pass* p = b->passes[members[i]];
            tile[i] = stage_is_pixel(S) ? b->tuning.tile(S, p->W, p->H) : 8u;
            start[i] = total;
            total += stage_items(S, p->W, p->H, tile[i]);
        }
        start[n] = total;
        P.items[st] = total;
        P.offStart[st] = P.tb.add(start);
        P.offTile[st] = P.tb.add(tile);
        const uint32_t resident = b->numSMs * (uint32_t)batched_blocks_per_sm(S, P.env);
        P.grid[st] = b->tuning.grid[st] == kGridFull ? total : std::min(total, std::max(resident, 1u));
    }
    P.offSlots = P.tb.add(slots);
    P.offTables = P.tb.add(tables);
    P.offVbuf = P.tb.add(vbuf);
    P.offCand = P.tb.add(cand);
    P.offReproj = P.tb.add(reproj);
    P.offWave = P.tb.add(wave);
    P.offWaveColor = P.tb.add(waveColor);
    for (uint32_t it = 0; it < P.iterations; it++)
    {
        P.offSpatial.push_back(P.tb.add(sp[it]));
        P.offSpatialColor.push_back(P.tb.add(spColor[it]));
    }
}

// One stage of a flattened frame: a launch over all instances (grid from the plan, or `gridOverride`).
static void launch_flat(const FlatPlan& P, uint8_t* dev, BatchStage st, size_t argsOff, cudaStream_t s, uint32_t gridOverride = 0)
{
    BatchQueue q;
    q.start = reinterpret_cast<const uint32_t*>(dev + P.offStart[st]);
    q.tile = reinterpret_cast<const uint32_t*>(dev + P.offTile[st]);
    q.slot = reinterpret_cast<const uint32_t*>(dev + P.offSlots);
    q.count = P.n;
    q.total = P.items[st];
    if (q.total == 0) return;
    const uint32_t grid = gridOverride ? gridOverride : P.grid[st];
    const uint32_t y = (st == kBatchSpCentral || st == kBatchSpNeighbor) ? P.neighborCount : 1u;
    launch_batched(st, P.env, dim3(grid, y), dim3(batched_threads(st)), s, q, dev + argsOff);
}

// Issues a flattened frame on `s` (and the batch's chain streams, joined back into s).  The members'
// contexts are uploaded from their graphCtx staging copies.  With `tune`, every tunable stage first
// runs each candidate tile width per resolution and each grid form, timed with events on `s`
// (everything then runs on `s` in order), and the tuning keeps the fastest; the frame's results
// are the same whichever configuration ran last.
static rs_status enqueue_flat(rs_batch* b, FlatPlan& P, uint8_t* dev, cudaStream_t s, const cudaStream_t* chains, cudaEvent_t forkEv,
                              const cudaEvent_t* joinEv, bool tune, uint32_t& launches)
{
    const size_t n = P.n;
    auto member = [&](size_t i) { return b->passes[P.members[i]]; };
    launches = 0;
    for (size_t i = 0; i < n; i++)
    {
        rs_pass* p = member(i);
        RS_CUDA(upload_ctx(p->slot, p->graphCtx, s));
        RS_CUDA(cudaMemsetAsync(p->fault.p, 0, sizeof(uint32_t), s));
    }
    kb_camera_table<<<(uint32_t)n, kMaxCameraKeyframes, 0, s>>>(reinterpret_cast<const uint32_t*>(dev + P.offSlots),
                                                                  reinterpret_cast<CameraTable* const*>(dev + P.offTables));
    launches++;
    cudaStream_t q[rs_batch::kChains];
    q[0] = s;
    for (int c = 1; c < rs_batch::kChains; c++) q[c] = tune ? s : chains[c - 1];
    auto fork = [&](int nch) {
        if (tune) return;
        cudaEventRecord(forkEv, s);
        for (int c = 1; c < nch; c++) cudaStreamWaitEvent(q[c], forkEv, 0);
    };
    auto join = [&](int nch) {
        if (tune) return;
        for (int c = 1; c < nch; c++)
        {
            cudaEventRecord(joinEv[c - 1], q[c]);
            cudaStreamWaitEvent(s, joinEv[c - 1], 0);
        }
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (tune)
    {
        RS_CUDA(cudaEventCreate(&e0));
        RS_CUDA(cudaEventCreate(&e1));
    }
    // The stage, tuned first when asked: for each resolution (instances sharing a width and
    // height) each tile width on that resolution's instances alone, then both grid forms on all.
    // Each trial is a full launch of the stage over its instances, timed by events on `s`; all
    // trials write the same values, so the last one leaves the stage's results in place.
    uint32_t* tq = nullptr; // trial queue: starts (n + 1) and tiles (n)
    if (tune) RS_CUDA(cudaMalloc(&tq, 4 * (2 * n + 1)));
    auto stage = [&](BatchStage st, size_t argsOff, cudaStream_t qs, const std::function<void()>& before) -> rs_status {
        if (!(tune && stage_tunable(st)))
        {
            if (before) before();
            launch_flat(P, dev, st, argsOff, qs);
            launches++;
            return RS_OK;
        }
        const uint32_t resident = std::max(1u, b->numSMs * (uint32_t)batched_blocks_per_sm(st, P.env));
        std::vector<uint32_t> tiles(n);
        for (size_t i = 0; i < n; i++) tiles[i] = stage_is_pixel(st) ? b->tuning.tile(st, member(i)->W, member(i)->H) : 8u;
        auto trial = [&](const std::vector<uint32_t>& tl, const std::vector<char>& on, uint32_t form, float& ms) -> rs_status {
            std::vector<uint32_t> start(n + 1);
            uint32_t total = 0;
            for (size_t i = 0; i < n; i++)
            {
                start[i] = total;
                if (on[i]) total += stage_items(st, member(i)->W, member(i)->H, tl[i]);
            }
            start[n] = total;
            RS_CUDA(cudaMemcpy(tq, start.data(), 4 * (n + 1), cudaMemcpyHostToDevice));
            RS_CUDA(cudaMemcpy(tq + n + 1, tl.data(), 4 * n, cudaMemcpyHostToDevice));
            BatchQueue qq;
            qq.start = tq; qq.tile = tq + n + 1;
            qq.slot = reinterpret_cast<const uint32_t*>(dev + P.offSlots);
            qq.count = (uint32_t)n; qq.total = total;
            const uint32_t grid = form == kGridFull ? total : std::min(total, resident);
            const uint32_t y = (st == kBatchSpCentral || st == kBatchSpNeighbor) ? P.neighborCount : 1u;
            if (before) before();
            RS_CUDA(cudaEventRecord(e0, s));
            if (total) launch_batched(st, P.env, dim3(grid, y), dim3(batched_threads(st)), s, qq, dev + argsOff);
            RS_CUDA(cudaEventRecord(e1, s));
            RS_CUDA(cudaEventSynchronize(e1));
            RS_CUDA(cudaGetLastError());
            RS_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            launches++;
            return RS_OK;
        };
        if (stage_is_pixel(st))
        {
            std::vector<std::pair<uint32_t, uint32_t>> res;
            for (size_t i = 0; i < n; i++)
                if (std::find(res.begin(), res.end(), std::make_pair(member(i)->W, member(i)->H)) == res.end()) res.push_back({member(i)->W, member(i)->H});
            for (auto wh : res)
            {
                std::vector<char> on(n, 0);
                for (size_t i = 0; i < n; i++) on[i] = member(i)->W == wh.first && member(i)->H == wh.second;
                uint32_t bestTile = 8u;
                float best = 3e38f;
                for (uint32_t tw : kBatchTileChoices)
                {
                    std::vector<uint32_t> tl = tiles;
                    for (size_t i = 0; i < n; i++) if (on[i]) tl[i] = tw;
                    float ms = 0.f;
                    rs_status r = trial(tl, on, kGridPersistent, ms);
                    if (r != RS_OK) return r;
                    if (ms < best) { best = ms; bestTile = tw; }
                }
                b->tuning.set_tile(st, wh.first, wh.second, bestTile, best);
                for (size_t i = 0; i < n; i++) if (on[i]) tiles[i] = bestTile;
            }
        }
        const std::vector<char> all(n, 1);
        float tp = 0.f, tf = 0.f;
        rs_status r = trial(tiles, all, kGridPersistent, tp);
        if (r == RS_OK) r = trial(tiles, all, kGridFull, tf); // the last trial: full grid, chosen tiles
        if (r != RS_OK) return r;
        b->tuning.grid[st] = tf < tp ? kGridFull : kGridPersistent;
        return RS_OK;
    };
    rs_status st = RS_OK;
    auto run = [&](rs_status r) { if (st == RS_OK) st = r; };

    // prologue: primary hits, candidates, and the previous frame's splats and cell lists
    fork(3);
    run(stage(kBatchVbuffer, P.offVbuf, q[0], nullptr));
    run(stage(kBatchCandidates, P.offCand, q[1], nullptr));
    auto clearCounts = [&]() {
        for (size_t i = 0; i < n; i++)
        {
            rs_pass* p = member(i);
            cudaMemsetAsync(p->counts.p, 0, (size_t)p->W * p->H * 4ull, q[2]);
        }
    };
    run(stage(kBatchReproject, P.offReproj, q[2], clearCounts));
    for (size_t i = 0; i < n; i++)
    {
        // the member's cell lists (buildCells of enqueue_frame)
        rs_pass* p = member(i);
        const uint32_t N = p->W * p->H;
        const uint32_t numTiles = (N + kScanTileElems - 1) / kScanTileElems;
        k_scan_tiles<<<numTiles, 1024, 0, q[2]>>>(p->counts.p, p->offsets.p, p->tileSums.p, N);
        k_scan_tile_sums<<<1, 1024, 0, q[2]>>>(p->tileSums.p, numTiles, p->total.p);
        k_scan_add<<<(N + 255) / 256, 256, 0, q[2]>>>(p->offsets.p, p->tileSums.p, N);
        cudaError_t e = radix_sort_indices_u32(p->targets.p, N, N, bit_length(N), p->sortedSplats.p, p->unsortedSplats.p, p->radixScratch.p, q[2]);
        if (e != cudaSuccess) run(fail(RS_CUDA_ERROR, std::string("batched cell lists: ") + cudaGetErrorString(e)));
        k_sorted_cells<<<(N + 255) / 256, 256, 0, q[2]>>>(p->targets.p, p->sortedSplats.p, p->sortedCell.p, N);
        launches += 4 + radix_sort_launches(N, bit_length(N));
    }
    join(3);
    // ScatterBackup shifts: four independent chains, then the combine
    fork(4);
    run(stage(kBatchSbCurrScatter, P.offWave, q[0], nullptr));
    run(stage(kBatchSbCurrGather, P.offWave, q[1], nullptr));
    run(stage(kBatchSbBackupGather, P.offWave, q[2], nullptr));
    run(stage(kBatchSbSplatScatter, P.offWave, q[3], nullptr));
    if (P.balance)
    {
        run(stage(kBatchSbBackupScatter, P.offWave, q[2], nullptr));
        run(stage(kBatchSbSplatGather, P.offWave, q[3], nullptr));
    }
    join(4);
    run(stage(kBatchSbCombine, P.offWaveColor, q[0], nullptr));
    for (uint32_t it = 0; it < P.iterations; it++)
    {
        fork(2);
        run(stage(kBatchSpCentral, P.offSpatial[it], q[0], nullptr));
        run(stage(kBatchSpNeighbor, P.offSpatial[it], q[1], nullptr));
        join(2);
        run(stage(kBatchSpCombine, P.offSpatialColor[it], q[0], nullptr));
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (tq) cudaFree(tq);
    RS_CUDA(cudaGetLastError());
    return st;
}

// Host-side frame setup of every member (begin_frame, staging of the contexts); the graph key.
static void batch_begin(rs_batch* b, const rs_frame_desc* frames, cudaStream_t s, std::vector<uint64_t>& key, std::vector<void*>& colors,
                        bool flat)
{
    const size_t n = b->passes.size();
    key.assign(n + 1, 0);
    colors.assign(3 * n, nullptr);
    for (size_t i = 0; i < n; i++)
    {
        rs_pass* p = b->passes[i];
        begin_frame(p, &frames[i]);
        *p->graphCtx = *p->hostCtx;
        p->lastStream = s;
        p->stageNames.clear();
        colors[3 * i] = frames[i].color;
        colors[3 * i + 1] = const_cast<float*>(frames[i].mvec);
        colors[3 * i + 2] = const_cast<uint32_t*>(frames[i].vbuffer);
        // the graph depends on the ping-pong buffers in use, on whether temporal stages run, on
        // which kernel variants run (environment light, depth of field in the gather) and on the
        // pass's buffers and options (its generation)
        const uint32_t shape = (uint32_t)p->currIdx * 3u + (uint32_t)p->prevIdx + 9u * (p->frameCount == 0 || frames[i].sceneShouldReset ? 1u : 0u) +
                               18u * (p->envHost.present ? 1u : 0u) + 36u * (p->camera.apertureRadius > 0.f ? 1u : 0u);
        key[i] = (p->generation << 8) | shape;
    }
    key[n] = flat ? (1ull << 63) | b->tuningVersion : 0ull;
}

static void batch_drop_stale(rs_batch* b)
{
    const size_t n = b->passes.size();
    if (!b->graphs.empty() && b->generations.size() == n)
    {
        bool changed = false;
        for (size_t i = 0; i < n; i++) changed = changed || b->generations[i] != b->passes[i]->generation;
        if (changed)
        {
            for (auto& g : b->graphs) cudaGraphExecDestroy(g.exec);
            b->graphs.clear();
        }
    }
    b->generations.resize(n);
    for (size_t i = 0; i < n; i++) b->generations[i] = b->passes[i]->generation;
}

// The groups of a flattened frame: the members of each resolution, in member order, in chunks of
// at most kFlatGroupMax.  Each group's stages are their own flattened launches on their own
// streams, so different groups' stages overlap (one group's latency-bound traversal with another's
// bandwidth-bound combine, and a group's slowest member holds back only its group at each stage).
// Measured on the 64-instance configuration: one group per resolution 246 instance-frames/s,
// chunks of 8 242, one group for all 242.
constexpr size_t kFlatGroupMax = 64;
static std::vector<std::vector<uint32_t>> flat_groups(const rs_batch* b)
{
    std::vector<std::vector<uint32_t>> byRes;
    std::vector<std::pair<uint32_t, uint32_t>> res;
    for (uint32_t i = 0; i < (uint32_t)b->passes.size(); i++)
    {
        const auto wh = std::make_pair(b->passes[i]->W, b->passes[i]->H);
        auto it = std::find(res.begin(), res.end(), wh);
        if (it == res.end()) { res.push_back(wh); byRes.push_back({i}); }
        else byRes[it - res.begin()].push_back(i);
    }
    std::vector<std::vector<uint32_t>> groups;
    for (const auto& r : byRes)
    {
        const size_t chunks = (r.size() + kFlatGroupMax - 1) / kFlatGroupMax;
        for (size_t c = 0; c < chunks; c++)
        {
            // near-equal chunks of the resolution's members
            const size_t a = r.size() * c / chunks, e = r.size() * (c + 1) / chunks;
            groups.emplace_back(r.begin() + a, r.begin() + e);
        }
    }
    return groups;
}

static rs_status ensure_group_streams(rs_batch* b, size_t groups)
{
    while (b->groupFork.size() < groups)
    {
        for (int c = 0; c < rs_batch::kChains; c++)
        {
            cudaStream_t q;
            cudaEvent_t e;
            RS_CUDA(cudaStreamCreateWithFlags(&q, cudaStreamNonBlocking));
            RS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            b->groupStream.push_back(q);
            b->groupJoin.push_back(e); // c = 0: the group's join into the caller's stream
        }
        cudaEvent_t f;
        RS_CUDA(cudaEventCreateWithFlags(&f, cudaEventDisableTiming));
        b->groupFork.push_back(f);
    }
    return RS_OK;
}

// frames[i] is the frame of passes[i]; each frames[i].color must be a device buffer (graphs keep
// the pointers; a new set of pointers captures a new graph).
extern "C" RS_API rs_status rs_batch_execute(rs_batch* b, const rs_frame_desc* frames, void* streamPtr)
{
    if (!b || !frames) return fail(RS_INVALID_ARG, "batch or frames is NULL");
    cudaStream_t s = (cudaStream_t)streamPtr;
    const size_t n = b->passes.size();
    for (size_t i = 0; i < n; i++)
        if (!frames[i].color) return fail(RS_INVALID_ARG, "batched frames need device colour buffers");
    // the previous replay reads the pinned host contexts; wait for it before rewriting them
    if (b->inFlight) RS_CUDA(cudaEventSynchronize(b->done));
    const bool flat = batch_flattenable(b, frames);
    std::vector<uint64_t> key;
    std::vector<void*> colors;
    batch_begin(b, frames, s, key, colors, flat);
    batch_drop_stale(b);
    cudaGraphExec_t exec = nullptr;
    for (auto& g : b->graphs)
        if (g.key == key && g.colors == colors) { exec = g.exec; break; }
    if (!exec)
    {
        std::shared_ptr<DeviceBlob> tables;
        std::vector<FlatPlan> plans;
        std::vector<size_t> planOff;
        if (flat)
        {
            // one plan per resolution group, all tables in one blob
            const auto groups = flat_groups(b);
            RS_CUDA_STATUS(ensure_group_streams(b, groups.size()));
            plans.resize(groups.size());
            size_t total = 0;
            for (size_t g = 0; g < groups.size(); g++)
            {
                build_flat_plan(b, frames, groups[g], plans[g]);
                planOff.push_back(total);
                total += (plans[g].tb.bytes.size() + 255) & ~(size_t)255;
            }
            tables.reset(new DeviceBlob());
            RS_CUDA(cudaMalloc(&tables->p, total));
            for (size_t g = 0; g < plans.size(); g++)
                RS_CUDA(cudaMemcpy(static_cast<uint8_t*>(tables->p) + planOff[g], plans[g].tb.bytes.data(), plans[g].tb.bytes.size(),
                                   cudaMemcpyHostToDevice));
        }
        cudaStream_t cs = b->capture; // capture never executes; the caller's stream may be the legacy default
        RS_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
        uint32_t launches = 0;
        rs_status st = RS_OK;
        if (flat)
        {
            cudaEventRecord(b->fork, cs);
            for (size_t g = 0; g < plans.size() && st == RS_OK; g++)
            {
                cudaStream_t* gs = &b->groupStream[g * rs_batch::kChains];
                cudaEvent_t* gj = &b->groupJoin[g * rs_batch::kChains];
                cudaStreamWaitEvent(gs[0], b->fork, 0);
                uint32_t l = 0;
                st = enqueue_flat(b, plans[g], static_cast<uint8_t*>(tables->p) + planOff[g], gs[0], gs + 1, b->groupFork[g], gj + 1, false, l);
                launches += l;
                cudaEventRecord(gj[0], gs[0]);
                cudaStreamWaitEvent(cs, gj[0], 0);
            }
        }
        else
        {
            cudaEventRecord(b->fork, cs);
            for (size_t i = 0; i < n && st == RS_OK; i++)
            {
                rs_pass* p = b->passes[i];
                cudaStreamWaitEvent(b->branch[i], b->fork, 0);
                bool timing = p->timing;
                p->timing = false;
                p->launches = 0;
                st = enqueue_frame(p, b->branch[i], reinterpret_cast<float4*>(frames[i].color), reinterpret_cast<const float2*>(frames[i].mvec),
                                   reinterpret_cast<const uint4*>(frames[i].vbuffer), true);
                p->timing = timing;
                launches += p->launches;
                cudaEventRecord(b->joins[i], b->branch[i]);
                cudaStreamWaitEvent(cs, b->joins[i], 0);
            }
        }
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(cs, &graph);
        if (st != RS_OK) { if (graph) cudaGraphDestroy(graph); return st; }
        if (e != cudaSuccess) return fail(RS_CUDA_ERROR, std::string("graph capture: ") + cudaGetErrorString(e));
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fail(RS_CUDA_ERROR, std::string("graph instantiate: ") + cudaGetErrorString(e));
        b->graphs.push_back({key, colors, exec, tables});
        b->lastLaunches = launches;
        b->lastFlattened = flat;
    }
    else
    {
        for (auto& g : b->graphs)
            if (g.exec == exec) b->lastFlattened = (g.key.back() >> 63) != 0;
    }
    RS_CUDA(cudaGraphLaunch(exec, s));
    RS_CUDA(cudaEventRecord(b->done, s));
    b->inFlight = true;
    for (size_t i = 0; i < n; i++) end_frame(b->passes[i]);
    return RS_OK;
}

// Renders one frame like rs_batch_execute, but eagerly and with the tile widths and grid forms of
// every tunable stage timed in place (the flattened form only); the choices replace the batch's
// tuning and cached graphs are recaptured.  Synchronous.
extern "C" RS_API rs_status rs_batch_tune(rs_batch* b, const rs_frame_desc* frames, void* streamPtr)
{
    if (!b || !frames) return fail(RS_INVALID_ARG, "batch or frames is NULL");
    cudaStream_t s = (cudaStream_t)streamPtr;
    const size_t n = b->passes.size();
    for (size_t i = 0; i < n; i++)
        if (!frames[i].color) return fail(RS_INVALID_ARG, "batched frames need device colour buffers");
    if (b->inFlight) RS_CUDA(cudaEventSynchronize(b->done));
    if (!batch_flattenable(b, frames))
        return fail(RS_INVALID_ARG, "rs_batch_tune needs a flattenable frame (every member ScatterBackup/Clamped, one sample per pixel, "
                                    "the same spatial settings, past its first frame)");
    std::vector<uint64_t> key;
    std::vector<void*> colors;
    batch_begin(b, frames, s, key, colors, true);
    rs_status st = RS_OK;
    for (const auto& members : flat_groups(b))
    {
        // each resolution group in turn, everything on `s`
        FlatPlan plan;
        build_flat_plan(b, frames, members, plan);
        DeviceBlob tables;
        RS_CUDA(cudaMalloc(&tables.p, plan.tb.bytes.size()));
        RS_CUDA(cudaMemcpy(tables.p, plan.tb.bytes.data(), plan.tb.bytes.size(), cudaMemcpyHostToDevice));
        uint32_t launches = 0;
        st = enqueue_flat(b, plan, static_cast<uint8_t*>(tables.p), s, nullptr, nullptr, nullptr, true, launches);
        RS_CUDA(cudaStreamSynchronize(s));
        if (st != RS_OK) break;
    }
    for (size_t i = 0; i < n; i++) end_frame(b->passes[i]);
    if (st != RS_OK) return st;
    b->tuningVersion++;
    for (auto& g : b->graphs) cudaGraphExecDestroy(g.exec);
    b->graphs.clear();
    b->inFlight = false;
    return RS_OK;
}

extern "C" RS_API rs_status rs_batch_get_tuning(rs_batch* b, rs_batch_tuning_entry* out, uint32_t* count)
{
    if (!b || !count) return fail(RS_INVALID_ARG, "batch or count is NULL");
    std::vector<rs_batch_tuning_entry> all = b->tuning.tiles;
    for (uint32_t st = 0; st < kBatchStageCount; st++)
    {
        rs_batch_tuning_entry e = {};
        e.stage = st; e.width = 0; e.height = 0; e.tile = 0; e.grid = b->tuning.grid[st]; e.ms = 0.f;
        all.push_back(e);
    }
    if (out)
        for (uint32_t i = 0; i < std::min<uint32_t>(*count, (uint32_t)all.size()); i++) out[i] = all[i];
    *count = (uint32_t)all.size();
    return RS_OK;
}

extern "C" RS_API rs_status rs_batch_set_tuning(rs_batch* b, const rs_batch_tuning_entry* in, uint32_t count)
{
    if (!b || (count && !in)) return fail(RS_INVALID_ARG, "batch or entries are NULL");
    for (uint32_t i = 0; i < count; i++)
    {
        const rs_batch_tuning_entry& e = in[i];
        if (e.stage >= kBatchStageCount) return fail(RS_INVALID_ARG, "tuning entry: unknown stage");
        if (e.width == 0 && e.height == 0)
        {
            if (e.grid > kGridFull) return fail(RS_INVALID_ARG, "tuning entry: grid form must be 0 (persistent) or 1 (one block per item)");
            b->tuning.grid[e.stage] = e.grid;
        }
        else
        {
            if (e.tile != 8u && e.tile != 16u && e.tile != 32u) return fail(RS_INVALID_ARG, "tuning entry: tile width must be 8, 16 or 32");
            b->tuning.set_tile((BatchStage)e.stage, e.width, e.height, e.tile, e.ms);
        }
    }
    b->tuningVersion++;
    return RS_OK;
}

extern "C" RS_API uint32_t rs_batch_launch_count(rs_batch* b)
{
    if (!b) return 0u;
    return b->lastLaunches;
}

extern "C" RS_API uint32_t rs_batch_last_flattened(rs_batch* b) { return b && b->lastFlattened ? 1u : 0u; }
