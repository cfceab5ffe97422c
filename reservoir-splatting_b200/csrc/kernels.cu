// sm_100a kernels of the Reservoir Splatting per-frame path.  One thread per
// pixel (or per source pixel / cell); all state lives in structure-of-arrays
// planes so every warp load and store is a coalesced 512-byte transaction.
// Nothing here is a dense contraction, so no tensor-core path exists; the
// bounds are HBM bandwidth (splat, scan, fill, resolve) and BVH traversal
// latency (candidates, reprojection visibility, resampling shifts).
#include "kernels.h"

namespace rs {

// Per-pass frame constants, one slot per live pass (kMaxPassSlots), indexed by a kernel argument.
// Reads with a warp-uniform slot are served by the constant cache; the host updates a slot with a
// stream-ordered copy (a memcpy node inside a captured graph).
__constant__ DevCtx c_ctx[kMaxPassSlots];

cudaError_t upload_ctx(uint32_t slot, const DevCtx* hostPinned, cudaStream_t s)
{
    return cudaMemcpyToSymbolAsync(c_ctx, hostPinned, sizeof(DevCtx), slot * sizeof(DevCtx), cudaMemcpyHostToDevice, s);
}

// ============================================================ primary hits + motion vectors
// VBufferRT.slang:71-150 (samplePattern Center, pinhole): hit of the pixel-centre ray of the
// frame's camera and mvec = prevScreen - (pixel + 0.5) / dim, prevScreen being the film
// projection of the hit point through the previous frame's camera.
__device__ __forceinline__ void vbuffer_body(uint32_t slot, uint4* __restrict__ vbuffer, float2* __restrict__ mvec, Blk blk)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t i;
    if (!tiled_pixel_at(C.W, C.H, blk, i)) return;
    uint32_t x = i % C.W, y = i / C.W;
    const CameraData& cam = C.camera;
    const CameraData& pc = C.prevCamera;
    f2 p = mk2(((float)x + 0.5f) / (float)C.W, ((float)y + 0.5f) / (float)C.H);
    f2 ndc = mk2(2.f * p.x + -1.f, -2.f * p.y + 1.f);
    f3 dir = normalize(cam.cameraU * ndc.x + cam.cameraV * ndc.y + cam.cameraW);
    HitInfo h; float t;
    if (trace_closest(C.bvh, mk_ray(cam.posW, dir, 0.f, kRayTMax), h, t, C.fault))
    {
        vbuffer[i] = make_uint4(h.w[0], h.w[1], h.w[2], h.w[3]);
        // Scene::getPrevPosW (VBufferRT.slang:84): the hit on the previous frame's geometry
        f3 prevPosW = hit_position(reinterpret_cast<const f4*>(C.prevTri), h);
        f3 d = prevPosW - pc.posW;
        f3 camRay = mk3(dot(pc.unitU, d), dot(pc.unitV, d), dot(pc.unitW, d));
        float lw = pc.lenW;
        f2 film = mk2(lw * (camRay.x / camRay.z), lw * (camRay.y / camRay.z));
        f2 pndc = mk2(film.x / pc.lenU, film.y / pc.lenV);
        f2 prevCrd = mk2(0.5f * pndc.x + 0.5f, -0.5f * pndc.y + 0.5f);
        mvec[i] = make_float2(prevCrd.x - p.x, prevCrd.y - p.y);
    }
    else
    {
        vbuffer[i] = make_uint4(0u, 0u, 0u, 0u);
        f2 mv = mk2(0.f, 0.f);
        if (C.env->present) mv = env_miss_motion_vector(cam, pc, dir, p); // writeMiss (VBufferRT.slang:128-149)
        mvec[i] = make_float2(mv.x, mv.y);
    }
}

__global__ void __launch_bounds__(256) k_vbuffer(uint32_t slot, uint4* __restrict__ vbuffer, float2* __restrict__ mvec)
{
    vbuffer_body(slot, vbuffer, mvec, Blk{blockIdx.x, 8u});
}

__global__ void __launch_bounds__(256) kb_vbuffer(BatchQueue q, const VbufArgs* __restrict__ args)
{
    for (uint32_t t = blockIdx.x; t < q.total; t += gridDim.x)
    {
        const uint32_t inst = batch_instance(q, t);
        const VbufArgs& a = args[inst];
        vbuffer_body(__ldg(q.slot + inst), a.vbuffer, a.mvec, batch_blk(q, inst, t));
    }
}

#ifdef RS_RAY_STATS
// Closest-hit and visibility queries counted by the frame kernels since the last call (reset).
cudaError_t ray_stats_take(unsigned long long out[2], cudaStream_t s)
{
    cudaError_t e = cudaMemcpyFromSymbolAsync(out, g_rayStats, 2 * sizeof(unsigned long long), 0, cudaMemcpyDeviceToHost, s);
    if (e != cudaSuccess) return e;
    e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return e;
    const unsigned long long zero[2] = {0ull, 0ull};
    e = cudaMemcpyToSymbolAsync(g_rayStats, zero, sizeof(zero), 0, cudaMemcpyHostToDevice, s);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(s);
}
#endif

// ============================================================ camera table
// The frame constants of orient_camera (CameraTable) for the context of `slot`; one block of
// kMaxCameraKeyframes threads, launched after the context upload of the frame.
__device__ __forceinline__ void camera_table_body(uint32_t slot, CameraTable* __restrict__ table)
{
    const DevCtx& C = c_ctx[slot];
    __shared__ f3 forward[kMaxCameraKeyframes];
    const int i = (int)threadIdx.x, K = (int)C.cm.keyframes;
    if (i < K) forward[i] = camera_table_forward(C.cm, i);
    __syncthreads();
    if (i < K)
    {
        table->forward[i] = forward[i];
        camera_table_pair(C.cm, forward, i, table->pairAxis[i], table->pairAngle[i]);
    }
    if (i == 0) camera_table_extents(C.camera, table->ulen, table->vlen);
    __syncthreads();
    if (i < 2)
    {
        const float t = i == 0 ? 0.f : C.cm.artificialFrameTime;
        CameraData c = C.camera;
        orient_camera_table(C.cm, *table, c, C.frameCount, t);
        table->time[i] = t;
        table->at[i] = c;
    }
}
__global__ void __launch_bounds__(kMaxCameraKeyframes) k_camera_table(uint32_t slot, CameraTable* __restrict__ table)
{
    camera_table_body(slot, table);
}

// One block per batch member: block b builds the camera table of context slots[b].
__global__ void __launch_bounds__(kMaxCameraKeyframes) kb_camera_table(const uint32_t* __restrict__ slots, CameraTable* const* __restrict__ tables)
{
    camera_table_body(slots[blockIdx.x], tables[blockIdx.x]);
}

// ============================================================ initial candidates
// Path state of the candidate tracer (PathStates.slang:85-219, the fields the pass uses).
struct PState
{
    uint32_t flags;      // PathFlags bits (unshifted)
    uint32_t vertex;     // vertex index
    uint32_t bounces;    // packed 8-bit counters: diffuse, specular, transmission
    f3 origin, dir;
    float pdf, totalPdf;
    HitInfo hit;
    f3 prevHitPos;
    f3 thp;
    f3 earlyThroughput;
    SampleGen sg;
    Recon rec;           // path.reconnection
    float candTotalWeight; // path.reservoir (CandidateReservoir)
    f3 candIntegrand;
    Recon candRec;       // path.reservoir.selectedReconnection (several samples per pixel)
    bool anySelected;    // a candidate was selected (one sample per pixel: its record is in the output)
};
enum : uint32_t { kPActive = 1u, kPHit = 2u, kPSpecular = 8u, kPDelta = 16u, kPLightUpper = 64u, kPLightLower = 128u };

__device__ __forceinline__ uint32_t pbounces(const PState& p, uint32_t type) { return (p.bounces >> (type << 3)) & 0xffu; }
// The bounce counters (two bits each: on entering x3 each is at most 2) and the path flags 4..128
// on entering the third vertex, in the 12 bits of Recon::suffixState.
__device__ __forceinline__ uint32_t suffix_state_pack(uint32_t bounces, uint32_t flags)
{
    return (bounces & 3u) | (((bounces >> 8) & 3u) << 2) | (((bounces >> 16) & 3u) << 4) | (((flags >> 2) & 0x3fu) << 6);
}
__device__ __forceinline__ void suffix_state_unpack(uint32_t st, uint32_t& bounces, uint32_t& flags)
{
    bounces = (st & 3u) | (((st >> 2) & 3u) << 8) | (((st >> 4) & 3u) << 16);
    flags = ((st >> 6) & 0x3fu) << 2;
}
__device__ __forceinline__ bool finished_bounces(const DevCtx& C, const PState& p) // PathTracer.slang:161-172
{
    uint32_t d = pbounces(p, 0), s = pbounces(p, 1), t = pbounces(p, 2);
    return (d + s + t) > C.maxSurfaceBounces || d > C.maxDiffuseBounces || s > C.maxSpecularBounces || t > C.maxTransmissionBounces;
}

// CandidateReservoir::addVertex (Reservoir.slang:43-58)
__device__ __forceinline__ bool cand_add_vertex(PState& p, float sampleMIS, f3 sampleIntegrand)
{
    float samplePHat = luminance(sampleIntegrand);
    float sampleWeight = sampleMIS * samplePHat;
    sampleWeight = f_isnan(sampleWeight) ? 0.f : sampleWeight;
    p.candTotalWeight += sampleWeight;
    float rng = sampleNext1D(p.sg);
    bool selected = (rng * p.candTotalWeight < sampleWeight);
    p.candIntegrand = selected ? sampleIntegrand : p.candIntegrand;
    return selected;
}

__device__ __forceinline__ void next_hit(const DevCtx& C, PState& p) // PathTracer.slang:278-299
{
    p.vertex += 1;
    HitInfo h; float t;
    const TraceHit th = C.bvh.numTris ? trace_closest_call(C.bvh, mk_ray(p.origin, p.dir, 0.f, kRayTMax), C.fault) : TraceHit{kInvalidIndex, 0.f, 0.f, 0.f};
    if (th.prim != kInvalidIndex) { h = hit_tri(th.prim, th.u, th.v); t = th.t; p.hit = h; p.flags |= kPHit; }
    else p.flags &= ~kPHit;
}

// handleHit (PathTracer.slang:783-1168)
// kDirect (one sample per pixel): a selected candidate's record is written straight to the
// output planes (outRec, pixel pix) instead of being carried in the path state; the output is the
// same, and ~28 registers of long-lived state are freed.
// A call, not inlined: the path tracer's loop then keeps fewer values live across the shading code
// (k_candidates_direct 4.50 -> 4.40 ms at 1080p, measured twice on separate boxes).
// generateAnalyticLightSample (PathTracer.slang:573-599) as a call: only scenes with analytic
// lights reach it, and inlined it would add its registers and code to every path tracer.
static __device__ __noinline__ bool nee_analytic(const DevCtx& C, f3 posW, f3 faceN, SampleGen& sg, f3& Li, float& pdf, f3& dir,
                                                 float& distance, f3& origin)
{
    AnalyticSample as;
    if (!analytic_light_sample(C.analytic, posW, sg, as)) return false;
    Li = as.Li;
    pdf = as.pdf;
    dir = as.dir;
    distance = as.distance;
    origin = computeRayOrigin(posW, dot(faceN, dir) >= 0.f ? faceN : -faceN);
    return true;
}

template <bool kDirect, bool kEnv, bool kAnalytic, bool kUniform>
__device__ __noinline__ void handle_hit(const DevCtx& C, PState& path, const RecPlanes& outRec, uint32_t pix)
{
    const bool isPrimaryHit = path.vertex == 1;
    ShadingData sd = dev_sd(C, path.hit, path.dir);
    float distanceToPrevVertex = length(sd.posW - path.prevHitPos);
    float geometryFactor = f_abs(dot(sd.faceN, sd.V)) / (distanceToPrevVertex * distanceToPrevVertex);
    float prevScatterPdf = path.pdf;
    path.prevHitPos = sd.posW;
    if (path.vertex == 1)
    {
        path.rec.firstHit = path.hit;
        path.rec.firstWi = -path.dir;
        CameraData cam; dev_orient(C, cam, 0.f); // path.time is never set by generatePath
        f3 x0 = camera_lens_point(cam, path.rec.lensSample);
        float dist = length(sd.posW - x0);
        float distSquared = dist * dist;
        float cosNormal = dot(-path.dir, sd.faceN);
        float cosSensor = dot(cam.unitW, path.dir);
        path.rec.subPixelJacobian = f_abs(cosNormal / distSquared) / f_abs(f_pow3(cosSensor));
        f3 camDir = cam.unitW;
        float camZ = dot(sd.posW - cam.posW, camDir);
        float d0 = (cam.lenW / f_abs(camZ) * dist);
        float d1 = dist - d0;
        path.rec.lensVertexJacobian = (d0 * d0) / (d1 * d1) * (f_abs(dot(-path.dir, sd.faceN))) / (f_abs(dot(-path.dir, camDir)));
    }
    else if (path.vertex == 2)
    {
        path.rec.secondHit = path.hit;
        path.rec.secondaryPathJacobian = prevScatterPdf * geometryFactor;
    }
    else if (path.vertex == 3)
    {
        path.rec.secondaryPathJacobian *= prevScatterPdf;
        path.rec.suffixSeed = (uint32_t)path.sg.state;
        path.rec.suffixState = suffix_state_pack(path.bounces, path.flags);
    }

    BsdfData d = dev_instance(C, sd);
    const bool isLightSamplable = !(path.flags & kPDelta);
    const bool isLightSampled = (path.flags & (kPLightUpper | kPLightLower)) != 0;
    const bool haveLights = C.lights.count > 0;
    bool computeEmissive = isPrimaryHit || (haveLights && (!isLightSampled || !isLightSamplable));
    if (computeEmissive && any_gt0(d.emission))
    {
        float misWeight = 1.f;
        float lightPdf = 0.f;
        if (haveLights && !isPrimaryHit && isLightSampled && isLightSamplable)
        {
            lightPdf = (kEnv || kAnalytic ? C.pEmissiveLight : 1.f) * eval_emissive_pdf(C.lights, path.origin, sd.lightIndex, sd.posW, sd_oriented_face_normal(sd));
            misWeight = dev_mis(C, path.totalPdf, lightPdf);
        }
        bool selected = cand_add_vertex(path, 1.f, path.earlyThroughput * path.thp * d.emission * misWeight);
        if (selected)
        {
            Recon sel = path.rec;
            sel.pathLength = path.vertex;
            sel.lightIsNEE = false;
            sel.lightIsDistant = false;
            sel.lightPdf = lightPdf;
            if (path.vertex == 2) sel.lightPdf *= geometryFactor;
            if (path.vertex == 2 || path.vertex == 3) sel.irradiance = d.emission;
            else sel.irradiance = path.thp * d.emission * misWeight;
            if (kDirect) { store_rec(outRec, pix, sel); path.anySelected = true; }
            else path.candRec = sel;
        }
    }

    if (finished_bounces(C, path)) { path.flags &= ~kPActive; return; }

    path.origin = sd_ray_origin(sd, true);

    const uint32_t lobeTypes = mi_lobe_types(d);
    path.flags &= ~(kPLightUpper | kPLightLower);
    if ((lobeTypes & kLobeNonDelta) != 0)
    {
        bool sampleUpper = (lobeTypes & kLobeNonDeltaReflection) != 0;
        bool sampleLower = (lobeTypes & kLobeNonDeltaTransmission) != 0;
        // generateLightSample (:668-701): the type-selection draw is always taken, then the env map
        // (p = pEnvLight), the emissive triangles (p = pEmissiveLight) or the analytic lights
        // (p = pAnalyticLight) are sampled.
        bool validSample = false, lsEnv = false, lsAnalytic = false;
        TriangleLightSample tls;
        f3 lsLi = mk3(0.f), lsOrigin = mk3(0.f), lsDir = mk3(0.f);
        float lsPdf = 0.f, lsDistance = 0.f, selectionPdf = 0.f;
        bool sampled = false;
        // with the emissive triangles alone p = {0, haveLights, 0} and the emissive sample's selection
        // pdf is 1; without an env map pEnv = 0, so u - pEnv is u (the reference's running subtraction)
        const float pEnv = kEnv ? C.pEnvLight : 0.f;
        const float pEmissive = (kEnv || kAnalytic) ? C.pEmissiveLight : (haveLights ? 1.f : 0.f);
        float u = sampleNext1D(path.sg);
        if (kEnv && u < pEnv)
        {
            // generateEnvMapSample (:516-534)
            selectionPdf = pEnv;
            lsEnv = true;
            f2 r2; r2.x = sampleNext1D(path.sg); r2.y = sampleNext1D(path.sg);
            const EnvSample es = dev_env_sample(C.env, r2);
            lsDir = es.dir; lsPdf = es.pdf;
            lsLi = lsPdf > 0.f ? es.Le / lsPdf : mk3(0.f);
            lsOrigin = computeRayOrigin(sd.posW, dot(sd.faceN, lsDir) >= 0.f ? sd.faceN : -sd.faceN);
            lsDistance = kRayTMax;
            sampled = any_gt0(lsLi);
        }
        else if (u - pEnv < pEmissive)
        {
            selectionPdf = (kEnv || kAnalytic) ? pEmissive : 1.f;
            if (kUniform ? sample_emissive_uniform(C.lights, sd.posW, path.sg, tls) : sample_emissive_power(C.lights, sd.posW, path.sg, tls))
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
        else if (kAnalytic && (u - pEnv) - pEmissive < C.pAnalyticLight)
        {
            // generateAnalyticLightSample (:573-599): no geometry, so the ray runs to the sampled
            // distance unshortened
            selectionPdf = C.pAnalyticLight;
            lsAnalytic = true;
            sampled = nee_analytic(C, sd.posW, sd.faceN, path.sg, lsLi, lsPdf, lsDir, lsDistance, lsOrigin);
        }
        if (sampled)
        {
            float NdotL = dot(sd_oriented_face_normal(sd), lsDir);
            if (!((!sampleUpper && NdotL >= -kMinCosTheta) || (!sampleLower && NdotL <= kMinCosTheta)))
            {
                lsPdf *= selectionPdf;
                lsLi /= selectionPdf;
                validSample = true;
            }
        }
        if (sampleUpper) path.flags |= kPLightUpper;
        if (sampleLower) path.flags |= kPLightLower;
        if (validSample)
        {
            f3 Le = lsLi * lsPdf;
            const BsdfPair bp = mi_eval_pair(sd, d, 0u, lsDir); // all lobes: the pair's total
            // analytic lights cannot be hit by scatter rays: MIS weight 1 (:1025-1031)
            float scatterPdf = bp.totalPdf;
            float misWeight = (kAnalytic && lsAnalytic) ? 1.f : dev_mis(C, lsPdf, scatterPdf);
            f3 weight = bp.totalBsdf;
            f3 Lr = weight * misWeight * lsLi;
            if (any_gt0(Lr) && dev_visible(C, mk_ray(lsOrigin, lsDir, 0.f, lsDistance)))
            {
                bool selected = cand_add_vertex(path, 1.f, path.earlyThroughput * path.thp * weight * lsLi * misWeight);
                if (selected)
                {
                    Recon sel = path.rec;
                    sel.pathLength = path.vertex + 1;
                    sel.lightIsNEE = true;
                    sel.irradiance = Le;
                    if (path.vertex == 1) sel.transmissionEvent = dot(sd.faceN, sd.V) * dot(sd.faceN, lsDir) < 0.f;
                    sel.lightIsDistant = lsEnv;
                    if (path.vertex == 1)
                    {
                        // an analytic light leaves the record's light vertex unset (:1079-1104):
                        // its second hit keeps the running record's (none)
                        if (kAnalytic && lsAnalytic) {}
                        else if (lsEnv)
                        {
                            sel.secondHit = hit_direction(lsDir);
                            sel.secondaryPathJacobian = lsPdf;
                            sel.lightPdf = lsPdf; // a distant light: no area measure
                        }
                        else
                        {
                            sel.secondHit = hit_tri(C.lights.tris[tls.triangleIndex].sceneTri, tls.uv.x, tls.uv.y);
                            sel.secondaryPathJacobian = lsPdf * tls.geometryTerm;
                            sel.lightPdf = lsPdf * tls.geometryTerm;
                        }
                    }
                    else if (path.vertex == 2)
                    {
                        sel.secondWo = lsDir;
                        sel.lightPdf = lsPdf;
                    }
                    else
                    {
                        sel.irradiance = path.thp * Lr;
                    }
                    if (kDirect) { store_rec(outRec, pix, sel); path.anySelected = true; }
                    else path.candRec = sel;
                }
            }
        }
    }

    if (C.useRussianRoulette)
    {
        float u = sampleNext1D(path.sg);
        const float rrVal = luminance(path.thp);
        const float prob = f_max(0.f, 1.f - rrVal);
        if (u < prob) { path.flags &= ~kPActive; return; }
        path.thp /= 1.f - prob;
    }

    // generateScatterRay (:331-382)
    BSDFSample result;
    result.wo = mk3(0.f); result.pdf = 0.f; result.weight = mk3(0.f); result.lobeType = 0;
    float totalPdf;
    bool valid = mi_sample_total_pdf(sd, d, 1u, path.sg, result, totalPdf); // and mi_pdf(sd, d, 0xF, result.wo)
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
    if (path.vertex == 1) path.rec.firstComp = componentType;
    else if (path.vertex == 2) { path.rec.secondComp = componentType; path.rec.secondWo = result.wo; }
    path.totalPdf = totalPdf;
    if (valid)
    {
        // generateScatterRay(bs, ...) (:391-471)
        path.dir = result.wo;
        path.thp *= result.weight;
        path.flags &= ~(4u | kPSpecular | kPDelta);
        if (result.lobeType & kLobeReflection)
        {
            float roughness = mi_roughness(d);
            bool isDiffuse = (result.lobeType & kLobeDiffuseReflection) || roughness > C.specularRoughnessThreshold;
            if (isDiffuse) path.bounces += 1u;
            else { path.bounces += (1u << 8); path.flags |= kPSpecular; }
        }
        if (result.lobeType & kLobeDelta) path.flags |= kPDelta;
    }
    if (path.vertex == 1 || path.vertex == 2)
    {
        path.earlyThroughput *= result.weight;
        path.thp = mk3(1.f);
    }
    const bool isLastVertex = finished_bounces(C, path);
    if (isLastVertex && !(path.flags & kPDelta)) valid = false;
    if (C.disableCaustics && pbounces(path, 0) > 0 && (path.flags & kPSpecular)) valid = false;
    if (!valid) path.flags &= ~kPActive;
}

// generatePath (PathTracer.slang:194-221): the path of pixel (x, y) up to its primary ray.
template <bool kDirect>
__device__ __forceinline__ void path_init(const DevCtx& C, uint32_t x, uint32_t y, PState& path)
{
    path.flags = kPActive;
    path.vertex = 0;
    path.bounces = 0;
    path.thp = mk3(1.f);
    path.earlyThroughput = mk3(1.f);
    path.pdf = 0.f; path.totalPdf = 0.f;
    path.hit = hit_none();
    path.rec = recon_default();
    path.candTotalWeight = 0.f;
    path.candIntegrand = mk3(0.f);
    if (!kDirect) path.candRec = recon_default();
    path.anySelected = false;
    path.sg = sg_create(x, y, C.useFixedSeed ? C.fixedSeed + 0 : kNumRenderPasses * (C.frameCount + C.seed) + 0, C.sgKind);
    CameraData cam = C.camera;
    path.rec.time = sampleNext1D(path.sg) * cam.shutterSpeed;
    path.rec.subPixel.x = sampleNext1D(path.sg);
    path.rec.subPixel.y = sampleNext1D(path.sg);
    if (cam.apertureRadius > 0.f)
    {
        f2 u; u.x = sampleNext1D(path.sg); u.y = sampleNext1D(path.sg);
        path.rec.lensSample = sample_disk(u);
    }
    else path.rec.lensSample = mk2(0.f, 0.f);
    dev_orient(C, cam, path.rec.time);
    Ray r = camera_ray_thinlens(cam, C.W, C.H, mk2((float)x + path.rec.subPixel.x, (float)y + path.rec.subPixel.y), path.rec.lensSample);
    path.origin = r.origin;
    path.dir = r.dir;
    path.prevHitPos = camera_lens_point(cam, path.rec.lensSample);
}

template <bool kDirect>
__device__ __forceinline__ void select_record(PState& path, const Recon& sel, const RecPlanes& outRec, uint32_t pix)
{
    if (kDirect) { store_rec(outRec, pix, sel); path.anySelected = true; }
    else path.candRec = sel;
}

// handlePrimaryMiss (PathTracer.slang:1529-1569): the environment seen straight through the pixel.
// The camera is the one at time 0 (generatePath leaves path.time unset).
template <bool kDirect>
__device__ void handle_primary_miss(const DevCtx& C, PState& path, const RecPlanes& outRec, uint32_t pix)
{
    if (!C.env->present) return;
    const f3 Le = dev_env_eval(C.env, path.dir);
    if (cand_add_vertex(path, 1.f, Le))
    {
        Recon sel = path.rec;
        sel.lightIsDistant = true;
        CameraData cam; dev_orient(C, cam, 0.f);
        const f3 camDir = cam.unitW;
        const float cosSensor = dot(camDir, path.dir);
        sel.subPixelJacobian = 1.f / f_abs(f_pow3(cosSensor));
        const float d0 = cam.lenW / dot(camDir, path.dir);
        sel.lensVertexJacobian = (d0 * d0) / f_abs(cosSensor);
        sel.firstWi = -path.dir;
        sel.pathLength = 1;
        sel.irradiance = Le;
        select_record<kDirect>(path, sel, outRec, pix);
    }
}

// handleMiss (PathTracer.slang:1433-1524): a scatter ray that leaves the scene sees the environment
// unless the previous vertex's light sample already covered it.
template <bool kDirect>
__device__ void handle_miss(const DevCtx& C, PState& path, const RecPlanes& outRec, uint32_t pix)
{
    if (path.vertex == 2) path.rec.secondaryPathJacobian = path.pdf * 1.f;
    else if (path.vertex == 3) path.rec.secondaryPathJacobian *= path.pdf;
    const bool isLightSamplable = !(path.flags & kPDelta);
    const bool isLightSampled = (path.flags & (kPLightUpper | kPLightLower)) != 0;
    if (!(C.env->present && (!isLightSampled || !isLightSamplable))) return;
    float misWeight = 1.f;
    float lightPdf = 0.f;
    if (isLightSampled && isLightSamplable)
    {
        lightPdf = C.pEnvLight * dev_env_eval_pdf(C.env, path.dir);
        misWeight = dev_mis(C, path.totalPdf, lightPdf);
    }
    const f3 Le = dev_env_eval(C.env, path.dir);
    const f3 emitterRadiance = misWeight * Le;
    if (cand_add_vertex(path, 1.f, path.earlyThroughput * path.thp * Le * misWeight))
    {
        Recon sel = path.rec;
        sel.pathLength = path.vertex;
        sel.lightIsNEE = false;
        sel.lightIsDistant = true;
        sel.lightPdf = lightPdf;
        if (path.vertex == 2) sel.secondHit = hit_direction(path.dir);
        if (path.vertex == 2 || path.vertex == 3) sel.irradiance = Le;
        else sel.irradiance = path.thp * emitterRadiance;
        select_record<kDirect>(path, sel, outRec, pix);
    }
}

// One vertex of the tracePath loop (InitialCandidates.cs.slang:80-141): the next closest hit, then
// handleHit, or handlePrimaryMiss / handleMiss, which end the path.
// kLights: bit 0 environment map, bit 1 analytic lights, bit 2 the uniform emissive sampler (the
// reference compiles its shaders per light configuration the same way: USE_ENV_LIGHT,
// USE_ANALYTIC_LIGHTS, _EMISSIVE_LIGHT_SAMPLER_TYPE)
template <bool kDirect, uint32_t kLights>
__device__ __forceinline__ void path_step(const DevCtx& C, PState& path, const RecPlanes& currRec, uint32_t i)
{
    constexpr bool kEnv = (kLights & 1u) != 0;
    next_hit(C, path);
    if (path.flags & kPHit) handle_hit<kDirect, kEnv, (kLights & 2u) != 0, (kLights & 4u) != 0>(C, path, currRec, i);
    else
    {
        if (!kEnv)
        {
            if (path.vertex == 2) path.rec.secondaryPathJacobian = path.pdf * 1.f;
            else if (path.vertex == 3) path.rec.secondaryPathJacobian *= path.pdf;
        }
        else if (path.vertex == 1) handle_primary_miss<kDirect>(C, path, currRec, i);
        else handle_miss<kDirect>(C, path, currRec, i);
        path.flags &= ~kPActive;
    }
}

// addCandidateReservoir (InitialCandidates.cs.slang:52-75) of sample sIdx of spp.
template <bool kDirect>
__device__ __forceinline__ void path_finish(PState& path, uint32_t sIdx, uint32_t spp, const ResPlanes& curr, const RecPlanes& currRec, uint32_t i)
{
    const bool isFirstSample = (sIdx == spp - 1) || spp == 1;
    Res ex = isFirstSample ? res_default() : load_res_rw(curr, i);
    float weight = (1.f / (float)spp) * path.candTotalWeight;
    ex.totalWeight = ex.totalWeight + weight;
    ex.confidence = f_min(ex.confidence + 1.f, kConfidenceCap);
    float rng = sampleNext1D(path.sg);
    bool selected = (rng * ex.totalWeight < weight);
    ex.integrand = selected ? path.candIntegrand : ex.integrand;
    ex.subPixel = selected ? path.rec.subPixel : ex.subPixel;
    ex.confidence = 1.f;
    store_res(curr, i, ex);
    if (kDirect)
    {
        // the output holds the last selected candidate's record when one was selected
        if (!(selected && path.anySelected)) store_rec(currRec, i, recon_default());
    }
    else
    {
        Recon exr = isFirstSample ? recon_default() : load_rec_rw(currRec, i);
        store_rec(currRec, i, selected ? path.candRec : exr);
    }
}

// InitialCandidates.cs.slang:80-141, several samples per pixel: one thread runs the pixel's paths.
template <uint32_t kLights>
__global__ void __launch_bounds__(128, 3) k_candidates(uint32_t slot, ResPlanes curr, RecPlanes currRec)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= C.W * C.H) return;
    const uint32_t x = i % C.W, y = i / C.W;
    for (uint32_t sIdx = 0; sIdx < C.spp; sIdx++)
    {
        PState path;
        path_init<false>(C, x, y, path);
        do path_step<false, kLights>(C, path, currRec, i);
        while (path.flags & kPActive);
        path_finish<false>(path, sIdx, C.spp, curr, currRec, i);
    }
}

// One sample per pixel (the reference default): records go straight to the output planes.
template <uint32_t kLights>
__device__ __forceinline__ void candidates_direct_body(uint32_t slot, const ResPlanes& curr, const RecPlanes& currRec, Blk blk)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t i;
    if (!tiled_pixel_at(C.W, C.H, blk, i)) return;
    PState path;
    path_init<true>(C, i % C.W, i / C.W, path);
    do path_step<true, kLights>(C, path, currRec, i);
    while (path.flags & kPActive);
    path_finish<true>(path, 0, 1, curr, currRec, i);
}

// kLights as in path_step: the default variant (emissive triangles, power sampler) carries no
// code of the other light configurations.
template <uint32_t kLights>
__global__ void __launch_bounds__(128, 8) k_candidates_direct(uint32_t slot, ResPlanes curr, RecPlanes currRec)
{
    candidates_direct_body<kLights>(slot, curr, currRec, Blk{blockIdx.x, 8u});
}

template <bool kEnv>
__global__ void __launch_bounds__(128, 8) kb_candidates_direct(BatchQueue q, const CandArgs* __restrict__ args)
{
    for (uint32_t t = blockIdx.x; t < q.total; t += gridDim.x)
    {
        const uint32_t inst = batch_instance(q, t);
        const CandArgs& a = args[inst];
        candidates_direct_body<kEnv ? 1u : 0u>(__ldg(q.slot + inst), a.curr, a.currRec, batch_blk(q, inst, t)); // flattened members: power sampler, no analytic lights
    }
}

// ============================================================ environment-map importance
// EnvMapSamplerSetup.cs.slang:48-76: one thread per texel of the 512 x 512 finest mip.
__global__ void __launch_bounds__(256) k_env_importance(EnvMapView E, float* __restrict__ importance)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= kEnvImportanceDim * kEnvImportanceDim) return;
    importance[i] = env_importance_texel(E, i % kEnvImportanceDim, i / kEnvImportanceDim);
}

// Mip m (>= 1) of the importance map from mip m - 1 (Texture::generateMips: 2 x 2 means).
__global__ void __launch_bounds__(256) k_env_reduce(float* __restrict__ importance, uint32_t m)
{
    const uint32_t d = kEnvImportanceDim >> m;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= d * d) return;
    importance[env_mip_offset(m) + i] = env_importance_reduce(importance, m, i % d, i / d);
}

// ============================================================ forward reprojection (splat)
// ReprojectTemporalSamples.rt.slang:64-175.  Writes the destination cell of every source pixel
// and counts splats per cell; the cell lists are built from the targets by a radix sort (pass.cu).
__device__ __forceinline__ void reproject_body(uint32_t slot, const ResPlanes& prev, const RecPlanes& prevRec, uint32_t* __restrict__ targets, uint32_t* __restrict__ counts, Blk blk)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ci;
    if (!tiled_pixel_at(C.W, C.H, blk, ci)) return;
    uint32_t target = kInvalidIndex;
    f3 integrand = load_integrand(prev, ci);
    if (!all_eq0(integrand))
    {
        const uint4* p = prevRec.p + ci;
        uint4 q0 = __ldg(p), q1 = __ldg(p + prevRec.stride), q2 = __ldg(p + 2 * prevRec.stride);
        f2 lensSample = mk2(u2f(q0.z), u2f(q0.w));
        float time = u2f(q1.x);
        HitInfo firstHit; firstHit.w[0] = q2.x; firstHit.w[1] = q2.y; firstHit.w[2] = q2.z; firstHit.w[3] = q2.w;
        const bool valid = hit_valid(firstHit);
        // an environment sample (no primary hit) reprojects by its direction (:110-118)
        if (valid || ((q1.y >> 14) & 1u))
        {
            CameraData cc; dev_orient(C, cc, time);
            f2 lensLocal = mk2(cc.apertureRadius * lensSample.x, cc.apertureRadius * lensSample.y);
            f3 lensWorld = cc.unitU * lensLocal.x + cc.unitV * lensLocal.y;
            Ray nr;
            nr.origin = cc.posW + lensWorld;
            if (valid)
            {
                f3 x1 = dev_sd(C, firstHit, mk3(0.f)).posW;
                nr.dir = normalize(x1 - nr.origin);
                nr.tMin = 0.001f * length(x1 - nr.origin);
                nr.tMax = 0.999f * length(x1 - nr.origin);
            }
            else
            {
                const uint4 q4 = __ldg(p + 4 * prevRec.stride);
                nr.dir = -mk3(u2f(q4.x), u2f(q4.y), u2f(q4.z));
                nr.tMin = 0.001f;
                nr.tMax = kRayTMax;
            }
            f3 camDir = mk3(dot(cc.unitU, nr.dir), dot(cc.unitV, nr.dir), dot(cc.unitW, nr.dir));
            if (camDir.z > 0.001f && dev_visible(C, nr))
            {
                float lw = cc.lenW;
                f2 film = mk2(lensLocal.x + lw * (camDir.x / camDir.z), lensLocal.y + lw * (camDir.y / camDir.z));
                f2 ndc = mk2(film.x / cc.lenU, film.y / cc.lenV);
                f2 nfp = mk2((0.5f * ndc.x + 0.5f) * (float)C.W, (-0.5f * ndc.y + 0.5f) * (float)C.H);
                if (valid_float(C, nfp)) target = (uint32_t)f_floor(nfp.y) * C.W + (uint32_t)f_floor(nfp.x);
            }
        }
    }
    targets[ci] = target;
    if (target != kInvalidIndex) atomicAdd(&counts[target], 1u);
}

__global__ void __launch_bounds__(256, 4) k_reproject(uint32_t slot, ResPlanes prev, RecPlanes prevRec,
                                                   uint32_t* __restrict__ targets, uint32_t* __restrict__ counts)
{
    reproject_body(slot, prev, prevRec, targets, counts, Blk{blockIdx.x, 8u});
}

__global__ void __launch_bounds__(256, 4) kb_reproject(BatchQueue q, const ReprojArgs* __restrict__ args)
{
    for (uint32_t t = blockIdx.x; t < q.total; t += gridDim.x)
    {
        const uint32_t inst = batch_instance(q, t);
        const ReprojArgs& a = args[inst];
        reproject_body(__ldg(q.slot + inst), a.prev, a.prevRec, a.targets, a.counts, batch_blk(q, inst, t));
    }
}

// MultiReprojectTemporalSamples.rt.slang:65-168 (P partitions; targets/counts hold P planes of N)
__global__ void __launch_bounds__(256) k_multi_reproject(uint32_t slot, ResPlanes prev, RecPlanes prevRec,
                                                         uint32_t* __restrict__ targets, uint32_t* __restrict__ counts)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ci;
    const uint32_t N = C.W * C.H;
    if (!tiled_pixel(C.W, C.H, ci)) return;
    const uint32_t P = C.numTimePartitions;
    for (uint32_t i = 0; i < P; i++) targets[(size_t)i * N + ci] = kInvalidIndex;
    f3 integrand = load_integrand(prev, ci);
    if (all_eq0(integrand)) return;
    const uint4* p = prevRec.p + ci;
    uint4 q1 = __ldg(p + prevRec.stride), q2 = __ldg(p + 2 * prevRec.stride);
    float time = u2f(q1.x);
    HitInfo firstHit; firstHit.w[0] = q2.x; firstHit.w[1] = q2.y; firstHit.w[2] = q2.z; firstHit.w[3] = q2.w;
    const bool valid = hit_valid(firstHit);
    // an environment sample (no primary hit) reprojects by its direction (:108-118)
    if (!valid && !((q1.y >> 14) & 1u)) return;
    float fractionalTime = time / C.camera.shutterSpeed;
    float timePartitions = C.camera.shutterSpeed / (float)P;
    f3 x1 = mk3(0.f), envDir = mk3(0.f);
    if (valid) x1 = dev_sd(C, firstHit, mk3(0.f)).posW;
    else
    {
        const uint4 q4 = __ldg(p + 4 * prevRec.stride);
        envDir = -mk3(u2f(q4.x), u2f(q4.y), u2f(q4.z));
    }
    for (uint32_t i = 0; i < P; i++)
    {
        float newTime = (fractionalTime + (float)i) * timePartitions;
        CameraData cc; dev_orient(C, cc, newTime);
        f3 rayDir = valid ? x1 - cc.posW : envDir;
        const float rayLength = valid ? 0.999f : kRayTMax;
        f3 nd = normalize(rayDir);
        float d = dot(nd, cc.unitW);
        if (d <= 0.001f) continue;
        if (!dev_visible(C, mk_ray(cc.posW, rayDir, 0.001f, rayLength))) continue;
        float tanFovY = cc.focalLength == 0.f ? 0.f : cc.frameHeight / cc.focalLength;
        d *= tanFovY;
        f2 offset = mk2(dot(nd, cc.unitU), -dot(nd, cc.unitV));
        f2 ndc = mk2(0.5f + offset.x / (d * cc.aspectRatio), 0.5f + offset.y / d);
        f2 nfp = mk2(ndc.x * (float)C.W, ndc.y * (float)C.H);
        if (!valid_float(C, nfp)) continue;
        uint32_t t = (uint32_t)f_floor(nfp.y) * C.W + (uint32_t)f_floor(nfp.x);
        targets[(size_t)i * N + ci] = t;
        atomicAdd(&counts[(size_t)i * N + t], 1u);
    }
}

// ============================================================ cell lists (canonical order)
// Exclusive scan of the per-cell counts: 1024 threads x 4 items per block, block sums scanned
// by one block, then added back.  Replaces the atomic offset allocation of
// SortReprojectedReservoirs.cs.slang:56-73 with a deterministic prefix sum.
constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* smem, uint32_t& total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1)
    {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem[warp] = x;
    __syncthreads();
    if (warp == 0)
    {
        uint32_t s = (lane < (int)(blockDim.x >> 5)) ? smem[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1)
        {
            uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        smem[lane] = s;
    }
    __syncthreads();
    uint32_t warpPrefix = warp > 0 ? smem[warp - 1] : 0u;
    total = smem[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warpPrefix + x - v;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_tiles(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                             uint32_t* __restrict__ tileSums, uint32_t n)
{
    __shared__ uint32_t smem[32];
    size_t base = (size_t)blockIdx.x * kScanTile + (size_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
    {
        v[k] = (base + k < n) ? in[base + k] : 0u;
        sum += v[k];
    }
    uint32_t total;
    uint32_t pre = block_exclusive_scan(sum, smem, total);
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
    {
        if (base + k < n) out[base + k] = pre;
        pre += v[k];
    }
    if (threadIdx.x == 0) tileSums[blockIdx.x] = total;
}

// One block scans the tile sums (up to kScanTile tiles = 16.7M cells) and writes the grand total.
__global__ void __launch_bounds__(kScanThreads) k_scan_tile_sums(uint32_t* __restrict__ tileSums, uint32_t numTiles, uint32_t* __restrict__ totalOut)
{
    __shared__ uint32_t smem[32];
    size_t base = (size_t)threadIdx.x * kScanItems;
    uint32_t v[kScanItems];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
    {
        v[k] = (base + k < numTiles) ? tileSums[base + k] : 0u;
        sum += v[k];
    }
    uint32_t total;
    uint32_t pre = block_exclusive_scan(sum, smem, total);
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
    {
        if (base + k < numTiles) tileSums[base + k] = pre;
        pre += v[k];
    }
    if (threadIdx.x == 0 && totalOut) *totalOut = total;
}

__global__ void __launch_bounds__(256) k_scan_add(uint32_t* __restrict__ out, const uint32_t* __restrict__ tileSums, uint32_t n)
{
    size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] += tileSums[i / kScanTile];
}

// The cell of each entry of the sorted splat list (the list holds source indices in (cell, source)
// order; entries whose source has no cell, after the last valid one, are left alone).
__global__ void __launch_bounds__(256) k_sorted_cells(const uint32_t* __restrict__ targets, const uint32_t* __restrict__ sorted,
                                                      uint32_t* __restrict__ sortedCell, uint32_t n)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = targets[sorted[i]];
    if (t < n) sortedCell[i] = t;
}

// ============================================================ backup gather (collect)
// CollectTemporalSamples.cs.slang:70-257
__device__ __forceinline__ f2 prev_pixel_from_mvec(const DevCtx& C, const float2* mvec, uint32_t x, uint32_t y)
{
    float2 m = __ldg(&mvec[y * C.W + x]);
    f2 mv = mk2(m.x, m.y);
    mv = (length(mv) < 1e-06f) ? mk2(0.f, 0.f) : mv;
    return mk2((float)x + mv.x * (float)C.W, (float)y + mv.y * (float)C.H);
}

__global__ void __launch_bounds__(128, 4) k_collect(uint32_t slot, const float2* __restrict__ mvec, ResPlanes prev, RecPlanes prevRec,
                                                 ResPlanes inter, RecPlanes interRec, float2* __restrict__ floatingCoords,
                                                 const Shifted* __restrict__ shiftedPaths)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ci;
    if (!tiled_pixel(C.W, C.H, ci)) return;
    uint32_t x = ci % C.W, y = ci / C.W;
    const bool useConf = C.useConfTemporal != 0;
    SampleGen sg = sg_create(x, y, pass_seed(C, 2), C.sgKind);
    f2 prevPixel = prev_pixel_from_mvec(C, mvec, x, y);
    Res dst = res_default();
    Recon dstR = recon_default();
    f2 dstFC = mk2(-1.f, -1.f);
    if (valid_float(C, prevPixel))
    {
        int tlx = (int)f_floor(prevPixel.x), tly = (int)f_floor(prevPixel.y);
        f2 frac = mk2(f_saturate(prevPixel.x - (float)tlx), f_saturate(prevPixel.y - (float)tly));
        if (C.gatherOption == 0u) // Fast
        {
            dstFC = prevPixel;
            float totalConfidence = 0.f;
            for (int ox = 0; ox < 2; ox++)
                for (int oy = 0; oy < 2; oy++)
                {
                    int nx = tlx + ox, ny = tly + oy;
                    if (!valid_int(C, nx, ny)) continue;
                    uint32_t ni = (uint32_t)ny * C.W + (uint32_t)nx;
                    Res nr = load_res(prev, ni);
                    f2 rel = mk2((float)ox + nr.subPixel.x - frac.x, (float)oy + nr.subPixel.y - frac.y);
                    float bw = f_lerp((float)(1 - ox), (float)ox, frac.x) * f_lerp((float)(1 - oy), (float)oy, frac.y);
                    totalConfidence += bw * (useConf ? nr.confidence : 1.f);
                    if (rel.x >= 0.f && rel.x < 1.f && rel.y >= 0.f && rel.y < 1.f)
                    {
                        nr.subPixel = rel;
                        bool sel = res_add_sample(dst, sg, 1.f, nr.integrand, 1.f, nr);
                        if (sel) dstR = load_rec(prevRec, ni);
                    }
                }
            dst.confidence = totalConfidence;
        }
        else if (C.gatherOption == 1u) // Clamped
        {
            float rx = f_round(prevPixel.x), ry = f_round(prevPixel.y);
            dstFC = mk2(rx, ry);
            if (valid_int(C, (int)rx, (int)ry))
            {
                uint32_t pi = (uint32_t)ry * C.W + (uint32_t)rx;
                dst = load_res(prev, pi);
                dstR = load_rec(prevRec, pi);
            }
        }
        else // Robust
        {
            dstFC = prevPixel;
            float totalConfidence = 0.f;
            for (int ox = 0; ox < 2; ox++)
                for (int oy = 0; oy < 2; oy++)
                {
                    int nx = tlx + ox, ny = tly + oy;
                    if (!valid_int(C, nx, ny)) continue;
                    uint32_t ni = (uint32_t)ny * C.W + (uint32_t)nx;
                    Res nr = load_res(prev, ni);
                    Recon nrd = load_rec(prevRec, ni);
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
                    Shifted sp;
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
                            if (!valid_int(C, px, py)) continue;
                            int dx = tx - ox, dy = ty - oy;
                            if (dx == 0 && dy == 0) continue;
                            float tbw = f_lerp((float)(1 - tx), (float)tx, frac.x) * f_lerp((float)(1 - ty), (float)ty, frac.y);
                            uint32_t tIdx = (uint32_t)((dx + 1) + 3 * (dy + 1));
                            tIdx = (tIdx > 4) ? tIdx - 1 : tIdx;
                            const Shifted& tp = shiftedPaths[8 * (size_t)ni + tIdx];
                            float tPHat = luminance(tp.radiance);
                            float tJac = tp.secondaryPathJacobian / nrd.secondaryPathJacobian;
                            float tConf = useConf ? load_confidence(prev, (uint32_t)py * C.W + (uint32_t)px) : 1.f;
                            totalPHat += tbw * tPHat * tJac * tConf;
                        }
                    float misWeight = (totalPHat > 0.f) ? sourceWeight / totalPHat : 0.f;
                    nr.subPixel = rel;
                    recon_update(nrd, sp);
                    nrd.subPixel = rel;
                    float lum = luminance(sp.radiance);
                    bool sel = res_add_sample(dst, sg, misWeight, mk3(lum), shiftedJacobian, nr);
                    if (sel) dstR = nrd;
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
    }
    store_res(inter, ci, dst);
    store_rec(interRec, ci, dstR);
    floatingCoords[ci] = make_float2(dstFC.x, dstFC.y);
}

// RobustReuseOptimization.rt.slang:63-89
// One thread per (pixel, neighbour): the eight lens-copy shifts are independent (the generator
// goes to the shift by value and is never advanced), so blockIdx.y is the neighbour k.
template <bool kEnv>
__global__ void __launch_bounds__(128, 10) k_robust(uint32_t slot, ResPlanes prev, RecPlanes prevRec, Shifted* __restrict__ shiftedPaths)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t idx;
    if (!tiled_pixel(C.W, C.H, idx)) return;
    const int k = (int)blockIdx.y;
    uint32_t x = idx % C.W, y = idx / C.W;
    const int kOff[8][2] = {{-1, -1}, {0, -1}, {1, -1}, {-1, 0}, {1, 0}, {-1, 1}, {0, 1}, {1, 1}};
    SampleGen sg = sg_create(x, y, pass_seed(C, 1), C.sgKind);
    Res pr = load_res(prev, idx);
    int nx = (int)x + kOff[k][0], ny = (int)y + kOff[k][1];
    bool neighborIsValid = valid_float(C, mk2((float)nx, (float)ny));
    bool canShift = any_gt0(pr.integrand);
    if (!(neighborIsValid && canShift)) { shiftedPaths[8 * (size_t)idx + k] = shifted_default(); return; }
    Recon rd = load_rec(prevRec, idx);
    shiftedPaths[8 * (size_t)idx + k] =
        dev_gather_lens_copy<kEnv>(C, sg, rd, rd.time + C.cm.artificialFrameTime, mk2((float)nx + pr.subPixel.x, (float)ny + pr.subPixel.y), rd.lensSample);
}

// ============================================================ temporal resampling
__device__ __forceinline__ float bilinear_confidence(const DevCtx& C, const float2* mvec, const ResPlanes& prev,
                                                     uint32_t x, uint32_t y, float newConfidence, bool useConf)
{
    f2 prevPixel = prev_pixel_from_mvec(C, mvec, x, y);
    int tlx = (int)f_floor(prevPixel.x), tly = (int)f_floor(prevPixel.y);
    f2 frac = mk2(f_saturate(prevPixel.x - (float)tlx), f_saturate(prevPixel.y - (float)tly));
    for (int ox = 0; ox < 2; ox++)
        for (int oy = 0; oy < 2; oy++)
        {
            int nx = tlx + ox, ny = tly + oy;
            if (!valid_int(C, nx, ny)) continue;
            float bw = f_lerp((float)(1 - ox), (float)ox, frac.x) * f_lerp((float)(1 - oy), (float)oy, frac.y);
            newConfidence += bw * (useConf ? load_confidence(prev, (uint32_t)ny * C.W + (uint32_t)nx) : 1.f);
        }
    return f_min(kConfidenceCap, newConfidence);
}

__device__ __forceinline__ void write_color(float4* color, uint32_t i, const Res& r)
{
    if (!color) return;
    f3 c = r.integrand * res_ucw(r); // ResolveReSTIR.cs.slang:45-63
    color[i] = make_float4(c.x, c.y, c.z, 1.f);
}


// GatherTemporalResampling.rt.slang:68-235
template <bool kEnv>
__global__ void __launch_bounds__(128, 6) k_gather_resample(uint32_t slot, const uint4* __restrict__ vbuffer, ResPlanes curr, RecPlanes currRec,
                                                         ResPlanes inter, RecPlanes interRec, const float2* __restrict__ floatingCoords,
                                                         float4* __restrict__ color)
{
    const DevCtx& C = c_ctx[slot];
    uint32_t ri;
    if (!tiled_pixel(C.W, C.H, ri)) return;
    uint32_t x = ri % C.W, y = ri / C.W;
    const bool useConf = C.useConfTemporal != 0;
    SampleGen sg = sg_create(x, y, pass_seed(C, 3), C.sgKind);
    const bool hasDoF = C.camera.apertureRadius > 0.f;
    f2 probs = pixel_dof_probs(C, vbuffer, ri);
    const bool doLensCopy = probs.x > 0.f;
    const bool doPrimaryReconnect = probs.y > 0.f;
    Res dst = res_default();
    Recon dstR = recon_default();
    float2 fcv = __ldg(&floatingCoords[ri]);
    f2 floatingCoord = mk2(fcv.x, fcv.y);
    Res currIn = load_res_rw(curr, ri);
    Recon currInR = load_rec_rw(currRec, ri);
    for (int stage = 0; stage < 2; stage++)
    {
        bool lens = stage == 0;
        if (lens && !doLensCopy) continue;
        if (!lens && !(hasDoF && doPrimaryReconnect)) continue;
        float prob = lens ? probs.x : probs.y;
        Res pr = load_res(inter, ri);
        Recon prd = load_rec(interRec, ri);
        Res cr = (lens || !doLensCopy) ? currIn : dst;
        Recon crd = (lens || !doLensCopy) ? currInR : dstR;
        if (!lens) { dst = res_default(); dstR = recon_default(); }
        float currSampleMIS = 0.f;
        f3 currPHat = mk3(0.f);
        if (any_gt0(cr.integrand))
        {
            float m1 = luminance(cr.integrand) * (useConf ? cr.confidence : 1.f);
            currPHat = cr.integrand;
            Shifted sc = lens ? dev_gather_lens_copy<kEnv>(C, sg, crd, crd.time + C.cm.artificialFrameTime, floatingCoord + cr.subPixel, crd.lensSample)
                              : dev_gather_primary_reconnect<kEnv>(C, sg, crd, crd.time + C.cm.artificialFrameTime, floatingCoord + cr.subPixel, crd.firstHit);
            float sj = lens ? sc.secondaryPathJacobian / crd.secondaryPathJacobian
                            : (sc.lensVertexJacobian * sc.secondaryPathJacobian) / (crd.lensVertexJacobian * crd.secondaryPathJacobian);
            float m2 = luminance(sc.radiance) * sj * (useConf ? pr.confidence : 1.f) * prob;
            m2 = f_isnan(m2) ? 0.f : m2;
            currSampleMIS = (m1 + m2 == 0.f) ? 0.f : m1 / (m1 + m2);
        }
        if (res_add_sample(dst, sg, currSampleMIS, currPHat, 1.f, cr)) dstR = crd;
        float prevSampleMIS = 0.f;
        f3 prevPHat = mk3(0.f);
        float sj = 1.f;
        if (any_gt0(pr.integrand))
        {
            f2 fp = mk2((float)x + pr.subPixel.x, (float)y + pr.subPixel.y);
            Shifted sp = lens ? dev_gather_lens_copy<kEnv>(C, sg, prd, prd.time, fp, prd.lensSample)
                              : dev_gather_primary_reconnect<kEnv>(C, sg, prd, prd.time, fp, prd.firstHit);
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
        if (res_add_sample(dst, sg, prevSampleMIS, prevPHat, sj, pr)) dstR = prd;
    }
    store_res(curr, ri, dst);
    store_rec(currRec, ri, dstR);
    write_color(color, ri, dst);
}

// ResolveReSTIR.cs.slang:45-63 (used when no resampling kernel wrote the colour)
__global__ void __launch_bounds__(256) k_resolve(uint32_t n, ResPlanes curr, float4* __restrict__ color)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Res r = load_res(curr, i);
    write_color(color, i, r);
}

} // namespace rs

// The wavefront kernels and the adjoint share the constant context table, so they live in this
// translation unit.
#include "wavefront.cuh"
#include "adjoint.cuh"

namespace rs {

// Launchers of both variants of the kernels that reach an environment-light branch: with
// env = false the kernel carries none of it (the reference compiles its shaders with USE_ENV_LIGHT
// 0 or 1 the same way).  They live beside the kernels so each launch finds its device code.
#define RS_LIGHT_VARIANTS(kernel)                                                                                  \
    switch (lights & 7u)                                                                                           \
    {                                                                                                              \
    case 0: kernel<0u><<<grid, block, 0, s>>>(slot, curr, currRec); break;                                        \
    case 1: kernel<1u><<<grid, block, 0, s>>>(slot, curr, currRec); break;                                        \
    case 2: kernel<2u><<<grid, block, 0, s>>>(slot, curr, currRec); break;                                        \
    case 3: kernel<3u><<<grid, block, 0, s>>>(slot, curr, currRec); break;                                        \
    case 4: kernel<4u><<<grid, block, 0, s>>>(slot, curr, currRec); break;                                        \
    case 5: kernel<5u><<<grid, block, 0, s>>>(slot, curr, currRec); break;                                        \
    case 6: kernel<6u><<<grid, block, 0, s>>>(slot, curr, currRec); break;                                        \
    default: kernel<7u><<<grid, block, 0, s>>>(slot, curr, currRec); break;                                       \
    }
// lights: bit 0 environment map, bit 1 analytic lights, bit 2 uniform emissive sampler
void launch_k_candidates(uint32_t lights, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, ResPlanes curr, RecPlanes currRec)
{
    RS_LIGHT_VARIANTS(k_candidates)
}
void launch_k_candidates_direct(uint32_t lights, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, ResPlanes curr, RecPlanes currRec)
{
    RS_LIGHT_VARIANTS(k_candidates_direct)
}
#undef RS_LIGHT_VARIANTS
void launch_k_robust(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, ResPlanes prev, RecPlanes prevRec, Shifted* __restrict__ shiftedPaths)
{
    if (env) k_robust<true><<<grid, block, 0, s>>>(slot, prev, prevRec, shiftedPaths);
    else k_robust<false><<<grid, block, 0, s>>>(slot, prev, prevRec, shiftedPaths);
}
void launch_k_gather_resample(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, const uint4* __restrict__ vbuffer, ResPlanes curr, RecPlanes currRec, ResPlanes inter, RecPlanes interRec, const float2* __restrict__ floatingCoords, float4* __restrict__ color)
{
    if (env) k_gather_resample<true><<<grid, block, 0, s>>>(slot, vbuffer, curr, currRec, inter, interRec, floatingCoords, color);
    else k_gather_resample<false><<<grid, block, 0, s>>>(slot, vbuffer, curr, currRec, inter, interRec, floatingCoords, color);
}
void launch_k_so_curr(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K)
{
    if (env) k_so_curr<true><<<grid, block, 0, s>>>(slot, K);
    else k_so_curr<false><<<grid, block, 0, s>>>(slot, K);
}
void launch_k_so_splat(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K)
{
    if (env) k_so_splat<true><<<grid, block, 0, s>>>(slot, K);
    else k_so_splat<false><<<grid, block, 0, s>>>(slot, K);
}
void launch_k_go_curr(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K)
{
    if (env) k_go_curr<true><<<grid, block, 0, s>>>(slot, K);
    else k_go_curr<false><<<grid, block, 0, s>>>(slot, K);
}
void launch_k_go_prev(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K)
{
    if (env) k_go_prev<true><<<grid, block, 0, s>>>(slot, K);
    else k_go_prev<false><<<grid, block, 0, s>>>(slot, K);
}
void launch_k_ms_curr(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, MultiCtx M)
{
    if (env) k_ms_curr<true><<<grid, block, 0, s>>>(slot, M);
    else k_ms_curr<false><<<grid, block, 0, s>>>(slot, M);
}
void launch_k_ms_splat(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, MultiCtx M)
{
    if (env) k_ms_splat<true><<<grid, block, 0, s>>>(slot, M);
    else k_ms_splat<false><<<grid, block, 0, s>>>(slot, M);
}
void launch_k_sb_curr_scatter(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K)
{
    if (env) k_sb_curr_scatter<true><<<grid, block, 0, s>>>(slot, K);
    else k_sb_curr_scatter<false><<<grid, block, 0, s>>>(slot, K);
}
void launch_k_sb_curr_gather(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K)
{
    if (env) k_sb_curr_gather<true><<<grid, block, 0, s>>>(slot, K);
    else k_sb_curr_gather<false><<<grid, block, 0, s>>>(slot, K);
}
void launch_k_sb_backup_gather(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K)
{
    if (env) k_sb_backup_gather<true><<<grid, block, 0, s>>>(slot, K);
    else k_sb_backup_gather<false><<<grid, block, 0, s>>>(slot, K);
}
void launch_k_sb_backup_scatter(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K)
{
    if (env) k_sb_backup_scatter<true><<<grid, block, 0, s>>>(slot, K);
    else k_sb_backup_scatter<false><<<grid, block, 0, s>>>(slot, K);
}
void launch_k_sb_splat_scatter(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K)
{
    if (env) k_sb_splat_scatter<true><<<grid, block, 0, s>>>(slot, K);
    else k_sb_splat_scatter<false><<<grid, block, 0, s>>>(slot, K);
}
void launch_k_sb_splat_gather(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K)
{
    if (env) k_sb_splat_gather<true><<<grid, block, 0, s>>>(slot, K);
    else k_sb_splat_gather<false><<<grid, block, 0, s>>>(slot, K);
}
void launch_k_sp_central(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, SpatialCtx S)
{
    if (env) k_sp_central<true><<<grid, block, 0, s>>>(slot, S);
    else k_sp_central<false><<<grid, block, 0, s>>>(slot, S);
}
void launch_k_sp_neighbor(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, SpatialCtx S)
{
    if (env) k_sp_neighbor<true><<<grid, block, 0, s>>>(slot, S);
    else k_sp_neighbor<false><<<grid, block, 0, s>>>(slot, S);
}

} // namespace rs

namespace rs {

template <typename Kern, typename Args>
static void launch_q(Kern k, dim3 grid, dim3 block, cudaStream_t s, const BatchQueue& q, const void* args)
{
    k<<<grid, block, 0, s>>>(q, static_cast<const Args*>(args));
}

void launch_batched(BatchStage stage, bool env, dim3 grid, dim3 block, cudaStream_t s, const BatchQueue& q, const void* args)
{
    switch (stage)
    {
    case kBatchCandidates:
        if (env) launch_q<decltype(&kb_candidates_direct<true>), CandArgs>(kb_candidates_direct<true>, grid, block, s, q, args);
        else launch_q<decltype(&kb_candidates_direct<false>), CandArgs>(kb_candidates_direct<false>, grid, block, s, q, args);
        break;
#define RS_BATCH_WAVE(st, kern)                                                                                      \
    case st:                                                                                                         \
        if (env) launch_q<decltype(&kern<true>), WaveCtx>(kern<true>, grid, block, s, q, args);                      \
        else launch_q<decltype(&kern<false>), WaveCtx>(kern<false>, grid, block, s, q, args);                        \
        break;
    RS_BATCH_WAVE(kBatchSbCurrScatter, kb_sb_curr_scatter)
    RS_BATCH_WAVE(kBatchSbCurrGather, kb_sb_curr_gather)
    RS_BATCH_WAVE(kBatchSbBackupGather, kb_sb_backup_gather)
    RS_BATCH_WAVE(kBatchSbBackupScatter, kb_sb_backup_scatter)
    RS_BATCH_WAVE(kBatchSbSplatScatter, kb_sb_splat_scatter)
    RS_BATCH_WAVE(kBatchSbSplatGather, kb_sb_splat_gather)
#undef RS_BATCH_WAVE
    case kBatchSpCentral:
        if (env) launch_q<decltype(&kb_sp_central<true>), SpatialCtx>(kb_sp_central<true>, grid, block, s, q, args);
        else launch_q<decltype(&kb_sp_central<false>), SpatialCtx>(kb_sp_central<false>, grid, block, s, q, args);
        break;
    case kBatchSpNeighbor:
        if (env) launch_q<decltype(&kb_sp_neighbor<true>), SpatialCtx>(kb_sp_neighbor<true>, grid, block, s, q, args);
        else launch_q<decltype(&kb_sp_neighbor<false>), SpatialCtx>(kb_sp_neighbor<false>, grid, block, s, q, args);
        break;
    case kBatchVbuffer: launch_q<decltype(&kb_vbuffer), VbufArgs>(kb_vbuffer, grid, block, s, q, args); break;
    case kBatchReproject: launch_q<decltype(&kb_reproject), ReprojArgs>(kb_reproject, grid, block, s, q, args); break;
    case kBatchSbCombine: launch_q<decltype(&kb_sb_combine), WaveColorArgs>(kb_sb_combine, grid, block, s, q, args); break;
    case kBatchSpCombine: launch_q<decltype(&kb_sp_combine), SpatialColorArgs>(kb_sp_combine, grid, block, s, q, args); break;
    default: break;
    }
}

uint32_t batched_threads(BatchStage stage) { return stage == kBatchVbuffer || stage == kBatchReproject ? 256u : 128u; }

template <typename Kern>
static int occupancy(Kern k, uint32_t threads)
{
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, (int)threads, 0) != cudaSuccess) n = 1;
    return n > 0 ? n : 1;
}

int batched_blocks_per_sm(BatchStage stage, bool env)
{
    const uint32_t t = batched_threads(stage);
    switch (stage)
    {
    case kBatchCandidates: return env ? occupancy(kb_candidates_direct<true>, t) : occupancy(kb_candidates_direct<false>, t);
    case kBatchSbCurrScatter: return env ? occupancy(kb_sb_curr_scatter<true>, t) : occupancy(kb_sb_curr_scatter<false>, t);
    case kBatchSbCurrGather: return env ? occupancy(kb_sb_curr_gather<true>, t) : occupancy(kb_sb_curr_gather<false>, t);
    case kBatchSbBackupGather: return env ? occupancy(kb_sb_backup_gather<true>, t) : occupancy(kb_sb_backup_gather<false>, t);
    case kBatchSbBackupScatter: return env ? occupancy(kb_sb_backup_scatter<true>, t) : occupancy(kb_sb_backup_scatter<false>, t);
    case kBatchSbSplatScatter: return env ? occupancy(kb_sb_splat_scatter<true>, t) : occupancy(kb_sb_splat_scatter<false>, t);
    case kBatchSbSplatGather: return env ? occupancy(kb_sb_splat_gather<true>, t) : occupancy(kb_sb_splat_gather<false>, t);
    case kBatchSpCentral: return env ? occupancy(kb_sp_central<true>, t) : occupancy(kb_sp_central<false>, t);
    case kBatchSpNeighbor: return env ? occupancy(kb_sp_neighbor<true>, t) : occupancy(kb_sp_neighbor<false>, t);
    case kBatchVbuffer: return occupancy(kb_vbuffer, t);
    case kBatchReproject: return occupancy(kb_reproject, t);
    case kBatchSbCombine: return occupancy(kb_sb_combine, t);
    case kBatchSpCombine: return occupancy(kb_sp_combine, t);
    default: return 1;
    }
}

} // namespace rs
