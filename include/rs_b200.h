/*
 * rs_b200.h - C ABI of the B200 Reservoir Splatting pass.
 *
 * One rs_pass is the drop-in replacement for one instance of the reference
 * render pass class `ReservoirSplatting : RenderPass`
 * (Source/RenderPasses/ReservoirSplatting/ReservoirSplatting.h:48-279).  The
 * calls map onto that class as follows:
 *
 *   rs_create / rs_destroy      registerPlugin + constructor           ReservoirSplatting.cpp:136-175
 *   rs_set_options              setProperties / parseProperties        ReservoirSplatting.cpp:177-261
 *   rs_set_scene                setScene (scene + light collection)    ReservoirSplatting.cpp:378-397
 *   rs_set_env_map              Scene envMap + EnvMapSampler setup     Scene/Lights/EnvMap.cpp:60-137, Rendering/Lights/EnvMapSampler.cpp:45-113
 *   rs_set_analytic_lights      Scene analytic lights (getLight)       Scene/Lights/Light.cpp:174-397, Rendering/Lights/LightHelpers.slang:67-284
 *   rs_execute                  execute (one frame)                    ReservoirSplatting.cpp:399-509
 *   rs_reset                    reset()                                ReservoirSplatting.cpp:813-820
 *   rs_set_seed                 Python useFixedSeed / fixedSeed        ReservoirSplatting.cpp:142-156
 *   rs_freeze                   Scene::isFrozen (no frame advance)     ReservoirSplatting.cpp:1672-1679
 *   rs_get_buffer / rs_set_buffer  read / restore the pass-owned buffers (reservoirs,
 *                               reconnection data, splat cell lists) ReservoirSplatting.h:236-278
 *   rs_default_options          the defaults of StaticParams / ReSTIRParams / CameraParams
 *                               ReservoirSplatting.h:124-184
 *
 * Threading: one host thread per rs_pass; all device work of a call is issued
 * on the caller's CUDA stream (passed as void*).  No call throws; every call
 * returns an rs_status and rs_last_error_string() describes the last failure
 * on the calling thread.
 */
#ifndef RS_B200_H
#define RS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(_WIN32)
#define RS_API __declspec(dllexport)
#else
#define RS_API __attribute__((visibility("default")))
#endif

typedef enum rs_status {
    RS_OK = 0,
    RS_INVALID_ARG = 1,   /* bad pointer, size or option value */
    RS_OOM = 2,           /* device allocation failed */
    RS_CUDA_ERROR = 3,    /* a CUDA runtime call failed */
    RS_DEVICE_FAULT = 4,  /* a kernel set the device status word (iteration cap hit) */
    RS_NOT_READY = 5      /* no scene set */
} rs_status;

/* TemporalReuse (ShiftOptions.slang:34-40) */
enum { RS_GATHER_ONLY = 0, RS_SCATTER_ONLY = 1, RS_SCATTER_BACKUP = 2, RS_MULTI_SCATTER = 3 };
/* GatherMechanism (ShiftOptions.slang:62-67) */
enum { RS_GATHER_FAST = 0, RS_GATHER_CLAMPED = 1, RS_GATHER_ROBUST = 2 };
/* ScatterBackupMIS (ShiftOptions.slang:49-53) */
enum { RS_MIS_BALANCE = 0, RS_MIS_PAIRWISE = 1 };
/* MISHeuristic (Params.slang:48-53); PowerExp uses rs_options.misPowerExponent (0.01 .. 10) */
enum { RS_MIS_HEURISTIC_BALANCE = 0, RS_MIS_HEURISTIC_POWER_TWO = 1, RS_MIS_HEURISTIC_POWER_EXP = 2 };
/* EmissiveLightSamplerType (EmissiveLightSamplerType.slangh:36-44): Uniform, LightBVH, Power (default) */
enum { RS_EMISSIVE_UNIFORM = 0, RS_EMISSIVE_LIGHT_BVH = 1, RS_EMISSIVE_POWER = 2 };
/* sampleGenerator: SAMPLE_GENERATOR_TINY_UNIFORM = 0 (reference default); 2 = PCG32 */
enum { RS_SG_TINY_UNIFORM = 0, RS_SG_PCG32 = 2 };

/* Property keys of ReservoirSplatting.cpp:99-131 plus the UI-only knobs of
 * ReservoirSplatting.h:159-184.  Field names follow the property names. */
typedef struct rs_options {
    uint32_t samplesPerPixel;            /* 1..16 */
    uint32_t maxSurfaceBounces;          /* <= 254 */
    uint32_t maxDiffuseBounces;
    uint32_t maxSpecularBounces;
    uint32_t maxTransmissionBounces;
    uint32_t sampleGenerator;            /* RS_SG_* */
    uint32_t useFixedSeed;
    uint32_t fixedSeed;
    uint32_t useRussianRoulette;
    uint32_t misHeuristic;               /* RS_MIS_HEURISTIC_* */
    float misPowerExponent;
    uint32_t disableCaustics;
    float specularRoughnessThreshold;
    uint32_t enableTemporalResampling;
    uint32_t enableSpatialResampling;
    uint32_t temporalReuse;              /* RS_GATHER_ONLY .. RS_MULTI_SCATTER */
    uint32_t scatterBackupMISOption;     /* RS_MIS_BALANCE / RS_MIS_PAIRWISE */
    uint32_t gatherOption;               /* RS_GATHER_FAST / CLAMPED / ROBUST */
    uint32_t numTimePartitions;          /* 1..8 */
    uint32_t useConfidenceWeightsTemporally;
    uint32_t numSpatialIterations;
    float spatialGatherRadius;
    uint32_t neighborCount;
    uint32_t useConfidenceWeightsSpatially;
    float artificialFrameTime;           /* seconds between two frames' cameras */
    uint32_t frameWidth;                 /* outputSize, <= 4096 */
    uint32_t frameHeight;                /* <= 4096 */
    uint32_t emissiveSampler;            /* RS_EMISSIVE_* (EmissiveLightSamplerType); LightBVH is not built */
} rs_options;

/* StandardMaterial parameters; 64 bytes.  flags bit 0 = double sided; bit 1 = the spec-gloss
 * shading model (ShadingModel::SpecGloss, StandardMaterial.slang:88-94, what Falcor's OBJ import
 * makes): baseColor is the diffuse colour, specular[3] the specular colour, `roughness` holds the
 * glossiness and metallic is derived; without bit 1 the model is metal-rough and specular[] is
 * unused. */
typedef struct rs_material {
    float baseColor[3];
    float roughness;                     /* glossiness with the spec-gloss model */
    float emissive[3];                   /* radiance, emissive factor included */
    float metallic;                      /* metal-rough only */
    float ior;
    uint32_t flags;
    float specular[3];                   /* spec-gloss only */
    float reserved[3];
} rs_material;

/* Flattened world-space triangle soup (the ray-traced geometry of a Falcor scene). */
typedef struct rs_scene_desc {
    uint32_t numTriangles;
    const float* positions;              /* host, 9 floats per triangle (p0, p1, p2) */
    const uint32_t* materialIds;         /* host, one per triangle */
    uint32_t numMaterials;
    const rs_material* materials;        /* host */
} rs_scene_desc;

/* Camera of the current frame (CameraData.slang:35-72 subset). */
typedef struct rs_camera {
    float position[3];
    float target[3];
    float up[3];
    float focalLength;                   /* mm */
    float frameHeight;                   /* mm */
    float aspectRatio;
    float focalDistance;
    float apertureRadius;
    float shutterSpeed;                  /* seconds */
    float nearZ;
    float farZ;
} rs_camera;

/* Per-frame inputs/outputs (the reflect() channels, ReservoirSplatting.cpp:64-96).
 *
 * mvec and vbuffer are the pass's two inputs (`mvec` RG32F and `vbuffer` PackedHitInfo,
 * ReservoirSplatting.cpp:64-72).  When given, the pass reads them in place of its own: the motion
 * vectors drive the backup gather and the scatter's motion checks; the primary hits give the
 * circle of confusion that splits depth-of-field gathers between the lens-vertex copy and the
 * primary-hit reconnection (GatherTemporalResampling.rt.slang:79, SpatialResampling.rt.slang:80).
 * A hit is four words (HitInfo.slang's type, primitive and barycentrics): word 0 = hit type
 * (0 miss, 1 triangle), word 1 = triangle index in the scene's order, words 2, 3 = barycentrics
 * u, v as float bits (the layout rs_get_buffer(RS_BUF_VBUFFER) returns).
 * When both are given the pass launches no primary-hit kernel of its own, and RS_BUF_MVEC /
 * RS_BUF_VBUFFER keep the values of the last frame that computed them. */
typedef struct rs_frame_desc {
    rs_camera camera;
    const float* mvec;                   /* optional device float2[W*H]; NULL: computed by the pass */
    const uint32_t* vbuffer;             /* optional device uint4[W*H] packed hits; NULL: computed by the pass */
    float* color;                        /* device float4[W*H] output (may be NULL if colorHost set) */
    float* colorHost;                    /* optional host float4[W*H]; copied back and synchronised */
    uint32_t sceneShouldReset;           /* Scene::shouldReset(): restart the temporal history */
} rs_frame_desc;

/* Buffers readable with rs_get_buffer (canonical host layouts):
 *   reservoirs      8 floats / pixel: integrand.xyz, totalWeight, subPixel.xy, confidence, 0
 *   reconnection    28 words / pixel (layout in rs_get_buffer's documentation)
 *   cellCounters    uint32 / pixel        cellOffsets  uint32 / pixel
 *   sortedSplats    uint32 source-pixel index per splat, cells in pixel order, sources ascending
 *   floatingCoords  float2 / pixel        mvec float2 / pixel      vbuffer uint4 / pixel
 *   splatTargets    uint32 / source pixel: destination cell or 0xffffffff */
typedef enum rs_buffer_id {
    RS_BUF_CURR_RESERVOIRS = 0,
    RS_BUF_CURR_RECONNECTION = 1,
    RS_BUF_PREV_RESERVOIRS = 2,
    RS_BUF_PREV_RECONNECTION = 3,
    RS_BUF_CELL_COUNTERS = 4,
    RS_BUF_CELL_OFFSETS = 5,
    RS_BUF_SORTED_SPLATS = 6,
    RS_BUF_FLOATING_COORDS = 7,
    RS_BUF_MVEC = 8,
    RS_BUF_VBUFFER = 9,
    RS_BUF_SPLAT_TARGETS = 10,
    RS_BUF_CANDIDATE_RESERVOIRS = 11,
    RS_BUF_CANDIDATE_RECONNECTION = 12,
    RS_BUF_BACKUP_RESERVOIRS = 13,
    RS_BUF_BACKUP_RECONNECTION = 14,
    RS_BUF_ENV_IMPORTANCE = 15           /* float, the env map's importance mips 512^2 .. 1 back to back */
} rs_buffer_id;

typedef struct rs_pass rs_pass;

RS_API void rs_default_options(rs_options* opts);
RS_API rs_status rs_create(const rs_options* opts, rs_pass** out);
RS_API rs_status rs_destroy(rs_pass* pass);
RS_API rs_status rs_set_options(rs_pass* pass, const rs_options* opts);
RS_API rs_status rs_set_scene(rs_pass* pass, const rs_scene_desc* scene);
/* Environment map light (Falcor EnvMap + EnvMapSampler).  A lat-long map of width x height RGBA
 * float texels (host, row-major, row 0 at the top: v = 0 looks along +y), centred on -z and wrapping
 * clockwise; radiance = bilinear texel value * intensity * tint, looked up after the rotation
 * (XYZ Euler angles in degrees, EnvMap::setRotation).  The pass builds the 512 x 512 importance map
 * with its mip chain on the device (64 luminance samples per texel) and samples the map for NEE in
 * proportion to it; light types are picked with equal probability when the scene also has emissive
 * triangles.  The light is used when intensity > 0 (Scene::useEnvLight).  NULL or width == 0 removes
 * it.  Synchronous; the next frame uses the new map. */
typedef struct rs_env_map {
    uint32_t width, height;
    const float* texels;                 /* host, 4 floats per texel (the fourth is ignored) */
    float intensity;
    float tint[3];
    float rotation[3];                   /* degrees */
} rs_env_map;
RS_API rs_status rs_set_env_map(rs_pass* pass, const rs_env_map* env);

/* Analytic lights (Scene::getLight / useAnalyticLights; Scene/Lights/Light.cpp, LightData.slang),
 * sampled by next-event estimation only (PathTracer.slang:567-599): uniform pick of a light, then
 * LightHelpers.slang's sample of its type.  The light-type selection gives the environment map,
 * the emissive triangles and the analytic lights equal probability when present.  As in the
 * reference, a light sampled at the primary hit leaves the reconnection record without a light
 * vertex (PathTracer.slang:1079-1104), and a point or directional light's stored radiance is
 * Li * pdf = 0, so shifts of such samples contribute nothing; the sample still counts at its own
 * pixel.  The reference's arithmetic for those records is kept as it is, and with it the few NaN
 * values it makes in shifts (a delta light sampled at the second vertex stores lightPdf = 0, so the
 * length-3 reconnection multiplies 0 by totalBsdf / 0, ShiftMapping.slang:479-493; a light vertex
 * left unset loads as a zero vertex, LoadShadingData.slang:69-74, whose Jacobian is 0 / 0): some
 * pixels of scenes with analytic lights and temporal or spatial reuse come out NaN, as they would
 * in the reference.  Synchronous; replaces the previous list (count 0 removes them).  rs_backward
 * rejects scenes with analytic lights. */
typedef enum rs_light_type {
    RS_LIGHT_POINT = 0,                  /* point, or spot when openingAngle < pi */
    RS_LIGHT_DIRECTIONAL = 1,
    RS_LIGHT_DISTANT = 2,                /* a cone of directions of half-angle `angle` */
    RS_LIGHT_RECT = 3,                   /* the quad [-1, 1]^2 x {0} of object space, one-sided (+z) */
    RS_LIGHT_DISC = 4,                   /* the unit disc of the z = 0 plane, one-sided (+z) */
    RS_LIGHT_SPHERE = 5                  /* the unit sphere */
} rs_light_type;
typedef struct rs_analytic_light {
    uint32_t type;                       /* rs_light_type */
    float intensity[3];                  /* point: intensity; the others: radiance */
    float position[3];                   /* point */
    float direction[3];                  /* point (spot axis), directional, distant: the direction light travels */
    float openingAngle;                  /* point: spot half-angle in radians, clamped to [0, pi] (pi: all directions) */
    float penumbraAngle;                 /* point: smooth edge inside the cone, clamped to [0, openingAngle] */
    float angle;                         /* distant: half-angle subtended, clamped to [0, pi/2] */
    float transform[16];                 /* rect, disc, sphere: row-major 4x4 object-to-world matrix */
    float scaling[3];                    /* rect, disc, sphere: object-space scale applied first */
} rs_analytic_light;
RS_API rs_status rs_set_analytic_lights(rs_pass* pass, const rs_analytic_light* lights, uint32_t count);
RS_API rs_status rs_execute(rs_pass* pass, const rs_frame_desc* frame, void* cudaStream);
/* Latency of host colour outputs (no reference counterpart: the reference presents on the GPU).
 * 0 (default): rs_execute with frame.colorHost returns once the image is in host memory.
 * 1: rs_execute renders into one of two pass-owned device images, queues the copy to
 * frame.colorHost on the pass's own copy stream behind the frame, and returns once the PREVIOUS
 * frame's copy is complete, so each copy overlaps the next frame's kernels; frame.colorHost must
 * stay valid until the next rs_execute or rs_wait_host_output returns, which also reports that
 * frame's device status (RS_DEVICE_FAULT).  frame.color, when also given, receives a device copy.
 * rs_wait_host_output completes the copy in flight and orders the last stream after it. */
RS_API rs_status rs_set_host_output_latency(rs_pass* pass, uint32_t frames);
RS_API rs_status rs_wait_host_output(rs_pass* pass);
RS_API rs_status rs_reset(rs_pass* pass);
RS_API rs_status rs_set_seed(rs_pass* pass, uint32_t useFixedSeed, uint32_t fixedSeed);
RS_API rs_status rs_freeze(rs_pass* pass, uint32_t frozen);
/* Copies a pass buffer to host memory (synchronises the pass's last stream).
 * *bytes is the destination capacity in, and the number of bytes written (or
 * needed when dst is NULL) out.
 *
 * Reservoirs (PathReservoir, Reservoir.slang:73-132): 8 words per pixel, float integrand.xyz,
 * totalWeight, subPixel.xy, confidence, 0.
 * Reconnection records (ReconnectionData.slang:89-166): 28 words per pixel,
 *   0-3   float subPixel.xy, lensSample.xy        4  float time
 *   5     flags: pathLength (bits 0-7), firstBSDFComponentType (8-9), secondBSDFComponentType
 *         (10-11), transmissionEvent (12), lightIsNEE (13), lightIsDistant (14), and the adjoint's
 *         suffix state on entering the third vertex (15-26: bounce counters diffuse, specular,
 *         transmission, two bits each, then path flags 4..128 shifted down by 2)
 *   6     float lightPdf                             7  float subPixelJacobian
 *   8-11  firstHit (HitInfo, four words)            12-15 secondHit
 *   16-18 float firstWi                              19 float lensVertexJacobian
 *   20-22 float secondWo                             23 float secondaryPathJacobian
 *   24-26 float irradiance                           27 the sample generator's state on entering
 *                                                       the third vertex (adjoint; 0 before it)
 * Bits 15-26 of word 5 and word 27 have no reference counterpart (its record has no such fields). */
RS_API rs_status rs_get_buffer(rs_pass* pass, rs_buffer_id id, void* dst, size_t* bytes);
/* Restores a reservoir / reconnection buffer from host memory (checkpoint restore). */
RS_API rs_status rs_set_buffer(rs_pass* pass, rs_buffer_id id, const void* src, size_t bytes);
/* Kernel timing of the last rs_execute: per-stage device milliseconds (CUDA events)
 * when timing is enabled with rs_enable_stage_timing.  Names are NUL-separated. */
RS_API rs_status rs_enable_stage_timing(rs_pass* pass, uint32_t enable);
RS_API rs_status rs_get_stage_times(rs_pass* pass, float* ms, uint32_t* count, char* names, size_t namesBytes);
/* Number of kernel launches issued by the last rs_execute. */
RS_API uint32_t rs_last_launch_count(rs_pass* pass);
RS_API const char* rs_last_error_string(void);

/* Batched instances (no reference counterpart: the reference renders one pass per render graph).
 * rs_batch_execute renders one frame of every member with one CUDA graph launch on `cudaStream`;
 * the members' stage chains are graph branches that run concurrently.  frames[i] belongs to
 * passes[i] and must carry a device colour buffer; graphs are cached per set of colour buffers and
 * per buffer-parity pattern, so keep the buffers stable across frames.  The call returns after the
 * launch; the previous batch frame is awaited before a member's context is rewritten.  frames[i].mvec
 * and .vbuffer work as in rs_execute; the graph holds their pointers too.  Changing a member's
 * options, scene, environment map or size between two calls drops the cached graphs. */
typedef struct rs_batch rs_batch;
RS_API rs_status rs_batch_create(rs_pass* const* passes, uint32_t count, rs_batch** out);
RS_API rs_status rs_batch_execute(rs_batch* batch, const rs_frame_desc* frames, void* cudaStream);
RS_API rs_status rs_batch_destroy(rs_batch* batch);
RS_API uint32_t rs_batch_launch_count(rs_batch* batch);

/* The flattened batch form.  When every member renders ScatterBackup with the Clamped gather and one
 * sample per pixel, with the same spatial settings and environment-light state, past its first
 * frame and not frozen, rs_batch_execute runs each stage as ONE launch over all members: a flattened
 * work queue (member k owns work items [start[k], start[k+1]), each one block of its own grid) that
 * persistent kernels stride over, reading each member's context and buffers from device tables
 * built at capture.  Otherwise (or with rs_batch_set_flatten(batch, 0)) each member's stage chain is
 * a graph branch.  Results are bit-identical either way.  rs_batch_last_flattened tells which form
 * the last rs_batch_execute used.
 *
 * Tuning: each stage's warp tile width (8, 16 or 32: a warp covers tw x 32/tw pixels) per
 * resolution and its grid form (0 persistent: SMs x resident blocks; 1: one block per work item).
 * rs_batch_tune renders one frame eagerly (synchronous) while timing every choice of every stage in
 * place and keeps the fastest; rs_batch_get_tuning / rs_batch_set_tuning read and restore the choices
 * (the Python layer caches them in a JSON file).  Entries with width = height = 0 carry a stage's
 * grid form; the others a tile width for that resolution.  Stages: 0 candidates, 1-6 the ScatterBackup
 * shifts (current scatter, current gather, backup gather, backup scatter, splat scatter, splat
 * gather), 7-8 spatial central and neighbour shifts, 9 primary hits, 10 reprojection, 11 ScatterBackup
 * combine (not tuned: it updates its input in place), 12 spatial combine. */
typedef struct rs_batch_tuning_entry {
    uint32_t stage;
    uint32_t width, height;  /* 0, 0: the stage's grid form */
    uint32_t tile;           /* 8, 16 or 32 */
    uint32_t grid;           /* 0 persistent, 1 one block per work item */
    float ms;                /* the tuning trial's time of the chosen tile (informative) */
} rs_batch_tuning_entry;
RS_API rs_status rs_batch_set_flatten(rs_batch* batch, uint32_t enable);
RS_API uint32_t rs_batch_last_flattened(rs_batch* batch);
RS_API rs_status rs_batch_tune(rs_batch* batch, const rs_frame_desc* frames, void* cudaStream);
RS_API rs_status rs_batch_get_tuning(rs_batch* batch, rs_batch_tuning_entry* out, uint32_t* count);
RS_API rs_status rs_batch_set_tuning(rs_batch* batch, const rs_batch_tuning_entry* entries, uint32_t count);

/* Moving geometry (Falcor's animated-scene update, done by the caller).  rs_update_geometry moves
 * every triangle to `positions` (9 floats per triangle, the scene's count; host memory, or device
 * memory of the current device when onDevice != 0) for the next rs_execute: the previous positions
 * give that frame's motion vectors (Scene::getPrevPosW, VBufferRT.slang:84), both BVHs are refitted
 * in place (the topology of rs_set_scene stays; rebuild with rs_set_scene after large changes) and
 * light records follow their triangles, with the power sampler's weights of the last
 * rs_set_scene / rs_set_materials.  Call it at most once per frame; stream-ordered on cudaStream. */
RS_API rs_status rs_update_geometry(rs_pass* pass, const float* positions, uint32_t numTriangles, uint32_t onDevice, void* cudaStream);

/* Ray-query diagnostics (no reference counterpart).  rs_debug_trace_rays: closest hits of n host
 * rays (8 floats each: origin.xyz, direction.xyz, tMin, tMax) against the pass's BVH: prim[n] (-1 on
 * a miss), tuv[3n], counts[2n] = nodes visited and triangles tested.  rs_debug_bvh_shape: {nodes,
 * depth, internal children, leaf children, leaf triangles, surface-area cost}.  Both synchronise. */
RS_API rs_status rs_debug_trace_rays(rs_pass* pass, const float* rays, uint32_t n, int32_t* prim, float* tuv, uint32_t* counts);
RS_API rs_status rs_debug_bvh_shape(rs_pass* pass, double* out6);
/* The library's own sort and scan on host data (no reference counterpart; synchronous, allocates):
 * rs_debug_sort_keys64: order[i] = the index of the i-th smallest of n keys over their low keyBits
 * bits, equal keys in ascending index order (the stable radix sort that orders the BVH build's
 * Morton codes); rs_debug_sort_keys32: the same for 32-bit keys with every key >= clampMax treated
 * as clampMax and sorted last (the cell-list sort of the temporal scatter, clampMax = cells);
 * rs_debug_scan: out[i] = values[0] + ... + values[i - 1]. */
RS_API rs_status rs_debug_sort_keys64(const uint64_t* keys, uint32_t n, uint32_t keyBits, uint32_t* order);
RS_API rs_status rs_debug_sort_keys32(const uint32_t* keys, uint32_t n, uint32_t clampMax, uint32_t* order);
RS_API rs_status rs_debug_scan(const uint32_t* values, uint32_t n, uint32_t* out);
/* Binary-tree builder for the next rs_set_scene (no reference counterpart: the reference traces with
 * the driver's RT acceleration structures): 0 = PLOC clustering (the default, the better tree),
 * 1 = LBVH (Karras 2012 radix tree over the same Morton order).  Hits do not depend on it. */
RS_API rs_status rs_set_bvh_builder(rs_pass* pass, uint32_t builder);
/* Ray-query counts per stage of the last frame rendered with stage timing on (no reference
 * counterpart): rays[2i], rays[2i+1] = closest-hit and visibility queries of stage i, in the order of
 * rs_get_stage_times; *count = stages.  Only a library built with -DRS_RAY_STATS counts (build.py
 * build_ray_stats; bench.py --ray-stats); the default library reports *count = 0.  Synchronises. */
RS_API rs_status rs_debug_stage_rays(rs_pass* pass, uint64_t* rays, uint32_t* count);

/* Path-replay adjoint (no reference counterpart: the reference pass renders forward only).
 *
 * A pixel's colour is f(y) * W, y being the path its final reservoir selected.  rs_backward holds
 * each pixel's y, W, sampling densities and MIS weights at their rendered values and
 * differentiates f(y) with respect to every material's baseColor (per channel), roughness, metallic
 * and emissive radiance (per channel).  E[df(y)/dtheta * W] is the derivative of the pixel integral, so
 * the gradient is unbiased.  Only the final reservoirs of a frame are needed: rs_checkpoint copies
 * them (rs_checkpoint_bytes = 144 bytes per pixel) and rs_backward recomputes the rest.  A path of
 * four or more vertices is re-run from its third vertex with the sample-generator state, bounce
 * counters and flags its record saved there (word 27 and bits 15-26 of word 5), which needs the
 * TinyUniform generator.  Where the suffix cannot be re-run (a delta lobe past x2, more than 8 BSDF
 * vertices, the PCG32 generator, or geometry moved since the record was made) it is held fixed at
 * the record's radiance, x1 and x2 are still differentiated, and the path is counted.  The scene may be lit by emissive triangles and an environment map, whose
 * radiance is held fixed (no analytic lights); ior is not differentiated.  For a spec-gloss
 * material baseColor is its diffuse colour and the roughness slot its glossiness; its specular
 * colour is held fixed and its metallic slot gets no gradient.
 *
 *   rs_set_materials   replace material parameters in place (same count; geometry and BVH stay)
 *   rs_checkpoint      copy the last frame's final reservoirs to caller device memory
 *   rs_backward        gradMaterials[m * 8 + k] += d loss / d (baseColor.xyz, roughness, emissive.xyz, metallic)
 *                      for d loss / d colour `gradColor` (device float4 per pixel); checkpoint NULL
 *                      means the last frame; the materials must be those the frame used
 *   rs_backward_stats  read and clear {paths replayed, suffixes held fixed, emitter not found, value mismatch} */
RS_API rs_status rs_set_materials(rs_pass* pass, const rs_material* materials, uint32_t count);
RS_API rs_status rs_checkpoint_bytes(rs_pass* pass, size_t* bytes);
RS_API rs_status rs_checkpoint(rs_pass* pass, void* dstDevice, void* cudaStream);
RS_API rs_status rs_backward(rs_pass* pass, const void* checkpointDevice, const float* gradColor, float* gradMaterials,
                             void* cudaStream);
RS_API rs_status rs_backward_stats(rs_pass* pass, uint64_t* stats4);

/* Frame output: the ToneMapper pass followed by the FrameDumper pass's 8-bit sRGB conversion
 * (RenderPasses/ToneMapper/ToneMapping.ps.slang:45-173, ToneMapper.cpp:538-550,
 * FrameDumper.cpp:80-90,151-158).  rs_tonemap reads width*height float4 colours (device memory,
 * e.g. rs_frame_desc.color) and writes width*height RGBA8 texels (device memory, R in the low
 * byte): auto exposure (key 0.042 over the mean log2 luminance, from the image itself), the
 * exposure scale 2^exposureCompensation (times filmSpeed/100 / (shutter * fNumber^2) without auto
 * exposure), the operator, the optional clamp, then sRGB encoding to 8 bits; alpha is stored
 * linearly.  With autoExposure, workspaceDev is device memory of rs_tonemap_workspace_bytes().
 * White balance is not implemented.  Work is enqueued on `cudaStream`; nothing is allocated. */
typedef enum rs_tonemap_operator {
    RS_TONEMAP_LINEAR = 0,
    RS_TONEMAP_REINHARD = 1,
    RS_TONEMAP_REINHARD_MODIFIED = 2,
    RS_TONEMAP_HEJI_HABLE_ALU = 3,
    RS_TONEMAP_HABLE_UC2 = 4,
    RS_TONEMAP_ACES = 5
} rs_tonemap_operator;

typedef struct rs_tonemap_options {
    uint32_t op;                /* rs_tonemap_operator (ToneMapperOperator) */
    float exposureCompensation; /* EV steps */
    uint32_t autoExposure;
    float filmSpeed, fNumber, shutter; /* manual exposure (shutter = reciprocal seconds) */
    uint32_t clamp;
    float whiteMaxLuminance;    /* ReinhardModified */
    float whiteScale;           /* HableUc2 */
    uint32_t whiteBalance;      /* colour grading: white balance to whitePoint (ToneMapper.cpp:530-536) */
    float whitePoint;           /* Kelvin, 1905 .. 25000 (default 6500: identity) */
} rs_tonemap_options;

RS_API void rs_tonemap_default_options(rs_tonemap_options* options);
RS_API size_t rs_tonemap_workspace_bytes(void);
/* The 3x3 colour transform rs_tonemap applies after auto exposure (row-major, out[9]): the white
 * balance matrix times the exposure scale (ToneMapper::updateColorTransform).  Host only. */
RS_API rs_status rs_tonemap_color_transform(const rs_tonemap_options* options, float* out9);
RS_API rs_status rs_tonemap(const void* colorDev, uint32_t width, uint32_t height, const rs_tonemap_options* options, void* rgba8Dev,
                            void* workspaceDev, void* cudaStream);

/* Allocation-free cell-list build.  This call has no counterpart in the reference.
 *
 * It exists for callers that cannot allocate device memory when they run: a host that hands
 * out all device memory from its own fixed pool, an allocator-free real-time loop, or a plug-in
 * invoked while its host captures a CUDA graph.  The rs_pass calls allocate their buffers on the
 * first frame at a given size; this call never calls cudaMalloc, cudaFree or any other
 * allocating routine.  Its temporaries live in a 9 MiB array compiled into the library, which
 * every GPU that loads the library holds until the process exits.
 *
 * Input:  targets[numSplats], device memory: the cell of each splat, or any value >= numCells
 *         (0xFFFFFFFF, say) for a splat that lands in no cell.
 * Output: counts[numCells] (splats per cell), offsets[numCells] (exclusive prefix sum of the
 *         counts) and sorted[numSplats] (splat indices grouped by cell, ascending within a cell,
 *         in the first sum(counts) entries; the splats without a cell follow in ascending order),
 *         all device memory on the current device.  The work per splat is bounded (a stable radix
 *         sort by cell), however many splats share one cell.
 * These are the lists rs_execute builds for the temporal scatter, in the same order.
 *
 * Limits: 1 <= numCells <= RS_CELL_LISTS_STATIC_MAX and numSplats <= RS_CELL_LISTS_STATIC_MAX
 * (2^21, enough for a 1920x1080 frame); larger sizes return RS_INVALID_ARG before any device work.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress with that
 * device current); make that first call before any stream capture begins.  Work is enqueued on
 * `cudaStream` and the call returns without waiting.  All calls on a device share the one array:
 * calls whose work overlaps on the GPU (other streams, other host threads) race and corrupt each
 * other's lists, so order them on one stream or with events. */
#define RS_CELL_LISTS_STATIC_MAX (1u << 21)
RS_API rs_status rs_build_cell_lists_static(const uint32_t* targets, uint32_t numSplats, uint32_t numCells,
                                            uint32_t* counts, uint32_t* offsets, uint32_t* sorted, void* cudaStream);

#ifdef __cplusplus
}
#endif

#endif /* RS_B200_H */
