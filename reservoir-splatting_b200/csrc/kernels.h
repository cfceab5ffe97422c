// Kernel declarations of the Reservoir Splatting pass (definitions in kernels.cu).
#pragma once
#include "pass_device.cuh"
#include "core/material_grad.h"

namespace rs {

__global__ void k_vbuffer(uint32_t slot, uint4* vbuffer, float2* mvec);
__global__ void k_camera_table(uint32_t slot, CameraTable* table);
#ifdef RS_RAY_STATS
cudaError_t ray_stats_take(unsigned long long out[2], cudaStream_t s);
#endif
__global__ void k_env_importance(EnvMapView E, float* importance);
__global__ void k_env_reduce(float* importance, uint32_t m);
__global__ void k_reproject(uint32_t slot, ResPlanes prev, RecPlanes prevRec, uint32_t* targets, uint32_t* counts);
__global__ void k_multi_reproject(uint32_t slot, ResPlanes prev, RecPlanes prevRec, uint32_t* targets, uint32_t* counts);
__global__ void k_scan_tiles(const uint32_t* in, uint32_t* out, uint32_t* tileSums, uint32_t n);
__global__ void k_scan_tile_sums(uint32_t* tileSums, uint32_t numTiles, uint32_t* totalOut);
__global__ void k_scan_add(uint32_t* out, const uint32_t* tileSums, uint32_t n);
__global__ void k_sorted_cells(const uint32_t* targets, const uint32_t* sorted, uint32_t* sortedCell, uint32_t n);
__global__ void k_collect(uint32_t slot, const float2* mvec, ResPlanes prev, RecPlanes prevRec, ResPlanes inter, RecPlanes interRec,
                          float2* floatingCoords, const Shifted* shiftedPaths);
__global__ void k_resolve(uint32_t n, ResPlanes curr, float4* color);

__global__ void k_backward(uint32_t slot, ResPlanes res, RecPlanes rec, const float4* gradColor, double* acc, uint32_t numMaterials,
                           unsigned long long* stats);
__global__ void k_grad_flush(const double* acc, float* grad, uint32_t n);
constexpr uint32_t kAdjointThreads = 128;        // k_backward block size
constexpr uint32_t kAdjointBlocksPerSm = 10;     // k_backward's resident blocks per SM (launch bounds and grid)
constexpr uint32_t kAdjointSharedDoubles = 6016; // k_backward stages numMaterials x 8 sums in shared memory up to this (47 KB)

// Blocks of `threads` (a multiple of 64) covering a W x H image for tiled_pixel.
inline uint32_t tiled_blocks(uint32_t W, uint32_t H, uint32_t threads)
{
    const uint32_t rows = (threads / 32u) * 2u;
    return ((W + 15u) / 16u) * ((H + rows - 1u) / rows);
}

constexpr uint32_t kMaxPassSlots = 64; // passes alive at once (size of the constant context table)
cudaError_t upload_ctx(uint32_t slot, const DevCtx* hostPinned, cudaStream_t s);

constexpr int kScanTileElems = 4096; // k_scan_tiles: 1024 threads x 4 items

// Stored shift results: five uint4 planes (radiance + jacobians + fractional pixel + primary hit +
// lens sample + first ray direction), plane k at p + k * stride.
struct ShiftPlanes { uint4* p; size_t stride; };

// Buffers of the wavefront ScatterBackup resampling (wavefront.cu).
struct WaveCtx
{
    bool fused;                 // Clamped gather read directly from the previous frame
    const float2* mvec;
    ResPlanes curr; RecPlanes currRec;
    ResPlanes prev; RecPlanes prevRec;
    ResPlanes inter; RecPlanes interRec;
    const float2* floatingCoords;
    const uint32_t* counts; const uint32_t* offsets; const uint32_t* sorted; const uint32_t* sortedCell;
    const uint32_t* totalSplats;
    float* m2curr; float* m3curr;
    ShiftPlanes backupShift; float4* backupTerms; float2* backupM;
    ShiftPlanes splatShift; float4* splatTerms; float4* splatM;
};

// Buffers of the wavefront MultiSplatting resampling: P partitions' cell lists (partition j at j * N)
// and, per splat position, its stored shift and terms.
struct MultiCtx
{
    const float2* mvec;
    ResPlanes curr; RecPlanes currRec;
    ResPlanes prev; RecPlanes prevRec;
    const uint32_t* counts; const uint32_t* offsets; const uint32_t* sorted; const uint32_t* sortedCell;
    const uint32_t* totals;        // splats per partition
    float* currMIS;                // per pixel: the current sample's MIS weight
    ShiftPlanes shift;             // per splat position (stride P * N)
    float4* terms;                 // per splat: prevPHat.xyz, Jacobian
    float4* misSub;                // per splat: prevMIS, shifted sub-pixel.xy, 0
};
__global__ void k_so_combine(uint32_t slot, WaveCtx K, float4* color);
__global__ void k_go_combine(uint32_t slot, WaveCtx K, float4* color);
__global__ void k_ms_combine(uint32_t slot, MultiCtx M, float4* color);

// Buffers of the wavefront spatial resampling (one iteration).
struct SpatialCtx
{
    uint32_t iteration;
    const uint4* vbuffer;
    const float2* neighborOffsets;
    ResPlanes src; RecPlanes srcRec;
    ResPlanes dst; RecPlanes dstRec;
    float* m1; ShiftPlanes shift; float4* terms; float* nw;
};

__global__ void k_sb_combine(uint32_t slot, WaveCtx K, float4* color);
__global__ void k_sp_combine(uint32_t slot, SpatialCtx S, float4* color);

// ---- batched stages: one persistent launch per stage over a BatchQueue of instances, each
// instance's own arguments at args[instance] in device memory (the kb_* kernels).
struct VbufArgs { uint4* vbuffer; float2* mvec; };
struct CandArgs { ResPlanes curr; RecPlanes currRec; };
struct ReprojArgs { ResPlanes prev; RecPlanes prevRec; uint32_t* targets; uint32_t* counts; };
struct WaveColorArgs { WaveCtx K; float4* color; };
struct SpatialColorArgs { SpatialCtx S; float4* color; };
__global__ void kb_camera_table(const uint32_t* slots, CameraTable* const* tables);
__global__ void kb_vbuffer(BatchQueue q, const VbufArgs* args);
__global__ void kb_reproject(BatchQueue q, const ReprojArgs* args);
__global__ void kb_sb_combine(BatchQueue q, const WaveColorArgs* args);
__global__ void kb_sp_combine(BatchQueue q, const SpatialColorArgs* args);
// Batched stages with environment-light variants: the stage is picked by `stage`, args points to
// the stage's argument array (CandArgs for candidates, WaveCtx for the six ScatterBackup shift
// stages, SpatialCtx for the two spatial shift stages).
enum BatchStage : uint32_t
{
    kBatchCandidates = 0, kBatchSbCurrScatter, kBatchSbCurrGather, kBatchSbBackupGather, kBatchSbBackupScatter,
    kBatchSbSplatScatter, kBatchSbSplatGather, kBatchSpCentral, kBatchSpNeighbor, kBatchVbuffer, kBatchReproject,
    kBatchSbCombine, kBatchSpCombine, kBatchStageCount
};
void launch_batched(BatchStage stage, bool env, dim3 grid, dim3 block, cudaStream_t s, const BatchQueue& q, const void* args);
// Threads per block and resident blocks per SM (for the persistent grid) of a batched stage kernel.
uint32_t batched_threads(BatchStage stage);
int batched_blocks_per_sm(BatchStage stage, bool env);


// The kernels that reach an environment-light branch are templates on it (kEnv), defined and
// launched in kernels.cu: launch one of the two variants (env: the pass has an environment light).
void launch_k_candidates(uint32_t lights, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, ResPlanes curr, RecPlanes currRec);
void launch_k_candidates_direct(uint32_t lights, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, ResPlanes curr, RecPlanes currRec);
void launch_k_robust(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, ResPlanes prev, RecPlanes prevRec, Shifted* __restrict__ shiftedPaths);
void launch_k_gather_resample(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, const uint4* __restrict__ vbuffer, ResPlanes curr, RecPlanes currRec, ResPlanes inter, RecPlanes interRec, const float2* __restrict__ floatingCoords, float4* __restrict__ color);
void launch_k_so_curr(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K);
void launch_k_so_splat(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K);
void launch_k_go_curr(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K);
void launch_k_go_prev(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K);
void launch_k_ms_curr(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, MultiCtx M);
void launch_k_ms_splat(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, MultiCtx M);
void launch_k_sb_curr_scatter(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K);
void launch_k_sb_curr_gather(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K);
void launch_k_sb_backup_gather(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K);
void launch_k_sb_backup_scatter(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K);
void launch_k_sb_splat_scatter(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K);
void launch_k_sb_splat_gather(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, WaveCtx K);
void launch_k_sp_central(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, SpatialCtx S);
void launch_k_sp_neighbor(bool env, dim3 grid, dim3 block, cudaStream_t s, uint32_t slot, SpatialCtx S);

} // namespace rs
