// Kernel declarations of the Reservoir Splatting pass (definitions in kernels.cu).
#pragma once
#include "pass_device.cuh"

namespace rs {

__global__ void k_vbuffer(DevCtx C, uint4* vbuffer, float2* mvec);
__global__ void k_candidates(DevCtx C, ResPlanes curr, RecPlanes currRec);
__global__ void k_reproject(DevCtx C, ResPlanes prev, RecPlanes prevRec, uint32_t* targets, uint32_t* counts);
__global__ void k_multi_reproject(DevCtx C, ResPlanes prev, RecPlanes prevRec, uint32_t* targets, uint32_t* counts);
__global__ void k_scan_tiles(const uint32_t* in, uint32_t* out, uint32_t* tileSums, uint32_t n);
__global__ void k_scan_tile_sums(uint32_t* tileSums, uint32_t numTiles, uint32_t* totalOut);
__global__ void k_scan_add(uint32_t* out, const uint32_t* tileSums, uint32_t n);
__global__ void k_fill(const uint32_t* targets, const uint32_t* offsets, uint32_t* cursor, uint32_t* unsorted, uint32_t n);
__global__ void k_rank_cells(const uint32_t* targets, const uint32_t* offsets, const uint32_t* counts, const uint32_t* unsorted,
                             uint32_t* sorted, uint32_t n);
__global__ void k_collect(DevCtx C, const float2* mvec, ResPlanes prev, RecPlanes prevRec, ResPlanes inter, RecPlanes interRec,
                          float2* floatingCoords, const Shifted* shiftedPaths);
__global__ void k_robust(DevCtx C, ResPlanes prev, RecPlanes prevRec, Shifted* shiftedPaths);
__global__ void k_scatter_resample(DevCtx C, const float2* mvec, ResPlanes prev, RecPlanes prevRec, ResPlanes curr, RecPlanes currRec,
                                   const uint32_t* counts, const uint32_t* offsets, const uint32_t* sorted, float4* color);
__global__ void k_scatter_backup_resample(DevCtx C, const float2* mvec, ResPlanes prev, RecPlanes prevRec, ResPlanes curr, RecPlanes currRec,
                                          ResPlanes inter, RecPlanes interRec, const float2* floatingCoords, const uint32_t* counts,
                                          const uint32_t* offsets, const uint32_t* sorted, float4* color);
// ScatterBackup with the Clamped gather: the collect pass is fused in (backup read from prev at round(prevPixel)).
__global__ void k_scatter_backup_resample_clamped(DevCtx C, const float2* mvec, ResPlanes prev, RecPlanes prevRec, ResPlanes curr,
                                                  RecPlanes currRec, const uint32_t* counts, const uint32_t* offsets, const uint32_t* sorted,
                                                  float4* color);
__global__ void k_gather_resample(DevCtx C, const uint4* vbuffer, ResPlanes curr, RecPlanes currRec, ResPlanes inter, RecPlanes interRec,
                                  const float2* floatingCoords, float4* color);
__global__ void k_multi_scatter_resample(DevCtx C, const float2* mvec, ResPlanes prev, RecPlanes prevRec, ResPlanes curr, RecPlanes currRec,
                                         const uint32_t* counts, const uint32_t* offsets, const uint32_t* sortedAll, float4* color);
__global__ void k_spatial(DevCtx C, uint32_t iteration, const uint4* vbuffer, const float2* neighborOffsets, ResPlanes src, RecPlanes srcRec,
                          ResPlanes dstP, RecPlanes dstRec, float4* color);
__global__ void k_resolve(uint32_t n, ResPlanes curr, float4* color);

constexpr int kScanTileElems = 4096; // k_scan_tiles: 1024 threads x 4 items

} // namespace rs
