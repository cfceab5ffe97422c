// rs_build_cell_lists_static: the splat cell-list build (count, exclusive scan, stable radix sort of
// the splat indices by cell) with its scratch memory in a fixed array that the library holds, so the
// call allocates nothing.
//
// Who needs it: callers that may not allocate device memory at the time they run.  A host that
// owns a fixed memory pool (and fails on any allocation it did not plan), an allocator-free
// real-time frame loop, or a plug-in that runs while its host is capturing a CUDA graph cannot
// call cudaMalloc, and the rs_pass entry points allocate their buffers on the first frame at a
// given size.  Such a caller passes its own input and output buffers; the temporaries (the sort's
// second index buffer and digit counts, the scan's tile sums) come from `g_cellScratch` below.
//
// The lists are the per-cell splat lists of the temporal scatter (the cell counters and splat
// indices that ReprojectTemporalSamples.rt.slang:64-175 fills, cleared at
// ReservoirSplatting.cpp:1759-1775), in the canonical order that rs_execute writes them: offsets
// are the exclusive prefix sum of the counts and each cell lists its splats by ascending index.
#include <cuda_runtime.h>
#include <mutex>
#include <string>
#include "../../include/rs_b200.h"
#include "kernels.h"
#include "radix_sort.h"

namespace rs {
void set_last_error(const std::string& msg);
}

using namespace rs;

namespace {

constexpr uint32_t kStaticMaxCells = RS_CELL_LISTS_STATIC_MAX;
constexpr uint32_t kStaticMaxSplats = RS_CELL_LISTS_STATIC_MAX;
constexpr uint32_t kStaticMaxTiles = (kStaticMaxCells + kScanTileElems - 1) / kScanTileElems;
// Word offsets inside the scratch array; each part starts on a 256-byte boundary.  The radix sort
// needs two 256-entry digit-count matrices over its tiles plus a little scan scratch
// (radix_scratch_words; at most 8-bit digits because keys have at most 22 bits here).
constexpr size_t kTmpWords = kStaticMaxSplats;
constexpr size_t kTileSumsOffset = kTmpWords;
constexpr size_t kRadixOffset = kTileSumsOffset + ((kStaticMaxTiles + 63) / 64) * 64;
constexpr size_t kRadixWords = 2 * 256 * ((kStaticMaxSplats + kSortTile - 1) / kSortTile) + 1024;
constexpr size_t kScratchWords = kRadixOffset + kRadixWords;
static_assert(kTileSumsOffset % 64 == 0 && kRadixOffset % 64 == 0, "scratch parts must be 256-byte aligned");
static_assert(kStaticMaxTiles <= kScanTileElems, "k_scan_tile_sums scans at most one tile of tile sums");

// Every GPU that loads the library holds this array (about 9 MiB) until the process exits.
// Host code must not pass `g_cellScratch` to a kernel: on the host the name is only a stand-in
// for the device symbol.  Its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) uint32_t g_cellScratch[kScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
uint32_t* g_scratchAddr[kMaxDevices] = {};

// Splats per cell.  A target outside [0, numCells) (kInvalidIndex included) means "no cell".
__global__ void __launch_bounds__(256) k_static_count(const uint32_t* __restrict__ targets, uint32_t n, uint32_t numCells,
                                                      uint32_t* __restrict__ counts)
{
    uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    uint32_t t = targets[s];
    if (t < numCells) atomicAdd(&counts[t], 1u);
}

rs_status static_fail(rs_status s, const std::string& msg)
{
    set_last_error(msg);
    return s;
}

rs_status cuda_fail(const char* what, cudaError_t e)
{
    return static_fail(RS_CUDA_ERROR, std::string("rs_build_cell_lists_static: ") + what + ": " + cudaGetErrorString(e));
}

// Once per device, with that device current: the device address of g_cellScratch.
rs_status scratch_for_current_device(uint32_t** out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail("cudaGetDevice", e);
    if (dev < 0 || dev >= kMaxDevices) return static_fail(RS_INVALID_ARG, "rs_build_cell_lists_static: device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_setupMutex);
    if (!g_scratchAddr[dev])
    {
        void* addr = nullptr;
        e = cudaGetSymbolAddress(&addr, g_cellScratch);
        if (e != cudaSuccess) return cuda_fail("cudaGetSymbolAddress", e);
        if (!addr) return static_fail(RS_CUDA_ERROR, "rs_build_cell_lists_static: null scratch address");
        g_scratchAddr[dev] = static_cast<uint32_t*>(addr);
    }
    *out = g_scratchAddr[dev];
    return RS_OK;
}

} // namespace

extern "C" RS_API rs_status rs_build_cell_lists_static(const uint32_t* targets, uint32_t numSplats, uint32_t numCells,
                                                       uint32_t* counts, uint32_t* offsets, uint32_t* sorted, void* cudaStream)
{
    if (numCells == 0 || numCells > kStaticMaxCells)
        return static_fail(RS_INVALID_ARG, "rs_build_cell_lists_static: numCells = " + std::to_string(numCells) +
                                               " is outside [1, " + std::to_string(kStaticMaxCells) + "] (the static scratch limit)");
    if (numSplats > kStaticMaxSplats)
        return static_fail(RS_INVALID_ARG, "rs_build_cell_lists_static: numSplats = " + std::to_string(numSplats) +
                                               " exceeds the static scratch limit of " + std::to_string(kStaticMaxSplats));
    if (!counts || !offsets || (numSplats > 0 && (!targets || !sorted)))
        return static_fail(RS_INVALID_ARG, "rs_build_cell_lists_static: null buffer");
    uint32_t* scratch = nullptr;
    rs_status st = scratch_for_current_device(&scratch);
    if (st != RS_OK) return st;
    uint32_t* tmp = scratch;
    uint32_t* tileSums = scratch + kTileSumsOffset;
    uint32_t* radixScratch = scratch + kRadixOffset;
    const uint32_t keyBits = bit_length(numCells); // targets >= numCells sort last as numCells
    if (radix_scratch_words(numSplats, keyBits) > kRadixWords)
        return static_fail(RS_INVALID_ARG, "rs_build_cell_lists_static: sort scratch larger than the static array");

    cudaStream_t s = static_cast<cudaStream_t>(cudaStream);
    const uint32_t numTiles = (numCells + kScanTileElems - 1) / kScanTileElems;
    const uint32_t cellBlocks = (numCells + 255) / 256, splatBlocks = (numSplats + 255) / 256;
    // The counts (an output) must start at zero; the scan and the sort overwrite everything else
    // they read (the array keeps the previous call's contents).
    cudaError_t e = cudaMemsetAsync(counts, 0, (size_t)numCells * 4, s);
    if (e != cudaSuccess) return cuda_fail("cudaMemsetAsync(counts)", e);
    if (splatBlocks) k_static_count<<<splatBlocks, 256, 0, s>>>(targets, numSplats, numCells, counts);
    k_scan_tiles<<<numTiles, 1024, 0, s>>>(counts, offsets, tileSums, numCells);
    k_scan_tile_sums<<<1, 1024, 0, s>>>(tileSums, numTiles, nullptr);
    k_scan_add<<<cellBlocks, 256, 0, s>>>(offsets, tileSums, numCells);
    // splat indices in (cell, index) order; the ones without a cell follow the last listed splat
    e = radix_sort_indices_u32(targets, numCells, numSplats, keyBits, sorted, tmp, radixScratch, s);
    if (e != cudaSuccess) return cuda_fail("radix sort launch", e);
    e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail("kernel launch", e);
    return RS_OK;
}
