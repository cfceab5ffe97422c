// Stable LSD radix sort of indices by a gathered key, and a hierarchical exclusive scan
// (declarations and the method in radix_sort.h).
//
// Per digit pass, for tiles of kSortTile elements in order:
//   k_rsort_count    digit histogram of each tile -> counts[digit * numTiles + tile]
//   scan             exclusive prefix over that digit-major matrix: the first destination of
//                    each (digit, tile) run, so digits stay grouped and tiles keep their order
//   k_rsort_scatter  each tile walks its elements in 16 rounds of 256 (element order); a round
//                    ranks equal digits within a warp with __match_any_sync, adds the counts of
//                    the earlier warps of the round from shared memory, and writes each index to
//                    its run's next free slot
// Element order inside a tile, tile order inside a digit and digit order overall are all fixed,
// so every pass is stable and the output is deterministic.
#include "radix_sort.h"

namespace rs {
namespace {

constexpr int kScanThreadsR = 1024;
constexpr int kScanItemsR = 4;
static_assert(kScanThreadsR * kScanItemsR == (int)kScanBlockElems, "scan tile");
constexpr int kSortThreads = 256;
constexpr int kSortRounds = (int)kSortTile / kSortThreads;
constexpr int kSortWarps = kSortThreads / 32;

inline size_t round64(size_t w) { return (w + 63) & ~(size_t)63; }

// Exclusive scan of v over the block (blockDim.x a multiple of 32, at most 1024); total = block sum.
__device__ __forceinline__ uint32_t block_scan_excl(uint32_t v, uint32_t* smem32, uint32_t& total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint32_t x = v;
    for (int o = 1; o < 32; o <<= 1)
    {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) smem32[warp] = x;
    __syncthreads();
    if (warp == 0)
    {
        uint32_t s = lane < (int)(blockDim.x >> 5) ? smem32[lane] : 0u;
        for (int o = 1; o < 32; o <<= 1)
        {
            const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        smem32[lane] = s;
    }
    __syncthreads();
    const uint32_t warpPrefix = warp > 0 ? smem32[warp - 1] : 0u;
    total = smem32[(blockDim.x >> 5) - 1];
    __syncthreads();
    return warpPrefix + x - v;
}

// One tile of the scan; `in` may equal `out` (every thread reads its items before the block scan
// and writes the same items after it).
__global__ void __launch_bounds__(kScanThreadsR) k_scan_block(const uint32_t* in, uint32_t* out, uint32_t* blockSums, uint32_t n)
{
    __shared__ uint32_t smem32[32];
    const size_t base = (size_t)blockIdx.x * kScanBlockElems + (size_t)threadIdx.x * kScanItemsR;
    uint32_t v[kScanItemsR];
    uint32_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItemsR; k++)
    {
        v[k] = base + k < n ? in[base + k] : 0u;
        sum += v[k];
    }
    uint32_t total;
    uint32_t pre = block_scan_excl(sum, smem32, total);
#pragma unroll
    for (int k = 0; k < kScanItemsR; k++)
    {
        if (base + k < n) out[base + k] = pre;
        pre += v[k];
    }
    if (threadIdx.x == 0) blockSums[blockIdx.x] = total;
}

// The whole scan in one block: 4096-element chunks in order, each scanned by the block and offset
// by the running total of the chunks before it.  `in` may equal `out`.
__global__ void __launch_bounds__(kScanThreadsR) k_scan_single(const uint32_t* in, uint32_t* out, uint32_t n)
{
    __shared__ uint32_t smem32[32];
    uint32_t carry = 0;
    for (size_t chunk = 0; chunk < n; chunk += kScanBlockElems)
    {
        const size_t base = chunk + (size_t)threadIdx.x * kScanItemsR;
        uint32_t v[kScanItemsR];
        uint32_t sum = 0;
#pragma unroll
        for (int k = 0; k < kScanItemsR; k++)
        {
            v[k] = base + k < n ? in[base + k] : 0u;
            sum += v[k];
        }
        uint32_t total;
        uint32_t pre = carry + block_scan_excl(sum, smem32, total);
#pragma unroll
        for (int k = 0; k < kScanItemsR; k++)
        {
            if (base + k < n) out[base + k] = pre;
            pre += v[k];
        }
        carry += total;
    }
}

__global__ void __launch_bounds__(256) k_scan_add_blocks(uint32_t* out, const uint32_t* blockSums, uint32_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] += blockSums[i / kScanBlockElems];
}

__global__ void __launch_bounds__(256) k_iota(uint32_t* out, uint32_t n)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (uint32_t)i;
}

struct KeyU32Clamp
{
    const uint32_t* k;
    uint32_t clampMax;
    __device__ __forceinline__ uint64_t operator()(uint32_t v) const
    {
        const uint32_t x = __ldg(k + v);
        return x < clampMax ? x : clampMax;
    }
};
struct KeyU64
{
    const uint64_t* k;
    __device__ __forceinline__ uint64_t operator()(uint32_t v) const { return __ldg(k + v); }
};

template <typename Key>
__global__ void __launch_bounds__(kSortThreads) k_rsort_count(Key key, const uint32_t* __restrict__ vin, uint32_t n, uint32_t shift,
                                                              uint32_t radix, uint32_t* __restrict__ counts, uint32_t numTiles)
{
    __shared__ uint32_t hist[256];
    for (uint32_t d = threadIdx.x; d < radix; d += kSortThreads) hist[d] = 0u;
    __syncthreads();
    const uint32_t tile = blockIdx.x;
    const uint32_t mask = radix - 1u;
#pragma unroll
    for (int r = 0; r < kSortRounds; r++)
    {
        const uint32_t i = tile * kSortTile + (uint32_t)r * kSortThreads + threadIdx.x;
        if (i < n)
        {
            const uint32_t v = vin ? vin[i] : i;
            atomicAdd(&hist[(uint32_t)(key(v) >> shift) & mask], 1u);
        }
    }
    __syncthreads();
    for (uint32_t d = threadIdx.x; d < radix; d += kSortThreads) counts[(size_t)d * numTiles + tile] = hist[d];
}

template <typename Key>
__global__ void __launch_bounds__(kSortThreads) k_rsort_scatter(Key key, const uint32_t* __restrict__ vin, uint32_t* __restrict__ vout,
                                                                uint32_t n, uint32_t shift, uint32_t radix,
                                                                const uint32_t* __restrict__ scanned, uint32_t numTiles)
{
    __shared__ uint32_t base[256];                 // next destination of each digit in this tile
    __shared__ uint32_t warpCount[kSortWarps][256]; // this round's elements per (warp, digit)
    const uint32_t tile = blockIdx.x;
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t mask = radix - 1u;
    for (uint32_t d = threadIdx.x; d < radix; d += kSortThreads)
    {
        base[d] = scanned[(size_t)d * numTiles + tile];
#pragma unroll
        for (int w = 0; w < kSortWarps; w++) warpCount[w][d] = 0u;
    }
    __syncthreads();
    const uint32_t lanesBelow = (1u << lane) - 1u;
    for (int r = 0; r < kSortRounds; r++)
    {
        const uint32_t i = tile * kSortTile + (uint32_t)r * kSortThreads + threadIdx.x;
        const bool valid = i < n;
        const uint32_t v = valid ? (vin ? vin[i] : i) : 0u;
        // lanes past the end form their own group (digit value `radix`, never stored)
        const uint32_t d = valid ? ((uint32_t)(key(v) >> shift) & mask) : radix;
        const uint32_t peers = __match_any_sync(0xffffffffu, d);
        const uint32_t rankInWarp = __popc(peers & lanesBelow);
        if (valid && rankInWarp == 0) warpCount[warp][d] = __popc(peers);
        __syncthreads();
        if (valid)
        {
            uint32_t before = 0;
            for (uint32_t w = 0; w < warp; w++) before += warpCount[w][d];
            vout[base[d] + before + rankInWarp] = v;
        }
        __syncthreads();
        for (uint32_t dd = threadIdx.x; dd < radix; dd += kSortThreads)
        {
            uint32_t t = 0;
#pragma unroll
            for (int w = 0; w < kSortWarps; w++)
            {
                t += warpCount[w][dd];
                warpCount[w][dd] = 0u;
            }
            base[dd] += t;
        }
        __syncthreads();
    }
}

template <typename Key>
cudaError_t radix_sort(Key key, uint32_t n, uint32_t keyBits, uint32_t* out, uint32_t* tmp, uint32_t* scratch, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    uint32_t passes, digitBits;
    radix_plan(keyBits, passes, digitBits);
    if (passes == 0)
    {
        k_iota<<<(n + 255) / 256, 256, 0, s>>>(out, n);
        return cudaGetLastError();
    }
    const uint32_t numTiles = (n + kSortTile - 1) / kSortTile;
    const uint32_t radix = 1u << digitBits;
    const uint32_t m = radix * numTiles;
    uint32_t* counts = scratch;
    uint32_t* scanned = counts + round64(m);
    uint32_t* scanScratch = scanned + round64(m);
    const uint32_t* src = nullptr; // the identity permutation
    for (uint32_t p = 0; p < passes; p++)
    {
        uint32_t* dst = ((passes - 1u - p) % 2u == 0u) ? out : tmp; // the last pass writes `out`
        const uint32_t shift = p * digitBits;
        k_rsort_count<Key><<<numTiles, kSortThreads, 0, s>>>(key, src, n, shift, radix, counts, numTiles);
        cudaError_t e = scan_exclusive_u32(counts, scanned, m, scanScratch, s);
        if (e != cudaSuccess) return e;
        k_rsort_scatter<Key><<<numTiles, kSortThreads, 0, s>>>(key, src, dst, n, shift, radix, scanned, numTiles);
        src = dst;
    }
    return cudaGetLastError();
}

} // namespace

size_t scan_scratch_words(uint32_t n)
{
    if (n <= kScanSingleMax) return 64;
    const uint32_t tiles = (n + kScanBlockElems - 1) / kScanBlockElems;
    return round64(tiles) + scan_scratch_words(tiles);
}

cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* scratch, cudaStream_t s)
{
    if (n == 0) return cudaSuccess;
    if (n <= kScanSingleMax)
    {
        k_scan_single<<<1, kScanThreadsR, 0, s>>>(in, out, n);
        return cudaGetLastError();
    }
    const uint32_t tiles = (n + kScanBlockElems - 1) / kScanBlockElems;
    uint32_t* sums = scratch;
    k_scan_block<<<tiles, kScanThreadsR, 0, s>>>(in, out, sums, n);
    if (tiles > 1)
    {
        cudaError_t e = scan_exclusive_u32(sums, sums, tiles, scratch + round64(tiles), s);
        if (e != cudaSuccess) return e;
        k_scan_add_blocks<<<(n + 255) / 256, 256, 0, s>>>(out, sums, n);
    }
    return cudaGetLastError();
}

void radix_plan(uint32_t keyBits, uint32_t& passes, uint32_t& digitBits)
{
    if (keyBits == 0) { passes = 0; digitBits = 0; return; }
    passes = (keyBits + 7u) / 8u;
    digitBits = (keyBits + passes - 1u) / passes;
}

size_t radix_scratch_words(uint32_t n, uint32_t keyBits)
{
    uint32_t passes, digitBits;
    radix_plan(keyBits, passes, digitBits);
    if (passes == 0 || n == 0) return 64;
    const size_t numTiles = (n + kSortTile - 1) / kSortTile;
    const size_t m = ((size_t)1 << digitBits) * numTiles;
    return 2 * round64(m) + scan_scratch_words((uint32_t)m);
}

uint32_t scan_launches(uint32_t n)
{
    if (n == 0) return 0;
    if (n <= kScanSingleMax) return 1;
    const uint32_t tiles = (n + kScanBlockElems - 1) / kScanBlockElems;
    return tiles > 1 ? 2 + scan_launches(tiles) : 1;
}

uint32_t radix_sort_launches(uint32_t n, uint32_t keyBits)
{
    uint32_t passes, digitBits;
    radix_plan(keyBits, passes, digitBits);
    if (n == 0) return 0;
    if (passes == 0) return 1;
    const uint32_t m = (1u << digitBits) * ((n + kSortTile - 1) / kSortTile);
    return passes * (2 + scan_launches(m));
}

cudaError_t radix_sort_indices_u32(const uint32_t* keys, uint32_t clampMax, uint32_t n, uint32_t keyBits, uint32_t* out, uint32_t* tmp,
                                   uint32_t* scratch, cudaStream_t s)
{
    return radix_sort(KeyU32Clamp{keys, clampMax}, n, keyBits, out, tmp, scratch, s);
}

cudaError_t radix_sort_indices_u64(const uint64_t* keys, uint32_t n, uint32_t keyBits, uint32_t* out, uint32_t* tmp, uint32_t* scratch,
                                   cudaStream_t s)
{
    return radix_sort(KeyU64{keys}, n, keyBits, out, tmp, scratch, s);
}

} // namespace rs

// ------------------------------------------------------------------ diagnostics (C ABI)
#include <string>
#include "../../include/rs_b200.h"

namespace rs { void set_last_error(const std::string& msg); }

namespace {

// Copies host keys to the device, runs `fn(deviceKeys, deviceOut, scratch)` and copies n results back.
template <typename K, typename Fn>
rs_status debug_run(const K* hostKeys, uint32_t n, size_t scratchWords, uint32_t* hostOut, Fn fn)
{
    K* dk = nullptr;
    uint32_t *dout = nullptr, *dtmp = nullptr, *dscr = nullptr;
    cudaError_t e = cudaMalloc(&dk, sizeof(K) * (n ? n : 1));
    if (e == cudaSuccess) e = cudaMalloc(&dout, 4ull * (n ? n : 1));
    if (e == cudaSuccess) e = cudaMalloc(&dtmp, 4ull * (n ? n : 1));
    if (e == cudaSuccess) e = cudaMalloc(&dscr, 4ull * scratchWords);
    if (e == cudaSuccess && n) e = cudaMemcpy(dk, hostKeys, sizeof(K) * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = fn(dk, dout, dtmp, dscr);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e == cudaSuccess && n) e = cudaMemcpy(hostOut, dout, 4ull * n, cudaMemcpyDeviceToHost);
    cudaFree(dk); cudaFree(dout); cudaFree(dtmp); cudaFree(dscr);
    if (e != cudaSuccess)
    {
        rs::set_last_error(std::string("radix sort diagnostics: ") + cudaGetErrorString(e));
        return RS_CUDA_ERROR;
    }
    return RS_OK;
}

} // namespace

// The library's stable radix sort on host data (no reference counterpart; synchronous, allocates):
// order[i] = index of the i-th smallest key (keys64 over keyBits bits; keys32 clamped to clampMax,
// which sorts last), ties in ascending index order.  rs_debug_scan: out = exclusive prefix sum.
extern "C" RS_API rs_status rs_debug_sort_keys64(const uint64_t* keys, uint32_t n, uint32_t keyBits, uint32_t* order)
{
    if ((n && (!keys || !order)) || keyBits > 64) { rs::set_last_error("rs_debug_sort_keys64: bad arguments"); return RS_INVALID_ARG; }
    return debug_run(keys, n, rs::radix_scratch_words(n, keyBits), order, [&](const uint64_t* dk, uint32_t* dout, uint32_t* dtmp, uint32_t* dscr) {
        return rs::radix_sort_indices_u64(dk, n, keyBits, dout, dtmp, dscr, 0);
    });
}

extern "C" RS_API rs_status rs_debug_sort_keys32(const uint32_t* keys, uint32_t n, uint32_t clampMax, uint32_t* order)
{
    if (n && (!keys || !order)) { rs::set_last_error("rs_debug_sort_keys32: bad arguments"); return RS_INVALID_ARG; }
    const uint32_t bits = rs::bit_length(clampMax);
    return debug_run(keys, n, rs::radix_scratch_words(n, bits), order, [&](const uint32_t* dk, uint32_t* dout, uint32_t* dtmp, uint32_t* dscr) {
        return rs::radix_sort_indices_u32(dk, clampMax, n, bits, dout, dtmp, dscr, 0);
    });
}

extern "C" RS_API rs_status rs_debug_scan(const uint32_t* values, uint32_t n, uint32_t* out)
{
    if (n && (!values || !out)) { rs::set_last_error("rs_debug_scan: bad arguments"); return RS_INVALID_ARG; }
    return debug_run(values, n, rs::scan_scratch_words(n), out, [&](const uint32_t* dk, uint32_t* dout, uint32_t*, uint32_t* dscr) {
        return rs::scan_exclusive_u32(dk, dout, n, dscr, 0);
    });
}
