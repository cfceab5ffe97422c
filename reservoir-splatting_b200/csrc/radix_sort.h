// Device sorting and scanning primitives of the pass, written for this library (no CUB):
//
//   scan_exclusive_u32      exclusive prefix sum of uint32 values: one block walking 4096-element
//                           chunks with a running carry up to kScanSingleMax elements, beyond that
//                           reduce-then-scan over tiles of 4096 (hierarchical, any length)
//   radix_sort_indices      stable LSD radix sort of element indices by a key read by gather
//
// The sort permutes indices only: the key of index v is read from the caller's key array at v
// every pass (the array stays where it is and, at the sizes used here, in L2), so no key
// ping-pong buffer is needed.  Passes use digits of up to 8 bits; each pass is a per-tile digit
// count, a scan of the digit-major count matrix and a stable scatter that ranks each tile's
// elements in shared memory (warp match + per-warp digit counts, in element order).  Nothing
// waits on another block, and the result does not depend on scheduling: equal keys keep
// ascending index order, which makes the sort a drop-in for a stable (key, index) pair sort.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace rs {

constexpr uint32_t kSortTile = 4096;     // elements per sort tile (256 threads x 16)
constexpr uint32_t kScanBlockElems = 4096; // elements per scan tile (1024 threads x 4)
constexpr uint32_t kScanSingleMax = 1u << 18; // longest scan done by one block

// Words of scratch scan_exclusive_u32 needs for n elements.
size_t scan_scratch_words(uint32_t n);
// out[i] = sum of in[0..i); in may equal out.  Returns the launch error, if any.
cudaError_t scan_exclusive_u32(const uint32_t* in, uint32_t* out, uint32_t n, uint32_t* scratch, cudaStream_t s);

// Digit passes and bits per digit for keys of keyBits significant bits.
void radix_plan(uint32_t keyBits, uint32_t& passes, uint32_t& digitBits);
// Words of scratch radix_sort_* needs for n elements of keyBits-bit keys.
size_t radix_scratch_words(uint32_t n, uint32_t keyBits);

// out = the indices 0..n-1 sorted stably by min(keys[i], clampMax) over its low keyBits bits
// (keyBits >= bit length of clampMax).  tmp holds n indices between passes.  A key at clampMax
// marks "no key" (an invalid splat target, say): those indices sort last.
cudaError_t radix_sort_indices_u32(const uint32_t* keys, uint32_t clampMax, uint32_t n, uint32_t keyBits, uint32_t* out, uint32_t* tmp,
                                   uint32_t* scratch, cudaStream_t s);
// The same for 64-bit keys (Morton codes), no clamp.
cudaError_t radix_sort_indices_u64(const uint64_t* keys, uint32_t n, uint32_t keyBits, uint32_t* out, uint32_t* tmp, uint32_t* scratch,
                                   cudaStream_t s);

// Kernel launches of scan_exclusive_u32 and of radix_sort_indices_* for these sizes.
uint32_t scan_launches(uint32_t n);
uint32_t radix_sort_launches(uint32_t n, uint32_t keyBits);

// Bit length of x (0 for 0).
inline uint32_t bit_length(uint64_t x)
{
    uint32_t b = 0;
    while (x) { b++; x >>= 1; }
    return b;
}

} // namespace rs
