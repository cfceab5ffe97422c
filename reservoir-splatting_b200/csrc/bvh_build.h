// GPU BVH build entry point (see bvh_build.cu).
#pragma once
#include <cuda_runtime.h>
#include "bvh.cuh"

namespace rs {

// The two trees of bvh.cuh and their leaf-order triangle array (device memory owned by the caller
// after a successful build; release with free_wide_bvh).
struct WideBvh
{
    float4* binNodes = nullptr; // binary tree (closest hit)
    uint32_t binRoot = 0;
    float4* nodes = nullptr;    // 4-wide tree (visibility)
    float4* leafTri = nullptr;
    uint32_t numNodes = 0;
    uint32_t depth = 0; // levels of nodes
    uint32_t numTris = 0;
    // refit data: the binary tree's parents, its arrival counters and, per 4-wide slot, the binary
    // reference the slot was made from (kInvalidIndex for an empty slot)
    uint32_t* parent = nullptr;
    uint32_t* leafParent = nullptr;
    uint32_t* arrivals = nullptr;
    uint4* binRef = nullptr;
};

// Builds the tree over n triangles (dTri: three float4 per triangle, geom.h layout); replaces
// *out.  Synchronises `s`.  n must be below kMaxBvhTriangles.
// Binary-tree builders: PLOC (the default) or the LBVH of Karras 2012 over the same Morton order.
enum BvhBuilder : uint32_t { kBvhPloc = 0, kBvhLbvh = 1 };
cudaError_t build_wide_bvh(const float4* dTri, uint32_t n, WideBvh* out, cudaStream_t s, BvhBuilder builder = kBvhPloc);
void free_wide_bvh(WideBvh* b);

// Refits both trees to moved triangles (same count and topology): leaf triangles, binary boxes
// bottom up, then the 4-wide boxes from the binary ones.  Stream-ordered on `s`.
cudaError_t refit_wide_bvh(const float4* dTri, WideBvh* b, cudaStream_t s);

// Diagnostics (bvh_debug.cu): rays are 8 floats (origin, direction, tMin, tMax); counts get the
// nodes visited and triangles tested per ray.
__global__ void k_debug_trace(BvhView bv, const float* rays, uint32_t n, int32_t* prim, float* tuv, uint32_t* counts, uint32_t* overflow);
void wide_bvh_shape(const WideBvh& b, double* out);

}
