// GPU LBVH build entry point (see bvh_build.cu).
#pragma once
#include <cuda_runtime.h>
#include "bvh.cuh"

namespace rs {
// dNodes must hold 4 float4 per internal node (n - 1 nodes).  *rootOut receives the
// root child index (0, or a leaf when n == 1).  Synchronises `s` before returning.
cudaError_t build_lbvh(const float4* dTri, uint32_t n, float4* dNodes, uint32_t* rootOut, cudaStream_t s);
}
