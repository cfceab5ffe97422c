// Diagnostics of the ray-query layer (no reference counterpart): the 4-wide tree's shape, and the
// closest hits of caller-given rays with the binary tree's per-ray traversal work.
#include <algorithm>
#include <vector>
#include "bvh_build.h"

namespace rs {

__global__ void k_debug_trace(BvhView bv, const float* __restrict__ rays, uint32_t n, int32_t* __restrict__ prim, float* __restrict__ tuv,
                              uint32_t* __restrict__ counts, uint32_t* overflow)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float* q = rays + 8 * (size_t)i;
    Ray r = mk_ray(mk3(q[0], q[1], q[2]), mk3(q[3], q[4], q[5]), q[6], q[7]);
    uint32_t c[2] = {0u, 0u};
    TraceHit h;
    if (bv.numTris == 0) { h.prim = kInvalidIndex; h.t = 0.f; h.u = 0.f; h.v = 0.f; }
    else h = trace_closest_bin<true>(bv, r, overflow, c);
    prim[i] = h.prim == kInvalidIndex ? -1 : (int32_t)h.prim;
    tuv[3 * i] = h.t; tuv[3 * i + 1] = h.u; tuv[3 * i + 2] = h.v;
    counts[2 * i] = c[0];
    counts[2 * i + 1] = c[1];
}

// Host-side shape of the tree: out = {nodes, depth, internal children, leaf children, leaf
// triangles, surface-area cost (node visits 1, triangle tests 1, weighted by box area / root area)}.
void wide_bvh_shape(const WideBvh& b, double* out)
{
    for (int k = 0; k < 6; k++) out[k] = 0.0;
    if (!b.nodes || b.numNodes == 0) return;
    std::vector<float4> h(7ull * b.numNodes);
    cudaMemcpy(h.data(), b.nodes, 112ull * b.numNodes, cudaMemcpyDeviceToHost);
    double internal = 0, leaves = 0, leafTris = 0, cost = 0;
    std::vector<double> area(b.numNodes, 0.0);
    double rootLo[3] = {3e38, 3e38, 3e38}, rootHi[3] = {-3e38, -3e38, -3e38};
    for (uint32_t i = 0; i < b.numNodes; i++)
    {
        const float4* n = &h[7ull * i];
        const float lo[3][4] = {{n[0].x, n[0].y, n[0].z, n[0].w}, {n[2].x, n[2].y, n[2].z, n[2].w}, {n[4].x, n[4].y, n[4].z, n[4].w}};
        const float hi[3][4] = {{n[1].x, n[1].y, n[1].z, n[1].w}, {n[3].x, n[3].y, n[3].z, n[3].w}, {n[5].x, n[5].y, n[5].z, n[5].w}};
        const uint32_t ref[4] = {f2u(n[6].x), f2u(n[6].y), f2u(n[6].z), f2u(n[6].w)};
        for (int k = 0; k < 4; k++)
        {
            if (ref[k] == kInvalidIndex) continue;
            double dx = hi[0][k] - lo[0][k], dy = hi[1][k] - lo[1][k], dz = hi[2][k] - lo[2][k];
            double ca = dx * dy + dy * dz + dz * dx;
            if (i == 0)
                for (int a = 0; a < 3; a++) { rootLo[a] = std::min(rootLo[a], (double)lo[a][k]); rootHi[a] = std::max(rootHi[a], (double)hi[a][k]); }
            if (ref[k] & kLeafBit) { leaves++; leafTris += (ref[k] & 3u) + 1; cost += ca * ((ref[k] & 3u) + 1); }
            else { internal++; area[ref[k]] = ca; }
        }
    }
    double dx = rootHi[0] - rootLo[0], dy = rootHi[1] - rootLo[1], dz = rootHi[2] - rootLo[2];
    double rootArea = dx * dy + dy * dz + dz * dx;
    area[0] = rootArea;
    for (uint32_t i = 0; i < b.numNodes; i++) cost += area[i];
    out[0] = b.numNodes; out[1] = b.depth; out[2] = internal; out[3] = leaves; out[4] = leafTris;
    out[5] = rootArea > 0 ? cost / rootArea : 0.0;
}

} // namespace rs
