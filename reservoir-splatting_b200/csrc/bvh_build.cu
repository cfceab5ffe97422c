// LBVH construction on the GPU (Karras 2012, "Maximizing parallelism in the
// construction of BVHs, octrees, and k-d trees"): 63-bit Morton codes (21 bits per axis) of the
// triangle centroids, a key/index sort, one thread per internal node to find its
// range and split, and a bottom-up box pass with per-node arrival counters.
// Built once per rs_set_scene; the per-frame path only traverses it.
#include <cub/device/device_radix_sort.cuh>
#include "bvh_build.h"

namespace rs {

// Spreads the low 21 bits of v so that two zero bits separate consecutive bits.
__device__ __forceinline__ uint64_t expand_bits21(uint64_t v)
{
    v &= 0x1fffffull;
    v = (v | (v << 32)) & 0x1f00000000ffffull;
    v = (v | (v << 16)) & 0x1f0000ff0000ffull;
    v = (v | (v << 8)) & 0x100f00f00f00f00full;
    v = (v | (v << 4)) & 0x10c30c30c30c30c3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__device__ __forceinline__ uint32_t ordered_bits(float f)
{
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float from_ordered_bits(uint32_t u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__global__ void k_centroid_bounds(const float4* __restrict__ tri, uint32_t n, uint32_t* __restrict__ bounds)
{
    float lo[3] = {3e38f, 3e38f, 3e38f}, hi[3] = {-3e38f, -3e38f, -3e38f};
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        float4 a = tri[3 * i], b = tri[3 * i + 1], c = tri[3 * i + 2];
        float cx = (a.x + b.x + c.x) * (1.f / 3.f), cy = (a.y + b.y + c.y) * (1.f / 3.f), cz = (a.z + b.z + c.z) * (1.f / 3.f);
        lo[0] = fminf(lo[0], cx); lo[1] = fminf(lo[1], cy); lo[2] = fminf(lo[2], cz);
        hi[0] = fmaxf(hi[0], cx); hi[1] = fmaxf(hi[1], cy); hi[2] = fmaxf(hi[2], cz);
    }
    for (int k = 0; k < 3; k++)
    {
        for (int off = 16; off > 0; off >>= 1)
        {
            lo[k] = fminf(lo[k], __shfl_xor_sync(0xffffffffu, lo[k], off));
            hi[k] = fmaxf(hi[k], __shfl_xor_sync(0xffffffffu, hi[k], off));
        }
    }
    if ((threadIdx.x & 31) == 0)
        for (int k = 0; k < 3; k++)
        {
            atomicMin(&bounds[k], ordered_bits(lo[k]));
            atomicMax(&bounds[3 + k], ordered_bits(hi[k]));
        }
}

__global__ void k_morton(const float4* __restrict__ tri, uint32_t n, const uint32_t* __restrict__ bounds,
                         uint64_t* __restrict__ keys, uint32_t* __restrict__ vals)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float lo[3], ext[3];
    for (int k = 0; k < 3; k++)
    {
        lo[k] = from_ordered_bits(bounds[k]);
        float hi = from_ordered_bits(bounds[3 + k]);
        ext[k] = hi > lo[k] ? hi - lo[k] : 1.f;
    }
    float4 a = tri[3 * i], b = tri[3 * i + 1], c = tri[3 * i + 2];
    float cx = (a.x + b.x + c.x) * (1.f / 3.f), cy = (a.y + b.y + c.y) * (1.f / 3.f), cz = (a.z + b.z + c.z) * (1.f / 3.f);
    const float Q = 2097152.f; // 2^21 cells per axis: 63-bit keys
    uint64_t qx = (uint64_t)fminf(fmaxf((cx - lo[0]) / ext[0] * Q, 0.f), Q - 1.f);
    uint64_t qy = (uint64_t)fminf(fmaxf((cy - lo[1]) / ext[1] * Q, 0.f), Q - 1.f);
    uint64_t qz = (uint64_t)fminf(fmaxf((cz - lo[2]) / ext[2] * Q, 0.f), Q - 1.f);
    keys[i] = (expand_bits21(qx) << 2) | (expand_bits21(qy) << 1) | expand_bits21(qz);
    vals[i] = i;
}

// Common-prefix length of sorted keys i and j (index bits break ties between equal keys).
__device__ __forceinline__ int delta(const uint64_t* keys, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    uint64_t a = keys[i], b = keys[j];
    if (a == b) return 64 + __clz((uint32_t)i ^ (uint32_t)j);
    return __clzll((long long)(a ^ b));
}

__global__ void k_karras(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ prim, int n,
                         float4* __restrict__ nodes, uint32_t* __restrict__ parent, uint32_t* __restrict__ leafParent)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta(keys, n, i, j);
    int s = 0;
    int len = l;
    for (int t = (len + 1) >> 1;; t = (t + 1) >> 1)
    {
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t == 1) break;
    }
    int gamma = i + s * d + (d < 0 ? -1 : 0);
    int lo = i < j ? i : j, hi = i < j ? j : i;
    uint32_t left = (lo == gamma) ? (kLeafBit | prim[gamma]) : (uint32_t)gamma;
    uint32_t right = (hi == gamma + 1) ? (kLeafBit | prim[gamma + 1]) : (uint32_t)(gamma + 1);
    nodes[4 * (size_t)i + 0].w = __uint_as_float(left);
    nodes[4 * (size_t)i + 1].w = __uint_as_float(right);
    if (lo == gamma) leafParent[gamma] = (uint32_t)i; else parent[gamma] = (uint32_t)i;
    if (hi == gamma + 1) leafParent[gamma + 1] = (uint32_t)i; else parent[gamma + 1] = (uint32_t)i;
}

__device__ __forceinline__ void tri_box(const float4* tri, uint32_t p, float lo[3], float hi[3])
{
    float4 a = tri[3 * p], b = tri[3 * p + 1], c = tri[3 * p + 2];
    lo[0] = fminf(a.x, fminf(b.x, c.x)); hi[0] = fmaxf(a.x, fmaxf(b.x, c.x));
    lo[1] = fminf(a.y, fminf(b.y, c.y)); hi[1] = fmaxf(a.y, fmaxf(b.y, c.y));
    lo[2] = fminf(a.z, fminf(b.z, c.z)); hi[2] = fmaxf(a.z, fmaxf(b.z, c.z));
    for (int k = 0; k < 3; k++)
    {
        float pad = (fabsf(lo[k]) + fabsf(hi[k]) + (hi[k] - lo[k])) * 1e-6f + 1e-30f;
        lo[k] -= pad; hi[k] += pad;
    }
}

__device__ __forceinline__ void child_box(const float4* tri, const float4* nodes, uint32_t c, float lo[3], float hi[3])
{
    if (c & kLeafBit) { tri_box(tri, c & ~kLeafBit, lo, hi); return; }
    const volatile float4* n = nodes + 4 * (size_t)c;
    float l0x = n[0].x, l0y = n[0].y, l0z = n[0].z, l1x = n[1].x, l1y = n[1].y, l1z = n[1].z;
    float r0x = n[2].x, r0y = n[2].y, r0z = n[2].z, r1x = n[3].x, r1y = n[3].y, r1z = n[3].z;
    lo[0] = fminf(l0x, r0x); lo[1] = fminf(l0y, r0y); lo[2] = fminf(l0z, r0z);
    hi[0] = fmaxf(l1x, r1x); hi[1] = fmaxf(l1y, r1y); hi[2] = fmaxf(l1z, r1z);
}

__global__ void k_refit(const float4* __restrict__ tri, int n, float4* nodes, const uint32_t* __restrict__ parent,
                        const uint32_t* __restrict__ leafParent, uint32_t* arrivals)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    uint32_t node = leafParent[k];
    while (true)
    {
        __threadfence();
        if (atomicAdd(&arrivals[node], 1u) == 0u) return; // the sibling subtree is not finished yet
        __threadfence();
        uint32_t cl = __float_as_uint(((volatile float4*)nodes)[4 * (size_t)node + 0].w);
        uint32_t cr = __float_as_uint(((volatile float4*)nodes)[4 * (size_t)node + 1].w);
        float llo[3], lhi[3], rlo[3], rhi[3];
        child_box(tri, nodes, cl, llo, lhi);
        child_box(tri, nodes, cr, rlo, rhi);
        volatile float4* o = (volatile float4*)(nodes + 4 * (size_t)node);
        o[0].x = llo[0]; o[0].y = llo[1]; o[0].z = llo[2];
        o[1].x = lhi[0]; o[1].y = lhi[1]; o[1].z = lhi[2];
        o[2].x = rlo[0]; o[2].y = rlo[1]; o[2].z = rlo[2];
        o[3].x = rhi[0]; o[3].y = rhi[1]; o[3].z = rhi[2];
        if (node == 0) return;
        node = parent[node];
    }
}

cudaError_t build_lbvh(const float4* dTri, uint32_t n, float4* dNodes, uint32_t* rootOut, cudaStream_t s)
{
    if (n == 0) { *rootOut = 0; return cudaSuccess; }
    if (n == 1) { *rootOut = kLeafBit | 0u; return cudaSuccess; }
    cudaError_t e;
    uint64_t *keys = nullptr, *keys2 = nullptr;
    uint32_t *vals = nullptr, *vals2 = nullptr, *bounds = nullptr;
    uint32_t *parent = nullptr, *leafParent = nullptr, *arrivals = nullptr;
    void* temp = nullptr;
    size_t tempBytes = 0;
#define RS_TRY(x) do { e = (x); if (e != cudaSuccess) goto done; } while (0)
    RS_TRY(cudaMalloc(&keys, n * 8ull)); RS_TRY(cudaMalloc(&vals, n * 4ull));
    RS_TRY(cudaMalloc(&keys2, n * 8ull)); RS_TRY(cudaMalloc(&vals2, n * 4ull));
    RS_TRY(cudaMalloc(&bounds, 6 * 4ull));
    RS_TRY(cudaMalloc(&parent, n * 4ull)); RS_TRY(cudaMalloc(&leafParent, n * 4ull)); RS_TRY(cudaMalloc(&arrivals, n * 4ull));
    {
        uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
        RS_TRY(cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, s));
        k_centroid_bounds<<<592, 256, 0, s>>>(dTri, n, bounds);
        k_morton<<<(n + 255) / 256, 256, 0, s>>>(dTri, n, bounds, keys, vals);
        RS_TRY(cub::DeviceRadixSort::SortPairs(nullptr, tempBytes, keys, keys2, vals, vals2, (int)n, 0, 63, s));
        RS_TRY(cudaMalloc(&temp, tempBytes));
        RS_TRY(cub::DeviceRadixSort::SortPairs(temp, tempBytes, keys, keys2, vals, vals2, (int)n, 0, 63, s));
        RS_TRY(cudaMemsetAsync(dNodes, 0, 64ull * (n - 1), s));
        k_karras<<<(n - 1 + 255) / 256, 256, 0, s>>>(keys2, vals2, (int)n, dNodes, parent, leafParent);
        RS_TRY(cudaMemsetAsync(arrivals, 0, n * 4ull, s));
        k_refit<<<(n + 255) / 256, 256, 0, s>>>(dTri, (int)n, dNodes, parent, leafParent, arrivals);
        RS_TRY(cudaGetLastError());
        RS_TRY(cudaStreamSynchronize(s));
        *rootOut = 0;
    }
done:
#undef RS_TRY
    cudaFree(keys); cudaFree(vals); cudaFree(keys2); cudaFree(vals2); cudaFree(bounds);
    cudaFree(parent); cudaFree(leafParent); cudaFree(arrivals); cudaFree(temp);
    return e;
}

} // namespace rs
