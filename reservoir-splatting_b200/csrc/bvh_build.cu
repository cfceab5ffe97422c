// BVH construction on the GPU, once per rs_set_scene.
//
// 1. Binary tree: 63-bit Morton codes (21 bits per axis) of the triangle centroids, a stable
//    radix sort of the triangle indices by key (radix_sort.cu), the triangles gathered in key order, then PLOC clustering of the ordered leaves
//    (below), or with kBvhLbvh the LBVH of k_karras (Karras 2012, "Maximizing parallelism in the
//    construction of BVHs, octrees, and k-d trees": the radix tree of the sorted keys) with its boxes
//    from k_refit, the bottom-up box pass with per-node arrival counters that also refits either
//    tree after geometry moves.
// 2. Collapse of the binary tree (kept for closest-hit queries) into the 4-wide tree of bvh.cuh, top down, one thread per node
//    and one launch per level: a node takes its binary node's two children and repeatedly opens
//    the child of largest surface area that holds more than four triangles, up to four children;
//    children of at most four triangles become leaves, which are ranges of the key-ordered
//    triangles (the leaf-order array).
#include <algorithm>
#include "radix_sort.h"
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

// keysOut[i] = keys[order[i]]
__global__ void k_gather_keys(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ order, uint32_t n, uint64_t* __restrict__ keysOut)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) keysOut[i] = keys[order[i]];
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

// Triangles in key order; the third record keeps the scene index in w.
__global__ void k_gather_sorted(const float4* __restrict__ tri, const uint32_t* __restrict__ order, uint32_t n, float4* __restrict__ sorted)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t t = order[i];
    sorted[3 * (size_t)i + 0] = tri[3 * (size_t)t + 0];
    sorted[3 * (size_t)i + 1] = tri[3 * (size_t)t + 1];
    float4 c = tri[3 * (size_t)t + 2];
    c.w = __uint_as_float(t);
    sorted[3 * (size_t)i + 2] = c;
}

// Binary node i: children in nodes[4i].w / nodes[4i+1].w (kLeafBit | sorted position for a leaf),
// its sorted range in range[i].
__global__ void k_karras(const uint64_t* __restrict__ keys, int n, float4* __restrict__ nodes, uint2* __restrict__ range,
                         uint32_t* __restrict__ parent, uint32_t* __restrict__ leafParent)
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
    uint32_t left = (lo == gamma) ? (kLeafBit | (uint32_t)gamma) : (uint32_t)gamma;
    uint32_t right = (hi == gamma + 1) ? (kLeafBit | (uint32_t)(gamma + 1)) : (uint32_t)(gamma + 1);
    nodes[4 * (size_t)i + 0].w = __uint_as_float(left);
    nodes[4 * (size_t)i + 1].w = __uint_as_float(right);
    range[i] = make_uint2((uint32_t)lo, (uint32_t)hi);
    if (lo == gamma) leafParent[gamma] = (uint32_t)i; else parent[gamma] = (uint32_t)i;
    if (hi == gamma + 1) leafParent[gamma + 1] = (uint32_t)i; else parent[gamma + 1] = (uint32_t)i;
}

__device__ __forceinline__ void tri_box(const float4* tri, uint32_t p, float lo[3], float hi[3])
{
    float4 a = tri[3 * (size_t)p], b = tri[3 * (size_t)p + 1], c = tri[3 * (size_t)p + 2];
    lo[0] = fminf(a.x, fminf(b.x, c.x)); hi[0] = fmaxf(a.x, fmaxf(b.x, c.x));
    lo[1] = fminf(a.y, fminf(b.y, c.y)); hi[1] = fmaxf(a.y, fmaxf(b.y, c.y));
    lo[2] = fminf(a.z, fminf(b.z, c.z)); hi[2] = fmaxf(a.z, fmaxf(b.z, c.z));
    for (int k = 0; k < 3; k++)
    {
        float pad = (fabsf(lo[k]) + fabsf(hi[k]) + (hi[k] - lo[k])) * 1e-6f + 1e-30f;
        lo[k] -= pad; hi[k] += pad;
    }
}

// Padded box of the triangle at leaf position p: tri is key ordered when leafTri is null, else scene
// ordered and reached through the scene index leafTri keeps.
__device__ __forceinline__ void leaf_box(const float4* tri, const float4* leafTri, uint32_t p, float lo[3], float hi[3])
{
    tri_box(tri, leafTri ? __float_as_uint(leafTri[3 * (size_t)p].w) : p, lo, hi);
}

__device__ __forceinline__ void child_box(const float4* tri, const float4* leafTri, const float4* nodes, uint32_t c, float lo[3], float hi[3])
{
    if (c & kLeafBit) { leaf_box(tri, leafTri, c & ~kLeafBit, lo, hi); return; }
    const volatile float4* n = nodes + 4 * (size_t)c;
    float l0x = n[0].x, l0y = n[0].y, l0z = n[0].z, l1x = n[1].x, l1y = n[1].y, l1z = n[1].z;
    float r0x = n[2].x, r0y = n[2].y, r0z = n[2].z, r1x = n[3].x, r1y = n[3].y, r1z = n[3].z;
    lo[0] = fminf(l0x, r0x); lo[1] = fminf(l0y, r0y); lo[2] = fminf(l0z, r0z);
    hi[0] = fmaxf(l1x, r1x); hi[1] = fmaxf(l1y, r1y); hi[2] = fmaxf(l1z, r1z);
}

__global__ void k_refit(const float4* __restrict__ tri, const float4* __restrict__ leafTri, int n, float4* nodes,
                        const uint32_t* __restrict__ parent, const uint32_t* __restrict__ leafParent, uint32_t* arrivals)
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
        child_box(tri, leafTri, nodes, cl, llo, lhi);
        child_box(tri, leafTri, nodes, cr, rlo, rhi);
        volatile float4* o = (volatile float4*)(nodes + 4 * (size_t)node);
        o[0].x = llo[0]; o[0].y = llo[1]; o[0].z = llo[2];
        o[1].x = lhi[0]; o[1].y = lhi[1]; o[1].z = lhi[2];
        o[2].x = rlo[0]; o[2].y = rlo[1]; o[2].z = rlo[2];
        o[3].x = rhi[0]; o[3].y = rhi[1]; o[3].z = rhi[2];
        if (node == 0) return;
        node = parent[node];
    }
}

// ------------------------------------------------------------------ PLOC (binary tree)
// Parallel locally-ordered clustering (Meister & Bittner 2018): the key-ordered leaves start as
// clusters; each round every cluster finds, among the kPlocRadius clusters on either side, the
// one whose merged box has the smallest surface area; mutual nearest neighbours merge into a new
// node; the clusters are compacted in order.  Node indices come from prefix sums of the merges,
// counting down from n - 2, so the numbering is deterministic and the last merge is the root, node 0.
constexpr int kPlocRadius = 24;

struct ClusterBox { float4 lo, hi; }; // lo.w = reference bits (kLeafBit | leaf, or node), hi.w = triangle count

__global__ void k_ploc_init(const float4* __restrict__ sorted, uint32_t n, ClusterBox* __restrict__ cl)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float lo[3], hi[3];
    tri_box(sorted, i, lo, hi);
    cl[i].lo = make_float4(lo[0], lo[1], lo[2], __uint_as_float(kLeafBit | i));
    cl[i].hi = make_float4(hi[0], hi[1], hi[2], __uint_as_float(1u));
}

__device__ __forceinline__ float union_area(const ClusterBox& a, const ClusterBox& b)
{
    float dx = fmaxf(a.hi.x, b.hi.x) - fminf(a.lo.x, b.lo.x);
    float dy = fmaxf(a.hi.y, b.hi.y) - fminf(a.lo.y, b.lo.y);
    float dz = fmaxf(a.hi.z, b.hi.z) - fminf(a.lo.z, b.lo.z);
    return dx * dy + dy * dz + dz * dx;
}

// Nearest neighbour of every cluster within the window; ties go to the lower index.
__global__ void k_ploc_nn(const ClusterBox* __restrict__ cl, uint32_t c, uint32_t* __restrict__ nn)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c) return;
    const ClusterBox me = cl[i];
    const uint32_t lo = i > (uint32_t)kPlocRadius ? i - kPlocRadius : 0u;
    const uint32_t hi = i + kPlocRadius < c - 1 ? i + kPlocRadius : c - 1;
    float best = 3e38f;
    uint32_t arg = i == 0 ? 1u : i - 1;
    for (uint32_t j = lo; j <= hi; j++)
    {
        if (j == i) continue;
        const float a = union_area(me, cl[j]);
        if (a < best) { best = a; arg = j; }
    }
    nn[i] = arg;
}

// merge[i]: i is the lower partner of a mutual pair (it creates the node); keep[i]: i survives the
// round (everything but the upper partner of a mutual pair).
__global__ void k_ploc_flags(const uint32_t* __restrict__ nn, uint32_t c, uint32_t* __restrict__ merge, uint32_t* __restrict__ keep)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c) return;
    const uint32_t j = nn[i];
    const bool mutual = nn[j] == i;
    merge[i] = (mutual && i < j) ? 1u : 0u;
    keep[i] = (mutual && i > j) ? 0u : 1u;
}

__global__ void k_ploc_merge(const ClusterBox* __restrict__ cl, uint32_t c, const uint32_t* __restrict__ nn, const uint32_t* __restrict__ merge,
                             const uint32_t* __restrict__ mergeOff, const uint32_t* __restrict__ keep, const uint32_t* __restrict__ keepOff,
                             uint32_t top, ClusterBox* __restrict__ out, float4* __restrict__ nodes, uint2* __restrict__ range,
                             uint32_t* __restrict__ parent, uint32_t* __restrict__ leafParent)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= c || !keep[i]) return;
    ClusterBox a = cl[i];
    if (merge[i])
    {
        const ClusterBox b = cl[nn[i]];
        const uint32_t node = top - mergeOff[i];
        const uint32_t ra = __float_as_uint(a.lo.w), rb = __float_as_uint(b.lo.w);
        float4* o = nodes + 4 * (size_t)node;
        o[0] = a.lo; o[1] = make_float4(a.hi.x, a.hi.y, a.hi.z, __uint_as_float(rb));
        o[2] = make_float4(b.lo.x, b.lo.y, b.lo.z, 0.f); o[3] = make_float4(b.hi.x, b.hi.y, b.hi.z, 0.f);
        const uint32_t count = __float_as_uint(a.hi.w) + __float_as_uint(b.hi.w);
        range[node] = make_uint2(0u, count - 1u); // only the triangle count is used for internal nodes
        if (ra & kLeafBit) leafParent[ra & ~kLeafBit] = node; else parent[ra] = node;
        if (rb & kLeafBit) leafParent[rb & ~kLeafBit] = node; else parent[rb] = node;
        a.lo = make_float4(fminf(a.lo.x, b.lo.x), fminf(a.lo.y, b.lo.y), fminf(a.lo.z, b.lo.z), __uint_as_float(node));
        a.hi = make_float4(fmaxf(a.hi.x, b.hi.x), fmaxf(a.hi.y, b.hi.y), fmaxf(a.hi.z, b.hi.z), __uint_as_float(count));
    }
    out[keepOff[i]] = a;
}

// ------------------------------------------------------------------ collapse to the 4-wide tree
struct WideChild
{
    uint32_t ref;          // binary reference (kLeafBit | sorted position, or internal node)
    uint32_t first, count; // sorted triangle range
    float lo[3], hi[3];
};

__device__ __forceinline__ float box_area(const WideChild& c)
{
    float dx = c.hi[0] - c.lo[0], dy = c.hi[1] - c.lo[1], dz = c.hi[2] - c.lo[2];
    return dx * dy + dy * dz + dz * dx;
}

__device__ __forceinline__ WideChild binary_child(const float4* nodes, const uint2* range, uint32_t b, int side)
{
    WideChild c;
    const float4* n = nodes + 4 * (size_t)b;
    float4 lo = n[2 * side], hi = n[2 * side + 1];
    c.ref = __float_as_uint(n[side].w);
    c.lo[0] = lo.x; c.lo[1] = lo.y; c.lo[2] = lo.z;
    c.hi[0] = hi.x; c.hi[1] = hi.y; c.hi[2] = hi.z;
    if (c.ref & kLeafBit) { c.first = c.ref & ~kLeafBit; c.count = 1; }
    else { uint2 r = range[c.ref]; c.first = r.x; c.count = r.y - r.x + 1; }
    return c;
}

constexpr uint32_t kWideLeafMax = 1; // triangles per leaf

__device__ __forceinline__ bool is_wide_leaf(const WideChild& c) { return (c.ref & kLeafBit) || c.count <= kWideLeafMax; }

// Writes node w for children c[0..n): internal children get consecutive node indices from
// childBase (returned through childOf), leaves reference their sorted range.
__device__ void write_wide_node(float4* wnodes, uint4* binRef, uint32_t w, const WideChild* c, int n, uint32_t childBase, uint32_t* childOf)
{
    float lo[3][4], hi[3][4];
    uint32_t ref[4], src[4];
    uint32_t nInternal = 0;
    for (int j = 0; j < 4; j++)
    {
        childOf[j] = kInvalidIndex;
        if (j >= n)
        {
            for (int a = 0; a < 3; a++) { lo[a][j] = __int_as_float(0x7f800000); hi[a][j] = __int_as_float(0xff800000); }
            ref[j] = kInvalidIndex;
            src[j] = kInvalidIndex;
            continue;
        }
        src[j] = c[j].ref;
        for (int a = 0; a < 3; a++) { lo[a][j] = c[j].lo[a]; hi[a][j] = c[j].hi[a]; }
        if (is_wide_leaf(c[j])) ref[j] = kLeafBit | (c[j].first << 2) | (c[j].count - 1u);
        else
        {
            ref[j] = childBase + nInternal;
            childOf[j] = childBase + nInternal;
            nInternal++;
        }
    }
    float4* o = wnodes + 7 * (size_t)w;
    o[0] = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
    o[1] = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
    o[2] = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
    o[3] = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
    o[4] = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
    o[5] = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
    o[6] = make_float4(__uint_as_float(ref[0]), __uint_as_float(ref[1]), __uint_as_float(ref[2]), __uint_as_float(ref[3]));
    binRef[w] = make_uint4(src[0], src[1], src[2], src[3]);
}

// counters: [0] nodes allocated, [1] unused, [2] next-level items, [3] unused
__global__ void k_collapse(const float4* __restrict__ nodes, const uint2* __restrict__ range, const uint2* __restrict__ qin, uint32_t nin,
                           uint2* __restrict__ qout, uint32_t* __restrict__ counters, float4* __restrict__ wnodes, uint4* __restrict__ binRef)
{
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nin) return;
    const uint2 item = qin[t]; // (binary internal node, wide node)
    WideChild c[4];
    int n = 2;
    c[0] = binary_child(nodes, range, item.x, 0);
    c[1] = binary_child(nodes, range, item.x, 1);
    while (n < 4)
    {
        int open = -1;
        float best = -1.f;
        for (int j = 0; j < n; j++)
            if (!is_wide_leaf(c[j]) && box_area(c[j]) > best) { best = box_area(c[j]); open = j; }
        if (open < 0) break;
        const uint32_t b = c[open].ref;
        c[open] = binary_child(nodes, range, b, 0);
        c[n++] = binary_child(nodes, range, b, 1);
    }
    uint32_t nInternal = 0;
    for (int j = 0; j < n; j++)
        if (!is_wide_leaf(c[j])) nInternal++;
    const uint32_t childBase = nInternal ? atomicAdd(&counters[0], nInternal) : 0u;
    uint32_t childOf[4];
    write_wide_node(wnodes, binRef, item.y, c, n, childBase, childOf);
    for (int j = 0; j < n; j++)
        if (childOf[j] != kInvalidIndex) qout[atomicAdd(&counters[2], 1u)] = make_uint2(c[j].ref, childOf[j]);
}

// A scene of one triangle: one node with one leaf.
__global__ void k_single_leaf(const float4* __restrict__ sorted, float4* __restrict__ wnodes, uint4* __restrict__ binRef)
{
    WideChild c;
    c.ref = kLeafBit;
    c.first = 0;
    c.count = 1;
    tri_box(sorted, 0, c.lo, c.hi);
    uint32_t childOf[4];
    write_wide_node(wnodes, binRef, 0, &c, 1, 0, childOf);
}

// Leaf-order triangles in the traversal form (p0, scene index), (p1 - p0), (p2 - p0).
__global__ void k_leaf_tris(const float4* __restrict__ sorted, uint32_t n, float4* __restrict__ leafTri)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = sorted[3 * (size_t)i], b = sorted[3 * (size_t)i + 1], c = sorted[3 * (size_t)i + 2];
    leafTri[3 * (size_t)i + 0] = make_float4(a.x, a.y, a.z, c.w);
    leafTri[3 * (size_t)i + 1] = make_float4(b.x - a.x, b.y - a.y, b.z - a.z, 0.f);
    leafTri[3 * (size_t)i + 2] = make_float4(c.x - a.x, c.y - a.y, c.z - a.z, 0.f);
}

// ------------------------------------------------------------------ refit to moved triangles
// Leaf triangles from the scene-order triangles through the scene index each one keeps.
__global__ void k_refit_leaf_tris(const float4* __restrict__ tri, uint32_t n, float4* __restrict__ leafTri)
{
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t t = __float_as_uint(leafTri[3 * (size_t)i].w);
    const float4 a = tri[3 * (size_t)t], b = tri[3 * (size_t)t + 1], c = tri[3 * (size_t)t + 2];
    leafTri[3 * (size_t)i + 0] = make_float4(a.x, a.y, a.z, __uint_as_float(t));
    leafTri[3 * (size_t)i + 1] = make_float4(b.x - a.x, b.y - a.y, b.z - a.z, 0.f);
    leafTri[3 * (size_t)i + 2] = make_float4(c.x - a.x, c.y - a.y, c.z - a.z, 0.f);
}

// Box of a binary reference: a leaf's padded triangle box, or the union of an internal node's children.
__device__ __forceinline__ void binary_ref_box(const float4* tri, const float4* leafTri, const float4* nodes, uint32_t ref, float lo[3], float hi[3])
{
    if (ref & kLeafBit) { leaf_box(tri, leafTri, ref & ~kLeafBit, lo, hi); return; }
    const float4* n = nodes + 4 * (size_t)ref;
    lo[0] = fminf(n[0].x, n[2].x); lo[1] = fminf(n[0].y, n[2].y); lo[2] = fminf(n[0].z, n[2].z);
    hi[0] = fmaxf(n[1].x, n[3].x); hi[1] = fmaxf(n[1].y, n[3].y); hi[2] = fmaxf(n[1].z, n[3].z);
}

__global__ void k_refit_wide(const float4* __restrict__ tri, const float4* __restrict__ leafTri, const float4* __restrict__ nodes,
                             const uint4* __restrict__ binRef, uint32_t numWide, float4* __restrict__ wnodes)
{
    uint32_t w = blockIdx.x * blockDim.x + threadIdx.x;
    if (w >= numWide) return;
    const uint4 src4 = binRef[w];
    const uint32_t src[4] = {src4.x, src4.y, src4.z, src4.w};
    float4* o = wnodes + 7 * (size_t)w;
    float lo[3][4], hi[3][4];
    for (int j = 0; j < 4; j++)
    {
        if (src[j] == kInvalidIndex)
        {
            for (int a = 0; a < 3; a++) { lo[a][j] = __int_as_float(0x7f800000); hi[a][j] = __int_as_float(0xff800000); }
            continue;
        }
        float l[3], h[3];
        binary_ref_box(tri, leafTri, nodes, src[j], l, h);
        for (int a = 0; a < 3; a++) { lo[a][j] = l[a]; hi[a][j] = h[a]; }
    }
    o[0] = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
    o[1] = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
    o[2] = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
    o[3] = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
    o[4] = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
    o[5] = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
}

cudaError_t refit_wide_bvh(const float4* dTri, WideBvh* b, cudaStream_t s)
{
    const uint32_t n = b->numTris;
    if (n == 0) return cudaSuccess;
    k_refit_leaf_tris<<<(n + 255) / 256, 256, 0, s>>>(dTri, n, b->leafTri);
    if (n > 1)
    {
        cudaError_t e = cudaMemsetAsync(b->arrivals, 0, n * 4ull, s);
        if (e != cudaSuccess) return e;
        k_refit<<<(n + 255) / 256, 256, 0, s>>>(dTri, b->leafTri, (int)n, b->binNodes, b->parent, b->leafParent, b->arrivals);
    }
    k_refit_wide<<<(b->numNodes + 127) / 128, 128, 0, s>>>(dTri, b->leafTri, b->binNodes, b->binRef, b->numNodes, b->nodes);
    return cudaGetLastError();
}

void free_wide_bvh(WideBvh* b)
{
    if (b->parent) cudaFree(b->parent);
    if (b->leafParent) cudaFree(b->leafParent);
    if (b->arrivals) cudaFree(b->arrivals);
    if (b->binRef) cudaFree(b->binRef);
    if (b->binNodes) cudaFree(b->binNodes);
    if (b->nodes) cudaFree(b->nodes);
    if (b->leafTri) cudaFree(b->leafTri);
    *b = WideBvh();
}

cudaError_t build_wide_bvh(const float4* dTri, uint32_t n, WideBvh* out, cudaStream_t s, BvhBuilder builder)
{
    free_wide_bvh(out);
    if (n == 0) return cudaSuccess;
    if (n >= kMaxBvhTriangles) return cudaErrorInvalidValue;
    cudaError_t e;
    uint64_t *keys = nullptr, *keys2 = nullptr;
    uint32_t *vals = nullptr, *vals2 = nullptr, *bounds = nullptr;
    uint32_t *parent = nullptr, *leafParent = nullptr, *arrivals = nullptr, *counters = nullptr;
    float4 *sorted = nullptr, *nodes = nullptr;
    uint2 *range = nullptr, *qa = nullptr, *qb = nullptr;
    void* temp = nullptr;
    size_t tempBytes = 0;
    const uint32_t maxWide = n / kWideLeafMax + 2; // every node but the root holds more than kWideLeafMax triangles
#define RS_TRY(x) do { e = (x); if (e != cudaSuccess) goto done; } while (0)
    RS_TRY(cudaMalloc(&out->nodes, 112ull * maxWide));
    RS_TRY(cudaMalloc(&out->binRef, 16ull * maxWide));
    RS_TRY(cudaMalloc(&out->leafTri, 48ull * n));
    RS_TRY(cudaMalloc(&keys, n * 8ull)); RS_TRY(cudaMalloc(&vals, n * 4ull));
    RS_TRY(cudaMalloc(&keys2, n * 8ull)); RS_TRY(cudaMalloc(&vals2, n * 4ull));
    RS_TRY(cudaMalloc(&bounds, 6 * 4ull));
    RS_TRY(cudaMalloc(&sorted, 48ull * n));
    RS_TRY(cudaMalloc(&counters, 4 * 4ull));
    RS_TRY(cudaMemsetAsync(counters, 0, 16, s));
    {
        uint32_t init[6] = {0xffffffffu, 0xffffffffu, 0xffffffffu, 0u, 0u, 0u};
        RS_TRY(cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, s));
        k_centroid_bounds<<<592, 256, 0, s>>>(dTri, n, bounds);
        k_morton<<<(n + 255) / 256, 256, 0, s>>>(dTri, n, bounds, keys, vals);
        // triangle indices in (Morton key, index) order, then the keys in that order for the Karras tree
        tempBytes = 4 * std::max(radix_scratch_words(n, 63), scan_scratch_words(n));
        RS_TRY(cudaMalloc(&temp, tempBytes));
        RS_TRY(radix_sort_indices_u64(keys, n, 63, vals2, vals, static_cast<uint32_t*>(temp), s));
        k_gather_keys<<<(n + 255) / 256, 256, 0, s>>>(keys, vals2, n, keys2);
        k_gather_sorted<<<(n + 255) / 256, 256, 0, s>>>(dTri, vals2, n, sorted);
        uint32_t levels = 0, numWide = 1;
        if (n == 1)
        {
            k_single_leaf<<<1, 1, 0, s>>>(sorted, out->nodes, out->binRef);
            levels = 1;
        }
        else
        {
            RS_TRY(cudaMalloc(&nodes, 64ull * (n - 1)));
            RS_TRY(cudaMalloc(&range, 8ull * (n - 1)));
            RS_TRY(cudaMalloc(&parent, n * 4ull)); RS_TRY(cudaMalloc(&leafParent, n * 4ull)); RS_TRY(cudaMalloc(&arrivals, n * 4ull));
            RS_TRY(cudaMalloc(&qa, 8ull * maxWide)); RS_TRY(cudaMalloc(&qb, 8ull * maxWide));
            RS_TRY(cudaMemsetAsync(nodes, 0, 64ull * (n - 1), s));
            k_leaf_tris<<<(n + 255) / 256, 256, 0, s>>>(sorted, n, out->leafTri);
            if (builder == kBvhLbvh)
            {
                // the radix tree of the sorted keys (node 0 = root), then its boxes bottom up
                k_karras<<<(n - 1 + 255) / 256, 256, 0, s>>>(keys2, (int)n, nodes, range, parent, leafParent);
                RS_TRY(cudaMemsetAsync(arrivals, 0, n * 4ull, s));
                k_refit<<<(n + 255) / 256, 256, 0, s>>>(dTri, out->leafTri, (int)n, nodes, parent, leafParent, arrivals);
                RS_TRY(cudaGetLastError());
            }
            else
            {
                // PLOC over the key-ordered leaves (node 0 = root); the binary tree the rest uses
                ClusterBox *ca = nullptr, *cb = nullptr;
                uint32_t *nn = nullptr, *mflag = nullptr, *kflag = nullptr, *moff = nullptr, *koff = nullptr;
                uint32_t* stemp = static_cast<uint32_t*>(temp); // the sort's scratch, sized for an n-element scan too
                RS_TRY(cudaMalloc(&ca, 32ull * n)); RS_TRY(cudaMalloc(&cb, 32ull * n));
                RS_TRY(cudaMalloc(&nn, 4ull * n)); RS_TRY(cudaMalloc(&mflag, 4ull * n)); RS_TRY(cudaMalloc(&kflag, 4ull * n));
                RS_TRY(cudaMalloc(&moff, 4ull * n)); RS_TRY(cudaMalloc(&koff, 4ull * n));
                k_ploc_init<<<(n + 255) / 256, 256, 0, s>>>(sorted, n, ca);
                uint32_t c = n, top = n - 2;
                while (c > 1 && e == cudaSuccess)
                {
                    k_ploc_nn<<<(c + 127) / 128, 128, 0, s>>>(ca, c, nn);
                    k_ploc_flags<<<(c + 255) / 256, 256, 0, s>>>(nn, c, mflag, kflag);
                    e = scan_exclusive_u32(mflag, moff, c, stemp, s);
                    if (e == cudaSuccess) e = scan_exclusive_u32(kflag, koff, c, stemp, s);
                    uint32_t tail[4] = {0, 0, 0, 0};
                    if (e == cudaSuccess) e = cudaMemcpyAsync(&tail[0], moff + c - 1, 4, cudaMemcpyDeviceToHost, s);
                    if (e == cudaSuccess) e = cudaMemcpyAsync(&tail[1], mflag + c - 1, 4, cudaMemcpyDeviceToHost, s);
                    if (e == cudaSuccess) e = cudaMemcpyAsync(&tail[2], koff + c - 1, 4, cudaMemcpyDeviceToHost, s);
                    if (e == cudaSuccess) e = cudaMemcpyAsync(&tail[3], kflag + c - 1, 4, cudaMemcpyDeviceToHost, s);
                    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
                    if (e != cudaSuccess) break;
                    const uint32_t merges = tail[0] + tail[1], kept = tail[2] + tail[3];
                    if (merges == 0 || kept + merges != c) { e = cudaErrorUnknown; break; } // a round always merges the globally closest pair
                    k_ploc_merge<<<(c + 255) / 256, 256, 0, s>>>(ca, c, nn, mflag, moff, kflag, koff, top, cb, nodes, range, parent, leafParent);
                    e = cudaGetLastError();
                    top -= merges;
                    c = kept;
                    std::swap(ca, cb);
                }
                cudaFree(ca); cudaFree(cb); cudaFree(nn); cudaFree(mflag); cudaFree(kflag); cudaFree(moff); cudaFree(koff);
                if (e != cudaSuccess) goto done;
            }
            const uint2 root = make_uint2(0u, 0u);
            const uint32_t one = 1u;
            RS_TRY(cudaMemcpyAsync(qa, &root, sizeof(root), cudaMemcpyHostToDevice, s));
            RS_TRY(cudaMemcpyAsync(counters, &one, 4, cudaMemcpyHostToDevice, s)); // node 0 is the root
            uint32_t nin = 1;
            while (nin > 0)
            {
                RS_TRY(cudaMemsetAsync(counters + 2, 0, 4, s));
                k_collapse<<<(nin + 127) / 128, 128, 0, s>>>(nodes, range, qa, nin, qb, counters, out->nodes, out->binRef);
                RS_TRY(cudaGetLastError());
                RS_TRY(cudaMemcpyAsync(&nin, counters + 2, 4, cudaMemcpyDeviceToHost, s));
                RS_TRY(cudaStreamSynchronize(s));
                std::swap(qa, qb);
                levels++;
            }
        }
        if (n == 1) k_leaf_tris<<<1, 256, 0, s>>>(sorted, n, out->leafTri);
        uint32_t host[4];
        RS_TRY(cudaMemcpyAsync(host, counters, 16, cudaMemcpyDeviceToHost, s));
        RS_TRY(cudaGetLastError());
        RS_TRY(cudaStreamSynchronize(s));
        numWide = n == 1 ? 1u : host[0];
        if (numWide > maxWide) { e = cudaErrorUnknown; goto done; }
        out->numNodes = numWide;
        out->depth = levels;
        out->binNodes = nodes; // the binary tree stays for closest-hit queries
        out->binRoot = n == 1 ? kLeafBit : 0u;
        out->numTris = n;
        out->parent = parent; out->leafParent = leafParent; out->arrivals = arrivals; // kept for refits
        nodes = nullptr; parent = nullptr; leafParent = nullptr; arrivals = nullptr;
    }
done:
#undef RS_TRY
    cudaFree(keys); cudaFree(vals); cudaFree(keys2); cudaFree(vals2); cudaFree(bounds); cudaFree(sorted); cudaFree(counters);
    cudaFree(nodes); cudaFree(range); cudaFree(parent); cudaFree(leafParent); cudaFree(arrivals); cudaFree(qa); cudaFree(qb);
    cudaFree(temp);
    if (e != cudaSuccess) free_wide_bvh(out);
    return e;
}

} // namespace rs
