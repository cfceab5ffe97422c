// The ray-query layer that replaces the reference's hardware acceleration structure
// (SceneRayQuery::traceRay / traceVisibilityRay, Scene/RaytracingInline.slang:86-362): two trees
// over the same triangles, each serving the query it traverses fastest.
//
// Closest hit: the binary tree (PLOC clustering of the Morton-ordered leaves), 64 bytes per
// internal node (four float4):
//   [0] left child box lo.xyz, left child reference   [1] left child box hi.xyz, right child reference
//   [2] right child box lo.xyz                         [3] right child box hi.xyz
// A reference with kLeafBit set is a single-triangle leaf (its position in the leaf-order array).
// The traversal visits the nearer child first and keeps the farther one on a stack.
//
// Visibility (any hit): the 4-wide tree collapsed from it, 112 bytes per node (seven float4),
// children's boxes as structure of arrays:
//   [0] lo.x of children 0-3   [1] hi.x   [2] lo.y   [3] hi.y   [4] lo.z   [5] hi.z
//   [6] child references (uint bits): an internal child's node index; a leaf
//       kLeafBit | first << 2 | (count - 1), count 1..4 triangles from leaf triangle `first`;
//       an empty slot kInvalidIndex with the box (+inf, -inf), which no ray enters.
// Leaf triangles are the scene's triangles in leaf order as (p0, scene index), (p1 - p0), (p2 - p0)
// (the edges the intersection test forms anyway).
//
// Child boxes are padded outward by a relative 1e-6 of their coordinates and a box counts as hit
// when its entry distance is within 2e-6 |exit distance| of the exit, so a box test only prunes
// triangles the exact intersection test rejects: the slab distances are off by a few ulp of the
// box coordinate (inside the padding) and of t (inside the slack).  A zero direction component
// uses 1/d = +-1e20, so the products stay finite and NaN-free.
// The closest hit is the (t, scene index) minimum over all triangles and does not depend on the
// tree; shading reads the scene-order triangle array.
#pragma once
#include "core/material.h"

namespace rs {

constexpr uint32_t kLeafBit = 0x80000000u;
constexpr uint32_t kMaxBvhTriangles = 1u << 29; // leaf references keep `first` in 29 bits
constexpr int kTraversalStack = 64;             // pending subtrees per ray

struct BvhView
{
    const float4* binNodes; // binary nodes, four float4 each
    uint32_t binRoot;       // 0, or kLeafBit | 0 for a scene of one triangle
    const float4* nodes;    // 4-wide nodes, seven float4 each; the root is node 0
    const float4* leafTri;  // leaf-order triangles, three float4 each
    const float4* tri;      // scene-order triangles (geom.h layout), for shading
    uint32_t numTris;
};

// A ray as values: the traversal keeps it in registers (a reference into local or constant
// memory could alias the traversal stack and force reloads).
struct RayQ
{
    float ox, oy, oz, dx, dy, dz;
    float ix, iy, iz; // 1/d, a zero component as +-1e20 (keeps the sign, no inf * 0)
    float ox_ix, oy_iy, oz_iz;
    float tMin, tMax;
    uint32_t nearX, farX, nearY, farY, nearZ, farZ; // node float4 holding each axis' entry / exit planes
};

__device__ __forceinline__ float safe_inv(float d) { return fabsf(d) > 1e-20f ? 1.f / d : copysignf(1e20f, d); }

__device__ __forceinline__ RayQ make_rayq(const Ray& r)
{
    RayQ q;
    q.ox = r.origin.x; q.oy = r.origin.y; q.oz = r.origin.z;
    q.dx = r.dir.x; q.dy = r.dir.y; q.dz = r.dir.z;
    q.ix = safe_inv(r.dir.x); q.iy = safe_inv(r.dir.y); q.iz = safe_inv(r.dir.z);
    q.ox_ix = q.ox * q.ix; q.oy_iy = q.oy * q.iy; q.oz_iz = q.oz * q.iz;
    q.tMin = r.tMin; q.tMax = r.tMax;
    const uint32_t sx = q.ix < 0.f ? 1u : 0u, sy = q.iy < 0.f ? 1u : 0u, sz = q.iz < 0.f ? 1u : 0u;
    q.nearX = sx; q.farX = 1u - sx; q.nearY = 2u + sy; q.farY = 3u - sy; q.nearZ = 4u + sz; q.farZ = 5u - sz;
    return q;
}

__device__ __forceinline__ float max3f(float a, float b, float c)
{
    float r;
    asm("max.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}
__device__ __forceinline__ float min3f(float a, float b, float c)
{
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// Entry distance into a child box given its entry planes (nx, ny, nz) and exit planes (fx, fy, fz)
// along the ray's direction, or kMissKey when the box is not entered before tmax.  With 1/d's
// sign the entry plane of each slab is known, so one fma per plane and two 3-way min / max give
// the interval (the same interval as min / max over both planes).
constexpr float kMissKey = 3e38f;
__device__ __forceinline__ float child_entry(float nx, float fx, float ny, float fy, float nz, float fz, const RayQ& r, float tmax)
{
    const float t0 = max3f(__fmaf_rn(nx, r.ix, -r.ox_ix), __fmaf_rn(ny, r.iy, -r.oy_iy), fmaxf(__fmaf_rn(nz, r.iz, -r.oz_iz), 0.f));
    const float t1 = min3f(__fmaf_rn(fx, r.ix, -r.ox_ix), __fmaf_rn(fy, r.iy, -r.oy_iy), fminf(__fmaf_rn(fz, r.iz, -r.oz_iz), tmax));
    return t0 <= __fmaf_rn(2e-6f, fabsf(t1), t1) ? t0 : kMissKey;
}

__device__ __forceinline__ bool leaf_tri_test(const float4* __restrict__ leafTri, uint32_t k, const RayQ& r, float& t, float& u, float& v,
                                              uint32_t& prim)
{
    const float4 a = __ldg(&leafTri[3 * (size_t)k + 0]);
    const float4 b = __ldg(&leafTri[3 * (size_t)k + 1]);
    const float4 c = __ldg(&leafTri[3 * (size_t)k + 2]);
    prim = __float_as_uint(a.w);
    return intersect_triangle_e(mk3(r.ox, r.oy, r.oz), mk3(r.dx, r.dy, r.dz), mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z), mk3(c.x, c.y, c.z),
                                r.tMin, r.tMax, t, u, v);
}

struct TraceHit { uint32_t prim; float t, u, v; };

// Binary-node box test: slab distances t = box * (1/d) - o * (1/d) by fma, entry as the 3-way
// max of the near planes (and 0), exit as the 3-way min of the far planes (and tmax).
__device__ __forceinline__ bool box_hit(float4 lo, float4 hi, const RayQ& r, float tmax, float& tEntry)
{
    const float ax = __fmaf_rn(lo.x, r.ix, -r.ox_ix), bx = __fmaf_rn(hi.x, r.ix, -r.ox_ix);
    const float ay = __fmaf_rn(lo.y, r.iy, -r.oy_iy), by = __fmaf_rn(hi.y, r.iy, -r.oy_iy);
    const float az = __fmaf_rn(lo.z, r.iz, -r.oz_iz), bz = __fmaf_rn(hi.z, r.iz, -r.oz_iz);
    const float t0 = max3f(fminf(ax, bx), fminf(ay, by), fmaxf(fminf(az, bz), 0.f));
    const float t1 = min3f(fmaxf(ax, bx), fmaxf(ay, by), fminf(fmaxf(az, bz), tmax));
    tEntry = t0;
    return t0 <= __fmaf_rn(2e-6f, fabsf(t1), t1);
}

// Closest hit on (tMin, tMax) over the binary tree; ties on t go to the lower scene triangle index;
// prim is kInvalidIndex on a miss.  kCount adds the nodes visited and triangles tested to
// counts[0..1].  *overflow is set when the stack would overflow (the subtree is skipped and the
// caller reports a device fault).
template <bool kCount>
__device__ __forceinline__ TraceHit trace_closest_bin(const BvhView& bv, const Ray& r, uint32_t* overflow, uint32_t* counts = nullptr)
{
    TraceHit best;
    best.prim = kInvalidIndex; best.t = r.tMax; best.u = 0.f; best.v = 0.f;
    if (ray_has_nan(r)) return best;
    const RayQ q = make_rayq(r);
    uint32_t stack[kTraversalStack];
    int sp = 0;
    uint32_t node = bv.binRoot;
    while (true)
    {
        if (node & kLeafBit)
        {
            const uint32_t k = node & ~kLeafBit;
            const float4 a = __ldg(&bv.leafTri[3 * (size_t)k + 0]);
            const float4 b = __ldg(&bv.leafTri[3 * (size_t)k + 1]);
            const float4 c = __ldg(&bv.leafTri[3 * (size_t)k + 2]);
            const uint32_t prim = __float_as_uint(a.w);
            float t, u, v;
            if (kCount) counts[1]++;
            if (intersect_triangle_e(r.origin, r.dir, mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z), mk3(c.x, c.y, c.z), r.tMin, r.tMax, t, u, v) &&
                (t < best.t || (t == best.t && prim < best.prim)))
            {
                best.t = t; best.prim = prim; best.u = u; best.v = v;
            }
            if (sp == 0) break;
            node = stack[--sp];
            continue;
        }
        if (kCount) counts[0]++;
        const float4* n = bv.binNodes + 4 * (size_t)node;
        const float4 l0 = __ldg(n + 0), l1 = __ldg(n + 1), r0 = __ldg(n + 2), r1 = __ldg(n + 3);
        float tl, tr;
        const bool hl = box_hit(l0, l1, q, best.t, tl);
        const bool hr = box_hit(r0, r1, q, best.t, tr);
        const uint32_t cl = __float_as_uint(l0.w), cr = __float_as_uint(l1.w);
        if (hl && hr)
        {
            const uint32_t nearC = tl <= tr ? cl : cr, farC = tl <= tr ? cr : cl;
            if (sp < kTraversalStack) stack[sp++] = farC;
            else *overflow = 1u;
            node = nearC;
        }
        else if (hl) node = cl;
        else if (hr) node = cr;
        else
        {
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
    return best;
}

// True when no triangle is hit on (tMin, tMax).
static __device__ __noinline__ bool trace_visible_q(const float4* __restrict__ nodes, const float4* __restrict__ leafTri, RayQ r,
                                                    uint32_t* overflow)
{
    uint32_t stack[kTraversalStack];
    int sp = 0;
    uint32_t node = 0;
    while (true)
    {
        const float4* n = nodes + 7 * (size_t)node;
        const float4 nx = __ldg(n + r.nearX), fx = __ldg(n + r.farX), ny = __ldg(n + r.nearY), fy = __ldg(n + r.farY);
        const float4 nz = __ldg(n + r.nearZ), fz = __ldg(n + r.farZ);
        const uint4 rf = __ldg(reinterpret_cast<const uint4*>(n + 6));
        const bool h[4] = {child_entry(nx.x, fx.x, ny.x, fy.x, nz.x, fz.x, r, r.tMax) != kMissKey,
                           child_entry(nx.y, fx.y, ny.y, fy.y, nz.y, fz.y, r, r.tMax) != kMissKey,
                           child_entry(nx.z, fx.z, ny.z, fy.z, nz.z, fz.z, r, r.tMax) != kMissKey,
                           child_entry(nx.w, fx.w, ny.w, fy.w, nz.w, fz.w, r, r.tMax) != kMissKey};
        const uint32_t c4[4] = {rf.x, rf.y, rf.z, rf.w};
        uint32_t next = kInvalidIndex;
#pragma unroll
        for (int c = 0; c < 4; c++)
        {
            if (!h[c] || c4[c] == kInvalidIndex) continue;
            if (c4[c] & kLeafBit)
            {
                const uint32_t first = (c4[c] & ~kLeafBit) >> 2, count = (c4[c] & 3u) + 1u;
                for (uint32_t j = 0; j < count; j++)
                {
                    float t, u, v;
                    uint32_t prim;
                    if (leaf_tri_test(leafTri, first + j, r, t, u, v, prim)) return false;
                }
            }
            else
            {
                if (next != kInvalidIndex)
                {
                    if (sp < kTraversalStack) stack[sp++] = next;
                    else *overflow = 1u;
                }
                next = c4[c];
            }
        }
        if (next != kInvalidIndex) { node = next; continue; }
        if (sp == 0) break;
        node = stack[--sp];
    }
    return true;
}

#ifdef RS_RAY_STATS
// Ray counting for workload measurement (a build with -DRS_RAY_STATS only): closest-hit and
// visibility queries, one warp-aggregated atomic per call site and warp.
static __device__ unsigned long long g_rayStats[2];
__device__ __forceinline__ void count_ray(int kind)
{
    const unsigned m = __activemask();
    if ((threadIdx.x & 31u) == (unsigned)(__ffs(m) - 1)) atomicAdd(&g_rayStats[kind], (unsigned long long)__popc(m));
}
#else
__device__ __forceinline__ void count_ray(int) {}
#endif

__device__ __forceinline__ bool trace_closest(const BvhView& bv, const Ray& r, HitInfo& hit, float& tHit, uint32_t* overflow)
{
    count_ray(0);
    if (bv.numTris == 0) return false;
    const TraceHit h = trace_closest_bin<false>(bv, r, overflow);
    if (h.prim == kInvalidIndex) return false;
    hit = hit_tri(h.prim, h.u, h.v);
    tHit = h.t;
    return true;
}

// The closest-hit traversal as a call: one copy in kernels with several ray sites and many live
// values around them (the path tracer), where inlining it raises register pressure.
static __device__ __noinline__ TraceHit trace_closest_call(BvhView bv, Ray r, uint32_t* overflow)
{
    count_ray(0);
    return trace_closest_bin<false>(bv, r, overflow);
}

__device__ __forceinline__ bool trace_visible(const BvhView& bv, const Ray& r, uint32_t* overflow)
{
    count_ray(1);
    if (bv.numTris == 0 || ray_has_nan(r)) return true;
    return trace_visible_q(bv.nodes, bv.leafTri, make_rayq(r), overflow);
}

} // namespace rs
