// Linear BVH over the triangle soup and its stack traversal: the ray-query
// layer that replaces the reference's hardware acceleration structure
// (SceneRayQuery::traceRay / traceVisibilityRay, Scene/RaytracingInline.slang:86-362).
//
// Node layout (64 B, one 4 x float4 record per internal node):
//   [0] = left child box lo.xyz,  left child index (uint bits)
//   [1] = left child box hi.xyz,  right child index (uint bits)
//   [2] = right child box lo.xyz, unused
//   [3] = right child box hi.xyz, unused
// A child index with bit 31 set is a leaf holding the triangle index in bits 0-30.
// Boxes are padded outward by a relative 1e-6 so a box test can only prune, never
// reject a triangle the exact intersection test accepts; the closest hit is the
// (t, triangle index) minimum over all triangles and does not depend on the tree.
#pragma once
#include "core/material.h"

namespace rs {

constexpr uint32_t kLeafBit = 0x80000000u;
constexpr int kTraversalStack = 64;

struct BvhView
{
    const float4* nodes;
    const float4* tri;      // 3 float4 per triangle (see geom.h TriangleView)
    uint32_t root;          // kLeafBit | tri when the scene has one triangle
    uint32_t numTris;
};

__device__ __forceinline__ bool slab_interval(float lo, float hi, float o, float inv, float& t0, float& t1)
{
    float a = (lo - o) * inv, b = (hi - o) * inv;
    if (a != a) a = -3e38f; // (0 * inf): origin on the slab plane, direction parallel
    if (b != b) b = 3e38f;
    t0 = fmaxf(t0, fminf(a, b));
    t1 = fminf(t1, fmaxf(a, b));
    return true;
}

__device__ __forceinline__ bool box_hit(float4 lo, float4 hi, f3 o, f3 inv, float tmax, float& tEntry)
{
    float t0 = 0.f, t1 = tmax;
    slab_interval(lo.x, hi.x, o.x, inv.x, t0, t1);
    slab_interval(lo.y, hi.y, o.y, inv.y, t0, t1);
    slab_interval(lo.z, hi.z, o.z, inv.z, t0, t1);
    tEntry = t0;
    return t0 <= t1 + 2e-6f * fabsf(t1);
}

__device__ __forceinline__ bool tri_test(const BvhView& bv, uint32_t prim, const Ray& r, float& t, float& u, float& v)
{
    float4 a = __ldg(&bv.tri[3 * prim + 0]);
    float4 b = __ldg(&bv.tri[3 * prim + 1]);
    float4 c = __ldg(&bv.tri[3 * prim + 2]);
    return intersect_triangle(r.origin, r.dir, mk3(a.x, a.y, a.z), mk3(b.x, b.y, b.z), mk3(c.x, c.y, c.z), r.tMin, r.tMax, t, u, v);
}

// Closest hit on (tMin, tMax); ties on t go to the lower triangle index.
// Returns false on a miss.  *overflow is set when the stack would overflow (the
// remaining subtree is skipped, the caller reports a device fault).
__device__ inline bool trace_closest(const BvhView& bv, const Ray& r, HitInfo& hit, float& tHit, uint32_t* overflow)
{
    if (bv.numTris == 0) return false;
    f3 inv = mk3(1.f / r.dir.x, 1.f / r.dir.y, 1.f / r.dir.z);
    float best = r.tMax;
    uint32_t bestPrim = kInvalidIndex;
    float bu = 0.f, bv_ = 0.f;
    uint32_t stack[kTraversalStack];
    int sp = 0;
    uint32_t node = bv.root;
    while (true)
    {
        if (node & kLeafBit)
        {
            uint32_t prim = node & ~kLeafBit;
            float t, u, v;
            if (tri_test(bv, prim, r, t, u, v) && (t < best || (t == best && prim < bestPrim)))
            {
                best = t; bestPrim = prim; bu = u; bv_ = v;
            }
            if (sp == 0) break;
            node = stack[--sp];
            continue;
        }
        const float4* n = bv.nodes + 4 * (size_t)node;
        float4 l0 = __ldg(n + 0), l1 = __ldg(n + 1), r0 = __ldg(n + 2), r1 = __ldg(n + 3);
        float tl, tr;
        bool hl = box_hit(l0, l1, r.origin, inv, best, tl);
        bool hr = box_hit(r0, r1, r.origin, inv, best, tr);
        uint32_t cl = __float_as_uint(l0.w), cr = __float_as_uint(l1.w);
        if (hl && hr)
        {
            uint32_t nearC = tl <= tr ? cl : cr, farC = tl <= tr ? cr : cl;
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
    if (bestPrim == kInvalidIndex) return false;
    hit = hit_tri(bestPrim, bu, bv_);
    tHit = best;
    return true;
}

// True when no triangle is hit on (tMin, tMax).
__device__ inline bool trace_visible(const BvhView& bv, const Ray& r, uint32_t* overflow)
{
    if (bv.numTris == 0) return true;
    f3 inv = mk3(1.f / r.dir.x, 1.f / r.dir.y, 1.f / r.dir.z);
    uint32_t stack[kTraversalStack];
    int sp = 0;
    uint32_t node = bv.root;
    while (true)
    {
        if (node & kLeafBit)
        {
            float t, u, v;
            if (tri_test(bv, node & ~kLeafBit, r, t, u, v)) return false;
            if (sp == 0) break;
            node = stack[--sp];
            continue;
        }
        const float4* n = bv.nodes + 4 * (size_t)node;
        float4 l0 = __ldg(n + 0), l1 = __ldg(n + 1), r0 = __ldg(n + 2), r1 = __ldg(n + 3);
        float tl, tr;
        bool hl = box_hit(l0, l1, r.origin, inv, r.tMax, tl);
        bool hr = box_hit(r0, r1, r.origin, inv, r.tMax, tr);
        uint32_t cl = __float_as_uint(l0.w), cr = __float_as_uint(l1.w);
        if (hl && hr)
        {
            if (sp < kTraversalStack) stack[sp++] = cr;
            else *overflow = 1u;
            node = cl;
        }
        else if (hl) node = cl;
        else if (hr) node = cr;
        else
        {
            if (sp == 0) break;
            node = stack[--sp];
        }
    }
    return true;
}

} // namespace rs
