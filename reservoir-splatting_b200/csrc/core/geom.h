// Scene geometry records, hit packing, ray/triangle intersection and shading
// data: the part of Falcor's Scene layer that the Reservoir Splatting pass uses.
//
//  * HitInfo: the uncompressed 128-bit triangle hit (Scene/HitInfo.slang:92-123):
//    word0 = hit type (0 none, 1 triangle), word1 = primitive index,
//    word2/3 = barycentrics (u, v) as float bits.  A distant (environment) light
//    reconnection reuses words 1-3 for a direction with type 0
//    (PathTracer.slang:1084-1085, 1505-1506).
//  * Triangles are a flattened world-space soup; the vertex interpolation and
//    face normal follow Scene/Scene.slang:440-475 with an identity world matrix.
//  * computeRayOrigin is Utils/Geometry/GeometryHelpers.slang:54-68.
//  * Ray/triangle intersection is Moller-Trumbore, two-sided, with the hit
//    accepted on the open interval (tMin, tMax).  The hardware intersector the
//    reference relies on (DXR) has no published arithmetic; this replaces it.
#pragma once
#include "vec.h"

namespace rs {

struct alignas(16) f4 { float x, y, z, w; };

enum HitType : uint32_t { kHitNone = 0, kHitTriangle = 1 };
constexpr uint32_t kInvalidIndex = 0xffffffffu;

struct HitInfo
{
    uint32_t w[4];
};

RS_HD HitInfo hit_none() { HitInfo h; h.w[0] = h.w[1] = h.w[2] = h.w[3] = 0; return h; }
RS_HD HitInfo hit_tri(uint32_t prim, float u, float v)
{
    HitInfo h; h.w[0] = kHitTriangle; h.w[1] = prim; h.w[2] = f2u(u); h.w[3] = f2u(v); return h;
}
RS_HD bool hit_valid(const HitInfo& h) { return h.w[0] != kHitNone; }
RS_HD uint32_t hit_prim(const HitInfo& h) { return h.w[1]; }
RS_HD f2 hit_bary(const HitInfo& h) { return mk2(u2f(h.w[2]), u2f(h.w[3])); }
RS_HD HitInfo hit_direction(f3 d)
{
    HitInfo h; h.w[0] = 0; h.w[1] = f2u(d.x); h.w[2] = f2u(d.y); h.w[3] = f2u(d.z); return h;
}
RS_HD f3 hit_as_direction(const HitInfo& h) { return mk3(u2f(h.w[1]), u2f(h.w[2]), u2f(h.w[3])); }

struct Ray
{
    f3 origin;
    float tMin;
    f3 dir;
    float tMax;
};
RS_HD Ray mk_ray(f3 o, f3 d, float tmin, float tmax) { Ray r; r.origin = o; r.dir = d; r.tMin = tmin; r.tMax = tmax; return r; }

// Triangle record: three float4 per triangle.
//   [0] = p0.xyz, material id (uint bits)
//   [1] = p1.xyz, emissive light index (uint bits, kInvalidIndex if not emissive)
//   [2] = p2.xyz, unused
struct TriangleView
{
    const f4* tri;
    uint32_t count;
};

// Moller-Trumbore, no culling.  Returns true and (t, u, v) when
// tMin < t < tMax and the barycentrics lie in the triangle.
// The test with the edges e1 = p1 - p0, e2 = p2 - p0 already formed (same result bit for bit).
RS_HD bool intersect_triangle_e(f3 o, f3 d, f3 p0, f3 e1, f3 e2, float tMin, float tMax, float& t, float& u, float& v)
{
    f3 pv = cross(d, e2);
    float det = dot(e1, pv);
    if (det == 0.f) return false;
    float inv = 1.f / det;
    f3 tv = o - p0;
    u = dot(tv, pv) * inv;
    if (!(u >= 0.f && u <= 1.f)) return false;
    f3 qv = cross(tv, e1);
    v = dot(d, qv) * inv;
    if (!(v >= 0.f && u + v <= 1.f)) return false;
    t = dot(e2, qv) * inv;
    return t > tMin && t < tMax;
}
// A ray with a NaN in its origin, direction or interval hits no triangle (every comparison in
// intersect_triangle_e fails on NaN) while min/max slab tests accept every box for it, so
// traversals return a miss for it before visiting any node: the result of a full traversal,
// without its cost (a NaN camera time makes such rays).
RS_HD bool ray_has_nan(const Ray& r)
{
    return !(r.origin.x == r.origin.x && r.origin.y == r.origin.y && r.origin.z == r.origin.z && r.dir.x == r.dir.x &&
             r.dir.y == r.dir.y && r.dir.z == r.dir.z && r.tMin == r.tMin && r.tMax == r.tMax);
}
RS_HD bool intersect_triangle(f3 o, f3 d, f3 p0, f3 p1, f3 p2, float tMin, float tMax, float& t, float& u, float& v)
{
    return intersect_triangle_e(o, d, p0, p1 - p0, p2 - p0, tMin, tMax, t, u, v);
}

// GeometryHelpers.slang:54-68 (integer ulp offset away from the surface).
RS_HD float offset_component(float p, float n)
{
    const float origin = 1.f / 16.f;
    const float fScale = 3.f / 65536.f;
    const float iScale = 3.f * 256.f;
    int32_t iOff = (int32_t)(n * iScale);
    float iPos = i2f_bits(f2i_bits(p) + (p < 0.f ? -iOff : iOff));
    float fOff = n * fScale;
    return f_abs(p) < origin ? p + fOff : iPos;
}
RS_HD f3 computeRayOrigin(f3 pos, f3 n)
{
    return mk3(offset_component(pos.x, n.x), offset_component(pos.y, n.y), offset_component(pos.z, n.z));
}

// Shading data for an opaque triangle hit (MaterialFactory.slang:78-100,
// ShadingData.slang:77-88).  The shading frame is the face normal with an
// invented tangent (ShadingFrame.slang:76-83, 138-156; MathHelpers.slang:542-554).
struct ShadingData
{
    f3 posW;
    f3 V;
    f3 faceN;
    f3 N, T, B; // shading frame (after the double-sided flip)
    bool frontFacing;
    uint32_t materialID;
    uint32_t lightIndex;
};

RS_HD f3 perp_stark(f3 u)
{
    f3 a = abs3(u);
    uint32_t uyx = (a.x - a.y) < 0.f ? 1u : 0u;
    uint32_t uzx = (a.x - a.z) < 0.f ? 1u : 0u;
    uint32_t uzy = (a.y - a.z) < 0.f ? 1u : 0u;
    uint32_t xm = uyx & uzx;
    uint32_t ym = (1u ^ xm) & uzy;
    uint32_t zm = 1u ^ (xm | ym);
    return normalize(cross(u, mk3((float)xm, (float)ym, (float)zm)));
}

// loadShadingData of a hit that is not a triangle hit (LoadShadingData.slang:69-74, 134-141): the
// zero VertexData and material 0.  A record whose light vertex was an analytic light holds such a
// hit; the reconnection then sees a vertex at the origin with a zero normal.
RS_HD ShadingData sd_zero_vertex()
{
    ShadingData sd;
    sd.posW = mk3(0.f); sd.V = mk3(0.f); sd.faceN = mk3(0.f);
    sd.N = mk3(0.f); sd.T = mk3(0.f); sd.B = mk3(0.f);
    sd.frontFacing = true; // dot(V, faceN) >= 0
    sd.materialID = 0; sd.lightIndex = kInvalidIndex;
    return sd;
}

RS_HD f3 sd_ray_origin(const ShadingData& sd, bool viewside = true)
{
    return computeRayOrigin(sd.posW, (sd.frontFacing == viewside) ? sd.faceN : -sd.faceN);
}
RS_HD f3 sd_oriented_face_normal(const ShadingData& sd) { return sd.frontFacing ? sd.faceN : -sd.faceN; }
RS_HD f3 sd_to_local(const ShadingData& sd, f3 v) { return mk3(dot(v, sd.T), dot(v, sd.B), dot(v, sd.N)); }
RS_HD f3 sd_from_local(const ShadingData& sd, f3 v) { return sd.T * v.x + sd.B * v.y + sd.N * v.z; }

RS_HD f3 f4xyz(const f4& a) { return mk3(a.x, a.y, a.z); }

} // namespace rs
