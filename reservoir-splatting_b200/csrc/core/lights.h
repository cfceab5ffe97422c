// Emissive-triangle light sampling for next-event estimation.
//
//   Rendering/Lights/EmissivePowerSampler.slang:61-96, 113-120  power-proportional pick via a
//       packed alias table (16-bit threshold, 2 x 24-bit indices) then uniform area sampling
//   Rendering/Lights/EmissiveLightSamplerHelpers.slang:54-85, 111-124  triangle sample / pdf
//   Utils/Math/MathHelpers.slang:391-396  sample_triangle
//   PathTracer.slang:543-565, 606-701     light-type selection (emissive only here) and the
//       hemisphere rejection applied to the sample
#pragma once
#include "material.h"

namespace rs {

// One emissive triangle of the light collection (LightCollectionShared.slang EmissiveTriangle +
// EmissiveFlux): positions, face normal, area, radiance, flux and the scene triangle it came from.
struct alignas(16) LightTriangle
{
    float p0[3]; uint32_t sceneTri;
    float p1[3]; float area;
    float p2[3]; float flux;
    float normal[3]; uint32_t materialID;
    float Le[3]; float pad;
};

// Geometry of a light record from its triangle's current vertices (LightCollection.cpp /
// BuildTriangleList.cs.slang:62: normal = N / |N|, area = |N| / 2 with N = (p1 - p0) x (p2 - p0)).
// The flux, and so the power sampler's selection weights, stay those of the last scene or
// material update; selection and its pdf both read them, so the estimator stays consistent.
RS_HD void light_set_vertices(LightTriangle& L, f3 p0, f3 p1, f3 p2)
{
    f3 N = cross(p1 - p0, p2 - p0);
    float len = length(N);
    L.p0[0] = p0.x; L.p0[1] = p0.y; L.p0[2] = p0.z;
    L.p1[0] = p1.x; L.p1[1] = p1.y; L.p1[2] = p1.z;
    L.p2[0] = p2.x; L.p2[1] = p2.y; L.p2[2] = p2.z;
    L.area = 0.5f * len;
    if (len > 0.f)
    {
        f3 n = N / len;
        L.normal[0] = n.x; L.normal[1] = n.y; L.normal[2] = n.z;
    }
}

// EmissiveLightSamplerType (EmissiveLightSamplerType.slangh:36-44): the uniform and power samplers.
enum : uint32_t { kEmissiveUniform = 0, kEmissiveLightBVH = 1, kEmissivePower = 2 };

struct LightView
{
    const LightTriangle* tris;
    const u2* aliasTable;
    uint32_t count;
    float invWeightsSum;
    uint32_t sampler; // kEmissiveUniform or kEmissivePower
};

// evalTriangleSelectionPdf of the sampler: flux / total flux (power) or 1 / count (uniform,
// EmissiveUniformSampler.slang:81-87).
RS_HD float emissive_selection_pdf(const LightView& L, uint32_t triangleIndex)
{
    if (L.sampler == kEmissiveUniform) return L.count > 0 ? 1.f / (float)L.count : 0.f;
    return L.tris[triangleIndex].flux * L.invWeightsSum;
}

struct TriangleLightSample
{
    uint32_t triangleIndex;
    f3 posW;
    f3 normalW;
    f3 dir;
    float distance;
    f3 Le;
    float pdf;
    f2 uv;
    float geometryTerm;
};

RS_HD bool sample_triangle_light(const LightView& L, f3 posW, uint32_t triangleIndex, f2 u, TriangleLightSample& ls)
{
    ls.triangleIndex = triangleIndex;
    const LightTriangle& tri = L.tris[triangleIndex];
    float su = f_sqrt(u.x);
    f2 b = mk2(1.f - su, u.y * su);
    f3 bary = mk3(1.f - b.x - b.y, b.x, b.y);
    f3 p0 = mk3(tri.p0[0], tri.p0[1], tri.p0[2]);
    f3 p1 = mk3(tri.p1[0], tri.p1[1], tri.p1[2]);
    f3 p2 = mk3(tri.p2[0], tri.p2[1], tri.p2[2]);
    ls.posW = p0 * bary.x + p1 * bary.y + p2 * bary.z;
    f3 toLight = ls.posW - posW;
    const float distSqr = f_max(kFltMin, dot(toLight, toLight));
    ls.distance = f_sqrt(distSqr);
    ls.dir = toLight / ls.distance;
    ls.normalW = mk3(tri.normal[0], tri.normal[1], tri.normal[2]);
    float cosTheta = dot(ls.normalW, -ls.dir);
    if (cosTheta <= 0.f) return false;
    ls.Le = mk3(tri.Le[0], tri.Le[1], tri.Le[2]);
    float denom = f_max(kFltMin, cosTheta * tri.area);
    ls.pdf = distSqr / denom;
    float su2 = f_sqrt(u.x);
    ls.uv = mk2(1.f - su2, u.y * su2);
    ls.geometryTerm = cosTheta / distSqr;
    return true;
}

// EmissivePowerSampler::sampleLight.  Draw order: uLight, uAlias, then 2D on the triangle.
RS_HD bool sample_emissive_power(const LightView& L, f3 posW, SampleGen& sg, TriangleLightSample& ls)
{
    if (L.count == 0) return false;
    float uLight = sampleNext1D(sg);
    uint32_t triangleCount = L.count;
    uint32_t idx = (uint32_t)(uLight * (float)triangleCount);
    uint32_t triangleIndex = idx < triangleCount - 1 ? idx : triangleCount - 1;
    u2 packed = L.aliasTable[triangleIndex];
    float threshold = f16_to_f32((uint16_t)(packed.x >> 16u));
    uint32_t selectAbove = ((packed.x & 0xFFFFu) << 8u) | ((packed.y >> 24u) & 0xFFu);
    uint32_t selectBelow = packed.y & 0xFFFFFFu;
    triangleIndex = (sampleNext1D(sg) >= threshold) ? selectAbove : selectBelow;
    float triangleSelectionPdf = L.tris[triangleIndex].flux * L.invWeightsSum;
    f2 u; u.x = sampleNext1D(sg); u.y = sampleNext1D(sg);
    if (!sample_triangle_light(L, posW, triangleIndex, u, ls)) return false;
    ls.pdf *= triangleSelectionPdf;
    return true;
}

// EmissiveUniformSampler::sampleLight (EmissiveUniformSampler.slang:55-75): a triangle with
// probability 1 / count, then a uniform point on it.  Draw order: uLight, then 2D on the triangle.
RS_HD bool sample_emissive_uniform(const LightView& L, f3 posW, SampleGen& sg, TriangleLightSample& ls)
{
    if (L.count == 0) return false;
    float uLight = sampleNext1D(sg);
    uint32_t triangleCount = L.count;
    uint32_t idx = (uint32_t)(uLight * (float)triangleCount);
    uint32_t triangleIndex = idx < triangleCount - 1 ? idx : triangleCount - 1;
    float triangleSelectionPdf = 1.f / (float)triangleCount;
    f2 u; u.x = sampleNext1D(sg); u.y = sampleNext1D(sg);
    if (!sample_triangle_light(L, posW, triangleIndex, u, ls)) return false;
    ls.pdf *= triangleSelectionPdf;
    return true;
}

// The scene's emissive sampler (EmissiveLightSampler.slang: the type the pass was compiled with).
RS_HD bool sample_emissive(const LightView& L, f3 posW, SampleGen& sg, TriangleLightSample& ls)
{
    return L.sampler == kEmissiveUniform ? sample_emissive_uniform(L, posW, sg, ls) : sample_emissive_power(L, posW, sg, ls);
}

// The material of the emissive triangles whose radiance is Le (each channel within 1e-5 relative),
// when exactly one material qualifies; kInvalidIndex otherwise.  The adjoint's fallback for a light
// sample it cannot find again by tracing (a ray through the seam between two triangles of a light).
RS_HD uint32_t emissive_material_with_radiance(const LightView& L, f3 Le)
{
    uint32_t found = kInvalidIndex;
    for (uint32_t i = 0; i < L.count; i++)
    {
        const LightTriangle& t = L.tris[i];
        const float a[3] = {t.Le[0], t.Le[1], t.Le[2]}, b[3] = {Le.x, Le.y, Le.z};
        bool match = true;
        for (int c = 0; c < 3; c++) match = match && f_abs(a[c] - b[c]) <= 1e-5f * f_max(f_abs(a[c]), 1e-30f);
        if (!match) continue;
        if (found != kInvalidIndex && found != t.materialID) return kInvalidIndex;
        found = t.materialID;
    }
    return found;
}

// evalPdf + evalTrianglePdf of the power or uniform sampler: solid-angle pdf at posW of a hit on
// light triangleIndex.
RS_HD float eval_emissive_pdf(const LightView& L, f3 posW, uint32_t triangleIndex, f3 hitPosW, f3 hitNormalW)
{
    if (triangleIndex == kInvalidIndex) return 0.f;
    float triangleSelectionPdf = emissive_selection_pdf(L, triangleIndex);
    f3 toLight = hitPosW - posW;
    const float distSqr = dot(toLight, toLight);
    float trianglePdf;
    if (distSqr <= kFltMin) trianglePdf = 0.f;
    else
    {
        f3 Ld = toLight / f_sqrt(distSqr);
        float cosTheta = dot(hitNormalW, -Ld);
        if (cosTheta <= 0.f) trianglePdf = 0.f;
        else
        {
            float denom = f_max(kFltMin, cosTheta * L.tris[triangleIndex].area);
            trianglePdf = distSqr / denom;
        }
    }
    return triangleSelectionPdf * trianglePdf;
}

} // namespace rs
