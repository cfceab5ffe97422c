// Analytic light sources (point / spot, directional, distant, rect, disc, sphere) for next-event
// estimation: the scene's analytic lights that the path tracer samples when the scene uses them
// (PathTracer.slang:567-599, USE_ANALYTIC_LIGHTS).
//
//   Scene/Lights/LightData.slang:34-69          light types and the per-light data
//   Scene/Lights/Light.cpp:174-397              host-side derived values (spot cone cosine,
//       subtended cone cosine, distant-light rotation, area-light transform and surface area)
//   Rendering/Lights/LightHelpers.slang:67-284  sampling of each type
//   Utils/Math/MathHelpers.slang:269-304        sample_disk / sample_cone / sample_sphere
//
// Analytic lights have no geometry: rays never hit them, so they are reached by light sampling
// only (the path tracer's MIS weight for them is 1), and a point or directional light has a Dirac
// solid-angle pdf, reported as 0.
#pragma once
#include <cmath>
#include "material.h"

namespace rs {

enum AnalyticLightType : uint32_t { kLightPoint = 0, kLightDirectional = 1, kLightDistant = 2, kLightRect = 3, kLightDisc = 4, kLightSphere = 5 };

// Device record of one light (LightData with the fields the sampling reads).
struct alignas(16) AnalyticLight
{
    uint32_t type;
    float posW[3];             // point: position
    float dirW[3];             // point: spot axis; directional / distant: direction the light travels
    float intensity[3];        // radiance (area, distant, directional) or intensity (point)
    float openingAngle;        // point: spot half-angle
    float cosOpeningAngle;
    float penumbraAngle;
    float cosSubtendedAngle;   // distant: cosine of the subtended half-angle
    float surfaceArea;         // rect / disc / sphere
    float transMat[12];        // rows 0-2 of the object-to-world matrix (distant: its rotation)
    float transMatIT[9];       // the 3 x 3 inverse transpose of transMat, for normals
};

struct AnalyticLightView
{
    const AnalyticLight* lights;
    uint32_t count;
};

constexpr float kMinLightDistSqr = 1e-9f;       // LightHelpers.slang:43
constexpr float kMaxLightDistance = 3.40282347e38f; // FLT_MAX (LightHelpers.slang:44)

// AnalyticLightSample (LightHelpers.slang:53-61).
struct AnalyticSample
{
    f3 posW, normalW, dir, Li;
    float distance, pdf;
};

RS_HD f3 al_f3(const float* p) { return mk3(p[0], p[1], p[2]); }

// mul(transMat, float4(p, 1)).xyz: each row's dot product with (p, 1), in that order.
RS_HD f3 al_transform_point(const AnalyticLight& L, f3 p)
{
    const float* m = L.transMat;
    return mk3(m[0] * p.x + m[1] * p.y + m[2] * p.z + m[3], m[4] * p.x + m[5] * p.y + m[6] * p.z + m[7],
               m[8] * p.x + m[9] * p.y + m[10] * p.z + m[11]);
}
// mul((float3x3)transMat, v)
RS_HD f3 al_rotate(const AnalyticLight& L, f3 v)
{
    const float* m = L.transMat;
    return mk3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[4] * v.x + m[5] * v.y + m[6] * v.z, m[8] * v.x + m[9] * v.y + m[10] * v.z);
}
// mul(transMatIT, float4(n, 0)).xyz
RS_HD f3 al_transform_normal(const AnalyticLight& L, f3 n)
{
    const float* m = L.transMatIT;
    return mk3(m[0] * n.x + m[1] * n.y + m[2] * n.z, m[3] * n.x + m[4] * n.y + m[5] * n.z, m[6] * n.x + m[7] * n.y + m[8] * n.z);
}

// sample_cone (MathHelpers.slang:285-291): uniform direction within the cone of half-angle
// acos(cosTheta) around +z.
RS_HD f3 sample_cone(f2 u, float cosTheta)
{
    const float z = u.x * (1.f - cosTheta) + cosTheta;
    const float r = f_sqrt(1.f - z * z);
    const float phi = k2Pi * u.y;
    float s, c;
    f_sincos(phi, s, c);
    return mk3(r * c, r * s, z);
}

// sample_sphere (MathHelpers.slang:298-304): uniform point on the unit sphere.
RS_HD f3 sample_sphere(f2 u)
{
    const float phi = k2Pi * u.y;
    const float cosTheta = 1.f - 2.f * u.x;
    const float sinTheta = f_sqrt(f_max(0.f, 1.f - cosTheta * cosTheta));
    float s, c;
    f_sincos(phi, s, c);
    return mk3(sinTheta * c, sinTheta * s, cosTheta);
}

// HLSL smoothstep: t = saturate((x - a) / (b - a)), t^2 (3 - 2t).
RS_HD float f_smoothstep(float a, float b, float x)
{
    const float t = f_saturate((x - a) / (b - a));
    return t * t * (3.f - 2.f * t);
}

// finalizeAreaLightSample (LightHelpers.slang:67-86): direction, distance, radiance and the
// solid-angle pdf of an area-light point whose posW and normalW are set; area lights are
// one-sided.
RS_HD bool al_finalize_area(f3 shadingPosW, const AnalyticLight& L, AnalyticSample& ls)
{
    const f3 toLight = ls.posW - shadingPosW;
    const float distSqr = f_max(dot(toLight, toLight), kMinLightDistSqr);
    ls.distance = f_sqrt(distSqr);
    ls.dir = toLight / ls.distance;
    const float cosTheta = dot(ls.normalW, -ls.dir);
    if (cosTheta <= 0.f) return false;
    ls.Li = al_f3(L.intensity) * (L.surfaceArea * cosTheta / distSqr);
    ls.pdf = distSqr / (cosTheta * L.surfaceArea);
    return true;
}

// samplePointLight (LightHelpers.slang:217-250): a point light, a spot light when its opening
// angle is below pi, with a smoothstep penumbra of penumbraAngle inside the cone's edge.
RS_HD bool al_sample_point(f3 shadingPosW, const AnalyticLight& L, AnalyticSample& ls)
{
    ls.posW = al_f3(L.posW);
    ls.normalW = al_f3(L.dirW);
    const f3 toLight = ls.posW - shadingPosW;
    const float distSqr = f_max(dot(toLight, toLight), kMinLightDistSqr);
    ls.distance = f_sqrt(distSqr);
    ls.dir = toLight / ls.distance;
    const float cosTheta = -dot(ls.dir, al_f3(L.dirW));
    float falloff = 1.f;
    if (cosTheta < L.cosOpeningAngle) falloff = 0.f;
    else if (L.penumbraAngle > 0.f)
    {
        const float deltaAngle = L.openingAngle - f_acos(cosTheta);
        falloff = f_smoothstep(0.f, L.penumbraAngle, deltaAngle);
    }
    ls.Li = al_f3(L.intensity) * falloff / distSqr;
    ls.pdf = 0.f;
    return true;
}

// sampleDirectionalLight (LightHelpers.slang:190-209).
RS_HD bool al_sample_directional(const AnalyticLight& L, AnalyticSample& ls)
{
    ls.posW = mk3(0.f);
    ls.normalW = al_f3(L.dirW);
    ls.distance = kMaxLightDistance;
    ls.dir = -al_f3(L.dirW);
    ls.Li = al_f3(L.intensity);
    ls.pdf = 0.f;
    return true;
}

// sampleDistantLight (LightHelpers.slang:161-182): a direction in the subtended cone, rotated
// onto the light; the intensity is radiance.
RS_HD bool al_sample_distant(const AnalyticLight& L, f2 u, AnalyticSample& ls)
{
    ls.posW = mk3(0.f);
    ls.dir = normalize(al_rotate(L, sample_cone(u, L.cosSubtendedAngle)));
    ls.normalW = -ls.dir;
    ls.distance = kMaxLightDistance;
    const float solidAngle = k2Pi * (1.f - L.cosSubtendedAngle);
    ls.Li = al_f3(L.intensity);
    ls.pdf = 1.f / solidAngle;
    return true;
}

// sampleRectAreaLight / sampleDiscAreaLight / sampleSphereAreaLight (LightHelpers.slang:94-152):
// a uniform point of the object-space shape ([-1, 1]^2 quad, unit disc, unit sphere) moved to
// world space.
RS_HD bool al_sample_area(f3 shadingPosW, const AnalyticLight& L, f2 u, AnalyticSample& ls)
{
    f3 pos, n;
    if (L.type == kLightRect) { pos = mk3(u.x * 2.f - 1.f, u.y * 2.f - 1.f, 0.f); n = mk3(0.f, 0.f, 1.f); }
    else if (L.type == kLightDisc) { const f2 d = sample_disk(u); pos = mk3(d.x, d.y, 0.f); n = mk3(0.f, 0.f, 1.f); }
    else { pos = sample_sphere(u); n = pos; }
    ls.posW = al_transform_point(L, pos);
    ls.normalW = normalize(al_transform_normal(L, n));
    return al_finalize_area(shadingPosW, L, ls);
}

// sampleLight (LightHelpers.slang:260-284): the area and distant types draw two numbers.
RS_HD bool al_sample(f3 shadingPosW, const AnalyticLight& L, SampleGen& sg, AnalyticSample& ls)
{
    ls.posW = mk3(0.f); ls.normalW = mk3(0.f); ls.dir = mk3(0.f); ls.Li = mk3(0.f); ls.distance = 0.f; ls.pdf = 0.f;
    switch (L.type)
    {
    case kLightPoint: return al_sample_point(shadingPosW, L, ls);
    case kLightDirectional: return al_sample_directional(L, ls);
    case kLightRect:
    case kLightDisc:
    case kLightSphere:
    {
        f2 u; u.x = sampleNext1D(sg); u.y = sampleNext1D(sg);
        return al_sample_area(shadingPosW, L, u, ls);
    }
    case kLightDistant:
    {
        f2 u; u.x = sampleNext1D(sg); u.y = sampleNext1D(sg);
        return al_sample_distant(L, u, ls);
    }
    default: return false;
    }
}

// generateAnalyticLightSample (PathTracer.slang:573-599) up to the ray origin: a light picked
// uniformly, its sample, and the pdf / radiance of the pick.  False when there is no light or no
// radiance.
RS_HD bool analytic_light_sample(const AnalyticLightView& V, f3 shadingPosW, SampleGen& sg, AnalyticSample& ls)
{
    if (V.count == 0) return false;
    const float fc = (float)V.count;
    uint32_t idx = (uint32_t)(sampleNext1D(sg) * fc);
    if (idx > V.count - 1) idx = V.count - 1;
    if (!al_sample(shadingPosW, V.lights[idx], sg, ls)) return false;
    ls.pdf = ls.pdf / fc;
    ls.Li = ls.Li * fc;
    return any_gt0(ls.Li);
}

// ---------------------------------------------------------------- host: lights from their description
// The host-side values Falcor's light classes keep in LightData (Light.cpp:174-397), from the
// description a scene gives: position, direction, intensity, spot opening and penumbra angles,
// distant subtended angle, and an area light's object-to-world transform and scaling (row-major
// 4 x 4; the light's matrix is transform x scaling).
struct AnalyticLightDesc
{
    uint32_t type;
    float intensity[3];
    float position[3];
    float direction[3];
    float openingAngle, penumbraAngle, angle;
    float transform[16];
    float scaling[3];
};

// Fills `out` from `d`; false for an unknown type or a zero-length direction where one is needed.
inline bool prepare_analytic_light(const AnalyticLightDesc& d, AnalyticLight& out)
{
    AnalyticLight L{};
    L.type = d.type;
    for (int k = 0; k < 3; k++) { L.intensity[k] = d.intensity[k]; L.posW[k] = d.position[k]; }
    L.openingAngle = (float)M_PI;
    L.cosOpeningAngle = -1.f;
    L.cosSubtendedAngle = 0.9999893f; // LightData default (the sun seen from the earth)
    for (int r = 0; r < 3; r++) L.transMat[4 * r + r] = 1.f, L.transMatIT[3 * r + r] = 1.f;
    if (d.type > kLightSphere) return false;
    if (d.type == kLightPoint || d.type == kLightDirectional || d.type == kLightDistant)
    {
        // setWorldDirection: a normalised direction (a zero or NaN length is rejected)
        const float x = d.direction[0], y = d.direction[1], z = d.direction[2];
        const float len = std::sqrt(x * x + y * y + z * z);
        if (!(len > 0.f)) return false;
        L.dirW[0] = x / len; L.dirW[1] = y / len; L.dirW[2] = z / len;
    }
    else { L.dirW[0] = 0.f; L.dirW[1] = -1.f; L.dirW[2] = 0.f; }
    if (d.type == kLightPoint)
    {
        // setOpeningAngle / setPenumbraAngle: clamped to [0, pi] and [0, openingAngle]
        const float open = std::fmin(std::fmax(d.openingAngle, 0.f), (float)M_PI);
        L.openingAngle = open;
        L.cosOpeningAngle = std::cos(open);
        L.penumbraAngle = std::fmin(std::fmax(d.penumbraAngle, 0.f), open);
    }
    if (d.type == kLightDistant)
    {
        // setAngle: the half-angle clamped to [0, pi/2]; update(): the rotation taking +z onto
        // -dirW (about up x -dirW by acos(up . -dirW)), identity when that axis vanishes
        const float angle = std::fmin(std::fmax(d.angle, 0.f), (float)M_PI_2);
        L.cosSubtendedAngle = std::cos(angle);
        const double w[3] = {-(double)L.dirW[0], -(double)L.dirW[1], -(double)L.dirW[2]};
        const double axis[3] = {-w[1], w[0], 0.0}; // (0, 0, 1) x w
        const double s = std::sqrt(axis[0] * axis[0] + axis[1] * axis[1]);
        if (s > 0.0)
        {
            const double th = std::acos(std::fmin(std::fmax(w[2], -1.0), 1.0));
            const double k[3] = {axis[0] / s, axis[1] / s, 0.0};
            const double c = std::cos(th), sn = std::sin(th), t = 1.0 - c;
            // Rodrigues: R = c I + sn [k]x + t k k^T
            const double R[9] = {c + t * k[0] * k[0], t * k[0] * k[1] - sn * k[2], t * k[0] * k[2] + sn * k[1],
                                 t * k[1] * k[0] + sn * k[2], c + t * k[1] * k[1], t * k[1] * k[2] - sn * k[0],
                                 t * k[2] * k[0] - sn * k[1], t * k[2] * k[1] + sn * k[0], c + t * k[2] * k[2]};
            for (int r = 0; r < 3; r++)
                for (int col = 0; col < 3; col++)
                {
                    L.transMat[4 * r + col] = (float)R[3 * r + col];
                    L.transMatIT[3 * r + col] = (float)R[3 * r + col]; // a rotation is its own inverse transpose
                }
        }
    }
    if (d.type >= kLightRect)
    {
        // AnalyticAreaLight::update: transMat = transform x scaling, transMatIT = (transMat^-1)^T
        double M[3][4];
        for (int r = 0; r < 3; r++)
        {
            for (int col = 0; col < 3; col++) M[r][col] = (double)d.transform[4 * r + col] * (double)d.scaling[col];
            M[r][3] = d.transform[4 * r + 3];
        }
        for (int r = 0; r < 3; r++)
            for (int col = 0; col < 4; col++) L.transMat[4 * r + col] = (float)M[r][col];
        const double det = M[0][0] * (M[1][1] * M[2][2] - M[1][2] * M[2][1]) - M[0][1] * (M[1][0] * M[2][2] - M[1][2] * M[2][0]) +
                           M[0][2] * (M[1][0] * M[2][1] - M[1][1] * M[2][0]);
        if (det == 0.0) return false;
        // inverse transpose = cofactor matrix / det
        const double C[9] = {M[1][1] * M[2][2] - M[1][2] * M[2][1], -(M[1][0] * M[2][2] - M[1][2] * M[2][0]), M[1][0] * M[2][1] - M[1][1] * M[2][0],
                             -(M[0][1] * M[2][2] - M[0][2] * M[2][1]), M[0][0] * M[2][2] - M[0][2] * M[2][0], -(M[0][0] * M[2][1] - M[0][1] * M[2][0]),
                             M[0][1] * M[1][2] - M[0][2] * M[1][1], -(M[0][0] * M[1][2] - M[0][2] * M[1][0]), M[0][0] * M[1][1] - M[0][1] * M[1][0]};
        for (int k = 0; k < 9; k++) L.transMatIT[k] = (float)(C[k] / det);
        // surface areas from the lengths of the transformed unit axes (Rect/Disc/SphereLight::update)
        auto axisLen = [&](int col) { return (float)std::sqrt(M[0][col] * M[0][col] + M[1][col] * M[1][col] + M[2][col] * M[2][col]); };
        const float rx = axisLen(0), ry = axisLen(1), rz = axisLen(2);
        if (d.type == kLightRect) L.surfaceArea = 4.0f * rx * ry;
        else if (d.type == kLightDisc) L.surfaceArea = (float)M_PI * rx * ry;
        else
            // Thomsen's ellipsoid area as SphereLight::update writes it, where only the third
            // term is divided by 3 (exact for no sphere; kept so that radiance matches)
            L.surfaceArea = 4.0f * (float)M_PI *
                            std::pow(std::pow(rx * ry, 1.6f) + std::pow(ry * rz, 1.6f) + std::pow(rx * rz, 1.6f) / 3.0f, 1.0f / 1.6f);
    }
    out = L;
    return true;
}

} // namespace rs
