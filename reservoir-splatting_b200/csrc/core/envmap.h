// Environment-map light: a lat-long RGB map, its hierarchical importance map, and the sampling,
// pdf and evaluation the path tracer and the shifts use.
//
//   Scene/Lights/EnvMap.slang:40-118          eval(dir) = texture(worldToUv(dir)) * intensity * tint,
//       worldToUv = world_to_latlong_map(invTransform * dir)
//   Scene/Lights/EnvMap.cpp:60-72, 130-137    transform from the XYZ rotation in degrees; bilinear
//       filtering, u wraps, v clamps
//   Utils/Math/MatrixMath.h:647-680           matrixFromRotationXYZ
//   Utils/Math/MathHelpers.slang:111-137, 213-255  lat-long and equal-area octahedral maps
//   Rendering/Lights/EnvMapSamplerSetup.cs.slang:48-76  importance texel = mean luminance of
//       8 x 8 stratified map samples over the texel's octahedral cell
//   Rendering/Lights/EnvMapSampler.cpp:36-37, 80-113    512 x 512 importance map, 64 samples per
//       texel, a full mip chain (each level the 2 x 2 mean of the one below)
//   Rendering/Lights/EnvMapSampler.slang:71-163  hierarchical sample warping and evalPdf
//   PathTracer.slang:516-534, 606-624          env light sample and light-type probabilities
//
// The texture unit's bilinear filter is restated in float arithmetic (full-precision weights),
// so host and device agree bit for bit.
#pragma once
#include "geom.h"
#include "camera.h"

namespace rs {

constexpr uint32_t kEnvImportanceDim = 512;     // EnvMapSampler.cpp:36
constexpr uint32_t kEnvImportanceMips = 10;     // 512 .. 1
constexpr uint32_t kEnvImportanceSide = 8;      // sqrt(64) samples per texel side (EnvMapSampler.cpp:37, 93-94)
constexpr uint32_t kEnvImportanceTexels = 349525u; // sum over the mips of (512 >> m)^2
constexpr float k1Over2Pi = 0.159154936671257019f; // 0x3e22f983
constexpr float k1Over4Pi = 0.0795774683356285095f; // 0x3da2f983
constexpr float k4Pi = 12.5663709640502930f;       // 0x41490fdb
constexpr float k2OverPi = 0.636619746685028076f;  // 0x3f22f983

struct EnvMapView
{
    const float* texels;     // RGBA float texels, w x h, row-major, row 0 at v = 0
    const float* importance; // importance mips 0..9 back to back (512^2, 256^2, ..., 1 texels)
    uint32_t w, h;
    uint32_t present;        // kUseEnvLight: a map is set and its intensity is > 0
    uint32_t pad;
    float toWorld[9];        // local -> world rotation, row-major (EnvMapData.transform)
    float toLocal[9];        // world -> local (EnvMapData.invTransform)
    float scale[3];          // intensity * tint
};

RS_HD uint32_t env_mip_offset(uint32_t m)
{
    uint32_t o = 0;
    for (uint32_t k = 0; k < m; k++) { const uint32_t d = kEnvImportanceDim >> k; o += d * d; }
    return o;
}

RS_HD f3 mat3_mul(const float* m, f3 v)
{
    return mk3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z, m[6] * v.x + m[7] * v.y + m[8] * v.z);
}

// world_to_latlong_map (MathHelpers.slang:111-119; its atan2/acos run in double there, in float here)
RS_HD f2 world_to_latlong_map(f3 dir)
{
    f3 p = normalize(dir);
    return mk2(f_atan2(p.x, -p.z) * k1Over2Pi + 0.5f, f_acos(p.y) * k1OverPi);
}

// oct_to_ndir_equal_area_unorm (MathHelpers.slang:237-255)
RS_HD f3 oct_to_ndir_equal_area_unorm(f2 p)
{
    p = mk2(p.x * 2.f - 1.f, p.y * 2.f - 1.f);
    float d = 1.f - (f_abs(p.x) + f_abs(p.y));
    float r = 1.f - f_abs(d);
    float phi = (r > 0.f) ? ((f_abs(p.y) - f_abs(p.x)) / r + 1.f) * kPiOver4 : 0.f;
    float f = r * f_sqrt(2.f - r * r);
    float s, c;
    f_sincos(phi, s, c);
    float x = f * f_sign(p.x) * c;
    float y = f * f_sign(p.y) * s;
    float z = f_sign(d) * (1.f - r * r);
    return mk3(x, y, z);
}

// ndir_to_oct_equal_area_unorm (MathHelpers.slang:213-230)
RS_HD f2 ndir_to_oct_equal_area_unorm(f3 n)
{
    float r = f_sqrt(1.f - f_abs(n.z));
    float phi = f_atan2(f_abs(n.y), f_abs(n.x));
    f2 p;
    p.y = r * phi * k2OverPi;
    p.x = r - p.y;
    if (n.z < 0.f) p = mk2(1.f - p.y, 1.f - p.x);
    p = mk2(p.x * f_sign(n.x), p.y * f_sign(n.y));
    return mk2(p.x * 0.5f + 0.5f, p.y * 0.5f + 0.5f);
}

RS_HD float env_bilerp(float c00, float c10, float c01, float c11, float tx, float ty)
{
    const float top = c00 * (1.f - tx) + c10 * tx;
    const float bot = c01 * (1.f - tx) + c11 * tx;
    return top * (1.f - ty) + bot * ty;
}

// Bilinear texel fetch of the lat-long map at uv (SampleLevel, lod 0): texel centres at
// (i + 0.5) / size, u wraps and v clamps to the edge texels.
RS_HD f3 env_lookup(const EnvMapView& E, f2 uv)
{
    float x = uv.x * (float)E.w - 0.5f, y = uv.y * (float)E.h - 0.5f;
    if (!(x > -1e7f && x < 1e7f)) x = 0.f; // NaN / out of range: any texel, the result is not used
    if (!(y > -1e7f && y < 1e7f)) y = 0.f;
    const float fx = f_floor(x), fy = f_floor(y);
    const float tx = x - fx, ty = y - fy;
    const int W = (int)E.w, H = (int)E.h;
    int x0 = (int)fx % W; if (x0 < 0) x0 += W;
    const int x1 = x0 + 1 == W ? 0 : x0 + 1;
    int y0 = (int)fy, y1 = y0 + 1;
    y0 = y0 < 0 ? 0 : (y0 >= H ? H - 1 : y0);
    y1 = y1 < 0 ? 0 : (y1 >= H ? H - 1 : y1);
    const float* t = E.texels;
    const float* c00 = t + 4 * ((size_t)y0 * W + x0);
    const float* c10 = t + 4 * ((size_t)y0 * W + x1);
    const float* c01 = t + 4 * ((size_t)y1 * W + x0);
    const float* c11 = t + 4 * ((size_t)y1 * W + x1);
    return mk3(env_bilerp(c00[0], c10[0], c01[0], c11[0], tx, ty), env_bilerp(c00[1], c10[1], c01[1], c11[1], tx, ty),
               env_bilerp(c00[2], c10[2], c01[2], c11[2], tx, ty));
}

// EnvMap::eval(dir): the radiance arriving from world direction dir.
RS_HD f3 env_eval(const EnvMapView& E, f3 dir)
{
    const f3 c = env_lookup(E, world_to_latlong_map(mat3_mul(E.toLocal, dir)));
    return mk3(c.x * E.scale[0], c.y * E.scale[1], c.z * E.scale[2]);
}

// handleReconnectionEnvMap (PathTracer.slang:1412-1416)
RS_HD f3 env_reconnection(const EnvMapView& E, f3 dir) { return E.present ? env_eval(E, dir) : mk3(0.f); }

// One texel of the importance map's finest mip (EnvMapSamplerSetup.cs.slang:48-76): the mean
// luminance of the map (without intensity) over 8 x 8 sample positions of its octahedral cell.
RS_HD float env_importance_texel(const EnvMapView& E, uint32_t px, uint32_t py)
{
    const float dimInSamples = (float)(kEnvImportanceDim * kEnvImportanceSide);
    float L = 0.f;
    for (uint32_t y = 0; y < kEnvImportanceSide; y++)
        for (uint32_t x = 0; x < kEnvImportanceSide; x++)
        {
            const uint32_t sx = px * kEnvImportanceSide + x, sy = py * kEnvImportanceSide + y;
            const f2 p = mk2(((float)sx + 0.5f) / dimInSamples, ((float)sy + 0.5f) / dimInSamples);
            L += luminance(env_lookup(E, world_to_latlong_map(oct_to_ndir_equal_area_unorm(p))));
        }
    return L * (1.f / (float)(kEnvImportanceSide * kEnvImportanceSide));
}

// Texel (x, y) of mip m >= 1 from the four texels of mip m - 1 below it.
RS_HD float env_importance_reduce(const float* importance, uint32_t m, uint32_t x, uint32_t y)
{
    const uint32_t d = kEnvImportanceDim >> (m - 1);
    const float* s = importance + env_mip_offset(m - 1);
    const float a = s[(2 * y) * d + 2 * x], b = s[(2 * y) * d + 2 * x + 1];
    const float c = s[(2 * y + 1) * d + 2 * x], e = s[(2 * y + 1) * d + 2 * x + 1];
    return ((a + b) + (c + e)) * 0.25f;
}

// EnvMapSampler::sample (EnvMapSampler.slang:71-140).
RS_HD bool env_sample(const EnvMapView& E, f2 rnd, f3& dirW, float& pdf, f3& Le)
{
    f2 p = rnd;
    uint32_t px = 0, py = 0;
    for (int mip = (int)kEnvImportanceMips - 2; mip >= 0; mip--)
    {
        px *= 2; py *= 2;
        const uint32_t d = kEnvImportanceDim >> mip;
        const float* lvl = E.importance + env_mip_offset((uint32_t)mip);
        const float w0 = lvl[py * d + px], w1 = lvl[py * d + px + 1];
        const float w2 = lvl[(py + 1) * d + px], w3 = lvl[(py + 1) * d + px + 1];
        const float q0 = w0 + w2, q1 = w1 + w3;
        uint32_t ox, oy;
        const float dd = q0 / (q0 + q1);
        if (p.x < dd) { ox = 0; p.x = p.x / dd; }
        else { ox = 1; p.x = (p.x - dd) / (1.f - dd); }
        const float e = ox == 0 ? (w0 / q0) : (w1 / q1);
        if (p.y < e) { oy = 0; p.y = p.y / e; }
        else { oy = 1; p.y = (p.y - e) / (1.f - e); }
        px += ox; py += oy;
    }
    const float invDim = 1.f / (float)kEnvImportanceDim;
    const f2 uv = mk2(((float)px + p.x) * invDim, ((float)py + p.y) * invDim);
    const f3 dir = oct_to_ndir_equal_area_unorm(uv);
    const float avg = E.importance[env_mip_offset(kEnvImportanceMips - 1)];
    const float pdfTexel = E.importance[py * kEnvImportanceDim + px] / avg;
    dirW = mat3_mul(E.toWorld, dir);
    pdf = pdfTexel * k1Over4Pi;
    Le = env_eval(E, dirW);
    return true;
}

// EnvMapSampler::evalPdf (EnvMapSampler.slang:149-162): point sampling, clamped to the edge.
RS_HD float env_eval_pdf(const EnvMapView& E, f3 dir)
{
    const f2 uv = ndir_to_oct_equal_area_unorm(mat3_mul(E.toLocal, dir));
    const float D = (float)kEnvImportanceDim;
    float fx = f_floor(uv.x * D), fy = f_floor(uv.y * D);
    fx = f_isnan(fx) ? 0.f : f_clamp(fx, 0.f, D - 1.f);
    fy = f_isnan(fy) ? 0.f : f_clamp(fy, 0.f, D - 1.f);
    const float avg = E.importance[env_mip_offset(kEnvImportanceMips - 1)];
    const float pdf = E.importance[(uint32_t)fy * kEnvImportanceDim + (uint32_t)fx] / avg;
    return pdf * (1.f / k4Pi);
}

// Motion vector of a primary miss when the environment light is on (VBufferRT.slang:128-149): the
// ray direction projected through the previous frame's camera basis, with this frame's focal
// length, frame height and aspect ratio; p is the pixel centre in [0,1]^2.
RS_HD f2 env_miss_motion_vector(const CameraData& cam, const CameraData& prev, f3 rayDir, f2 p)
{
    float d = dot(rayDir, normalize(prev.cameraW));
    const float tanFovY = cam.focalLength == 0.f ? 0.f : cam.frameHeight / cam.focalLength;
    d *= tanFovY;
    const f2 offset = mk2(dot(rayDir, normalize(prev.cameraU)), -dot(rayDir, normalize(prev.cameraV)));
    const f2 newNDC = mk2(0.5f + offset.x / (d * cam.aspectRatio), 0.5f + offset.y / d);
    return mk2(newNDC.x - p.x, newNDC.y - p.y);
}

// EnvMap transform from XYZ Euler angles in degrees (EnvMap::setRotation, EnvMap.cpp:60-72, with
// matrixFromRotationXYZ, MatrixMath.h:647-680), computed in double; the world -> local matrix is
// its transpose (the inverse of a rotation).  Host only.
inline void env_transform(const float rotationDeg[3], float toWorld[9], float toLocal[9])
{
    const double k = 3.14159265358979323846 / 180.0;
    const double c1 = cos(-rotationDeg[0] * k), c2 = cos(-rotationDeg[1] * k), c3 = cos(-rotationDeg[2] * k);
    const double s1 = sin(-rotationDeg[0] * k), s2 = sin(-rotationDeg[1] * k), s3 = sin(-rotationDeg[2] * k);
    const double m[9] = {c2 * c3, c2 * s3, -s2,
                         -c1 * s3 + s1 * s2 * c3, c1 * c3 + s1 * s2 * s3, s1 * c2,
                         s1 * s3 + c1 * s2 * c3, -s1 * c3 + c1 * s2 * s3, c1 * c2};
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++)
        {
            toWorld[3 * r + c] = (float)m[3 * r + c];
            toLocal[3 * c + r] = (float)m[3 * r + c];
        }
}

// getLightTypeSelectionProbabilities (PathTracer.slang:606-622): equal probabilities for the
// light types the scene has (environment map, emissive triangles, analytic lights).
RS_HD void light_type_probabilities(bool env, bool emissive, bool analytic, float& pEnv, float& pEmissive, float& pAnalytic)
{
    pEnv = env ? 1.f : 0.f;
    pEmissive = emissive ? 1.f : 0.f;
    pAnalytic = analytic ? 1.f : 0.f;
    const float sum = pEnv + pEmissive + pAnalytic;
    if (sum == 0.f) return;
    const float invSum = 1.f / sum;
    pEnv *= invSum;
    pEmissive *= invSum;
    pAnalytic *= invSum;
}

} // namespace rs
