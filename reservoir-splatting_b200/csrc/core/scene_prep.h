// Host-side scene preparation shared by the pass and its CPU checker: the
// triangle records, the emissive light collection and the power-sampler alias
// table.
//
//   Scene/Lights/LightCollection.cpp + BuildTriangleList.cs.slang:62   per-triangle
//       face normal and area (normal = N / |N|, area = |N| / 2, N = cross(p1 - p0, p2 - p0))
//   Scene/Lights/FinalizeIntegration.cs.slang:108   flux = luminance(Le) * area * pi
//   Rendering/Lights/EmissivePowerSampler.cpp:86-172   alias table: weights scaled to
//       mean 1, sorted, two-pointer pairing, a seeded shuffle (std::mt19937, default seed),
//       packed as 16-bit threshold + 2 x 24-bit indices
#pragma once
#include <algorithm>
#include <random>
#include <vector>
#include "lights.h"

namespace rs {

struct PreparedScene
{
    std::vector<f4> tri;                  // 3 per triangle
    std::vector<MaterialData> materials;
    std::vector<LightTriangle> lights;
    std::vector<u2> alias;
    float invWeightsSum = 0.f;
    double weightSum = 0.0;
};

inline bool material_is_emissive(const MaterialData& m)
{
    return m.emissive[0] > 0.f || m.emissive[1] > 0.f || m.emissive[2] > 0.f;
}

// EmissivePowerSampler::generateAliasTable
inline void build_alias_table(std::vector<float> weights, std::vector<u2>& table, double& sumOut)
{
    uint32_t N = (uint32_t)weights.size();
    table.assign(N, u2{0, 0});
    sumOut = 0.0;
    if (N == 0) return;
    std::mt19937 rng; // default seed, as the reference sampler's member RNG
    double sum = 0.0;
    for (float f : weights) sum += f;
    for (float& f : weights) f *= (float)N / (float)sum;
    std::vector<uint32_t> permutation(N);
    for (uint32_t i = 0; i < N; ++i) permutation[i] = i;
    std::sort(permutation.begin(), permutation.end(), [&](uint32_t a, uint32_t b) { return weights[a] < weights[b]; });
    std::vector<float> thresholds(N, 0.f);
    std::vector<uint32_t> redirect(N, 0);
    uint32_t head = 0, tail = N - 1;
    while (head != tail)
    {
        uint32_t i = permutation[head];
        uint32_t j = permutation[tail];
        thresholds[i] = weights[i];
        redirect[i] = j;
        weights[j] -= 1.0f - weights[i];
        if (head == tail - 1)
        {
            thresholds[j] = 1.0f;
            redirect[j] = j;
            break;
        }
        else if (weights[j] < 1.0f)
        {
            std::swap(permutation[head], permutation[tail]);
            tail--;
        }
        else
        {
            head++;
        }
    }
    for (uint32_t i = 0; i < N; ++i) permutation[i] = i;
    for (uint32_t i = 0; i < N; ++i)
    {
        uint32_t r = (uint32_t)rng();
        uint32_t dst = i + (r % (N - i));
        std::swap(thresholds[i], thresholds[dst]);
        std::swap(redirect[i], redirect[dst]);
        std::swap(permutation[i], permutation[dst]);
    }
    for (uint32_t i = 0; i < N; ++i)
    {
        uint32_t prob = ((uint32_t)f32_to_f16(thresholds[i])) << 16u;
        uint32_t lx = redirect[i] & 0xFFFFFFu, ly = permutation[i] & 0xFFFFFFu;
        table[i].x = prob | ((lx >> 8u) & 0xFFFFu);
        table[i].y = ((lx & 0xFFu) << 24u) | ly;
    }
    sumOut = sum;
}

// Builds the triangle records and the light collection from a triangle soup.
// Returns false when a material id is out of range.
inline bool prepare_scene(uint32_t numTris, const float* pos, const uint32_t* mtlIds, uint32_t numMaterials,
                          const MaterialData* mtls, PreparedScene& out)
{
    out.materials.assign(mtls, mtls + numMaterials);
    out.tri.resize(3 * (size_t)numTris);
    out.lights.clear();
    std::vector<float> weights;
    for (uint32_t t = 0; t < numTris; t++)
    {
        uint32_t m = mtlIds[t];
        if (m >= numMaterials) return false;
        const float* p = pos + 9 * (size_t)t;
        f4 a = {p[0], p[1], p[2], u2f(m)};
        f4 b = {p[3], p[4], p[5], u2f(kInvalidIndex)};
        f4 c = {p[6], p[7], p[8], 0.f};
        if (material_is_emissive(mtls[m]))
        {
            f3 p0 = mk3(p[0], p[1], p[2]), p1 = mk3(p[3], p[4], p[5]), p2 = mk3(p[6], p[7], p[8]);
            f3 N = cross(p1 - p0, p2 - p0);
            float len = length(N);
            LightTriangle L;
            memset(&L, 0, sizeof(L));
            for (int k = 0; k < 3; k++) { L.p0[k] = p[k]; L.p1[k] = p[3 + k]; L.p2[k] = p[6 + k]; }
            L.area = 0.5f * len;
            f3 n = N / len;
            L.normal[0] = n.x; L.normal[1] = n.y; L.normal[2] = n.z;
            L.Le[0] = mtls[m].emissive[0]; L.Le[1] = mtls[m].emissive[1]; L.Le[2] = mtls[m].emissive[2];
            L.flux = luminance(mk3(L.Le[0], L.Le[1], L.Le[2])) * L.area * kPi;
            L.sceneTri = t;
            L.materialID = m;
            if (len > 0.f && L.flux > 0.f)
            {
                b.w = u2f((uint32_t)out.lights.size());
                out.lights.push_back(L);
                weights.push_back(L.flux);
            }
        }
        out.tri[3 * (size_t)t + 0] = a;
        out.tri[3 * (size_t)t + 1] = b;
        out.tri[3 * (size_t)t + 2] = c;
    }
    build_alias_table(weights, out.alias, out.weightSum);
    out.invWeightsSum = out.lights.empty() ? 0.f : 1.0f / (float)out.weightSum;
    return true;
}

} // namespace rs
