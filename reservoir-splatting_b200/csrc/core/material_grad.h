// Derivatives of the StandardBSDF evaluation (material.h) with respect to the
// material parameters that the path-replay adjoint differentiates: baseColor (per
// channel), the roughness slot and metallic.  ior and the specular colour are held fixed.
//
// With metallic m and F0 = ((ior - 1) / (ior + 1))^2 (StandardMaterial.slang:48-115):
//   diffuse albedo  = baseColor * (1 - m)          d/d baseColor.c = (1 - m)   d/dm = -baseColor
//   specular colour = F0 + (baseColor - F0) * m    d/d baseColor.c = m         d/dm = baseColor - F0
//   GGX alpha       = max(roughness^2, 0.0064)     d/d roughness   = 2 * roughness above the clamp
// Spec-gloss (kMtlSpecGloss, ShadingUtils.slang:57-71): diffuse albedo = baseColor (d/d baseColor.c
//   = 1), specular colour = the material's specular (no baseColor term), roughness = 1 - the stored
//   glossiness (d/d slot = -d/d roughness); its derived metallic only sets the lobe probabilities
//   and has no derivative of its own.
// The lobe probabilities depend on metallic too; like the gates they are sampling densities.
// Frostbite diffuse (FrostbiteDiffuseBRDF.slang): albedo * Fi * Fo * E / pi * cos(wo) with
//   fd90 = 0.5 r + 2 (wo.h)^2 r, F(c) = 1 + (fd90 - 1) (1 - c)^5, E = 1 + (1/1.51 - 1) r.
// GGX reflection (SpecularMicrofacet.slang:49-200): F * D * G / (4 cos(wi)) with
//   D = a2 / (pi d^2), d = c^2 (a2 - 1) + 1, a2 = alpha^2:  dD/da2 = (d - 2 a2 c^2) / (pi d^3)
//   G = 1 / (1 + Li + Lo), L = (sqrt(1 + a2 tan^2) - 1) / 2:  dL/da2 = tan^2 / (4 sqrt(1 + a2 tan^2))
// Lobe-selection probabilities and the validity gates are piecewise constant
// in the parameters and are not differentiated (they are sampling densities).
#pragma once
#include "material.h"

namespace rs {

struct BsdfGrad
{
    f3 value;  // mi_eval(sd, d, lobeMask, wo)
    f3 dBase;  // d value.c / d baseColor.c (channel c depends only on baseColor.c)
    f3 dRough; // d value / d roughness
    f3 dMetal; // d value / d metallic (zero for spec-gloss)
};

// tan^2 of a unit local direction from its tangent-plane components (no 1 - cos^2 cancellation).
RS_HD float ggx_tan2(f3 w)
{
    return (w.x * w.x + w.y * w.y) / (w.z * w.z);
}

// Value and derivatives of mi_eval(sd, d, lobeMask, wo).  The value uses forms without
// cancellation (the GGX denominator as sin^2 + cos^2 alpha^2 of the half vector, Smith's Lambda as
// x / (2 (sqrt(1 + x) + 1))), so near a sharp specular peak it is more accurate than the pass's own
// float evaluation; both agree wherever that one is well conditioned.
RS_HD BsdfGrad mi_eval_grad(const ShadingData& sd, const BsdfData& d, const MaterialData& m, uint32_t lobeMask, f3 wo)
{
    BsdfGrad g;
    g.value = mk3(0.f); g.dBase = mk3(0.f); g.dRough = mk3(0.f); g.dMetal = mk3(0.f);
    const bool specGloss = (m.flags & kMtlSpecGloss) != 0;
    const f3 base = mk3(m.baseColor[0], m.baseColor[1], m.baseColor[2]);
    const float fr = (m.ior - 1.f) / (m.ior + 1.f), F0 = fr * fr;
    f3 wi = sd_to_local(sd, sd.V);
    f3 wl = sd_to_local(sd, wo);
    if (!valid_hemisphere(sd, wi, wl, wo)) return g;
    if (f_min(wi.z, wl.z) < kMinCosTheta) return g;
    StandardBSDF b = make_bsdf(wi, d, lobeMask);
    const uint32_t mask = lobeMask == 0 ? 0xfu : lobeMask;
    f3 h = normalize(wi + wl);
    if (b.pDiffuseReflection > 0.f && (mask & 0x1u))
    {
        float woDotH = dot(wl, h);
        float r = b.diffRoughness;
        float E = f_lerp(1.f, 1.f / 1.51f, r);
        float fd90 = f_lerp(0.f, 0.5f, r) + 2.f * woDotH * woDotH * r;
        float Pi = f_pow5(f_max(1.f - wi.z, 0.f));
        float Po = f_pow5(f_max(1.f - wl.z, 0.f));
        float Fi = 1.f + (fd90 - 1.f) * Pi;
        float Fo = 1.f + (fd90 - 1.f) * Po;
        float k = k1OverPi * wl.z;
        float S = Fi * Fo * E * k;
        float dfd90 = 0.5f + 2.f * woDotH * woDotH;
        float dS = (dfd90 * (Pi * Fo + Fi * Po) * E + Fi * Fo * (1.f / 1.51f - 1.f)) * k;
        g.value += b.diffAlbedo * S;
        g.dBase += mk3(specGloss ? S : (1.f - d.metallic) * S);
        g.dRough += b.diffAlbedo * dS;
        if (!specGloss) g.dMetal = g.dMetal - base * S;
    }
    if (b.pSpecularReflection > 0.f && (mask & 0x4u) && b.alpha != 0.f)
    {
        float a = b.alpha, a2 = a * a;
        float c2 = h.z * h.z;
        float dd = (h.x * h.x + h.y * h.y) + c2 * a2;
        float D = a2 / (dd * dd * kPi);
        float dD = (dd - 2.f * a2 * c2) / (kPi * dd * dd * dd);
        float ti = ggx_tan2(wi), to = ggx_tan2(wl);
        float xi = a2 * ti, xo = a2 * to;
        float si = f_sqrt(1.f + xi), so = f_sqrt(1.f + xo);
        float G = 1.f / (1.f + 0.5f * xi / (si + 1.f) + 0.5f * xo / (so + 1.f));
        float dG = -G * G * (0.25f * ti / si + 0.25f * to / so);
        float P = f_pow5(f_max(1.f - dot(wi, h), 0.f));
        f3 F = b.specAlbedo + (mk3(1.f) - b.specAlbedo) * P;
        float k = 0.25f / wi.z;
        g.value += F * (D * G * k);
        if (!specGloss)
        {
            g.dBase += mk3(d.metallic * (1.f - P) * D * G * k);
            g.dMetal += (base - mk3(F0)) * ((1.f - P) * D * G * k);
        }
        float r = d.roughness;
        float dAlpha = (lobeMask != 5u && r * r > kMinGGXAlpha) ? 2.f * r : 0.f;
        g.dRough += F * (k * (dD * G + D * dG) * 2.f * a * dAlpha);
    }
    if (specGloss) g.dRough = -g.dRough;
    return g;
}

// Layout of one material's gradient record: the first eight floats of the material record
// (baseColor.xyz, roughness, emissive.xyz, metallic).
enum : uint32_t { kGradBase = 0, kGradRough = 3, kGradEmissive = 4, kGradMetal = 7, kGradStride = 8 };

} // namespace rs
