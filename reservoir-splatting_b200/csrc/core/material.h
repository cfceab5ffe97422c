// Falcor StandardMaterial (metal-rough, opaque) and its StandardBSDF with the
// lobe mask that the Reservoir Splatting pass adds.
//
//   StandardMaterial.slang:48-115        material instance setup (diffuse/specular/roughness,
//                                         emission only on the front face, double-sided flip)
//   StandardMaterialInstance.slang:64-160 eval / sample / evalPdf / getProperties / lobe types
//   BSDFs/StandardBSDF.slang:96-347      lobe probabilities, lobe-masked eval / sample / pdf
//   BSDFs/FrostbiteDiffuseBRDF.slang     diffuse lobe (the default DiffuseBrdf, BSDFConfig.slangh)
//   BSDFs/SpecularMicrofacet.slang:49-200 GGX reflection, VNDF sampling, correlated Smith G
//   IsotropicGGX.slang                   D, G1, Lambda, VNDF sampling (spherical caps)
//   Fresnel.slang:42-51                  Schlick
//   Scene/Material/ShadingUtils.slang:111-122, 214-247  double-sided flip, hemisphere validity
//
// Transmission lobes are not built: every material here is opaque
// (specularTransmission = diffuseTransmission = 0), so their sampling
// probabilities are identically zero in the reference as well.
#pragma once
#include "geom.h"
#include "rng.h"

namespace rs {

// LobeType.slang
enum LobeType : uint32_t
{
    kLobeDiffuseReflection = 0x01,
    kLobeSpecularReflection = 0x02,
    kLobeDeltaReflection = 0x04,
    kLobeDiffuseTransmission = 0x10,
    kLobeSpecularTransmission = 0x20,
    kLobeDeltaTransmission = 0x40,
    kLobeSpecular = 0x22,
    kLobeDelta = 0x44,
    kLobeNonDelta = 0x33,
    kLobeReflection = 0x0f,
    kLobeTransmission = 0xf0,
    kLobeNonDeltaReflection = 0x03,
    kLobeNonDeltaTransmission = 0x30,
};

constexpr float kMinCosTheta = 1e-6f;   // IBSDF.slang:35
constexpr float kMinGGXAlpha = 0.0064f; // StandardBSDF.slang:52

enum MaterialFlags : uint32_t { kMtlDoubleSided = 1u, kMtlSpecGloss = 2u };

// One material: 16 floats.  Metal-rough (StandardMaterial's default shading model): baseColor,
// roughness, metallic, ior.  Spec-gloss (kMtlSpecGloss, the model Falcor's OBJ import uses):
// baseColor is the diffuse colour, specular the specular colour and `roughness` holds the
// glossiness.  emissive already includes the emissive factor.
struct alignas(16) MaterialData
{
    float baseColor[3];
    float roughness;
    float emissive[3];
    float metallic;
    float ior;
    uint32_t flags;
    float specular[3];
    float pad[3];
};

// Material instance parameters (StandardMaterial.slang:48-115, opaque subset).
struct BsdfData
{
    f3 diffuse;
    f3 specular;
    float roughness;
    float metallic;
    f3 emission;
};

// The metallic factor of a spec-gloss material (ShadingUtils.slang:57-71): the metallic m for which
// the UE4 metal-rough conversion with specular level 0.5 (F0 = 0.04) gives the two colours'
// luminances, the root of 0.04 m^2 + (s + d - 0.08) m + (0.04 - s) = 0; 0 without specular.  Like
// the reference it can return a negative value or NaN for colour pairs no metallic produces.
RS_HD float spec_gloss_metallic(f3 diffuse, f3 specular)
{
    const float d = luminance(diffuse), s = luminance(specular);
    if (s == 0.f) return 0.f;
    const float b = s + d - 0.08f;
    const float c = 0.04f - s;
    const float root = f_sqrt(b * b - 0.16f * c);
    return (root - b) * 12.5f;
}

RS_HD BsdfData setup_material(const MaterialData& m, bool frontFacing)
{
    BsdfData d;
    f3 baseColor = mk3(m.baseColor[0], m.baseColor[1], m.baseColor[2]);
    if (m.flags & kMtlSpecGloss)
    {
        d.diffuse = baseColor;
        d.specular = mk3(m.specular[0], m.specular[1], m.specular[2]);
        d.roughness = 1.f - m.roughness; // the stored glossiness
        d.metallic = spec_gloss_metallic(d.diffuse, d.specular);
    }
    else
    {
        float f = (m.ior - 1.f) / (m.ior + 1.f);
        float F0 = f * f;
        float metallic = m.metallic;
        d.diffuse = lerp(baseColor, mk3(0.f), metallic);
        d.specular = lerp(mk3(F0), baseColor, metallic);
        d.roughness = m.roughness;
        d.metallic = metallic;
    }
    d.emission = frontFacing ? mk3(m.emissive[0], m.emissive[1], m.emissive[2]) : mk3(0.f);
    return d;
}

// loadShadingData (LoadShadingData.slang:134-142) for a triangle hit of the soup.
// World position of a triangle hit with the arithmetic of load_shading_data (used with the
// previous frame's triangles for motion vectors: Scene::getPrevPosW, VBufferRT.slang:84).
RS_HD f3 hit_position(const f4* tri, const HitInfo& hit)
{
    uint32_t prim = hit_prim(hit);
    f3 p0 = f4xyz(tri[3 * prim + 0]), p1 = f4xyz(tri[3 * prim + 1]), p2 = f4xyz(tri[3 * prim + 2]);
    f2 bc = hit_bary(hit);
    float b0 = 1.f - bc.x - bc.y;
    f3 pos = p0 * b0;
    pos += p1 * bc.x;
    pos += p2 * bc.y;
    return pos;
}

RS_HD ShadingData load_shading_data(const f4* tri, const MaterialData* mtl, const HitInfo& hit, f3 rayDir)
{
    ShadingData sd;
    uint32_t prim = hit_prim(hit);
    f4 a = tri[3 * prim + 0], b = tri[3 * prim + 1], c = tri[3 * prim + 2];
    f3 p0 = f4xyz(a), p1 = f4xyz(b), p2 = f4xyz(c);
    f2 bc = hit_bary(hit);
    float b0 = 1.f - bc.x - bc.y;
    sd.posW = p0 * b0;
    sd.posW += p1 * bc.x;
    sd.posW += p2 * bc.y;
    sd.faceN = normalize(cross(p1 - p0, p2 - p0));
    sd.V = -rayDir;
    sd.frontFacing = dot(sd.V, sd.faceN) >= 0.f;
    sd.materialID = f2u(a.w);
    sd.lightIndex = f2u(b.w);
    // ShadingFrame::createSafe with no tangent: N = normalize(normal), T = perp_stark(N), B = cross(N, T).
    sd.N = normalize(sd.faceN);
    sd.T = perp_stark(sd.N);
    sd.B = cross(sd.N, sd.T);
    if (!sd.frontFacing && (mtl[sd.materialID].flags & kMtlDoubleSided)) sd.N = -sd.N;
    return sd;
}

// ---- GGX helpers (IsotropicGGX.slang) ----
RS_HD float evalNdfGGX(float alpha, float cosTheta)
{
    float a2 = alpha * alpha;
    float d = ((cosTheta * a2 - cosTheta) * cosTheta + 1.f);
    return a2 / (d * d * kPi);
}
RS_HD float evalG1GGX(float alphaSqr, float cosTheta)
{
    if (cosTheta <= 0.f) return 0.f;
    float cosThetaSqr = cosTheta * cosTheta;
    float tanThetaSqr = f_max(1.f - cosThetaSqr, 0.f) / cosThetaSqr;
    return 2.f / (1.f + f_sqrt(1.f + alphaSqr * tanThetaSqr));
}
RS_HD float evalLambdaGGX(float alphaSqr, float cosTheta)
{
    if (cosTheta <= 0.f) return 0.f;
    float cosThetaSqr = cosTheta * cosTheta;
    float tanThetaSqr = f_max(1.f - cosThetaSqr, 0.f) / cosThetaSqr;
    return 0.5f * (-1.f + f_sqrt(1.f + alphaSqr * tanThetaSqr));
}
RS_HD float evalMaskingSmithGGXCorrelated(float alpha, float cosThetaI, float cosThetaO)
{
    float alphaSqr = alpha * alpha;
    float lambdaI = evalLambdaGGX(alphaSqr, cosThetaI);
    float lambdaO = evalLambdaGGX(alphaSqr, cosThetaO);
    return 1.f / (1.f + lambdaI + lambdaO);
}
RS_HD float evalPdfGGX_VNDF(float alpha, f3 wi, f3 h)
{
    float G1 = evalG1GGX(alpha * alpha, wi.z);
    float D = evalNdfGGX(alpha, h.z);
    return G1 * D * f_max(0.f, dot(wi, h)) / wi.z;
}
// Spherical-cap VNDF sampling (Dupuy & Benyoub 2023), IsotropicGGX.slang SampleVndf_Hemisphere.
// The reference writes z = fma(1 - u.y, 1 + Vh.z, -Vh.z); here the product and sum are
// rounded separately (the restatement never fuses).
RS_HD f3 sampleGGX_VNDF(float alpha, f3 wi, f2 u, float& pdf)
{
    f3 Vh = normalize(mk3(alpha * wi.x, alpha * wi.y, wi.z));
    float phi = k2Pi * u.x;
    float z = (1.f - u.y) * (1.f + Vh.z) - Vh.z;
    float sinTheta = f_sqrt(f_saturate(1.f - z * z));
    float s, c;
    f_sincos(phi, s, c);
    f3 Nh = mk3(sinTheta * c, sinTheta * s, z) + Vh;
    f3 h = normalize(mk3(alpha * Nh.x, alpha * Nh.y, Nh.z));
    pdf = evalPdfGGX_VNDF(alpha, wi, h);
    return h;
}

RS_HD f3 evalFresnelSchlick3(f3 f0, float f90, float cosTheta)
{
    float p = f_pow5(f_max(1.f - cosTheta, 0.f));
    return mk3(f0.x + (f90 - f0.x) * p, f0.y + (f90 - f0.y) * p, f0.z + (f90 - f0.z) * p);
}
RS_HD float evalFresnelSchlick1(float f0, float f90, float cosTheta)
{
    return f0 + (f90 - f0) * f_pow5(f_max(1.f - cosTheta, 0.f));
}

// ---- sampling helpers (MathHelpers.slang:269-277, 323-355, 391-396) ----
RS_HD f2 sample_disk(f2 u)
{
    float r = f_sqrt(u.x);
    float phi = k2Pi * u.y;
    float s, c;
    f_sincos(phi, s, c);
    return mk2(r * c, r * s);
}
RS_HD f2 sample_disk_concentric(f2 u)
{
    u = mk2(2.f * u.x - 1.f, 2.f * u.y - 1.f);
    if (u.x == 0.f && u.y == 0.f) return u;
    float phi, r;
    if (f_abs(u.x) > f_abs(u.y))
    {
        r = u.x;
        phi = (u.y / u.x) * kPiOver4;
    }
    else
    {
        r = u.y;
        phi = kPiOver2 - (u.x / u.y) * kPiOver4;
    }
    float s, c;
    f_sincos(phi, s, c);
    return mk2(r * c, r * s);
}
RS_HD f3 sample_cosine_hemisphere_concentric(f2 u, float& pdf)
{
    f2 d = sample_disk_concentric(u);
    float z = f_sqrt(f_max(0.f, 1.f - dot(d, d)));
    pdf = z * k1OverPi;
    return mk3(d.x, d.y, z);
}

// ---- StandardBSDF (opaque: Frostbite diffuse + GGX reflection) ----
struct StandardBSDF
{
    f3 diffAlbedo;
    float diffRoughness;
    f3 specAlbedo;
    float alpha;
    float pDiffuseReflection;
    float pSpecularReflection;
    uint32_t lobeMask;
};

RS_HD StandardBSDF make_bsdf(f3 wi, const BsdfData& d, uint32_t lobeMask)
{
    StandardBSDF b;
    b.lobeMask = lobeMask;
    b.diffAlbedo = d.diffuse;
    b.diffRoughness = d.roughness;
    float alpha = d.roughness * d.roughness;
    alpha = f_max(alpha, kMinGGXAlpha);
    alpha = lobeMask == 5u ? 0.f : alpha;
    b.specAlbedo = d.specular;
    b.alpha = alpha;
    // With specTrans = diffTrans = 0 the factors (1 - specTrans) and (1 - diffTrans) are exactly 1.
    float metallicBRDF = d.metallic;
    float dielectricBSDF = 1.f - d.metallic;
    float diffuseWeight = luminance(d.diffuse);
    float specularWeight = luminance(evalFresnelSchlick3(d.specular, 1.f, wi.z));
    b.pDiffuseReflection = diffuseWeight * dielectricBSDF;
    b.pSpecularReflection = specularWeight * (metallicBRDF + dielectricBSDF);
    float normFactor = b.pDiffuseReflection + b.pSpecularReflection;
    if (normFactor > 0.f)
    {
        normFactor = 1.f / normFactor;
        b.pDiffuseReflection *= normFactor;
        b.pSpecularReflection *= normFactor;
    }
    return b;
}

// FrostbiteDiffuseBRDF::evalWeight
RS_HD f3 frostbite_weight(const StandardBSDF& b, f3 wi, f3 wo)
{
    f3 h = normalize(wi + wo);
    float woDotH = dot(wo, h);
    float energyBias = f_lerp(0.f, 0.5f, b.diffRoughness);
    float energyFactor = f_lerp(1.f, 1.f / 1.51f, b.diffRoughness);
    float fd90 = energyBias + 2.f * woDotH * woDotH * b.diffRoughness;
    float fd0 = 1.f;
    float wiScatter = evalFresnelSchlick1(fd0, fd90, wi.z);
    float woScatter = evalFresnelSchlick1(fd0, fd90, wo.z);
    return b.diffAlbedo * wiScatter * woScatter * energyFactor;
}
RS_HD f3 diffuse_eval(const StandardBSDF& b, f3 wi, f3 wo)
{
    if (f_min(wi.z, wo.z) < kMinCosTheta) return mk3(0.f);
    return frostbite_weight(b, wi, wo) * k1OverPi * wo.z;
}
RS_HD float diffuse_pdf(f3 wi, f3 wo)
{
    if (f_min(wi.z, wo.z) < kMinCosTheta) return 0.f;
    return k1OverPi * wo.z;
}
RS_HD f3 specular_eval(const StandardBSDF& b, f3 wi, f3 wo)
{
    if (f_min(wi.z, wo.z) < kMinCosTheta) return mk3(0.f);
    if (b.alpha == 0.f) return mk3(0.f);
    f3 h = normalize(wi + wo);
    float wiDotH = dot(wi, h);
    float D = evalNdfGGX(b.alpha, h.z);
    float G = evalMaskingSmithGGXCorrelated(b.alpha, wi.z, wo.z);
    f3 F = evalFresnelSchlick3(b.specAlbedo, 1.f, wiDotH);
    return F * D * G * 0.25f / wi.z;
}
RS_HD float specular_pdf(const StandardBSDF& b, f3 wi, f3 wo)
{
    if (f_min(wi.z, wo.z) < kMinCosTheta) return 0.f;
    if (b.alpha == 0.f) return 0.f;
    f3 h = normalize(wi + wo);
    float wiDotH = dot(wi, h);
    float pdf = evalPdfGGX_VNDF(b.alpha, wi, h);
    return pdf / (4.f * wiDotH);
}

RS_HD f3 bsdf_eval_local(const StandardBSDF& b, f3 wi, f3 wo)
{
    uint32_t mask = b.lobeMask;
    if (b.lobeMask == 0) mask = 0xfu;
    f3 result = mk3(0.f);
    if (b.pDiffuseReflection > 0.f && (mask & 0x1u)) result += diffuse_eval(b, wi, wo);
    if (b.pSpecularReflection > 0.f && (mask & 0x4u)) result += specular_eval(b, wi, wo);
    return result;
}
RS_HD float bsdf_pdf_local(const StandardBSDF& b, f3 wi, f3 wo)
{
    float pdf = 0.f;
    uint32_t mask = b.lobeMask;
    if (b.lobeMask == 0) mask = 0xfu;
    if (b.pDiffuseReflection > 0.f && (mask & 0x1u)) pdf += b.pDiffuseReflection * diffuse_pdf(wi, wo);
    if (b.pSpecularReflection > 0.f && (mask & 0x4u)) pdf += b.pSpecularReflection * specular_pdf(b, wi, wo);
    return pdf;
}

// StandardBSDF::sample restricted to the two reflection lobes.  Draw order:
// lobe select (1D) then the lobe's 2D sample.
RS_HD bool bsdf_sample_local(const StandardBSDF& b, f3 wi, f3& wo, float& pdf, f3& weight, uint32_t& lobeType, SampleGen& sg)
{
    wo = mk3(0.f);
    weight = mk3(0.f);
    pdf = 0.f;
    lobeType = kLobeDiffuseReflection;
    bool valid = false;
    float uSelect = sampleNext1D(sg);
    if (uSelect < b.pDiffuseReflection)
    {
        f2 u; u.x = sampleNext1D(sg); u.y = sampleNext1D(sg);
        wo = sample_cosine_hemisphere_concentric(u, pdf);
        lobeType = kLobeDiffuseReflection;
        if (f_min(wi.z, wo.z) < kMinCosTheta) { weight = mk3(0.f); valid = false; }
        else { weight = frostbite_weight(b, wi, wo); valid = true; }
        weight = weight / b.pDiffuseReflection;
        pdf *= b.pDiffuseReflection;
        if (b.lobeMask == 0)
        {
            if (b.pSpecularReflection > 0.f) pdf += b.pSpecularReflection * specular_pdf(b, wi, wo);
        }
    }
    else if (uSelect < b.pDiffuseReflection + b.pSpecularReflection)
    {
        // SpecularMicrofacetBRDF::sample
        lobeType = kLobeSpecularReflection;
        valid = false;
        if (wi.z < kMinCosTheta) { valid = false; }
        else if (b.alpha == 0.f)
        {
            wo = mk3(-wi.x, -wi.y, wi.z);
            pdf = 0.f;
            weight = evalFresnelSchlick3(b.specAlbedo, 1.f, wi.z);
            lobeType = kLobeDeltaReflection;
            valid = true;
        }
        else
        {
            f2 u; u.x = sampleNext1D(sg); u.y = sampleNext1D(sg);
            float hpdf;
            f3 h = sampleGGX_VNDF(b.alpha, wi, u, hpdf);
            pdf = hpdf;
            float wiDotH = dot(wi, h);
            wo = h * (2.f * wiDotH) - wi;
            if (wo.z < kMinCosTheta) { valid = false; }
            else
            {
                float G = evalMaskingSmithGGXCorrelated(b.alpha, wi.z, wo.z);
                float GOverG1wo = G * (1.f + evalLambdaGGX(b.alpha * b.alpha, wi.z));
                f3 F = evalFresnelSchlick3(b.specAlbedo, 1.f, wiDotH);
                pdf /= (4.f * wiDotH);
                weight = F * GOverG1wo;
                lobeType = kLobeSpecularReflection;
                valid = true;
            }
        }
        weight = weight / b.pSpecularReflection;
        pdf *= b.pSpecularReflection;
        if (b.lobeMask == 0)
        {
            if (b.pDiffuseReflection > 0.f) pdf += b.pDiffuseReflection * diffuse_pdf(wi, wo);
        }
    }
    return valid;
}

// Material instance: shading frame + BSDF parameters (StandardMaterialInstance.slang).
struct MaterialInstance
{
    BsdfData data;
};

// isValidHemisphereReflectionOrTransmission with FALCOR_BACKFACE_BLACK, fullSphere = false.
RS_HD bool valid_hemisphere(const ShadingData& sd, f3 wiLocal, f3 woLocal, f3 wo)
{
    const bool isTransmission = wiLocal.z * woLocal.z < 0.f;
    float cosThetaI = wiLocal.z;
    if (f_min(cosThetaI, f_abs(woLocal.z)) < kMinCosTheta) return false;
    bool wiTop = sd.frontFacing;
    bool woTop = dot(wo, sd.faceN) >= 0.f;
    if (isTransmission) { if (wiTop == woTop) return false; }
    else { if (wiTop != woTop) return false; }
    bool shadingTop = dot(sd.N, sd.faceN) >= 0.f;
    if (wiTop != shadingTop) return false;
    return true;
}

RS_HD f3 mi_eval(const ShadingData& sd, const BsdfData& d, uint32_t lobeMask, f3 wo)
{
    f3 wiLocal = sd_to_local(sd, sd.V);
    f3 woLocal = sd_to_local(sd, wo);
    if (!valid_hemisphere(sd, wiLocal, woLocal, wo)) return mk3(0.f);
    StandardBSDF b = make_bsdf(wiLocal, d, lobeMask);
    return bsdf_eval_local(b, wiLocal, woLocal);
}
RS_HD float mi_pdf(const ShadingData& sd, const BsdfData& d, uint32_t lobeMask, f3 wo)
{
    f3 wiLocal = sd_to_local(sd, sd.V);
    f3 woLocal = sd_to_local(sd, wo);
    if (!valid_hemisphere(sd, wiLocal, woLocal, wo)) return 0.f;
    StandardBSDF b = make_bsdf(wiLocal, d, lobeMask);
    return bsdf_pdf_local(b, wiLocal, woLocal);
}
// mi_eval and mi_pdf for the single lobe 1 << comp (comp < 4) and for all lobes (mask 0 or 0xF) in
// one pass.  The per-lobe values do not depend on the mask (make_bsdf changes alpha only for mask
// 5, which no single lobe has), so they are computed once and summed in the order of
// bsdf_eval_local / bsdf_pdf_local: every result has the bits of the four separate calls.
struct BsdfPair
{
    f3 lobeBsdf;
    float lobePdf;
    f3 totalBsdf;
    float totalPdf;
};
RS_HD BsdfPair mi_eval_pair(const ShadingData& sd, const BsdfData& d, uint32_t comp, f3 wo)
{
    BsdfPair r;
    r.lobeBsdf = mk3(0.f); r.totalBsdf = mk3(0.f);
    r.lobePdf = 0.f; r.totalPdf = 0.f;
    f3 wiLocal = sd_to_local(sd, sd.V);
    f3 woLocal = sd_to_local(sd, wo);
    if (!valid_hemisphere(sd, wiLocal, woLocal, wo)) return r;
    const uint32_t mask = 1u << comp;
    StandardBSDF b = make_bsdf(wiLocal, d, mask);
    if (b.pDiffuseReflection > 0.f)
    {
        const f3 v = diffuse_eval(b, wiLocal, woLocal);
        const float p = b.pDiffuseReflection * diffuse_pdf(wiLocal, woLocal);
        r.totalBsdf += v; r.totalPdf += p;
        if (mask & 0x1u) { r.lobeBsdf += v; r.lobePdf += p; }
    }
    if (b.pSpecularReflection > 0.f)
    {
        const f3 v = specular_eval(b, wiLocal, woLocal);
        const float p = b.pSpecularReflection * specular_pdf(b, wiLocal, woLocal);
        r.totalBsdf += v; r.totalPdf += p;
        if (mask & 0x4u) { r.lobeBsdf += v; r.lobePdf += p; }
    }
    return r;
}

struct BSDFSample
{
    f3 wo;
    float pdf;
    f3 weight;
    uint32_t lobeType;
};
RS_HD bool mi_sample(const ShadingData& sd, const BsdfData& d, uint32_t lobeMask, SampleGen& sg, BSDFSample& r)
{
    f3 wiLocal = sd_to_local(sd, sd.V);
    f3 woLocal;
    StandardBSDF b = make_bsdf(wiLocal, d, lobeMask);
    if (!bsdf_sample_local(b, wiLocal, woLocal, r.pdf, r.weight, r.lobeType, sg)) return false;
    r.wo = sd_from_local(sd, woLocal);
    if (!valid_hemisphere(sd, wiLocal, woLocal, r.wo)) return false;
    return true;
}
// mi_sample(sd, d, lobeMask, sg, r) and, in `totalPdf`, mi_pdf(sd, d, 0xF, r.wo) in one pass: the
// local incident direction and the BSDF parameters are shared (make_bsdf's mask changes alpha only
// for mask 5, so lobeMask != 5 is required), the sampled direction is brought back to the local
// frame from its world value as mi_pdf does; every result has the bits of the two calls.  r.wo must
// hold the caller's value for a failed sample (mi_sample leaves it unchanged then).
RS_HD bool mi_sample_total_pdf(const ShadingData& sd, const BsdfData& d, uint32_t lobeMask, SampleGen& sg, BSDFSample& r, float& totalPdf)
{
    const f3 wiLocal = sd_to_local(sd, sd.V);
    StandardBSDF b = make_bsdf(wiLocal, d, lobeMask);
    f3 woLocal;
    bool ok = bsdf_sample_local(b, wiLocal, woLocal, r.pdf, r.weight, r.lobeType, sg);
    if (ok)
    {
        r.wo = sd_from_local(sd, woLocal);
        ok = valid_hemisphere(sd, wiLocal, woLocal, r.wo);
    }
    const f3 woTotal = sd_to_local(sd, r.wo);
    b.lobeMask = 0xFu;
    totalPdf = valid_hemisphere(sd, wiLocal, woTotal, r.wo) ? bsdf_pdf_local(b, wiLocal, woTotal) : 0.f;
    return ok;
}

// getLobeTypes for an opaque StandardBSDFData (StandardBSDF.slang:210-232).
RS_HD uint32_t mi_lobe_types(const BsdfData& d)
{
    uint32_t lobeTypes = kLobeSpecularReflection;
    if (any_gt0(d.diffuse)) lobeTypes |= kLobeDiffuseReflection;
    return lobeTypes;
}
// getProperties().roughness (StandardMaterialInstance.slang:128-131)
RS_HD float mi_roughness(const BsdfData& d)
{
    float alpha = d.roughness * d.roughness;
    return alpha < kMinGGXAlpha ? 0.f : d.roughness;
}

} // namespace rs
