"""Property tests of the shared shading core (csrc/core: BSDF, emissive light sampling, camera),
checked against independent float64 numpy restatements of the reference's formulas and against the
sampling tests the reference runs on its own BSDFs.

The CUDA kernels and the oracle compile the same csrc/core headers, so a GPU-vs-oracle comparison
cannot see a mistake in them.  These tests pin that layer from outside:

* BSDF sampling: the chi^2 test of Source/Tools/FalcorTest/Tests/Scene/Material/BSDFTests.cpp
  (directions binned into 130 phi x 65 cos(theta) cells, expected counts from the pdf integrated
  over each cell with 64 x 64 midpoint samples, Pearson's statistic with cells of expected count < 5 pooled, significance 0.01
  with a Sidak correction over the configurations), on the same configurations (Frostbite diffuse
  at roughness 0.5; GGX reflection at alpha 0.05 and 0.5; incident directions perpendicular,
  oblique and grazing), plus the opaque StandardBSDF mix.  Also its weight check (the sample weight
  against eval / evalPdf) and pdf check (the sample pdf against evalPdf), both to 1e-3.
* BSDF values: eval and evalPdf against a numpy restatement of FrostbiteDiffuseBRDF.slang,
  SpecularMicrofacet.slang / IsotropicGGX.slang (GGX D, height-correlated Smith G, VNDF pdf),
  Fresnel.slang (Schlick) and StandardBSDF.slang's lobe probabilities; reciprocity; the directional
  albedo against a numpy quadrature of the restated BSDF (and <= 1 where the model conserves energy).
* Emissive sampling (EmissivePowerSampler.slang, EmissiveLightSamplerHelpers.slang): the sample
  pdf equals evalPdf at the sampled point, triangles are picked in proportion to their flux
  (chi^2), and E[1/pdf] over a light's samples equals its solid angle (Van Oosterom & Strackee).
* Camera: the basis of Camera.cpp:179-185 and orientCamera / angularLerp of
  CameraManager.slang:50-113 (with the quaternion helpers of Utils/Math/Quaternion.slang).
"""
import ctypes as C
import math

import numpy as np
import pytest
from scipy import stats

LUM = np.array([0.2126, 0.7152, 0.0722])
K_MIN_COS = 1e-6
K_MIN_GGX_ALPHA = 0.0064


@pytest.fixture(scope="module")
def lib(oracle_mod):
    L = oracle_mod.load()
    vp, u32, f32 = C.c_void_p, C.c_uint32, C.c_float
    L.ro_test_bsdf_sample.argtypes = [u32, vp, vp, u32, u32, vp, vp, vp, vp, vp]
    L.ro_test_bsdf_eval.argtypes = [u32, vp, vp, vp, u32, vp, vp]
    L.ro_test_bsdf_histogram.argtypes = [u32, vp, vp, u32, u32, u32, u32, u32, vp, vp, vp]
    L.ro_test_emissive.argtypes = [vp, vp, u32, u32, vp, vp, vp, vp]
    L.ro_test_emissive.restype = C.c_int
    L.ro_test_lights.argtypes = [vp, vp]
    L.ro_test_lights.restype = u32
    L.ro_test_camera_basis.argtypes = [vp, vp]
    L.ro_test_orient_camera.argtypes = [vp, u32, vp, vp, f32, u32, f32, vp]
    return L


# ---------------------------------------------------------------- independent restatements (float64)
def _normalize(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def _schlick(f0, f90, cos_theta):
    return f0 + (f90 - f0) * np.maximum(1.0 - cos_theta, 0.0) ** 5


def _ggx_d(alpha, cos_h):
    a2 = alpha * alpha
    d = (cos_h * a2 - cos_h) * cos_h + 1.0
    return a2 / (d * d * math.pi)


def _ggx_lambda(a2, c):
    c = np.asarray(c, np.float64)
    tan2 = np.maximum(1.0 - c * c, 0.0) / np.where(c > 0, c * c, 1.0)
    return np.where(c > 0, 0.5 * (-1.0 + np.sqrt(1.0 + a2 * tan2)), 0.0)


def _ggx_g1(a2, c):
    return np.where(np.asarray(c) > 0, 1.0 / (1.0 + _ggx_lambda(a2, c)), 0.0)


def _spec_eval(alpha, f0, wi, wo):
    """SpecularMicrofacetBRDF::eval: F D G / (4 cos_i) (the cosine of wo folded in)."""
    h = _normalize(wi + wo)
    wi_h = np.sum(wi * h, -1)
    D = _ggx_d(alpha, h[..., 2])
    G = 1.0 / (1.0 + _ggx_lambda(alpha * alpha, wi[..., 2]) + _ggx_lambda(alpha * alpha, wo[..., 2]))
    F = _schlick(np.asarray(f0)[None, :], 1.0, wi_h[:, None])
    ok = np.minimum(wi[..., 2], wo[..., 2]) >= K_MIN_COS
    return np.where(ok[:, None], F * (D * G * 0.25 / wi[..., 2])[:, None], 0.0)


def _spec_pdf(alpha, wi, wo):
    """VNDF pdf of the half vector over the reflection Jacobian 4 (wi . h)."""
    h = _normalize(wi + wo)
    wi_h = np.sum(wi * h, -1)
    pdf_h = _ggx_g1(alpha * alpha, wi[..., 2]) * _ggx_d(alpha, h[..., 2]) * np.maximum(0.0, wi_h) / wi[..., 2]
    ok = np.minimum(wi[..., 2], wo[..., 2]) >= K_MIN_COS
    return np.where(ok, pdf_h / (4.0 * wi_h), 0.0)


def _frostbite_eval(rough, albedo, wi, wo):
    h = _normalize(wi + wo)
    wo_h = np.sum(wo * h, -1)
    energy_bias = 0.5 * rough
    energy_factor = 1.0 + (1.0 / 1.51 - 1.0) * rough
    fd90 = energy_bias + 2.0 * wo_h * wo_h * rough
    s = _schlick(1.0, fd90, wi[..., 2]) * _schlick(1.0, fd90, wo[..., 2]) * energy_factor
    ok = np.minimum(wi[..., 2], wo[..., 2]) >= K_MIN_COS
    return np.where(ok[:, None], np.asarray(albedo)[None, :] * (s * wo[..., 2] / math.pi)[:, None], 0.0)


def _frostbite_pdf(wi, wo):
    ok = np.minimum(wi[..., 2], wo[..., 2]) >= K_MIN_COS
    return np.where(ok, wo[..., 2] / math.pi, 0.0)


def _standard(params, wi):
    """StandardMaterial (metal-rough, opaque) -> StandardBSDF lobe parameters and probabilities for
    each incident direction."""
    base, rough, metallic, ior = params
    f = (ior - 1.0) / (ior + 1.0)
    F0 = f * f
    diffuse = np.full(3, base * (1.0 - metallic))
    specular = np.full(3, F0 + (base - F0) * metallic)
    alpha = max(rough * rough, K_MIN_GGX_ALPHA)
    p_d = np.full(len(wi), float(LUM @ diffuse) * (1.0 - metallic))
    p_s = (_schlick(specular[None, :], 1.0, wi[:, 2:3]) @ LUM) * (metallic + (1.0 - metallic))
    norm = p_d + p_s
    p_d, p_s = np.where(norm > 0, p_d / norm, p_d), np.where(norm > 0, p_s / norm, p_s)
    return diffuse, specular, rough, alpha, p_d, p_s


def ref_eval_pdf(kind, params, wi, wo):
    if kind == 0:
        return _frostbite_eval(params[0], np.ones(3), wi, wo), _frostbite_pdf(wi, wo)
    if kind == 1:
        return _spec_eval(params[0], np.ones(3), wi, wo), _spec_pdf(params[0], wi, wo)
    diffuse, specular, rough, alpha, p_d, p_s = _standard(params, wi)
    v = np.where((p_d > 0)[:, None], _frostbite_eval(rough, diffuse, wi, wo), 0.0) + \
        np.where((p_s > 0)[:, None], _spec_eval(alpha, specular, wi, wo), 0.0)
    pdf = np.where(p_d > 0, p_d * _frostbite_pdf(wi, wo), 0.0) + np.where(p_s > 0, p_s * _spec_pdf(alpha, wi, wo), 0.0)
    return v, pdf


# ---------------------------------------------------------------- product hooks
def _params(p):
    return np.asarray(list(p) + [0.0] * (4 - len(p)), np.float32)


def product_eval(lib, kind, params, wi, wo):
    wi = np.ascontiguousarray(wi, np.float32)
    wo = np.ascontiguousarray(wo, np.float32)
    n = len(wi)
    v = np.zeros((n, 3), np.float32)
    pdf = np.zeros(n, np.float32)
    pp = _params(params)
    lib.ro_test_bsdf_eval(kind, pp.ctypes.data, wi.ctypes.data, wo.ctypes.data, n, v.ctypes.data, pdf.ctypes.data)
    return v, pdf


def product_samples(lib, kind, params, wi, n, seed=1):
    pp = _params(params)
    w = np.ascontiguousarray(wi, np.float32)
    wo = np.zeros((n, 3), np.float32)
    pdf = np.zeros(n, np.float32)
    weight = np.zeros((n, 3), np.float32)
    valid = np.zeros(n, np.uint32)
    lobe = np.zeros(n, np.uint32)
    lib.ro_test_bsdf_sample(kind, pp.ctypes.data, w.ctypes.data, n, seed, wo.ctypes.data, pdf.ctypes.data, weight.ctypes.data,
                            valid.ctypes.data, lobe.ctypes.data)
    return wo, pdf, weight, valid.astype(bool), lobe


def chi2_test(obs, exp, sample_count, min_exp=5.0, significance=0.01, test_count=1):
    """Pearson's chi^2 with pooling of low-expectation cells (the procedure of Jakob's `hypothesis`
    helpers that the reference's BSDF test calls): returns (passed, p-value, message)."""
    order = np.argsort(exp, kind="stable")
    chsq, dof = 0.0, 0
    pooled_obs = pooled_exp = 0.0
    for i in order:
        o, e = float(obs[i]), float(exp[i])
        if e == 0.0:
            if o > sample_count * 1e-5:
                return False, 0.0, f"cell {i}: {o} samples where the pdf integrates to 0"
        elif e < min_exp:
            pooled_obs += o
            pooled_exp += e
        elif 0.0 < pooled_exp < min_exp:
            pooled_obs += o
            pooled_exp += e
        else:
            chsq += (o - e) ** 2 / e
            dof += 1
    if pooled_exp > 0.0 or pooled_obs > 0.0:
        chsq += (pooled_obs - pooled_exp) ** 2 / pooled_exp
        dof += 1
    dof -= 1
    if dof < 1:
        return False, 0.0, "too few cells"
    pval = float(stats.chi2.sf(chsq, dof))
    alpha = 1.0 - (1.0 - significance) ** (1.0 / test_count)
    return pval >= alpha, pval, f"chi2 {chsq:.1f} dof {dof} p {pval:.4g} (threshold {alpha:.3g})"


PERP = (0.0, 0.0, 1.0)
OBLIQUE = tuple(np.array([0.5, 0.0, 0.5]) / np.linalg.norm([0.5, 0.0, 0.5]))
GRAZING = tuple(np.array([0.0, 1.0, 0.01]) / np.linalg.norm([0.0, 1.0, 0.01]))
SAMPLING_CONFIGS = [
    ("frostbite_perp", 0, [0.5], PERP), ("frostbite_oblique", 0, [0.5], OBLIQUE), ("frostbite_grazing", 0, [0.5], GRAZING),
    ("ggx_smooth_perp", 1, [0.05], PERP), ("ggx_smooth_oblique", 1, [0.05], OBLIQUE), ("ggx_smooth_grazing", 1, [0.05], GRAZING),
    ("ggx_rough_perp", 1, [0.5], PERP), ("ggx_rough_oblique", 1, [0.5], OBLIQUE), ("ggx_rough_grazing", 1, [0.5], GRAZING),
    ("standard_perp", 2, [0.5, 0.5, 0.3, 1.5], PERP), ("standard_oblique", 2, [0.5, 0.5, 0.3, 1.5], OBLIQUE),
    ("standard_metal_oblique", 2, [0.9, 0.35, 1.0, 1.5], OBLIQUE),
]
PHI_BINS, COS_BINS, BIN_SAMPLES = 130, 65, 64
SAMPLE_COUNT = 8 * 1024 * 1024


@pytest.mark.parametrize("name,kind,params,wi", SAMPLING_CONFIGS, ids=[c[0] for c in SAMPLING_CONFIGS])
def test_bsdf_sampling_chi2_weight_and_pdf(lib, name, kind, params, wi):
    pp = _params(params)
    w = np.asarray(wi, np.float32)
    hist = np.zeros(PHI_BINS * COS_BINS)
    exp = np.zeros(PHI_BINS * COS_BINS)
    err = np.zeros(2)
    lib.ro_test_bsdf_histogram(kind, pp.ctypes.data, w.ctypes.data, SAMPLE_COUNT, PHI_BINS, COS_BINS, BIN_SAMPLES, 5,
                               hist.ctypes.data, exp.ctypes.data, err.ctypes.data)
    ok, pval, msg = chi2_test(hist, exp, SAMPLE_COUNT, test_count=len(SAMPLING_CONFIGS))
    assert ok, f"{name}: sampled directions do not follow evalPdf: {msg}"
    if kind != 2:
        # a single lobe: weight = eval / pdf.  The StandardBSDF mix returns the picked lobe's weight
        # over its selection probability with the mixture's pdf (StandardBSDF.slang sample), so for
        # it only the mean weight is pinned (test_white_furnace_albedo).
        assert err[0] <= 1e-3, f"{name}: sample weight vs eval/evalPdf relative error {err[0]:.3g}"
    assert err[1] <= 1e-3, f"{name}: sample pdf vs evalPdf relative error {err[1]:.3g}"


def _hemisphere_pairs(n, seed, min_cos=0.05):
    rng = np.random.default_rng(seed)

    def dirs():
        z = rng.uniform(min_cos, 1.0, n)
        phi = rng.uniform(0.0, 2.0 * math.pi, n)
        s = np.sqrt(1.0 - z * z)
        return np.stack([s * np.cos(phi), s * np.sin(phi), z], 1)
    return dirs().astype(np.float32), dirs().astype(np.float32)


EVAL_CONFIGS = [(0, [0.0]), (0, [0.5]), (0, [1.0]), (1, [0.05]), (1, [0.3]), (1, [1.0]),
                (2, [0.5, 0.5, 0.0, 1.5]), (2, [0.8, 0.2, 1.0, 1.5]), (2, [0.3, 0.9, 0.5, 1.33])]


@pytest.mark.parametrize("kind,params", EVAL_CONFIGS, ids=[f"k{k}-{p}" for k, p in EVAL_CONFIGS])
def test_bsdf_eval_and_pdf_match_restatement(lib, kind, params):
    wi, wo = _hemisphere_pairs(20000, 3 + kind)
    v, pdf = product_eval(lib, kind, params, wi, wo)
    rv, rpdf = ref_eval_pdf(kind, params, wi.astype(np.float64), wo.astype(np.float64))
    scale_v = np.maximum(np.abs(rv), 1e-6)
    assert np.all(np.abs(v - rv) <= 5e-4 * scale_v + 1e-7), float(np.max(np.abs(v - rv) / scale_v))
    assert np.all(np.abs(pdf - rpdf) <= 5e-4 * np.maximum(rpdf, 1e-6) + 1e-7), float(np.max(np.abs(pdf - rpdf) / np.maximum(rpdf, 1e-6)))


@pytest.mark.parametrize("kind,params", EVAL_CONFIGS, ids=[f"k{k}-{p}" for k, p in EVAL_CONFIGS])
def test_bsdf_reciprocity(lib, kind, params):
    """f(wi, wo) = f(wo, wi): eval carries cos(wo), so eval(wi, wo) / wo.z = eval(wo, wi) / wi.z."""
    wi, wo = _hemisphere_pairs(20000, 11 + kind)
    a, _ = product_eval(lib, kind, params, wi, wo)
    b, _ = product_eval(lib, kind, params, wo, wi)
    fa = a / wo[:, 2:3]
    fb = b / wi[:, 2:3]
    assert np.all(np.abs(fa - fb) <= 1e-4 * np.maximum(np.abs(fa), 1e-6) + 1e-7)


def _albedo_quadrature(kind, params, wi, n_cos=1024, n_phi=512):
    """Directional albedo = integral of eval over the hemisphere, by the midpoint rule in (cos, phi)."""
    c = (np.arange(n_cos) + 0.5) / n_cos
    phi = (np.arange(n_phi) + 0.5) / n_phi * 2.0 * math.pi
    cc, pp = np.meshgrid(c, phi, indexing="ij")
    s = np.sqrt(1.0 - cc * cc)
    wo = np.stack([s * np.cos(pp), s * np.sin(pp), cc], -1).reshape(-1, 3)
    wiv = np.broadcast_to(np.asarray(wi, np.float64), wo.shape).copy()
    v, _ = ref_eval_pdf(kind, params, wiv, wo)
    return float(v[:, 0].sum() * (1.0 / n_cos) * (2.0 * math.pi / n_phi))


FURNACE = [(0, [0.0]), (0, [0.5]), (0, [1.0]), (1, [0.3]), (1, [0.6]), (1, [1.0]), (2, [1.0, 0.6, 0.0, 1.5]),
           (2, [1.0, 0.5, 1.0, 1.5])]


@pytest.mark.parametrize("kind,params", FURNACE, ids=[f"k{k}-{p}" for k, p in FURNACE])
@pytest.mark.parametrize("cos_i", [1.0, 0.5, 0.1])
def test_white_furnace_albedo(lib, kind, params, cos_i):
    """The mean sample weight (the Monte Carlo directional albedo of the product's sampler) equals an
    independent quadrature of the restated BSDF.  The GGX lobe (Smith masking) and the Frostbite lobe
    at roughness <= 0.5 keep it <= 1 at white albedo; Frostbite's normalisation is an average over
    incident directions, so at roughness 1 and grazing incidence (and in the StandardBSDF sum of a
    white diffuse and a dielectric coat) a directional albedo slightly above 1 is the model's own."""
    wi = np.array([math.sqrt(1.0 - cos_i * cos_i), 0.0, cos_i])
    n = 1 << 20
    _, _, weight, valid, _ = product_samples(lib, kind, params, wi, n, seed=21)
    x = np.where(valid, weight[:, 0], 0.0).astype(np.float64)
    mc, se = x.mean(), x.std() / math.sqrt(n)
    q = _albedo_quadrature(kind, params, wi)
    assert abs(mc - q) <= 5.0 * se + 2e-3 * q, (mc, se, q)
    if kind == 1 or (kind == 0 and params[0] <= 0.5):
        assert mc <= 1.0 + 5.0 * se and q <= 1.0 + 1e-3


def _solid_angle(p0, p1, p2, x):
    """Solid angle of triangle (p0, p1, p2) seen from x (Van Oosterom & Strackee 1983)."""
    a, b, c = (np.asarray(p, np.float64) - x for p in (p0, p1, p2))
    la, lb, lc = (np.linalg.norm(v) for v in (a, b, c))
    num = abs(np.dot(a, np.cross(b, c)))
    den = la * lb * lc + np.dot(a, b) * lc + np.dot(a, c) * lb + np.dot(b, c) * la
    return 2.0 * math.atan2(num, den)


@pytest.mark.parametrize("sampler", ["Power", "Uniform"])
def test_emissive_sampling_pdf_selection_and_solid_angle(lib, oracle_mod, rs, sampler):
    """EmissivePowerSampler (triangles in proportion to their flux) and EmissiveUniformSampler
    (each triangle with probability 1 / count): the sample's pdf is evalPdf, the selection follows
    the sampler, and E[1 / pdf] over a light's samples is its solid angle."""
    import reservoir_splatting_b200.scenes as S
    # a floor and five emissive triangles of different radiance, area and orientation
    tris, mats, mids = [], [S.material((0.5, 0.5, 0.5))], []
    tris += [[-5, 0, -5, 5, 0, -5, 5, 0, 5], [-5, 0, -5, 5, 0, 5, -5, 0, 5]]
    mids += [0, 0]
    rng = np.random.default_rng(4)
    for k in range(5):
        c = np.array([rng.uniform(-2, 2), rng.uniform(1.5, 3.0), rng.uniform(-2, 2)])
        d1, d2 = rng.normal(0, 0.4, 3), rng.normal(0, 0.4, 3)
        p0, p1, p2 = c, c + d1, c + d2
        if np.cross(p1 - p0, p2 - p0)[1] > 0:  # face down, toward the floor point
            p1, p2 = p2, p1
        tris.append(np.concatenate([p0, p1, p2]).tolist())
        mats.append(S.material((0, 0, 0), emissive=tuple(rng.uniform(2.0, 30.0, 3))))
        mids.append(len(mats) - 1)
    # one light facing up: never visible from below, so its samples are rejected
    tris.append([0, 2.0, 0, 0.3, 2.0, 0.3, 0.3, 2.0, 0])
    mats.append(S.material((0, 0, 0), emissive=(10.0, 10.0, 10.0)))
    mids.append(len(mats) - 1)
    sc = S.Scene(np.asarray(tris, np.float32), np.asarray(mids, np.uint32), np.stack(mats).astype(np.float32))
    ora = oracle_mod.OraclePass({"temporalReuse": "GatherOnly", "emissiveSampler": sampler}, 8, 8)
    ora.set_scene(sc)
    n_l = lib.ro_test_lights(ora._h, None)
    rec = np.zeros((n_l, 20), np.float32)
    lib.ro_test_lights(ora._h, rec.ctypes.data)
    flux = rec[:, 11].astype(np.float64)
    x = np.array([0.3, 0.0, -0.2], np.float32)
    n = 1 << 21
    tri = np.zeros(n, np.uint32)
    pdf = np.zeros(n, np.float32)
    epdf = np.zeros(n, np.float32)
    pos = np.zeros((n, 3), np.float32)
    assert lib.ro_test_emissive(ora._h, x.ctypes.data, n, 7, tri.ctypes.data, pdf.ctypes.data, epdf.ctypes.data, pos.ctypes.data) == 0
    ok = pdf > 0
    # the sample's pdf is evalPdf at the sampled point
    assert np.all(np.abs(pdf[ok] - epdf[ok]) <= 1e-5 * epdf[ok])
    # triangles are picked in proportion to their flux, or uniformly (before the facing test)
    counts = np.bincount(tri, minlength=n_l).astype(np.float64)
    expected = flux / flux.sum() * n if sampler == "Power" else np.full(n_l, n / n_l)
    passed, pval, msg = chi2_test(counts, expected, n)
    assert passed, msg
    # E[1 / pdf; sample of light t] = solid angle of t (a light facing away contributes 0)
    for t in range(n_l):
        est = np.where(ok & (tri == t), 1.0 / np.where(ok, pdf, 1.0), 0.0).astype(np.float64)
        mean, se = est.mean(), est.std() / math.sqrt(n)
        p = rec[t]
        facing = np.dot(p[12:15], x - p[0:3]) > 0
        omega = _solid_angle(p[0:3], p[4:7], p[8:11], x.astype(np.float64)) if facing else 0.0
        assert abs(mean - omega) <= 5.0 * se + 1e-3 * omega, (t, mean, se, omega)


# ---------------------------------------------------------------- camera
def _fov_y(focal_length, frame_height):
    return 0.0 if focal_length == 0.0 else 2.0 * math.atan(0.5 * frame_height / focal_length)


def ref_basis(pos, target, up, focal_length, frame_height, aspect, focal_distance, forward=None):
    """Camera.cpp:179-185 (forward = normalize(target - pos)) / recalculateCameraVectors (given forward)."""
    f = _normalize(np.asarray(target, np.float64) - pos) if forward is None else forward
    W = f * focal_distance
    U = _normalize(np.cross(W, up))
    V = _normalize(np.cross(U, W))
    t = math.tan(_fov_y(focal_length, frame_height) * 0.5)
    return U * focal_distance * t * aspect, V * focal_distance * t, W


def _camera(rs, pos, target, up=(0.0, 1.0, 0.0), focal_length=21.0, frame_height=24.0, aspect=1.5, focal_distance=3.0):
    c = rs.abi.RsCamera()
    for k in range(3):
        c.position[k], c.target[k], c.up[k] = pos[k], target[k], up[k]
    c.focalLength, c.frameHeight, c.aspectRatio, c.focalDistance = focal_length, frame_height, aspect, focal_distance
    return c


def test_camera_basis_matches_restatement(lib, rs):
    rng = np.random.default_rng(2)
    for _ in range(500):
        pos = rng.uniform(-10, 10, 3)
        target = pos + rng.normal(0, 1, 3) * rng.uniform(0.5, 20)
        fl, fh, asp, fd = rng.uniform(10, 80), 24.0, rng.uniform(0.5, 2.5), rng.uniform(0.5, 30)
        cam = _camera(rs, pos, target, focal_length=fl, frame_height=fh, aspect=asp, focal_distance=fd)
        out = np.zeros(9, np.float32)
        lib.ro_test_camera_basis(C.byref(cam), out.ctypes.data)
        U, V, W = ref_basis(pos.astype(np.float32).astype(np.float64), target.astype(np.float32).astype(np.float64),
                            np.array([0.0, 1.0, 0.0]), np.float32(fl), fh, np.float32(asp), np.float32(fd))
        ref = np.concatenate([U, V, W])
        assert np.allclose(out, ref, rtol=2e-5, atol=2e-5 * np.abs(ref).max())


def _quat_rotate(v, axis, angle):
    """rotate_vector(v, rotate_angle_axis(angle, axis)) of Quaternion.slang: q v q*."""
    s, c = math.sin(angle * 0.5), math.cos(angle * 0.5)
    q = np.concatenate([axis * s, [c]])

    def qmul(a, b):
        return np.concatenate([b[:3] * a[3] + a[:3] * b[3] + np.cross(a[:3], b[:3]), [a[3] * b[3] - np.dot(a[:3], b[:3])]])
    qc = q * np.array([-1.0, -1.0, -1.0, 1.0])
    return qmul(q, qmul(np.concatenate([v, [0.0]]), qc))[:3]


def ref_orient(positions, targets, aft, frame_count, time, fl, fh, asp, fd):
    """CameraManager.slang orientCamera: camera at `time` before the current frame."""
    K = len(positions)
    curr = frame_count % K
    frame_index = int(math.floor(time / aft))
    first = (curr - frame_index - 1 + K) % K
    second = (first + 1 + K) % K
    t = (time - frame_index * aft) / aft
    pos = positions[second] + (positions[first] - positions[second]) * t
    f1 = _normalize(targets[first] - positions[first])
    f2 = _normalize(targets[second] - positions[second])
    axis = _normalize(np.cross(f2, f1))
    angle = math.acos(min(1.0, max(-1.0, float(np.dot(f2, f1)))))
    fwd = f2 if angle < 0.001 else _quat_rotate(f2, axis, angle * t)
    U, V, W = ref_basis(pos, None, np.array([0.0, 1.0, 0.0]), fl, fh, asp, fd, forward=fwd)
    return pos, U, V, W


def test_orient_camera_matches_restatement(lib, rs):
    rng = np.random.default_rng(9)
    aft = np.float32(1.0 / 48.0)
    checked = 0
    for trial in range(300):
        K = int(rng.integers(2, 6))
        base = rng.uniform(-5, 5, 3)
        positions = (base + np.cumsum(rng.normal(0, 0.05, (K, 3)), 0)).astype(np.float32)
        yaw = rng.uniform(0, 2 * math.pi) + np.cumsum(rng.normal(0, 0.05, K))
        targets = (positions + np.stack([np.cos(yaw), rng.normal(0, 0.2, K), np.sin(yaw)], 1) * 5.0).astype(np.float32)
        frame_count = int(rng.integers(0, 100))
        time = np.float32(rng.uniform(0.0, (K - 1) * float(aft)))
        q = float(time) / float(aft)
        if abs(q - round(q)) < 1e-3:  # float32 and float64 floor may differ at a keyframe boundary
            continue
        cam = _camera(rs, positions[0], targets[0], focal_length=35.0, aspect=1.7, focal_distance=2.0)
        out = np.zeros(12, np.float32)
        lib.ro_test_orient_camera(C.byref(cam), K, positions.ctypes.data, targets.ctypes.data, aft, frame_count, time, out.ctypes.data)
        ref = np.concatenate(ref_orient(positions.astype(np.float64), targets.astype(np.float64), float(aft), frame_count,
                                        float(time), 35.0, 24.0, np.float32(1.7), 2.0))
        assert np.allclose(out, ref, rtol=1e-4, atol=2e-4), (trial, out, ref)
        checked += 1
    assert checked > 250
