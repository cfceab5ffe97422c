"""Analytic lights (rs_set_analytic_lights; PathTracer.slang:567-599, LightHelpers.slang) through
the CUDA pass against the oracle: every light type, with and without the emissive triangles and
the environment map beside them (the light-type selection of :606-656 over one, two or three
types), in every temporal mode with spatial reuse; plus the records they make: a light sampled at
the primary hit leaves the record without a light vertex, a delta light stores zero radiance."""
import numpy as np
import pytest

import parity as P

pytestmark = pytest.mark.gpu


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def _down(tx, ty, tz, s):
    """Object-to-world matrix of an area light at (tx, ty, tz) facing -y (object +z onto -y)."""
    T = np.eye(4)
    T[:3, :3] = [[1, 0, 0], [0, 0, -1], [0, 1, 0]]  # rotation by 90 degrees about x
    T[:3, 3] = (tx, ty, tz)
    return {"transform": T, "scaling": (s, s, 1.0)}


LIGHTS = {
    "spot": {"type": "point", "position": (0.5, 0.9, 0.5), "direction": (0.0, -1.0, 0.1), "intensity": (1.5, 1.2, 1.0),
             "openingAngle": 0.7, "penumbraAngle": 0.25},
    "point": {"type": "point", "position": (0.2, 0.55, 0.8), "intensity": (0.3, 0.3, 0.35)},
    "directional": {"type": "directional", "direction": (0.3, -1.0, -0.6), "intensity": (0.6, 0.6, 0.5)},
    "distant": {"type": "distant", "direction": (-0.2, -0.6, -1.0), "intensity": (0.8, 0.7, 0.6), "angle": 0.12},
    "rect": dict({"type": "rect", "intensity": (6.0, 5.0, 4.0)}, **_down(0.3, 0.96, 0.3, 0.08)),
    "disc": dict({"type": "disc", "intensity": (5.0, 6.0, 7.0)}, **_down(0.7, 0.96, 0.7, 0.07)),
    "sphere": {"type": "sphere", "intensity": (4.0, 3.0, 3.0), "transform": np.array([[1, 0, 0, 0.8], [0, 1, 0, 0.3], [0, 0, 1, 0.2], [0, 0, 0, 1.0]]),
               "scaling": (0.05, 0.05, 0.05)},
}
ALL = list(LIGHTS.values())

MODES = [
    ("ScatterBackup-Clamped", {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped"}),
    ("ScatterBackup-Fast-Pairwise", {"temporalReuse": "ScatterBackup", "gatherOption": "Fast", "scatterBackupMISOption": "Pairwise"}),
    ("ScatterOnly", {"temporalReuse": "ScatterOnly"}),
    ("GatherOnly-Robust", {"temporalReuse": "GatherOnly", "gatherOption": "Robust"}),
    ("MultiScatter", {"temporalReuse": "MultiScatter", "numTimePartitions": 3}),
]


def _mostly_finite(img, frac=0.05):
    """The reference's reuse of analytic-light samples makes a few non-finite values (checked
    against the oracle above, which reproduces them value for value): a delta light sampled at the
    second vertex stores lightPdf = 0, and the length-3 reconnection forms misWeight (0) x thp x
    totalBsdf / lightPdf (inf) x irradiance (0) (ShiftMapping.slang:479-493); a light sampled at
    the primary hit leaves no light vertex, whose zero normal gives a 0 / 0 Jacobian."""
    bad = ~np.isfinite(img).all(-1)
    return bad.mean() <= frac


def _lit(scenes, emissive=True):
    sc = scenes.cornell_box(0)
    if not emissive:
        mats = sc.materials.copy()
        mats[:, 4:7] = 0.0
        sc = scenes.Scene(sc.positions, sc.material_ids, mats, "cornell_analytic")
    return sc


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("name,props", MODES, ids=[m[0] for m in MODES])
def test_all_light_types_in_every_mode(rs, oracle_mod, scenes, name, props):
    props = dict(props, maxSurfaceBounces=2, enableSpatialResampling=True)
    shutter = 0.04 if props["temporalReuse"] == "MultiScatter" else 0.0
    report, img = P.run_pair(rs, oracle_mod, _lit(scenes), scenes.cornell_camera, props, frames=4, width=48, height=40,
                             shutter=shutter, setup=lambda p: p.set_analytic_lights(ALL))
    assert _mostly_finite(img) and np.nanmean(img[..., :3]) > 0.02


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("kind", list(LIGHTS), ids=list(LIGHTS))
@pytest.mark.parametrize("emissive", [False, True], ids=["analytic_only", "with_emissive"])
def test_each_light_type(rs, oracle_mod, scenes, kind, emissive):
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 2, "enableSpatialResampling": True}
    report, img = P.run_pair(rs, oracle_mod, _lit(scenes, emissive), scenes.cornell_camera, props, frames=3, width=40, height=32,
                             setup=lambda p: p.set_analytic_lights([LIGHTS[kind]]))
    assert _mostly_finite(img) and np.nanmax(img[..., :3]) > 0.0


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("name,props", [MODES[0], ("GatherOnly-Fast", {"temporalReuse": "GatherOnly", "gatherOption": "Fast"})],
                         ids=["ScatterBackup-Clamped", "GatherOnly-Fast"])
def test_depth_of_field_with_analytic_lights(rs, oracle_mod, scenes, name, props):
    """An open aperture: the gather's depth-of-field split between the lens-vertex copy and the
    primary-hit reconnection (k_gather_resample) and the spatial shifts over analytic-light records."""
    props = dict(props, maxSurfaceBounces=2, enableSpatialResampling=True)
    report, img = P.run_pair(rs, oracle_mod, _lit(scenes), scenes.cornell_camera, props, frames=4, width=40, height=32, aperture=0.02,
                             setup=lambda p: p.set_analytic_lights([LIGHTS["spot"], LIGHTS["disc"], LIGHTS["directional"]]))
    assert _mostly_finite(img)


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_three_light_types_with_env_map(rs, oracle_mod, scenes):
    """Environment map, emissive triangles and analytic lights: selection probability 1/3 each."""
    sky = scenes.sky_env_map(128, 64, seed=2)

    def setup(p):
        p.set_env_map(sky, 1.0)
        p.set_analytic_lights([LIGHTS["spot"], LIGHTS["rect"], LIGHTS["distant"]])
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 2, "enableSpatialResampling": True}
    report, img = P.run_pair(rs, oracle_mod, _lit(scenes), scenes.cornell_camera, props, frames=4, width=48, height=32, setup=setup)
    assert _mostly_finite(img)


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_analytic_records_follow_the_reference(rs, scenes):
    """Candidates lit by a point light at the primary hit: length-2 NEE records with no light vertex
    (second hit of type none), not distant, and zero stored radiance (Le = Li * pdf, pdf 0)."""
    W, H = 48, 40
    p = rs.ReservoirSplatting({"temporalReuse": "ScatterBackup", "maxSurfaceBounces": 1}, W, H)
    p.set_scene(_lit(scenes, emissive=False))
    p.set_analytic_lights([LIGHTS["point"]])
    p.keep_candidates(True)
    p.render(scenes.cornell_camera(0, W, H))
    rec = p.get_buffer("candidate_reconnection").reshape(-1, 28)  # word 4k + j = plane k, word j
    res = p.get_buffer("candidate_reservoirs").reshape(-1, 8)
    flags = rec[:, 5]
    path_len, nee, distant = flags & 0xff, (flags >> 13) & 1, (flags >> 14) & 1
    lit = (res[:, 3] > 0) & (path_len == 2)
    assert lit.sum() > W * H // 4
    assert np.all(nee[lit] == 1) and np.all(distant[lit] == 0)
    assert np.all(rec[lit, 12] == 0) and np.all(rec[lit, 13] == 0)  # second hit: type none, primitive 0
    irr = rec[lit][:, 24:27].view(np.float32)
    assert np.all(irr == 0.0)
    p.set_analytic_lights([])
    p.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_analytic_light_validation(rs, scenes):
    p = rs.ReservoirSplatting({}, 16, 16)
    with pytest.raises(rs.RsError):
        p.set_analytic_lights([{"type": "directional", "direction": (0.0, 0.0, 0.0)}])
    with pytest.raises(rs.RsError):
        p.set_analytic_lights([{"type": "rect", "scaling": (0.0, 1.0, 1.0)}])
    p.set_analytic_lights([])
    p.close()
