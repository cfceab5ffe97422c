"""Environment-map lighting, CUDA pass vs CPU oracle through the C ABI.

The env light of the reference (Falcor EnvMap + EnvMapSampler, PathTracer.slang:516-534 light
sample, :1433-1569 handleMiss / handlePrimaryMiss, :1412-1416 handleReconnectionEnvMap, the
distant-light branches of ShiftMapping.slang:90-421 and ReprojectTemporalSamples.rt.slang:110-118):
the importance map and every temporal mode with the Cornell box open to a sky, with and without
emissive triangles, pinhole and thin lens, spatial reuse on.
"""
import numpy as np
import pytest

import parity as P
from test_parity_gpu import run_pair

pytestmark = pytest.mark.gpu


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def _with_env(rs, oracle_mod, scenes, env_kw):
    """set_scene replacements for both passes that also set the same env map."""
    orig_gpu, orig_ora = rs.ReservoirSplatting.set_scene, oracle_mod.OraclePass.set_scene
    env = scenes.sky_env_map(128, 64, seed=2)

    def gpu_set_scene(self, scene):
        orig_gpu(self, scene)
        self.set_env_map(env, **env_kw)

    def ora_set_scene(self, scene):
        orig_ora(self, scene)
        self.set_env_map(env, **env_kw)
    return gpu_set_scene, ora_set_scene


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_env_importance_map_matches_oracle(rs, oracle_mod, scenes):
    env = scenes.sky_env_map(200, 100, seed=4)
    gpu = rs.ReservoirSplatting({}, 16, 16)
    ora = oracle_mod.OraclePass({}, 16, 16)
    gpu.set_env_map(env, intensity=2.0, rotation=(10.0, 30.0, 0.0))
    ora.set_env_map(env, intensity=2.0, rotation=(10.0, 30.0, 0.0))
    g = gpu.get_buffer("env_importance")
    o = ora.env_importance()
    gpu.close()
    P.assert_equal("env_importance", g.view(np.uint32), o.view(np.uint32))
    assert g[-1] > 0


MODES = [
    ("ScatterBackup-Clamped", {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped"}, 0.0),
    ("ScatterBackup-Robust-Pairwise", {"temporalReuse": "ScatterBackup", "gatherOption": "Robust", "scatterBackupMISOption": "Pairwise"}, 0.0),
    ("ScatterOnly", {"temporalReuse": "ScatterOnly"}, 0.0),
    ("GatherOnly-Fast", {"temporalReuse": "GatherOnly", "gatherOption": "Fast"}, 0.0),
    ("GatherOnly-Robust", {"temporalReuse": "GatherOnly", "gatherOption": "Robust"}, 0.0),
    ("GatherOnly-Clamped-DoF", {"temporalReuse": "GatherOnly", "gatherOption": "Clamped"}, 0.05),
    ("ScatterBackup-DoF", {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped"}, 0.05),
    ("MultiScatter", {"temporalReuse": "MultiScatter", "numTimePartitions": 3}, 0.0),
]


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("name,props,aperture", MODES, ids=[m[0] for m in MODES])
@pytest.mark.parametrize("emissive", [True, False], ids=["sky+emissive", "sky-only"])
def test_env_modes(rs, oracle_mod, scenes, monkeypatch, name, props, aperture, emissive):
    gs, os_ = _with_env(rs, oracle_mod, scenes, {"intensity": 1.5, "tint": (1.0, 0.95, 0.9), "rotation": (0.0, 35.0, 0.0)})
    monkeypatch.setattr(rs.ReservoirSplatting, "set_scene", gs)
    monkeypatch.setattr(oracle_mod.OraclePass, "set_scene", os_)
    sc = scenes.cornell_box(0)
    if not emissive:
        mats = sc.materials.copy()
        mats[:, 4:7] = 0.0
        sc = scenes.Scene(sc.positions, sc.material_ids, mats, "cornell_sky")
    shutter = 0.04 if props["temporalReuse"] == "MultiScatter" else 0.0
    props = dict(props, maxSurfaceBounces=2, enableSpatialResampling=True)
    report, img = run_pair(rs, oracle_mod, sc, scenes.cornell_camera, props, frames=4, width=48, height=32,
                           shutter=shutter, aperture=aperture)
    assert np.isfinite(img).all()
    assert img[..., :3].mean() > 0.05


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_env_records_are_made(rs, scenes):
    """Sky pixels select primary-miss records (length 1, distant) and lit surfaces select
    environment NEE records, so the distant-light shift branches above are exercised."""
    sc = scenes.cornell_box(0)
    p = rs.ReservoirSplatting({"temporalReuse": "ScatterBackup", "maxSurfaceBounces": 2}, 48, 32)
    p.set_scene(sc)
    p.set_env_map(scenes.sky_env_map(128, 64, seed=2))
    p.keep_candidates(True)
    for f in range(2):
        p.render(scenes.cornell_camera(f, 48, 32))
    rec = p.get_buffer("candidate_reconnection").reshape(-1, 28)
    flags = rec[:, 5]
    distant = ((flags >> 14) & 1) == 1
    length = flags & 0xff
    p.close()
    assert (distant & (length == 1)).sum() > 0
    assert (distant & (length >= 2)).sum() > 0


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_zero_intensity_env_is_no_env(rs, scenes):
    sc = scenes.cornell_box(0)
    imgs = []
    for env in (False, True):
        p = rs.ReservoirSplatting({"temporalReuse": "ScatterBackup", "maxSurfaceBounces": 2}, 32, 24)
        p.set_scene(sc)
        if env:
            p.set_env_map(scenes.sky_env_map(64, 32), intensity=0.0)
        for f in range(3):
            img = p.render(scenes.cornell_camera(f, 32, 24))
        imgs.append(img)
        p.close()
    assert np.array_equal(imgs[0].view(np.uint32), imgs[1].view(np.uint32))


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("mode", ["ScatterBackup", "GatherOnly"])
def test_imported_pbrt_scene(rs, oracle_mod, scenes, monkeypatch, tmp_path, mode):
    """A PBRT v4 file through importers.load_pbrt (area light, conductor, coated diffuse, dielectric,
    instanced PLY, constant infinite light as the env map) rendered by the pass and the oracle."""
    import reservoir_splatting_b200.importers as I
    from test_importers_cpu import _write_pbrt
    sc = I.load_pbrt(_write_pbrt(tmp_path))
    env = sc.info["env"]
    orig_gpu, orig_ora = rs.ReservoirSplatting.set_scene, oracle_mod.OraclePass.set_scene

    def gpu_set_scene(self, scene):
        orig_gpu(self, scene)
        self.set_env_map(env)

    def ora_set_scene(self, scene):
        orig_ora(self, scene)
        self.set_env_map(env)
    monkeypatch.setattr(rs.ReservoirSplatting, "set_scene", gpu_set_scene)
    monkeypatch.setattr(oracle_mod.OraclePass, "set_scene", ora_set_scene)

    def camera_fn(f, w, h):
        c = I.pbrt_camera(sc, w, h)
        c.position = (c.position[0] + 0.02 * f, c.position[1], c.position[2])
        return c
    props = {"temporalReuse": mode, "gatherOption": "Clamped", "maxSurfaceBounces": 2, "enableSpatialResampling": True}
    _, img = run_pair(rs, oracle_mod, sc, camera_fn, props, frames=3, width=48, height=36)
    assert np.isfinite(img).all() and img[..., :3].mean() > 0.01


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_imported_mitsuba_scene(rs, oracle_mod, scenes, monkeypatch, tmp_path):
    """A Mitsuba 3 XML scene through importers.load_mitsuba, its constant emitter as the env map."""
    import reservoir_splatting_b200.importers as I
    from test_importers_cpu import _write_mitsuba
    sc = I.load_mitsuba(_write_mitsuba(tmp_path))
    env = sc.info["env"]
    orig_gpu, orig_ora = rs.ReservoirSplatting.set_scene, oracle_mod.OraclePass.set_scene

    def gpu_set_scene(self, scene):
        orig_gpu(self, scene)
        self.set_env_map(env)

    def ora_set_scene(self, scene):
        orig_ora(self, scene)
        self.set_env_map(env)
    monkeypatch.setattr(rs.ReservoirSplatting, "set_scene", gpu_set_scene)
    monkeypatch.setattr(oracle_mod.OraclePass, "set_scene", ora_set_scene)
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 2, "enableSpatialResampling": True}
    _, img = run_pair(rs, oracle_mod, sc, lambda f, w, h: I.pbrt_camera(sc, w, h), props, frames=3, width=48, height=36)
    assert np.isfinite(img).all() and img[..., :3].mean() > 0.01
