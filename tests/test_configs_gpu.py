"""CUDA pass vs CPU oracle on the benchmark configurations at their stated settings.

* Cornell box, 256 x 256, 16 frames, ScatterOnly, Balance MIS, PCG32, maximum path length 3, a
  pinhole camera translating 0.01 units per frame along +x (the small plain-method configuration,
  exactly as specified; spatial reuse off and on).
* The headline scene itself (seeded 512 x 512 fBm terrain + 500 icospheres at subdivision 4 + 64
  emissive triangles, 3.08M triangles) at 480 x 270 for 4 frames: ScatterBackup, Clamped gather,
  Balance MIS, path length 4, spatial reuse on, the benchmark's orbiting camera.
* The motion-blur configuration at 240 x 135: the 3.84M-triangle scene with 200 spheres moving at
  U[0, 0.05] units per frame, MultiSplatting with 4 shutter partitions, shutter 1/24 s, artificial
  frame time 1/48 s, aperture radius 0.02.

Splat targets, cell lists, hits, path lengths and flags are compared bit for bit; float fields
and colour within 1e-4 relative (parity.REL_TOL); the colour is also required to be bit-exact,
which is what the shared float expressions deliver.
"""
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


@pytest.fixture(scope="module")
def oracle_threads(oracle_mod):
    import os
    oracle_mod.set_threads(os.cpu_count() or 1)
    return oracle_mod


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("spatial", [False, True], ids=["nospatial", "spatial"])
def test_cornell_256_scatter_only_pcg32_16_frames(rs, oracle_threads, scenes, spatial):
    props = {"temporalReuse": "ScatterOnly", "misHeuristic": "Balance", "sampleGenerator": "PCG32", "maxSurfaceBounces": 1,
             "enableSpatialResampling": spatial}
    report, img = P.run_pair(rs, oracle_threads, scenes.cornell_box(0), scenes.cornell_camera, props, frames=16, width=256, height=256)
    assert all(report[f"bits{f}"] == 0.0 for f in range(16)), report
    assert report["splats"] > 0.5 * 256 * 256
    assert img[..., :3].mean() > 0.01


@pytest.fixture(scope="module")
def headline_scene(scenes):
    return scenes.terrain_spheres(seed=1, grid=512, spheres=500, subdiv=4, lights=64)


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_headline_scene_480x270(rs, oracle_threads, scenes, headline_scene):
    assert headline_scene.num_triangles == 3_082_306
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "scatterBackupMISOption": "Balance",
             "maxSurfaceBounces": 2, "enableSpatialResampling": True}
    report, img = P.run_pair(rs, oracle_threads, headline_scene, scenes.orbit_camera, props, frames=4, width=480, height=270)
    assert all(report[f"bits{f}"] == 0.0 for f in range(4)), report
    assert np.isfinite(img).all() and img[..., :3].mean() > 0.0


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_motion_blur_config_240x135(rs, oracle_threads, scenes):
    sc = scenes.motion_blur_scene()
    motion = scenes.SphereMotion(sc, moving=200, max_speed=0.05, seed=4)
    props = {"temporalReuse": "MultiScatter", "numTimePartitions": 4, "artificialFrameTime": 1.0 / 48.0,
             "maxSurfaceBounces": 2, "enableSpatialResampling": True}
    W, H = 240, 135
    gpu = rs.ReservoirSplatting(props, W, H)
    ora = oracle_threads.OraclePass(props, W, H)
    gpu.set_scene(sc)
    ora.set_scene(sc)
    for f in range(4):
        cam = scenes.orbit_camera(f, W, H)
        cam.shutter_speed = 1.0 / 24.0
        cam.aperture_radius = 0.02
        if f > 0:
            pos = motion.positions(f)
            gpu.update_geometry(pos)
            ora.update_geometry(pos)
        img_g = gpu.render(cam)
        img_o = ora.execute(cam)
        P.assert_equal(f"frame{f}.vbuffer", gpu.get_buffer("vbuffer"), ora.get_buffer("vbuffer"))
        P.assert_equal(f"frame{f}.mvec", gpu.get_buffer("mvec").view(np.uint32), ora.get_buffer("mvec").view(np.uint32))
        P.compare_reservoirs(f"frame{f}.reservoirs", gpu.get_buffer("curr_reservoirs"), ora.get_buffer("curr_reservoirs"))
        P.compare_recon(f"frame{f}.reconnection", gpu.get_buffer("curr_reconnection"), ora.get_buffer("curr_reconnection"))
        P.assert_close(f"frame{f}.color", img_g, img_o)
        assert P.bit_mismatch_fraction(img_g, img_o) == 0.0, f"frame {f}"
    gpu.close()
