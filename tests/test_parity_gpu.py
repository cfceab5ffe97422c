"""CUDA pass vs CPU oracle, frame by frame, through the C ABI (include/rs_b200.h).

Every temporal mode of the reference pass (TemporalReuse x GatherMechanism x
ScatterBackupMIS, ShiftOptions.slang:34-67), spatial reuse on and off, on the
seeded Cornell box (36 triangles) and a small terrain-and-spheres scene.
"""
import numpy as np
import pytest

import parity as P

pytestmark = pytest.mark.gpu

W = H = 64
FRAMES = 5
run_pair = P.run_pair


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


MODES = [
    ("ScatterOnly", {"temporalReuse": "ScatterOnly"}),
    ("ScatterBackup-Clamped-Balance", {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped"}),
    ("ScatterBackup-Fast-Pairwise", {"temporalReuse": "ScatterBackup", "gatherOption": "Fast", "scatterBackupMISOption": "Pairwise"}),
    ("ScatterBackup-Robust-Balance", {"temporalReuse": "ScatterBackup", "gatherOption": "Robust"}),
    ("GatherOnly-Fast", {"temporalReuse": "GatherOnly", "gatherOption": "Fast"}),
    ("GatherOnly-Clamped", {"temporalReuse": "GatherOnly", "gatherOption": "Clamped"}),
    ("GatherOnly-Robust", {"temporalReuse": "GatherOnly", "gatherOption": "Robust"}),
]


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("name,props", MODES, ids=[m[0] for m in MODES])
@pytest.mark.parametrize("spatial", [False, True], ids=["nospatial", "spatial"])
def test_cornell_modes(rs, oracle_mod, scenes, name, props, spatial):
    props = dict(props, maxSurfaceBounces=1, enableSpatialResampling=spatial)
    report, img = run_pair(rs, oracle_mod, scenes.cornell_box(0), scenes.cornell_camera, props)
    assert np.isfinite(img).all()
    assert img[..., :3].mean() > 0.01


ODD_MODES = MODES + [("MultiScatter", {"temporalReuse": "MultiScatter", "numTimePartitions": 3})]


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("name,props", ODD_MODES, ids=[m[0] for m in ODD_MODES])
@pytest.mark.parametrize("size", [(37, 23), (1, 1), (4096, 3), (3, 4096)], ids=["37x23", "1x1", "4096x3", "3x4096"])
def test_odd_image_sizes(rs, oracle_mod, scenes, name, props, size):
    """Images that are not a multiple of the 8 x 4 warp tile, a single pixel, and the largest width
    and height the pass accepts (4096): the tile-edge guards of every pixel kernel, the bounds of
    the per-splat kernels and the cell indices at the extremes, in every temporal mode."""
    w, h = size
    props = dict(props, maxSurfaceBounces=2, enableSpatialResampling=True)
    shutter = 0.04 if name == "MultiScatter" else 0.0
    report, img = run_pair(rs, oracle_mod, scenes.cornell_box(0), scenes.cornell_camera, props, frames=4, width=w, height=h,
                           shutter=shutter)
    assert img.shape == (h, w, 4) and np.isfinite(img).all()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_multiscatter_motion_blur(rs, oracle_mod, scenes):
    props = {"temporalReuse": "MultiScatter", "numTimePartitions": 4, "maxSurfaceBounces": 1, "enableSpatialResampling": False,
             "artificialFrameTime": 1.0 / 48.0}
    run_pair(rs, oracle_mod, scenes.cornell_box(0), scenes.cornell_camera, props, shutter=1.0 / 24.0)


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_depth_of_field_gather_and_spatial(rs, oracle_mod, scenes):
    props = {"temporalReuse": "GatherOnly", "gatherOption": "Fast", "maxSurfaceBounces": 1, "enableSpatialResampling": True,
             "neighborCount": 3}
    run_pair(rs, oracle_mod, scenes.cornell_box(0), scenes.cornell_camera, props, aperture=0.02)


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_pcg32_and_longer_paths(rs, oracle_mod, scenes):
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 3, "sampleGenerator": "PCG32"}
    run_pair(rs, oracle_mod, scenes.cornell_box(3), scenes.cornell_camera, props)


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("builder", ["PLOC", "LBVH"])
def test_terrain_scene_scatter_backup(rs, oracle_mod, scenes, builder):
    sc = scenes.terrain_spheres(seed=7, grid=48, spheres=12, subdiv=2, lights=8, extent=40.0, height=4.0)
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 2}
    cam = lambda f, w, h: scenes.orbit_camera(f, w, h, radius=30.0, height_above=12.0)
    run_pair(rs, oracle_mod, sc, cam, props, frames=4, width=96, height=64, builder=builder)


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("mode", ["ScatterBackup", "GatherOnly", "MultiScatter"])
def test_uniform_emissive_sampler(rs, oracle_mod, scenes, mode):
    """emissiveSampler = Uniform (EmissiveUniformSampler): NEE picks each emissive triangle with
    probability 1 / count and the BSDF-hit MIS uses the same selection pdf, on the GPU as in the oracle."""
    sc = scenes.terrain_spheres(seed=7, grid=48, spheres=12, subdiv=2, lights=8, extent=40.0, height=4.0)
    props = {"temporalReuse": mode, "gatherOption": "Clamped", "maxSurfaceBounces": 2, "emissiveSampler": "Uniform",
             "enableSpatialResampling": True}
    cam = lambda f, w, h: scenes.orbit_camera(f, w, h, radius=30.0, height_above=12.0)
    report, img = run_pair(rs, oracle_mod, sc, cam, props, frames=4, width=80, height=48,
                           shutter=0.04 if mode == "MultiScatter" else 0.0)
    assert np.isfinite(img).all() and img[..., :3].mean() > 0.0


OPTION_CASES = [
    ("numSpatialIterations=3", {"numSpatialIterations": 3}),
    ("spatialGatherRadius=5", {"spatialGatherRadius": 5.0, "neighborCount": 3}),
    ("noConfidenceTemporal", {"useConfidenceWeightsTemporally": False}),
    ("noConfidenceSpatial", {"useConfidenceWeightsSpatially": False, "neighborCount": 2}),
    ("noRussianRoulette", {"useRussianRoulette": False}),
    ("disableCaustics", {"disableCaustics": True, "maxSurfaceBounces": 3}),
    ("specularRoughnessThreshold=0.6", {"specularRoughnessThreshold": 0.6, "maxSpecularBounces": 1}),
    ("maxDiffuseBounces=1", {"maxSurfaceBounces": 3, "maxDiffuseBounces": 1}),
    ("maxSpecularBounces=0", {"maxSurfaceBounces": 3, "maxSpecularBounces": 0}),
]


def _glossy_cornell(scenes):
    """The Cornell box with a mirror-like tall box (metallic, roughness 0.05) and a glossy short box
    (roughness 0.3): specular vertices for the caustics and roughness-threshold options."""
    sc = scenes.cornell_box(0)
    mats = np.concatenate([sc.materials, scenes.material((0.9, 0.8, 0.6), roughness=0.05, metallic=1.0)[None],
                           scenes.material((0.5, 0.6, 0.7), roughness=0.3)[None]]).astype(np.float32)
    mids = sc.material_ids.copy()
    mids[22:34] = len(mats) - 2  # the tall box (triangles 22-33: the second box)
    mids[10:22] = len(mats) - 1  # the short box
    return scenes.Scene(sc.positions, mids, mats, "cornell_glossy")


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("mode", ["ScatterBackup", "GatherOnly"])
@pytest.mark.parametrize("name,extra", OPTION_CASES, ids=[c[0] for c in OPTION_CASES])
def test_option_values(rs, oracle_mod, scenes, mode, name, extra):
    """Each option of ReservoirSplatting.h:124-184 at a non-default value, on a scene with specular
    surfaces, against the oracle."""
    base = {"temporalReuse": mode, "gatherOption": "Clamped", "maxSurfaceBounces": 2, "enableSpatialResampling": True}
    props = dict(base, **extra)
    sc = _glossy_cornell(scenes)
    report, img = run_pair(rs, oracle_mod, sc, scenes.cornell_camera, props, frames=4, width=40, height=32)
    assert np.isfinite(img).all() and img[..., :3].mean() > 0.0
    # the option takes effect: without it (the companion settings kept) the frames differ
    companion = {k: v for k, v in extra.items() if k in ("maxSurfaceBounces", "neighborCount")}
    other = rs.ReservoirSplatting(dict(base, **companion), 40, 32)
    other.set_scene(sc)
    for f in range(4):
        ref = other.render(scenes.cornell_camera(f, 40, 32))
    other.close()
    assert not np.array_equal(ref, img), f"{name} changed nothing" 


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("spp", [2, 5, 16])
@pytest.mark.parametrize("lights", ["emissive", "env+analytic", "uniform"])
def test_several_samples_per_pixel(rs, oracle_mod, scenes, spp, lights):
    """samplesPerPixel > 1 (InitialCandidates.cs.slang:80-141: the pixel's paths stream into one
    candidate reservoir; k_candidates, one thread per pixel) up to the maximum of 16, with each light
    configuration the path tracer is compiled for."""
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 2, "enableSpatialResampling": True,
             "samplesPerPixel": spp}
    if lights == "uniform":
        props["emissiveSampler"] = "Uniform"
    sky = scenes.sky_env_map(64, 32, seed=5)
    spot = {"type": "point", "position": (0.5, 0.9, 0.5), "direction": (0.0, -1.0, 0.0), "intensity": (1.0, 1.0, 1.0),
            "openingAngle": 0.7, "penumbraAngle": 0.2}

    def setup(p):
        if lights == "env+analytic":
            p.set_env_map(sky, 0.8)
            p.set_analytic_lights([spot])
    report, img = run_pair(rs, oracle_mod, scenes.cornell_box(0), scenes.cornell_camera, props, frames=3, width=32, height=24, setup=setup)
    assert np.nanmax(img[..., :3]) > 0.0


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_imported_pyscene(rs, oracle_mod, scenes, tmp_path):
    """A Falcor .pyscene (generated meshes, a node hierarchy, an emissive quad, a spot and a distant
    light) imported and rendered with its analytic lights, on the GPU as in the oracle."""
    import dataclasses
    import reservoir_splatting_b200.importers as I
    from test_importers_cpu import PYSCENE
    path = tmp_path / "room.pyscene"
    path.write_text(PYSCENE)
    sc = I.load_pyscene(path)

    def cam(f, w, h):
        c = I.pyscene_camera(sc, w, h)
        return dataclasses.replace(c, position=(c.position[0] + 0.01 * f, c.position[1], c.position[2]))
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 2, "enableSpatialResampling": True}
    report, img = run_pair(rs, oracle_mod, sc, cam, props, frames=4, width=48, height=36,
                           setup=lambda p: p.set_analytic_lights(sc.info["lights"]))
    assert np.nanmax(img[..., :3]) > 0.0


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_imported_pyscene_with_hdr_environment(rs, oracle_mod, scenes, tmp_path):
    """The pyscene's EnvMap read from a Radiance .hdr image, with its intensity, tint and rotation
    given to rs_set_env_map, on the GPU as in the oracle."""
    import dataclasses
    import reservoir_splatting_b200.importers as I
    from test_importers_cpu import PYSCENE, _write_hdr
    _write_hdr(tmp_path / "sky.hdr", scenes.sky_env_map(64, 32, seed=3), True)
    path = tmp_path / "room.pyscene"
    path.write_text(PYSCENE + "e = EnvMap('sky.hdr')\ne.intensity = 0.7\ne.rotation = float3(0, 40, 0)\ne.tint = float3(1, 0.9, 0.8)\n"
                    "sceneBuilder.envMap = e\n")
    sc = I.load_pyscene(path)
    env, ep = sc.info["env"], sc.info["env_params"]

    def setup(p):
        p.set_env_map(env, ep["intensity"], ep["tint"], ep["rotation"])
        p.set_analytic_lights(sc.info["lights"])

    def cam(f, w, h):
        c = I.pyscene_camera(sc, w, h)
        return dataclasses.replace(c, position=(c.position[0] + 0.01 * f, c.position[1], c.position[2]))
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 2, "enableSpatialResampling": True}
    report, img = run_pair(rs, oracle_mod, sc, cam, props, frames=3, width=40, height=30, setup=setup)
    assert np.nanmax(img[..., :3]) > 0.0


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("mode", ["ScatterBackup", "GatherOnly"])
def test_imported_obj_spec_gloss_scene(rs, oracle_mod, scenes, tmp_path, mode):
    """A Cornell box written as OBJ + MTL and imported with the Assimp importer's OBJ mapping:
    spec-gloss materials (diffuse, specular colour, glossiness from the Phong exponent, derived
    metallic), shaded the same on the GPU and in the oracle.  The adjoint differentiates its diffuse
    colours and glossiness like the oracle's replay."""
    import torch
    import reservoir_splatting_b200.importers as I
    sc = scenes.cornell_box(0)
    I.save_obj(sc, tmp_path / "cb.obj", ["white", "red", "green", "light"],
               {"white": {"Kd": (0.7, 0.7, 0.7), "Ks": (0.05, 0.05, 0.05), "Ns": 30.0},
                "red": {"Kd": (0.6, 0.05, 0.05), "Ks": (0.3, 0.3, 0.3), "Ns": 400.0},
                "green": {"Kd": (0.1, 0.4, 0.1), "Ks": (0.02, 0.02, 0.02), "Ns": 5.0},
                "light": {"Kd": (0, 0, 0), "Ke": (17, 12, 4)}})
    imported = I.load_obj(tmp_path / "cb.obj")
    props = {"temporalReuse": mode, "gatherOption": "Clamped", "maxSurfaceBounces": 2, "enableSpatialResampling": True}
    run_pair(rs, oracle_mod, imported, scenes.cornell_camera, props, frames=4)
    p = rs.ReservoirSplatting(props, W, H)
    p.set_scene(imported)
    ora = oracle_mod.OraclePass(props, W, H)
    ora.set_scene(imported)
    img = p.render(scenes.cornell_camera(0, W, H))
    np.testing.assert_array_equal(img, ora.execute(scenes.cornell_camera(0, W, H)))
    gc = np.random.default_rng(5).uniform(-1.0, 1.0, img.shape).astype(np.float32)
    gm = torch.zeros((len(imported.materials), 8), device="cuda")
    p.backward(torch.from_numpy(gc).cuda().data_ptr(), gm.data_ptr())
    torch.cuda.synchronize()
    O, ost = ora.backward(gc, len(imported.materials))
    st = p.backward_stats()
    assert st[0] > 0 and st[0] == ost[0] and st[1] == 0 and st[2] == 0
    assert np.abs(gm.cpu().numpy() - O).max() <= 1e-4 * np.abs(O).max()
    p.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("props", [{"temporalReuse": "ScatterBackup", "gatherOption": "Clamped"},
                                   {"temporalReuse": "GatherOnly", "gatherOption": "Robust"}],
                         ids=["ScatterBackup", "GatherOnly-Robust"])
def test_bit_exact_against_oracle(rs, oracle_mod, scenes, props):
    """Host and device evaluate the same float expressions without contraction, so the CUDA pass
    reproduces the oracle bit for bit (the 1e-4 tolerance elsewhere is the contract, not the need)."""
    props = dict(props, maxSurfaceBounces=2, enableSpatialResampling=True)
    gpu = rs.ReservoirSplatting(props, 48, 40)
    ora = oracle_mod.OraclePass(props, 48, 40)
    sc = scenes.cornell_box(1)
    gpu.set_scene(sc)
    ora.set_scene(sc)
    for f in range(4):
        cam = scenes.cornell_camera(f, 48, 40)
        a, b = gpu.render(cam), ora.execute(cam)
        assert P.bit_mismatch_fraction(a, b) == 0.0, f"frame {f}"
        np.testing.assert_array_equal(gpu.get_buffer("curr_reservoirs").view(np.uint32), ora.get_buffer("curr_reservoirs").view(np.uint32))
        np.testing.assert_array_equal(gpu.get_buffer("curr_reconnection"), ora.get_buffer("curr_reconnection"))
    gpu.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("name", ["cornell_scatteronly", "cornell_scatterbackup"])
def test_gpu_matches_committed_golden(rs, scenes, name):
    import sys
    from pathlib import Path
    golden = Path(__file__).resolve().parent / "golden"
    sys.path.insert(0, str(golden))
    import make_golden
    ref = np.load(golden / f"{name}.npz")
    size = make_golden.GOLDEN_SIZE
    gpu = rs.ReservoirSplatting(make_golden.GOLDEN_RUNS[name], size, size)
    gpu.set_scene(scenes.cornell_box(0))
    for f in range(make_golden.GOLDEN_FRAMES):
        img = gpu.render(scenes.cornell_camera(f, size, size))
    P.assert_close("color", img, ref["color"])
    P.compare_reservoirs("reservoirs", gpu.get_buffer("curr_reservoirs"), ref["reservoirs"])
    P.compare_recon("reconnection", gpu.get_buffer("curr_reconnection"), ref["reconnection"])
    gpu.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("mode,builder", [("ScatterBackup", "PLOC"), ("MultiScatter", "PLOC"), ("ScatterBackup", "LBVH")])
def test_moving_spheres(rs, oracle_mod, scenes, mode, builder):
    """Spheres moving linearly each frame (rs_update_geometry: refitted trees, previous-frame motion
    vectors) against the oracle, which rebuilds its own tree every frame."""
    sc = scenes.terrain_spheres(seed=5, grid=40, spheres=10, subdiv=2, lights=6, extent=30.0, height=3.0)
    motion = scenes.SphereMotion(sc, moving=6, max_speed=0.3, seed=2)
    props = {"temporalReuse": mode, "gatherOption": "Clamped", "maxSurfaceBounces": 2, "numTimePartitions": 4,
             "artificialFrameTime": 1.0 / 48.0, "enableSpatialResampling": True}
    W, H = 80, 56
    gpu = rs.ReservoirSplatting(props, W, H)
    gpu.set_bvh_builder(builder)
    ora = oracle_mod.OraclePass(props, W, H)
    gpu.set_scene(sc)
    ora.set_scene(sc)
    for f in range(5):
        cam = scenes.orbit_camera(f, W, H, radius=24.0, height_above=9.0)
        cam.shutter_speed = 1.0 / 24.0 if mode == "MultiScatter" else 0.0
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
        P.assert_close(f"frame{f}.color", img_g, img_o)
    gpu.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("mode", ["ScatterOnly", "ScatterBackup"])
def test_zoom_out_crowded_cells(rs, oracle_mod, scenes, mode):
    """A zoom-out by 32x between frames (the focal length drops from 32x to 1x the base): the
    previous frame's pixels splat into a small patch, hundreds of splats per cell.  The cell lists
    (a stable radix sort by cell, bounded work per splat) and the resampling over them match the
    oracle bit for bit."""
    base = scenes.cornell_camera(0, 64, 64).focal_length

    def cam(f, w, h):
        c = scenes.cornell_camera(0, w, h)
        c.focal_length = base * (32.0 if f % 2 == 0 else 1.0)
        return c

    props = {"temporalReuse": mode, "gatherOption": "Clamped", "maxSurfaceBounces": 1, "enableSpatialResampling": False}
    gpu = rs.ReservoirSplatting(props, 64, 64)
    gpu.keep_candidates(True)
    ora = oracle_mod.OraclePass(props, 64, 64)
    sc = scenes.cornell_box(0)
    gpu.set_scene(sc)
    ora.set_scene(sc)
    most = 0
    for f in range(4):
        c = cam(f, 64, 64)
        a, b = gpu.render(c), ora.execute(c)
        if f > 0:
            counts = gpu.get_buffer("cell_counters")
            P.assert_equal(f"frame{f}.cell_counters", counts, ora.get_buffer("cell_counters"))
            P.assert_equal(f"frame{f}.sorted_splats", gpu.get_buffer("sorted_splats"), ora.get_buffer("sorted_splats"))
            most = max(most, int(counts.max()))
        P.compare_reservoirs(f"frame{f}.reservoirs", gpu.get_buffer("curr_reservoirs"), ora.get_buffer("curr_reservoirs"))
        assert P.bit_mismatch_fraction(a, b) == 0.0, f"frame {f}"
    assert most >= 256, most
    gpu.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("mode", ["ScatterBackup", "GatherOnly"])
def test_power_exp_mis(rs, oracle_mod, scenes, mode):
    """misHeuristic PowerExp (PathTracer.slang:498-503) with a non-integer exponent: the NEE / BSDF
    MIS weights of the candidates and of every shift that re-evaluates them, GPU against the oracle."""
    props = {"temporalReuse": mode, "gatherOption": "Clamped", "maxSurfaceBounces": 2, "misHeuristic": "PowerExp",
             "misPowerExponent": 1.5, "enableSpatialResampling": True}
    report, img = run_pair(rs, oracle_mod, scenes.cornell_box(0), scenes.cornell_camera, props, frames=4, width=48, height=40)
    assert all(report[f"bits{f}"] == 0.0 for f in range(4)), report
