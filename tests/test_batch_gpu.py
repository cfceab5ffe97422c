"""Batched instances (one CUDA graph launch per frame for all members) give the same results as
rendering each pass on its own."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("env_frame", [None, 5], ids=["no-env", "env-from-frame-5"])
def test_batch_matches_individual_passes(rs, scenes, env_frame):
    """With env_frame, the first instance gets a sky environment map at that frame: graphs captured
    before it (the same buffer pattern recurs) must not be replayed with the kernels without it."""
    import torch
    terrain = scenes.terrain_spheres(seed=4, grid=32, spheres=6, subdiv=2, lights=6, extent=30.0, height=3.0)
    cfgs = [
        (scenes.cornell_box(0), scenes.cornell_camera, {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 2}, 48, 32),
        (terrain, lambda f, w, h: scenes.orbit_camera(f, w, h, radius=25.0, height_above=10.0),
         {"temporalReuse": "ScatterOnly", "enableSpatialResampling": False, "maxSurfaceBounces": 1}, 64, 40),
        (scenes.cornell_box(2), scenes.cornell_camera, {"temporalReuse": "GatherOnly", "gatherOption": "Fast", "maxSurfaceBounces": 1}, 32, 32),
    ]
    solo, batched = [], []
    for sc, _, props, w, h in cfgs:
        a = rs.ReservoirSplatting(props, w, h); a.set_scene(sc); solo.append(a)
        b = rs.ReservoirSplatting(props, w, h); b.set_scene(sc); batched.append(b)
    outs = [torch.zeros((h, w, 4), dtype=torch.float32, device="cuda") for _, _, _, w, h in cfgs]
    batch = rs.Batch(batched)
    stream = torch.cuda.current_stream().cuda_stream
    for f in range(5 if env_frame is None else 8):
        if f == env_frame:
            sky = scenes.sky_env_map(64, 32, seed=1)
            solo[0].set_env_map(sky)
            batched[0].set_env_map(sky)
        cams = [cfg[1](f, cfg[3], cfg[4]) for cfg in cfgs]
        ref = [p.render(c) for p, c in zip(solo, cams)]
        batch.execute(cams, [o.data_ptr() for o in outs], stream=stream)
        torch.cuda.synchronize()
        for k in range(len(cfgs)):
            np.testing.assert_array_equal(outs[k].cpu().numpy(), ref[k], err_msg=f"instance {k} frame {f}")
            np.testing.assert_array_equal(batched[k].get_buffer("curr_reservoirs"), solo[k].get_buffer("curr_reservoirs"))
    assert batch.launch_count() > 0
    batch.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_batch_member_changes_options_size_and_aperture(rs, scenes):
    """A member's options and frame size change between two batch calls (rs_set_options
    reallocates its buffers), and another member's camera opens its aperture (the gather switches to
    its depth-of-field kernel): the batch must capture new graphs, not replay the stale ones, and
    still match the passes rendered on their own."""
    import torch
    cfgs = [
        (scenes.cornell_box(0), {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 1}, 40, 32),
        (scenes.cornell_box(1), {"temporalReuse": "GatherOnly", "gatherOption": "Fast", "maxSurfaceBounces": 1}, 32, 24),
    ]
    solo, batched = [], []
    for sc, props, w, h in cfgs:
        a = rs.ReservoirSplatting(props, w, h); a.set_scene(sc); solo.append(a)
        b = rs.ReservoirSplatting(props, w, h); b.set_scene(sc); batched.append(b)
    sizes = [(w, h) for _, _, w, h in cfgs]
    batch = rs.Batch(batched)
    stream = torch.cuda.current_stream().cuda_stream
    new_props = {"temporalReuse": "ScatterOnly", "enableSpatialResampling": False, "maxSurfaceBounces": 2}
    for f in range(8):
        if f == 3:  # member 0: new mode and a new size
            sizes[0] = (24, 40)
            solo[0].set_properties(new_props, *sizes[0])
            batched[0].set_properties(new_props, *sizes[0])
        outs = [torch.zeros((h, w, 4), dtype=torch.float32, device="cuda") for w, h in sizes]
        cams = []
        for k, (w, h) in enumerate(sizes):
            c = scenes.cornell_camera(f, w, h)
            if k == 1 and f >= 5:
                c.aperture_radius = 0.02
            cams.append(c)
        ref = [p.render(c) for p, c in zip(solo, cams)]
        batch.execute(cams, [o.data_ptr() for o in outs], stream=stream)
        torch.cuda.synchronize()
        for k in range(len(cfgs)):
            np.testing.assert_array_equal(outs[k].cpu().numpy(), ref[k], err_msg=f"instance {k} frame {f}")
    batch.close()
    for p in solo + batched:
        p.close()


def _uniform_members(rs, scenes, env=False):
    terrain = scenes.terrain_spheres(seed=4, grid=32, spheres=6, subdiv=2, lights=6, extent=30.0, height=3.0)
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 2, "enableSpatialResampling": True,
             "neighborCount": 2}
    cfgs = [(scenes.cornell_box(0), scenes.cornell_camera, 48, 32), (terrain, lambda f, w, h: scenes.orbit_camera(f, w, h, radius=25.0, height_above=10.0), 64, 40),
            (scenes.cornell_box(2), scenes.cornell_camera, 37, 23), (scenes.cornell_box(1), scenes.cornell_camera, 48, 32)]
    solo, batched = [], []
    sky = scenes.sky_env_map(64, 32, seed=1) if env else None
    for sc, _, w, h in cfgs:
        for lst in (solo, batched):
            p = rs.ReservoirSplatting(props, w, h)
            p.set_scene(sc)
            if env:
                p.set_env_map(sky)
            lst.append(p)
    return cfgs, solo, batched


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("env", [False, True], ids=["emissive", "env"])
def test_flattened_batch_matches_individual_passes(rs, scenes, env):
    """Members in one ScatterBackup/Clamped configuration run the flattened form (one persistent launch
    per stage over a work queue of all members, uneven resolutions) from their second frame on, and
    give bit for bit the images and reservoirs of the passes rendered alone, at every tile width and
    grid form, and after rs_batch_tune."""
    import torch
    cfgs, solo, batched = _uniform_members(rs, scenes, env)
    outs = [torch.zeros((h, w, 4), dtype=torch.float32, device="cuda") for _, _, w, h in cfgs]
    batch = rs.Batch(batched)
    stream = torch.cuda.current_stream().cuda_stream
    settings = [None, (16, 0), (32, 1), (8, 1), "tune", None]
    for f in range(len(settings) + 1):
        cams = [cfg[1](f, cfg[2], cfg[3]) for cfg in cfgs]
        ref = [p.render(c) for p, c in zip(solo, cams)]
        setting = settings[f - 1] if f > 0 else None
        if setting == "tune":
            batch.tune(cams, [o.data_ptr() for o in outs], stream=stream)
            tuning = batch.tuning()
            assert any(e["width"] > 0 for e in tuning) and all(e["tile"] in (0, 8, 16, 32) for e in tuning)
        else:
            if isinstance(setting, tuple):
                tw, grid = setting
                entries = [{"stage": st, "width": w, "height": h, "tile": tw, "grid": 0} for st in rs.abi.BATCH_STAGES for _, _, w, h in cfgs]
                entries += [{"stage": st, "width": 0, "height": 0, "tile": 0, "grid": grid} for st in rs.abi.BATCH_STAGES]
                batch.set_tuning(entries)
            batch.execute(cams, [o.data_ptr() for o in outs], stream=stream)
        torch.cuda.synchronize()
        assert batch.last_flattened() == (f > 0 and setting != "tune") or setting == "tune"
        for k in range(len(cfgs)):
            np.testing.assert_array_equal(outs[k].cpu().numpy(), ref[k], err_msg=f"instance {k} frame {f} setting {setting}")
            np.testing.assert_array_equal(batched[k].get_buffer("curr_reservoirs"), solo[k].get_buffer("curr_reservoirs"))
    batch.close()
    for p in solo + batched:
        p.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_batch_member_with_analytic_lights(rs, scenes):
    """A member with analytic lights keeps the batch on per-member graphs (the flattened kernels
    are built without them), and every member still matches its pass rendered alone."""
    import torch
    cfgs, solo, batched = _uniform_members(rs, scenes)
    spot = {"type": "point", "position": (0.5, 0.9, 0.5), "direction": (0.0, -1.0, 0.0), "intensity": (1.0, 1.0, 1.0),
            "openingAngle": 0.8, "penumbraAngle": 0.2}
    for p in (solo[0], batched[0]):
        p.set_analytic_lights([spot])
    outs = [torch.zeros((h, w, 4), dtype=torch.float32, device="cuda") for _, _, w, h in cfgs]
    batch = rs.Batch(batched)
    stream = torch.cuda.current_stream().cuda_stream
    for f in range(4):
        cams = [cfg[1](f, cfg[2], cfg[3]) for cfg in cfgs]
        ref = [p.render(c) for p, c in zip(solo, cams)]
        batch.execute(cams, [o.data_ptr() for o in outs], stream=stream)
        torch.cuda.synchronize()
        assert not batch.last_flattened()
        for k in range(len(cfgs)):
            np.testing.assert_array_equal(outs[k].cpu().numpy(), ref[k], err_msg=f"instance {k} frame {f}")
    batch.close()
    for p in solo + batched:
        p.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_tuning_cache_round_trip(rs, scenes, tmp_path):
    import torch
    cfgs, solo, batched = _uniform_members(rs, scenes)
    outs = [torch.zeros((h, w, 4), dtype=torch.float32, device="cuda") for _, _, w, h in cfgs]
    cache = tmp_path / "tuning.json"
    batch = rs.Batch(batched, tuning_cache=str(cache))
    stream = torch.cuda.current_stream().cuda_stream
    for f in range(2):
        cams = [cfg[1](f, cfg[2], cfg[3]) for cfg in cfgs]
        if f == 0:
            batch.execute(cams, [o.data_ptr() for o in outs], stream=stream)
        else:
            tuned = batch.tune(cams, [o.data_ptr() for o in outs], stream=stream)
    assert cache.exists()
    form = batch.choose_form([[cfg[1](f, cfg[2], cfg[3]) for cfg in cfgs] for f in range(2, 4)], [o.data_ptr() for o in outs], stream=stream)
    assert set(form) == {"flattened_ms", "branches_ms", "flatten"} and form["flattened_ms"] > 0 and form["branches_ms"] > 0
    again = rs.Batch(batched, tuning_cache=str(cache))
    assert again.flatten == form["flatten"]
    assert again.tuning() == [dict(e, ms=e["ms"]) for e in tuned]
    with pytest.raises(rs.RsError, match="tile width"):
        again.set_tuning([{"stage": "candidates", "width": 48, "height": 32, "tile": 12, "grid": 0}])
    again.close()
    batch.close()
    for p in solo + batched:
        p.close()
