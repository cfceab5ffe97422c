"""Path-replay adjoint on the CPU: the BSDF derivatives and the oracle's analytic replay gradient
against FP64 central differences.

The differentiated function is the replay estimator of the pass (selections, contribution weights,
sampling densities and MIS weights held at the rendered values; BSDF factors and emitted radiance
re-evaluated), written out in FP64 by the oracle.  Central differences use h = 1e-3 and h = 5e-4
combined by Richardson extrapolation: a plain h = 1e-3 difference has an O(h^2) truncation error
near 1e-3 on the roughness of sharp GGX lobes, the size of the tolerance itself.
"""
import numpy as np
import pytest

GRAD_TOL = 1e-3  # relative error of a gradient against FP64 central differences


def _cd(f, x, h):
    return (f(x + h) - f(x - h)) / (2 * h)


def _richardson(f, x, h=1e-3):
    return (4 * _cd(f, x, h / 2) - _cd(f, x, h)) / 3


@pytest.mark.parametrize("model", ["metal_rough", "spec_gloss"])
def test_bsdf_derivatives_match_fp64_differences(oracle_mod, model):
    """Derivatives with respect to baseColor, roughness and (metal-rough) metallic.  Spec-gloss:
    baseColor is the diffuse albedo, the specular colour is held fixed and the roughness slot holds
    the glossiness (roughness = 1 - slot)."""
    rng = np.random.default_rng(0)
    worst = 0.0
    for _ in range(300):
        mat = np.array([*rng.uniform(0.05, 0.95, 3), rng.uniform(0.12, 0.95), rng.choice([0.0, 0.3, 1.0]), 1.5])
        spec = None
        if model == "spec_gloss":
            mat[3] = 1.0 - mat[3]
            spec = rng.uniform(0.02, 0.9, 3)

        def unit():
            v = rng.normal(size=3)
            v[2] = abs(v[2]) + 0.1
            return v / np.linalg.norm(v)

        wi, wo = unit(), unit()
        mask = int(rng.choice([0, 1, 4, 0xF]))
        value, d_base, d_rough, value64, d_metal = oracle_mod.bsdf_grad(mat, wi, wo, mask, spec)
        scale = max(np.abs(value64).max(), 1e-9)
        assert np.abs(value - value64).max() <= 1e-5 * scale

        def val(k):
            def f(x):
                m = mat.copy()
                m[k] = x
                return oracle_mod.bsdf_grad(m, wi, wo, mask, spec)[3]
            return f

        fd_base = np.array([_richardson(val(c), mat[c])[c] for c in range(3)])
        fd_rough = _richardson(val(3), mat[3])
        err = max(np.abs(fd_base - d_base).max() / max(np.abs(fd_base).max(), 1e-9),
                  np.abs(fd_rough - d_rough).max() / max(np.abs(fd_rough).max(), 1e-3 * scale))
        if model == "metal_rough" and mat[4] < 1.0:
            # metallic = 1 switches the diffuse lobe off: a one-sided point, not differenced
            fd_metal = _richardson(val(4), mat[4])
            err = max(err, np.abs(fd_metal - d_metal).max() / max(np.abs(fd_metal).max(), 1e-3 * scale))
        elif model == "spec_gloss":
            assert np.all(d_metal == 0.0)  # the derived metallic has no derivative of its own
        worst = max(worst, err)
    assert worst < GRAD_TOL, worst


def _replay_check(oracle_mod, scene, camera_fn, width, height, frames, props, perturb_seed=1, env=None, motion=None):
    """Analytic oracle gradient vs FP64 Richardson differences of the replay L2 loss against a
    target rendered with perturbed parameters; returns (max error / max |grad|, stats, gradient,
    differences, the number of final reservoirs holding paths of more than three vertices)."""
    mats = np.array(scene.materials, np.float32).reshape(len(scene.materials), -1)
    emissive = mats[:, 4:7].max(1) > 0
    rng = np.random.default_rng(perturb_seed)
    pert = mats.copy()
    pert[~emissive, :3] = np.clip(pert[~emissive, :3] + rng.normal(0, 0.05, (int((~emissive).sum()), 3)), 0.0, 1.0)
    pert[~emissive, 3] = np.clip(pert[~emissive, 3] + rng.normal(0, 0.05, int((~emissive).sum())), 0.1, 1.0)
    pert[emissive, 4:7] *= 1.0 + rng.normal(0, 0.05, (int(emissive.sum()), 3))
    tgt = oracle_mod.OraclePass(props, width, height)
    tgt.set_scene(scene)
    tgt.set_materials(pert)
    ora = oracle_mod.OraclePass(props, width, height)
    ora.set_scene(scene)
    if env is not None:
        tgt.set_env_map(env)
        ora.set_env_map(env)
    P0 = mats[:, :8].astype(np.float64)
    metal_rough = (mats[:, 9].view(np.uint32) & 2) == 0  # kMtlSpecGloss clear
    # metallic too where it is below 1 (at 1 the diffuse lobe is switched off: a one-sided point)
    params = [(m, k) for m in range(len(mats))
              for k in (list(range(4, 7)) if emissive[m] else list(range(4)) + ([7] if metal_rough[m] and mats[m, 7] < 1.0 else []))]
    G = np.zeros((len(mats), 8))
    FD = np.zeros((len(mats), 8))
    stats = np.zeros(4, np.uint64)
    long_paths = 0
    for f in range(frames):
        cam = camera_fn(f, width, height)
        if motion is not None and f > 0:  # the frame's triangle positions (rs_update_geometry)
            pos = motion(f)
            tgt.update_geometry(pos)
            ora.update_geometry(pos)
        target = tgt.execute(cam)
        img = ora.execute(cam)
        g, st = ora.backward(2.0 * (img - target), len(mats))
        G += g
        stats += st
        long_paths += int(((ora.get_buffer("curr_reconnection").reshape(-1, 28)[:, 5] & 0xff) > 3).sum())
        for m, k in params:
            def loss(x):
                q = P0.copy()
                q[m, k] = x
                return ora.replay_loss(target, q)
            FD[m, k] += _richardson(loss, P0[m, k])
    return np.abs(G - FD).max() / np.abs(FD).max(), stats, G, FD, long_paths


@pytest.mark.parametrize("case,bounces", [("cornell", 1), ("inverse_scene", 1), ("cornell", 2), ("cornell", 3), ("inverse_scene", 2)])
def test_oracle_replay_gradient_matches_fp64_differences(oracle_mod, scenes, case, bounces):
    """With more than one bounce the final reservoirs hold paths of four and five vertices, whose
    suffix the replay re-runs from x3 (the records' sample-generator state, bounce counters and
    flags there); every one of them is replayed and differentiated."""
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": bounces,
             "enableSpatialResampling": True}
    if case == "cornell":
        err, stats, G, FD, long_paths = _replay_check(oracle_mod, scenes.cornell_box(0), scenes.cornell_camera, 32, 32, 3, props)
    else:
        sc = scenes.inverse_scene(grid=64, spheres=6, subdiv=2)
        err, stats, G, FD, long_paths = _replay_check(oracle_mod, sc, scenes.translate_camera, 40, 40, 3, props)
    assert stats[0] > 0 and stats[1] == 0
    if bounces > 1:
        assert long_paths > (100 if case == "cornell" else 5)
    assert err < GRAD_TOL, err
    big = np.abs(FD) > 1e-2 * np.abs(FD).max()
    assert (np.abs(G - FD)[big] / np.abs(FD)[big]).max() < GRAD_TOL


def test_set_materials_equals_a_fresh_scene(oracle_mod, scenes):
    """Replacing the materials in place renders exactly what a scene built with them renders."""
    props = {"temporalReuse": "ScatterBackup", "maxSurfaceBounces": 1}
    sc = scenes.cornell_box(0)
    mats = np.array(sc.materials, np.float32).reshape(len(sc.materials), -1).copy()
    mats[0, :3] = (0.3, 0.6, 0.2)
    mats[3, 4:7] = (9.0, 14.0, 6.0)
    a = oracle_mod.OraclePass(props, 24, 24)
    a.set_scene(sc)
    a.set_materials(mats)
    sc2 = scenes.cornell_box(0)
    sc2.materials[:] = mats
    b = oracle_mod.OraclePass(props, 24, 24)
    b.set_scene(sc2)
    for f in range(2):
        cam = scenes.cornell_camera(f, 24, 24)
        np.testing.assert_array_equal(a.execute(cam), b.execute(cam))


@pytest.mark.parametrize("case,bounces", [("inverse_scene", 1), ("inverse_scene", 2), ("cornell", 3)])
def test_oracle_replay_gradient_with_an_env_map(oracle_mod, scenes, case, bounces):
    """An environment map beside the emissive triangles: paths that end at it (a primary-hit light
    sample stores a direction as its second hit; longer ones a direction out of x2 or a suffix light
    sample) carry its radiance, held fixed, and have no emitter material; the light-type selection
    of the suffix replay takes the env branch too.  The BSDF gradients still match FP64 differences."""
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": bounces,
             "enableSpatialResampling": True}
    sky = scenes.sky_env_map(64, 32, seed=3)
    if case == "cornell":  # open at the front: 100-200 of its final reservoirs per frame end at the sky, some after x3
        err, stats, G, FD, long_paths = _replay_check(oracle_mod, scenes.cornell_box(0), scenes.cornell_camera, 32, 32, 3, props, env=sky)
    else:
        sc = scenes.inverse_scene(grid=64, spheres=6, subdiv=2)
        err, stats, G, FD, long_paths = _replay_check(oracle_mod, sc, scenes.translate_camera, 40, 40, 3, props, env=sky)
    assert stats[0] > 0 and stats[1] == 0 and stats[2] == 0
    assert err < GRAD_TOL, err
    big = np.abs(FD) > 1e-2 * np.abs(FD).max()
    assert (np.abs(G - FD)[big] / np.abs(FD)[big]).max() < GRAD_TOL


@pytest.mark.parametrize("bounces", [1, 2])
def test_oracle_replay_gradient_spec_gloss(oracle_mod, scenes, tmp_path, bounces):
    """The Cornell box through the OBJ importer, whose materials are spec-gloss (Falcor's OBJ
    model): the diffuse colour and the glossiness slot are differentiated, the specular colour is
    held fixed; the replay gradient matches FP64 differences."""
    import reservoir_splatting_b200.importers as I
    sc = scenes.cornell_box(0)
    I.save_obj(sc, tmp_path / "cb.obj", ["white", "red", "green", "light"],
               {"white": {"Kd": (0.7, 0.7, 0.7), "Ks": (0.05, 0.05, 0.05), "Ns": 30.0},
                "red": {"Kd": (0.6, 0.05, 0.05), "Ks": (0.3, 0.3, 0.3), "Ns": 400.0},
                "green": {"Kd": (0.1, 0.4, 0.1), "Ks": (0.02, 0.02, 0.02), "Ns": 5.0},
                "light": {"Kd": (0, 0, 0), "Ke": (17, 12, 4)}})
    imported = I.load_obj(tmp_path / "cb.obj")
    flags = np.array(imported.materials, np.float32).reshape(len(imported.materials), -1)[:, 9].view(np.uint32)
    assert np.all((flags & 2) != 0)  # kMtlSpecGloss
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": bounces,
             "enableSpatialResampling": True}
    err, stats, G, FD, long_paths = _replay_check(oracle_mod, imported, scenes.cornell_camera, 32, 32, 3, props)
    assert stats[0] > 0 and stats[1] == 0 and stats[2] == 0
    assert err < GRAD_TOL, err
    big = np.abs(FD) > 1e-2 * np.abs(FD).max()
    assert (np.abs(G - FD)[big] / np.abs(FD)[big]).max() < GRAD_TOL


@pytest.mark.parametrize("mode", [{"temporalReuse": "GatherOnly", "gatherOption": "Robust"},
                                  {"temporalReuse": "GatherOnly", "gatherOption": "Fast"},
                                  {"temporalReuse": "ScatterOnly"},
                                  {"temporalReuse": "ScatterBackup", "gatherOption": "Fast", "scatterBackupMISOption": "Pairwise"},
                                  {"temporalReuse": "MultiScatter", "numTimePartitions": 3}],
                         ids=["GatherOnly-Robust", "GatherOnly-Fast", "ScatterOnly", "ScatterBackup-Pairwise", "MultiScatter"])
def test_oracle_replay_gradient_in_every_temporal_mode(oracle_mod, scenes, mode):
    """The suffix-replay state travels with the record through every mode's shifts and copies: the
    final reservoirs of four-vertex paths replay exactly (no value mismatch) and the gradient
    matches FP64 differences."""
    props = dict(mode, maxSurfaceBounces=2, enableSpatialResampling=True)
    err, stats, G, FD, long_paths = _replay_check(oracle_mod, scenes.cornell_box(0), scenes.cornell_camera, 32, 32, 3, props)
    assert stats[0] > 0 and stats[1] == 0 and stats[2] == 0 and stats[3] == 0
    assert long_paths > 100
    assert err < GRAD_TOL, err


def _dof_camera(scenes):
    def cam(f, w, h):
        c = scenes.cornell_camera(f, w, h)
        c.aperture_radius = 0.03
        c.focal_distance = 1.6
        return c
    return cam


@pytest.mark.parametrize("mode", [{"temporalReuse": "ScatterBackup", "gatherOption": "Clamped"},
                                  {"temporalReuse": "GatherOnly", "gatherOption": "Fast"}], ids=["ScatterBackup", "GatherOnly"])
def test_oracle_replay_gradient_with_depth_of_field(oracle_mod, scenes, mode):
    """An open aperture: the final records come through the lens-vertex copy and primary-hit
    reconnection shifts, and the replay at each pixel's own primary hit still differentiates them."""
    props = dict(mode, maxSurfaceBounces=2, enableSpatialResampling=True)
    err, stats, G, FD, long_paths = _replay_check(oracle_mod, scenes.cornell_box(0), _dof_camera(scenes), 32, 32, 3, props)
    assert stats[0] > 0 and stats[1] == 0 and stats[2] == 0
    assert long_paths > 100
    assert err < GRAD_TOL, err


def test_oracle_replay_gradient_with_moving_geometry(oracle_mod, scenes):
    """The two boxes of the Cornell box slide each frame (refitted trees, previous-frame motion
    vectors): the final reservoirs replay against the frame's own geometry, and the few suffixes
    that were traced in an earlier frame's geometry are held fixed at the records' radiance."""
    sc = scenes.cornell_box(0)
    base = np.array(sc.positions, np.float32).reshape(len(sc.positions), -1).copy()
    boxes = (np.arange(len(base)) >= 10) & (np.arange(len(base)) < 34)  # walls first, the light last

    def motion(f):
        pos = base.copy()
        pos[boxes, 0::3] += 0.01 * f
        return pos.reshape(np.shape(sc.positions))
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 2, "enableSpatialResampling": True}
    err, stats, G, FD, long_paths = _replay_check(oracle_mod, sc, scenes.cornell_camera, 32, 32, 3, props, motion=motion)
    # a record reused from an earlier frame keeps a suffix traced in that frame's geometry: where the
    # replay in the moved geometry does not give its radiance back, the suffix is held fixed
    assert stats[0] > 0 and stats[2] == 0 and 0 < stats[1] < stats[0] // 20, stats
    assert err < GRAD_TOL, err


def test_suffix_fields_of_the_records(oracle_mod, scenes):
    """The record's suffix fields (word 27 and bits 15-26 of word 5): zero for paths that end before
    x3; for longer ones the bounce counters on entering x3 count the two scatter samples at x1 and
    x2 (reflection lobes only in these scenes), and the generator state is the TinyUniform LCG's."""
    props = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 3}
    o = oracle_mod.OraclePass(props, 32, 32)
    o.set_scene(scenes.cornell_box(0))
    o.execute(scenes.cornell_camera(0, 32, 32))
    rec = o.get_buffer("curr_reconnection").reshape(-1, 28)
    length = rec[:, 5] & 0xff
    state = (rec[:, 5] >> 15) & 0xfff
    short, long_ = length <= 3, length > 3
    assert long_.sum() > 50
    assert np.all(state[short] == 0) and np.all(rec[short, 27] == 0)
    diffuse, specular, transmission = state & 3, (state >> 2) & 3, (state >> 4) & 3
    assert np.all((diffuse + specular)[long_] == 2) and np.all(transmission[long_] == 0)
    assert np.all(rec[long_, 27] != 0)
