"""rs_backward (CUDA, through the C ABI) against the oracle's replay gradient and FP64 differences,
and the torch.autograd layer over it.

The forward passes are bit-exact between GPU and oracle, so both differentiate the same selected
paths.  The GPU sums per-pixel terms in FP32 with atomics in arbitrary order; the oracle sums them
in FP64.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-3    # against FP64 central differences (Richardson, h = 1e-3 and 5e-4)
ORACLE_TOL = 1e-4  # against the oracle's analytic gradient, relative to the largest component


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


PROPS = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 1,
         "enableSpatialResampling": True}


def _setup(rs, oracle_mod, scenes, width=64, height=64, props=PROPS, scene=None):
    sc = scene if scene is not None else scenes.inverse_scene(grid=80, spheres=8, subdiv=2)
    gpu = rs.ReservoirSplatting(props, width, height)
    gpu.set_scene(sc)
    ora = oracle_mod.OraclePass(props, width, height)
    ora.set_scene(sc)
    mats = np.array(sc.materials, np.float32).reshape(len(sc.materials), -1)
    return sc, gpu, ora, mats


def _richardson(f, x, h=1e-3):
    cd = lambda hh: (f(x + hh) - f(x - hh)) / (2 * hh)
    return (4 * cd(h / 2) - cd(h)) / 3


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("case,bounces,env", [("inverse_scene", 1, False), ("inverse_scene", 2, False), ("cornell", 2, False),
                                              ("cornell", 3, False), ("inverse_scene", 2, True), ("cornell", 3, True),
                                              ("cornell_dof", 2, False)])
def test_backward_matches_oracle_and_fp64_differences(rs, oracle_mod, scenes, case, bounces, env):
    """With more than one bounce, paths of four and five vertices are differentiated through the
    suffix replay from x3; none is skipped, and the replayed suffix radiance is the record's.  With
    an environment map, the paths that end at it carry its radiance (held fixed) and have no emitter
    material, and the suffix replay's light-type selection takes the env branch too."""
    import torch
    W = H = 64 if case == "inverse_scene" else 40
    props = dict(PROPS, maxSurfaceBounces=bounces)
    sc, gpu, ora, mats = _setup(rs, oracle_mod, scenes, W, H, props, None if case == "inverse_scene" else scenes.cornell_box(0))
    if env:
        sky = scenes.sky_env_map(64, 32, seed=3)
        gpu.set_env_map(sky)
        ora.set_env_map(sky)
    camera = scenes.translate_camera if case == "inverse_scene" else scenes.cornell_camera
    if case == "cornell_dof":  # an open aperture: lens-vertex copies and primary-hit reconnections
        def camera(f, w, h):
            c = scenes.cornell_camera(f, w, h)
            c.aperture_radius = 0.03
            c.focal_distance = 1.6
            return c
    rng = np.random.default_rng(2)
    n = len(mats)
    G = torch.zeros((n, 8), dtype=torch.float32, device="cuda")
    O = np.zeros((n, 8))
    FD = np.zeros((n, 8))
    P0 = mats[:, :8].astype(np.float64)
    emissive = mats[:, 4:7].max(1) > 0
    metal_rough = (mats[:, 9].view(np.uint32) & 2) == 0  # kMtlSpecGloss clear
    # metallic too where it is below 1 (at 1 the diffuse lobe is switched off: a one-sided point)
    params = [(m, k) for m in range(n)
              for k in (list(range(4, 7)) if emissive[m] else list(range(4)) + ([7] if metal_rough[m] and mats[m, 7] < 1.0 else []))]
    stats = np.zeros(4, np.uint64)
    long_paths = 0
    for f in range(3):
        cam = camera(f, W, H)
        img = gpu.render(cam)
        np.testing.assert_array_equal(img, ora.execute(cam))
        long_paths += int(((gpu.get_buffer("curr_reconnection").reshape(-1, 28)[:, 5] & 0xff) > 3).sum())
        target = (img * rng.uniform(0.9, 1.1, img.shape)).astype(np.float32)
        gc = (2.0 * (img - target)).astype(np.float32)
        gpu.backward(torch.from_numpy(gc).cuda().data_ptr(), G.data_ptr())
        torch.cuda.synchronize()
        stats += gpu.backward_stats()
        O += ora.backward(gc, n)[0]
        for m, k in params:
            def loss(x):
                q = P0.copy()
                q[m, k] = x
                return ora.replay_loss(target, q)
            FD[m, k] += _richardson(loss, P0[m, k])
    g = G.cpu().numpy().astype(np.float64)
    assert stats[0] > 0 and stats[1] == 0
    assert stats[2] == 0, f"{stats[2]} replayed paths without an identified emitter"
    if bounces > 1:
        assert long_paths > (20 if case == "inverse_scene" else 100), long_paths
    assert np.abs(g - O).max() <= ORACLE_TOL * np.abs(O).max()
    assert np.abs(g - FD).max() <= GRAD_TOL * np.abs(FD).max()
    big = np.abs(FD) > 1e-2 * np.abs(FD).max()
    assert (np.abs(g - FD)[big] / np.abs(FD)[big]).max() < GRAD_TOL
    gpu.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_checkpoint_replays_an_earlier_frame(rs, scenes):
    """Backward from a checkpoint taken at frame f equals backward run right after frame f."""
    import torch
    W = H = 48
    sc = scenes.inverse_scene(grid=64, spheres=6, subdiv=2)
    p = rs.ReservoirSplatting(PROPS, W, H)
    p.set_scene(sc)
    n = len(sc.materials)
    gc = torch.rand((H, W, 4), device="cuda")
    p.render(scenes.translate_camera(0, W, H))
    ck = torch.empty(p.checkpoint_bytes(), dtype=torch.uint8, device="cuda")
    p.checkpoint(ck.data_ptr())
    direct = torch.zeros((n, 8), device="cuda")
    p.backward(gc.data_ptr(), direct.data_ptr())
    p.render(scenes.translate_camera(1, W, H))
    later = torch.zeros((n, 8), device="cuda")
    p.backward(gc.data_ptr(), later.data_ptr(), checkpoint_ptr=ck.data_ptr())
    torch.cuda.synchronize()
    scale = direct.abs().max().item()
    assert scale > 0
    assert (direct - later).abs().max().item() <= 1e-5 * scale
    p.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_set_materials_renders_like_the_oracle(rs, oracle_mod, scenes):
    W = H = 40
    sc, gpu, ora, mats = _setup(rs, oracle_mod, scenes, W, H)
    new = mats.copy()
    new[:32, :3] = np.clip(new[:32, :3] * 0.8 + 0.1, 0, 1)
    new[32:, 4:7] *= 1.3
    gpu.set_materials(new)
    ora.set_materials(new)
    for f in range(3):
        cam = scenes.translate_camera(f, W, H)
        np.testing.assert_array_equal(gpu.render(cam), ora.execute(cam))
    gpu.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_suffix_replay_needs_the_tiny_uniform_generator(rs, oracle_mod, scenes):
    """A record keeps 32 bits of the sample generator's state at x3: PCG32's 64-bit state cannot be
    re-run, so with PCG32 the paths of four or more vertices have their suffix held fixed at the
    record's radiance (x1 and x2 are still differentiated) and are counted, by the GPU and the oracle
    alike."""
    import torch
    W = H = 40
    props = dict(PROPS, maxSurfaceBounces=2, sampleGenerator="PCG32")
    sc, gpu, ora, mats = _setup(rs, oracle_mod, scenes, W, H, props, scenes.cornell_box(0))
    n = len(mats)
    img = gpu.render(scenes.cornell_camera(0, W, H))
    np.testing.assert_array_equal(img, ora.execute(scenes.cornell_camera(0, W, H)))
    gc = np.ones_like(img)
    G = torch.zeros((n, 8), dtype=torch.float32, device="cuda")
    gpu.backward(torch.from_numpy(gc).cuda().data_ptr(), G.data_ptr())
    torch.cuda.synchronize()
    st = gpu.backward_stats()
    O, ost = ora.backward(gc, n)
    assert st[1] > 0 and st[1] == ost[1] and st[0] == ost[0]
    assert np.abs(G.cpu().numpy() - O).max() <= ORACLE_TOL * np.abs(O).max()
    gpu.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_autograd_l2_loss_matches_direct_backward(rs, scenes):
    """torch autograd over render_sequence gives the summed rs_backward gradient of the L2 loss."""
    import torch
    import reservoir_splatting_b200.adjoint as adj
    W = H = 48
    sc = scenes.inverse_scene(grid=64, spheres=6, subdiv=2)
    renderer = adj.Renderer(sc, PROPS, W, H)
    cams = [scenes.translate_camera(f, W, H) for f in range(3)]
    theta = renderer.params().clone()
    target, _ = renderer.render(cams, keep_checkpoints=False)
    target = target * 1.05
    p = theta.clone().requires_grad_(True)
    images = adj.render_sequence(p, renderer, cams)
    loss = ((images - target)[..., :3] ** 2).sum()
    loss.backward()
    # direct: the same frames, rs_backward with d loss / d image = 2 (image - target)
    imgs, ckpts = renderer.render(cams)
    torch.testing.assert_close(imgs, images.detach(), rtol=0, atol=0)
    gimg = 2.0 * (imgs - target)
    gimg[..., 3] = 0.0
    direct = renderer.backward(gimg, ckpts).cpu()
    scale = direct.abs().max().item()
    assert scale > 0
    assert (p.grad - direct).abs().max().item() <= 1e-5 * scale
    assert p.grad[:, 7].abs().max().item() > 0  # metallic is differentiated


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("bounces", [1, 2])
def test_replay_gradient_is_unbiased_over_seeds(rs, scenes, bounces):
    """The estimator itself, not just the replay: for a linear loss (the sum of the last frame's
    pixels), the mean over K seeds of rs_backward's gradient equals the central difference of the
    mean image over the same seeds, to within the statistical error of the paired per-seed
    differences.  Each seed fixes the random numbers (useFixedSeed), so the differences move only
    the parameters; the resampling decisions still change with them, which is what the replay
    estimator must average out (E[df(y)/dtheta W] = dI/dtheta because W is a contribution weight of y
    for every theta)."""
    import torch
    import reservoir_splatting_b200.adjoint as adj
    W = H = 24
    K = 192
    sc = scenes.inverse_scene(grid=40, spheres=6, subdiv=2, emitters=4)
    renderer = adj.Renderer(sc, dict(PROPS, maxSurfaceBounces=bounces), W, H)
    cams = [scenes.translate_camera(f, W, H) for f in range(2)]
    theta = renderer.params().clone()
    n = renderer.num_materials
    # the terrain bands' albedos, one sphere material's roughness, one emitter's radiance
    checks = [(0, 0), (1, 1), (2, 2), (3, 0), (5, 3), (n - 1, 4), (n - 2, 5)]
    hs = {0: 0.02, 1: 0.02, 2: 0.02, 3: 0.02, 4: 0.5, 5: 0.5}
    gsum = np.zeros(len(checks))
    dsum = np.zeros(len(checks))
    d2sum = np.zeros(len(checks))
    gimg = torch.ones((len(cams), H, W, 4), device="cuda")
    gimg[:-1] = 0.0
    gimg[..., 3] = 0.0

    def last_sum(params):
        renderer.apply(params)
        imgs, _ = renderer.render(cams, keep_checkpoints=False)
        return float(imgs[-1, ..., :3].double().sum().item())

    for k in range(K):
        renderer.pass_.useFixedSeed = True
        renderer.pass_.fixedSeed = 7919 * (k + 1)
        renderer.apply(theta)
        imgs, ckpts = renderer.render(cams)
        g = renderer.backward(gimg, ckpts).cpu().numpy()
        for j, (m, c) in enumerate(checks):
            h = hs[c]
            tp, tm = theta.clone(), theta.clone()
            tp[m, c] += h
            tm[m, c] -= h
            fd = (last_sum(tp) - last_sum(tm)) / (2 * h)
            gsum[j] += g[m, c]
            d = g[m, c] - fd
            dsum[j] += d
            d2sum[j] += d * d
    renderer.pass_.close()
    gmean = gsum / K
    dmean = dsum / K
    se = np.sqrt(np.maximum(d2sum / K - dmean ** 2, 0.0) / (K - 1))
    for j, (m, c) in enumerate(checks):
        assert abs(dmean[j]) <= 4.0 * se[j] + 1e-3 * abs(gmean[j]) + 1e-6, \
            f"material {m} param {c}: mean gradient {gmean[j]:.6g}, mean (gradient - difference) {dmean[j]:.3g} +- {se[j]:.3g}"
    assert np.abs(gmean).max() > 0


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_differentiation_config_at_its_stated_size(rs, oracle_mod, scenes):
    """The differentiation configuration as specified: 512 x 512, the seeded 199k-triangle scene with
    32 materials and 8 emitters, ScatterBackup with paths of up to four vertices (the headline path
    length, as the bench measures it) over 8 frames of a translating camera, L2 loss against a
    target rendered with the parameters perturbed by N(0, 0.05).  Every frame's image is bit-exact
    with the oracle, and the summed rs_backward gradient matches the oracle's FP64-summed replay
    gradient within 1e-4 of its largest component; no replayed path lacks an emitter."""
    import os
    import torch
    import reservoir_splatting_b200.adjoint as adj
    oracle_mod.set_threads(os.cpu_count() or 1)
    W = H = 512
    sc = scenes.inverse_scene()
    assert sc.num_triangles == 199_298
    props = dict(PROPS, maxSurfaceBounces=2)
    renderer = adj.Renderer(sc, props, W, H)
    ora = oracle_mod.OraclePass(props, W, H)
    ora.set_scene(sc)
    cams = [scenes.translate_camera(f, W, H) for f in range(8)]
    theta = renderer.params().clone()
    rng = np.random.default_rng(7)
    pert = theta.clone()
    pert[:, :7] += torch.from_numpy(rng.normal(0.0, 0.05, (len(pert), 7)).astype(np.float32))
    emissive = theta[:, 4:7].amax(1) > 0
    pert[~emissive, 4:7] = 0.0
    pert[emissive, :4] = theta[emissive, :4]
    pert[:, :3] = pert[:, :3].clamp(0.0, 1.0)
    pert[:, 3] = pert[:, 3].clamp(0.1, 1.0)
    pert[:, 7] = theta[:, 7]
    renderer.apply(pert)
    target, _ = renderer.render(cams, keep_checkpoints=False)
    renderer.apply(theta)
    images, ckpts = renderer.render(cams)
    gimg = 2.0 * (images - target)
    gimg[..., 3] = 0.0
    g = renderer.backward(gimg, ckpts).cpu().numpy().astype(np.float64)
    stats = renderer.pass_.backward_stats()
    n = renderer.num_materials
    O = np.zeros((n, 8))
    gi = gimg.cpu().numpy()
    for f, cam in enumerate(cams):
        img = ora.execute(cam, should_reset=(f == 0))
        np.testing.assert_array_equal(img, images[f].cpu().numpy(), err_msg=f"frame {f}")
        o, st = ora.backward(gi[f], n)
        O += o
        assert st[2] == 0
    assert stats[0] > 0 and stats[1] == 0 and stats[2] == 0
    assert np.abs(g - O).max() <= 1e-4 * np.abs(O).max()
    renderer.pass_.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_backward_with_moving_geometry_matches_oracle(rs, oracle_mod, scenes):
    """The Cornell box's two boxes slide each frame (rs_update_geometry): frames bit-exact with the
    oracle, and each frame's gradient equals the oracle's, including the suffixes held fixed because
    they were traced in an earlier frame's geometry (counted alike)."""
    import torch
    W = H = 40
    props = dict(PROPS, maxSurfaceBounces=2)
    sc, gpu, ora, mats = _setup(rs, oracle_mod, scenes, W, H, props, scenes.cornell_box(0))
    base = np.array(sc.positions, np.float32).reshape(len(sc.positions), -1).copy()
    boxes = (np.arange(len(base)) >= 10) & (np.arange(len(base)) < 34)
    n = len(mats)
    rng = np.random.default_rng(4)
    for f in range(4):
        if f > 0:
            pos = base.copy()
            pos[boxes, 0::3] += 0.01 * f
            gpu.update_geometry(pos)
            ora.update_geometry(pos)
        cam = scenes.cornell_camera(f, W, H)
        img = gpu.render(cam)
        np.testing.assert_array_equal(img, ora.execute(cam), err_msg=f"frame {f}")
        gc = rng.uniform(-1.0, 1.0, img.shape).astype(np.float32)
        G = torch.zeros((n, 8), dtype=torch.float32, device="cuda")
        gpu.backward(torch.from_numpy(gc).cuda().data_ptr(), G.data_ptr())
        torch.cuda.synchronize()
        st = gpu.backward_stats()
        O, ost = ora.backward(gc, n)
        assert list(st) == list(ost), (f, st, ost)
        assert np.abs(G.cpu().numpy() - O).max() <= ORACLE_TOL * np.abs(O).max()
    gpu.close()
