"""Environment-map light on the CPU: the oracle's importance sampler against a quadrature of the
map (EnvMapSampler.slang:71-163), its pdf against evalPdf, the light-type probabilities, and the
ABI struct the Python wrapper builds."""
import numpy as np
import pytest


@pytest.fixture(scope="module")
def env_pass(oracle_mod, scenes):
    o = oracle_mod.OraclePass({"temporalReuse": "ScatterBackup"}, 16, 16)
    env = scenes.sky_env_map(256, 128, seed=0)
    o.set_env_map(env, intensity=1.5, tint=(1.0, 0.9, 0.8), rotation=(0.0, 30.0, 0.0))
    return o, env


def test_importance_mips_are_means(env_pass):
    o, _ = env_pass
    imp = o.env_importance()
    assert imp.shape == (349525,)
    mip0 = imp[:512 * 512].reshape(512, 512)
    mip1 = imp[512 * 512:512 * 512 + 256 * 256].reshape(256, 256)
    ref = ((mip0[0::2, 0::2] + mip0[0::2, 1::2]) + (mip0[1::2, 0::2] + mip0[1::2, 1::2])) * np.float32(0.25)
    assert np.array_equal(mip1, ref)
    assert abs(imp[-1] - mip0.astype(np.float64).mean()) < 1e-4 * imp[-1]


def test_sampler_matches_quadrature(env_pass):
    o, env = env_pass
    rng = np.random.default_rng(1)
    smp = o.env_samples(rng.random((100000, 2), dtype=np.float32))
    pdf = smp[:, 3]
    assert np.all(pdf > 0)
    assert np.abs(np.linalg.norm(smp[:, :3], axis=1) - 1).max() < 1e-5
    # the sample's pdf is evalPdf of its direction, up to texel-boundary rounding
    assert np.mean(pdf == smp[:, 7]) > 0.999
    # the returned radiance is eval of the direction
    assert np.array_equal(smp[:, 4:7], smp[:, 8:11])
    est = (smp[:, 4:7] / pdf[:, None]).mean(0)
    H, W = env.shape[:2]
    theta = np.pi * (np.arange(H) + 0.5) / H
    wgt = np.sin(theta)[:, None] * (np.pi / H) * (2 * np.pi / W)
    quad = (env * wgt[..., None]).sum((0, 1)) * 1.5 * np.array([1.0, 0.9, 0.8])
    assert np.allclose(est, quad, rtol=0.01)


def test_zero_intensity_env_is_no_env(oracle_mod, scenes):
    imgs = []
    for env in (False, True):
        o = oracle_mod.OraclePass({"temporalReuse": "ScatterBackup", "maxSurfaceBounces": 2}, 24, 16)
        o.set_scene(scenes.cornell_box(0))
        if env:
            o.set_env_map(scenes.sky_env_map(64, 32), intensity=0.0)
        for f in range(2):
            img = o.execute(scenes.cornell_camera(f, 24, 16))
        imgs.append(img)
    assert np.array_equal(imgs[0].view(np.uint32), imgs[1].view(np.uint32))


def test_sky_pixels_and_env_records(oracle_mod, scenes):
    o = oracle_mod.OraclePass({"temporalReuse": "GatherOnly", "gatherOption": "Clamped", "maxSurfaceBounces": 2}, 32, 24)
    o.set_scene(scenes.cornell_box(0))
    o.set_env_map(scenes.sky_env_map(128, 64, seed=2))
    for f in range(2):
        img = o.execute(scenes.cornell_camera(f, 32, 24))
    vb = o.get_buffer("vbuffer").reshape(-1, 4)
    sky = vb[:, 0] == 0
    assert sky.any()
    assert np.isfinite(img).all()
    # a sky pixel's jittered candidate ray can still hit the box at its silhouette
    assert (img.reshape(-1, 4)[sky, :3] > 0).all(1).mean() > 0.9
    flags = o.get_buffer("curr_reconnection").reshape(-1, 28)[:, 5]
    assert (((flags >> 14) & 1) == 1).sum() > 0


def test_env_map_struct(rs):
    import reservoir_splatting_b200.abi as A
    with pytest.raises(ValueError):
        A.env_map_struct(np.zeros((4, 4), np.float32))
    e, keep = A.env_map_struct(np.ones((2, 3, 3), np.float32), intensity=2.0, tint=(1, 0.5, 0.25), rotation=(0, 90, 0))
    assert (e.width, e.height) == (3, 2) and keep.shape == (2, 3, 4) and keep[..., 3].sum() == 0
    assert abs(e.intensity - 2.0) < 1e-7 and list(e.rotation) == [0.0, 90.0, 0.0]
    e, keep = A.env_map_struct(None)
    assert e.width == 0 and keep is None
