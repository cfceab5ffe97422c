"""Comparison helpers for the CUDA-vs-oracle parity tests.

Parity contract: splat targets, surviving splats, in-cell order and
selected-reservoir data (hits, path lengths, flags) are bit-exact; radiance, W and
the other float fields agree within REL_TOL relative error.
"""
import numpy as np

REL_TOL = 1e-4
ABS_TOL = 1e-6

# float words of the 28-word reconnection record; the others are integers / packed hits
RECON_FLOAT_WORDS = [0, 1, 2, 3, 4, 6, 7, 16, 17, 18, 19, 20, 21, 22, 23, 24, 25, 26]
RECON_INT_WORDS = [5, 8, 9, 10, 11, 12, 13, 14, 15, 27]
# barycentric words of the hits are floats stored as bits
RECON_HIT_FLOAT_WORDS = [10, 11, 14, 15]


def close(a, b, rel=REL_TOL, abs_=ABS_TOL):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    both_nan = np.isnan(a) & np.isnan(b)
    ok = (np.abs(a - b) <= abs_ + rel * np.maximum(np.abs(a), np.abs(b))) | both_nan
    return ok


def assert_close(name, a, b, rel=REL_TOL, abs_=ABS_TOL):
    assert a.shape == b.shape, f"{name}: shape {a.shape} vs {b.shape}"
    ok = close(a, b, rel, abs_)
    if not ok.all():
        idx = np.argwhere(~ok)[:5]
        raise AssertionError(f"{name}: {int((~ok).sum())} of {ok.size} values differ beyond {rel} rel; first {idx.tolist()} "
                             f"gpu={a[tuple(idx[0])]!r} oracle={b[tuple(idx[0])]!r}")


def assert_equal(name, a, b):
    assert a.shape == b.shape, f"{name}: shape {a.shape} vs {b.shape}"
    bad = a != b
    if bad.any():
        idx = np.argwhere(bad)[:5]
        raise AssertionError(f"{name}: {int(bad.sum())} of {bad.size} values differ; first {idx.tolist()} "
                             f"gpu={a[tuple(idx[0])]!r} oracle={b[tuple(idx[0])]!r}")


def compare_reservoirs(name, g, o):
    assert_close(name, g[:, :7], o[:, :7])


def compare_recon(name, g, o):
    ints = [w for w in RECON_INT_WORDS if w not in RECON_HIT_FLOAT_WORDS]
    assert_equal(name + ".int", g[:, ints], o[:, ints])
    fw = RECON_FLOAT_WORDS + RECON_HIT_FLOAT_WORDS
    # words of invalid hits / distant directions are compared as floats too (0 for both)
    assert_close(name + ".float", g[:, fw].view(np.float32), o[:, fw].view(np.float32))


def bit_mismatch_fraction(g, o):
    return float((g.view(np.uint32) != o.view(np.uint32)).mean())


def run_pair(rs, oracle_mod, scene, camera_fn, props, frames=5, width=64, height=64, shutter=0.0, aperture=0.0,
             check_candidates=True, builder="PLOC", setup=None):
    gpu = rs.ReservoirSplatting(props, width, height)
    gpu.set_bvh_builder(builder)
    gpu.keep_candidates(True)
    ora = oracle_mod.OraclePass(props, width, height)
    gpu.set_scene(scene)
    ora.set_scene(scene)
    if setup is not None:  # scene extras given to both passes alike (env map, analytic lights)
        setup(gpu)
        setup(ora)
    mode = gpu.options.temporalReuse
    report = {}
    for f in range(frames):
        cam = camera_fn(f, width, height)
        cam.shutter_speed = shutter
        cam.aperture_radius = aperture
        img_g = gpu.render(cam)
        img_o = ora.execute(cam)
        assert_equal(f"frame{f}.vbuffer", gpu.get_buffer("vbuffer"), ora.get_buffer("vbuffer"))
        assert_equal(f"frame{f}.mvec", gpu.get_buffer("mvec").view(np.uint32), ora.get_buffer("mvec").view(np.uint32))
        if check_candidates:
            compare_reservoirs(f"frame{f}.candidates", gpu.get_buffer("candidate_reservoirs"), ora.get_buffer("candidate_reservoirs"))
            compare_recon(f"frame{f}.candidate_recon", gpu.get_buffer("candidate_reconnection"), ora.get_buffer("candidate_reconnection"))
        if f > 0 and mode in (1, 2):  # ScatterOnly / ScatterBackup: the splat cell lists
            assert_equal(f"frame{f}.splat_targets", gpu.get_buffer("splat_targets"), ora.get_buffer("splat_targets"))
            assert_equal(f"frame{f}.cell_counters", gpu.get_buffer("cell_counters"), ora.get_buffer("cell_counters"))
            assert_equal(f"frame{f}.cell_offsets", gpu.get_buffer("cell_offsets"), ora.get_buffer("cell_offsets"))
            assert_equal(f"frame{f}.sorted_splats", gpu.get_buffer("sorted_splats"), ora.get_buffer("sorted_splats"))
            report["splats"] = int(gpu.get_buffer("cell_counters").sum())
        compare_reservoirs(f"frame{f}.reservoirs", gpu.get_buffer("curr_reservoirs"), ora.get_buffer("curr_reservoirs"))
        compare_recon(f"frame{f}.reconnection", gpu.get_buffer("curr_reconnection"), ora.get_buffer("curr_reconnection"))
        assert_close(f"frame{f}.color", img_g, img_o)
        report[f"bits{f}"] = bit_mismatch_fraction(img_g, img_o)
    gpu.close()
    return report, img_g
