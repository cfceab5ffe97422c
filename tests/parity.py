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
