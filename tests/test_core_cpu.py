"""Known-answer and accuracy tests of the shared float/RNG core (compiled into the oracle library).

The random streams are pinned against tests/golden/rng_kat.json, produced by a pure-Python
restatement of TEA / interleave / LCG (Utils/Sampling/Pseudorandom/LCG.slang:50-56, the
constants the reference's Source/Tools/FalcorTest/Tests/Sampling/PseudorandomTests.cpp pins)
and PCG32.
"""
import ctypes as C
import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def lib(oracle_mod):
    L = oracle_mod.load()
    L.ro_test_rng.argtypes = [C.c_uint32] * 5 + [C.c_void_p]
    L.ro_test_tea.argtypes = [C.c_uint32, C.c_uint32, C.c_void_p]
    L.ro_test_interleave.argtypes = [C.c_uint32, C.c_uint32]
    L.ro_test_interleave.restype = C.c_uint32
    L.ro_test_fmath.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_uint32]
    L.ro_test_f16.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
    L.ro_test_alias.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
    L.ro_test_alias.restype = C.c_double
    return L


def test_rng_known_answers(lib):
    kat = json.loads((GOLDEN / "rng_kat.json").read_text())
    for case in kat["cases"]:
        px, py = case["pixel"]
        seed = case["seed"]
        assert lib.ro_test_interleave(px, py) == case["interleave"]
        t = np.zeros(2, np.uint32)
        lib.ro_test_tea(case["interleave"], seed, t.ctypes.data)
        assert t.tolist() == case["tea"]
        for kind, key in ((0, "tiny_uniform"), (2, "pcg32")):
            out = np.zeros(16, np.uint32)
            lib.ro_test_rng(kind, px, py, seed, 16, out.ctypes.data)
            assert out.tolist() == case[key], (key, case["pixel"], seed)


def test_sample_next_1d_is_24_bit(lib):
    # SampleGeneratorInterface.slang:50-56: u = (next >> 8) * 2^-24, so u < 1 exactly
    out = np.zeros(4096, np.uint32)
    lib.ro_test_rng(0, 3, 5, 99, 4096, out.ctypes.data)
    u = (out >> 8).astype(np.float64) * 2.0 ** -24
    assert (u >= 0).all() and (u < 1).all()
    assert abs(u.mean() - 0.5) < 0.02


def _fmath(lib, kind, x):
    x = np.ascontiguousarray(x, np.float32)
    y = np.empty_like(x)
    lib.ro_test_fmath(kind, x.ctypes.data, y.ctypes.data, x.size)
    return y


def _ulp(v):
    return np.spacing(np.abs(v).astype(np.float32)).astype(np.float64)


def test_sin_cos_tan_accuracy(lib):
    x = np.linspace(-24.0, 24.0, 200001).astype(np.float32)
    xd = x.astype(np.float64)
    s, c = _fmath(lib, 0, x), _fmath(lib, 1, x)
    assert np.max(np.abs(s - np.sin(xd))) < 4e-7
    assert np.max(np.abs(c - np.cos(xd))) < 4e-7
    xt = np.linspace(-1.4, 1.4, 100001).astype(np.float32)
    t = _fmath(lib, 2, xt)
    ref = np.tan(xt.astype(np.float64))
    assert np.max(np.abs(t - ref) / _ulp(ref)) < 8


def test_atan_acos_accuracy(lib):
    x = np.concatenate([np.linspace(-50, 50, 100001), np.geomspace(1e-6, 1e6, 10001)]).astype(np.float32)
    a = _fmath(lib, 3, x)
    ref = np.arctan(x.astype(np.float64))
    assert np.max(np.abs(a - ref) / _ulp(ref)) < 4
    y = np.linspace(-1, 1, 200001).astype(np.float32)
    ac = _fmath(lib, 4, y)
    assert np.max(np.abs(ac - np.arccos(y.astype(np.float64)))) < 6e-7
    # arguments that round above 1 are clamped (acos of a dot product of unit vectors)
    assert _fmath(lib, 4, np.array([1.0000001, -1.0000001], np.float32)).tolist() == pytest.approx([0.0, np.pi], abs=1e-6)


def test_f16_round_trip_matches_ieee(lib):
    rng = np.random.default_rng(0)
    x = np.concatenate([rng.standard_normal(100000) * 10.0 ** rng.integers(-9, 6, 100000),
                        [0.0, -0.0, 65504.0, 65520.0, 1e6, -1e6, 5.96e-8, 2.98e-8, 6.1e-5]]).astype(np.float32)
    h = np.empty(x.size, np.uint16)
    back = np.empty_like(x)
    lib.ro_test_f16(x.ctypes.data, h.ctypes.data, back.ctypes.data, x.size)
    ref = x.astype(np.float16)
    np.testing.assert_array_equal(h, ref.view(np.uint16))
    np.testing.assert_array_equal(back, ref.astype(np.float32))


def test_alias_table_reproduces_the_weights(lib):
    rng = np.random.default_rng(3)
    for n in (1, 2, 7, 64, 1000):
        w = rng.uniform(0.01, 5.0, n).astype(np.float32)
        table = np.zeros(2 * n, np.uint32)
        s = lib.ro_test_alias(w.ctypes.data, n, table.ctypes.data)
        assert s == pytest.approx(float(w.astype(np.float64).sum()), rel=1e-6)
        x, y = table[0::2], table[1::2]
        thr = (x >> 16).astype(np.uint16).view(np.float16).astype(np.float64)
        above = ((x & 0xFFFF) << 8) | ((y >> 24) & 0xFF)
        below = y & 0xFFFFFF
        p = np.zeros(n)
        np.add.at(p, below, thr / n)
        np.add.at(p, above, (1 - thr) / n)
        np.testing.assert_allclose(p, w / w.sum(), atol=2e-3 / max(n, 1) ** 0.5 + 1e-3 / n)


def test_pow_for_power_exp_mis(lib):
    """f_pow_pos (csrc/core/fmath.h: 2^(e log2 x) in binary64 from the atanh and exponential series)
    against numpy's float64 power: within 1 ulp of binary32 over the pdf products and exponents the
    PowerExp heuristic sees; 0 at 0, NaN for NaN and negative bases."""
    lib.ro_test_pow.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
    rng = np.random.default_rng(3)
    n = 200_000
    x = np.exp(rng.uniform(np.log(1e-30), np.log(1e30), n)).astype(np.float32)
    e = rng.uniform(0.01, 10.0, n).astype(np.float32)
    x[:8] = [0.0, 1.0, 2.0, 0.5, 1e-38, 3e38, np.nan, -1.0]
    y = np.empty(n, np.float32)
    lib.ro_test_pow(x.ctypes.data, e.ctypes.data, y.ctypes.data, n)
    ref = np.power(x.astype(np.float64), e.astype(np.float64))
    assert y[0] == 0.0 and y[1] == 1.0 and y[2] == np.float32(2.0 ** np.float64(e[2]))
    assert np.isnan(y[6]) and np.isnan(y[7])
    ok = np.isfinite(ref) & (ref > 1e-37) & (ref < 3e38)
    ulp = np.spacing(np.abs(ref[ok]).astype(np.float32)).astype(np.float64)
    err = np.abs(y[ok].astype(np.float64) - ref[ok]) / ulp
    assert err.max() <= 1.0, float(err.max())
