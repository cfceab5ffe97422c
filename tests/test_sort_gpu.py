"""The library's own device sort and scan (csrc/radix_sort.cu), which order the BVH build's Morton
codes, the PLOC merge offsets and the temporal scatter's cell lists: against numpy's stable
argsort and cumsum, on edge-case key distributions (empty, one element, all keys equal, every key
in one cell, keys at and beyond the clamp, sizes that are not a multiple of the tile)."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def _sort64(lib, keys, bits):
    keys = np.ascontiguousarray(keys, np.uint64)
    out = np.zeros(len(keys), np.uint32)
    assert lib.rs_debug_sort_keys64(keys.ctypes.data, len(keys), bits, out.ctypes.data) == 0
    return out


def _sort32(lib, keys, clamp):
    keys = np.ascontiguousarray(keys, np.uint32)
    out = np.zeros(len(keys), np.uint32)
    assert lib.rs_debug_sort_keys32(keys.ctypes.data, len(keys), clamp, out.ctypes.data) == 0
    return out


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("n", [0, 1, 2047, 2048, 2049, 100_003, 3_082_306])
def test_sort64_morton_like_keys(rs, n):
    lib = rs.load_library()
    rng = np.random.default_rng(n)
    keys = rng.integers(0, 1 << 63, n, dtype=np.uint64)
    if n > 10:  # duplicates, as triangles sharing a centroid cell have
        keys[rng.integers(0, n, n // 4)] = keys[rng.integers(0, n, n // 4)]
    np.testing.assert_array_equal(_sort64(lib, keys, 63), np.argsort(keys, kind="stable").astype(np.uint32))


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_sort64_all_equal_and_few_bits(rs):
    lib = rs.load_library()
    n = 50_000
    np.testing.assert_array_equal(_sort64(lib, np.full(n, 7, np.uint64), 63), np.arange(n, dtype=np.uint32))
    keys = np.random.default_rng(1).integers(0, 16, n).astype(np.uint64)
    np.testing.assert_array_equal(_sort64(lib, keys, 4), np.argsort(keys, kind="stable").astype(np.uint32))


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("case", ["uniform", "one_cell", "few_cells", "invalid_mix", "beyond_clamp"])
def test_sort32_cell_targets(rs, case):
    """Splat targets as the temporal scatter makes them: the sort puts splats in (cell, source)
    order with every target >= the cell count (0xffffffff, cells, cells + 5) last."""
    lib = rs.load_library()
    rng = np.random.default_rng(3)
    n, cells = 1920 * 1080, 1920 * 1080
    if case == "uniform":
        t = rng.integers(0, cells, n).astype(np.uint32)
    elif case == "one_cell":  # a zoom that lands every source pixel in one cell
        t = np.full(n, 12345, np.uint32)
    elif case == "few_cells":
        t = rng.integers(0, 300, n).astype(np.uint32) * 997
    elif case == "invalid_mix":
        t = rng.integers(0, cells, n).astype(np.uint32)
        t[rng.random(n) < 0.3] = 0xFFFFFFFF
    else:
        cells = 5000
        t = rng.integers(0, cells + 10, n).astype(np.uint32)
        t[::7] = cells
        t[::11] = cells + 5
    expect = np.argsort(np.minimum(t, cells), kind="stable").astype(np.uint32)
    np.testing.assert_array_equal(_sort32(lib, t, cells), expect)


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("n", [0, 1, 4095, 4096, 4097, 16_777_217])
def test_scan(rs, n):
    lib = rs.load_library()
    v = np.random.default_rng(n).integers(0, 200, n).astype(np.uint32)
    out = np.zeros(n, np.uint32)
    assert lib.rs_debug_scan(v.ctypes.data, n, out.ctypes.data) == 0
    ref = np.concatenate([[0], np.cumsum(v, dtype=np.uint64)[:-1]]).astype(np.uint32) if n else out
    np.testing.assert_array_equal(out, ref)
