"""rs_build_cell_lists_static: the splat cell lists built with no device allocation.

Callers that cannot allocate device memory when they run (a host that owns a fixed memory pool,
an allocator-free real-time loop, a plug-in called during its host's graph capture) build the
temporal scatter's cell lists with this call instead; its temporaries live in a fixed array inside
the library.  The GPU test checks that two calls in a row reproduce, exactly, the lists that
rs_execute built for the same frames (integer lists: bit-exact is the tolerance, as for every
index buffer in these tests).  The array keeps the previous call's contents, so the second call
also shows that whatever must start at zero is cleared.

The file is named to be collected last, so that a run stopping at the first failure has run every
other test before this one.
"""
import ctypes as C

import numpy as np
import pytest

RS_INVALID_ARG = 1


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def test_sizes_beyond_the_static_limit_are_rejected(rs):
    """Rejected before any device work, so this runs without a GPU."""
    lib = rs.load_library()
    limit = 1 << 21
    f = lib.rs_build_cell_lists_static
    assert f(None, 0, limit + 1, None, None, None, None) == RS_INVALID_ARG
    assert b"static scratch limit" in lib.rs_last_error_string()
    assert f(None, limit + 1, 16, None, None, None, None) == RS_INVALID_ARG
    assert b"static scratch limit" in lib.rs_last_error_string()
    assert f(None, 0, 0, None, None, None, None) == RS_INVALID_ARG


@pytest.mark.gpu
@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_static_cell_lists_match_rs_execute_on_two_calls(rs, scenes):
    import torch

    torch.cuda.set_device(0)
    lib = rs.load_library()
    W, H = 160, 120  # 19,200 cells: five scan tiles
    N = W * H
    p = rs.ReservoirSplatting({"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 1,
                               "enableSpatialResampling": False}, W, H)
    p.set_scene(scenes.cornell_box(0))
    # The caller owns every input and output buffer; the entry point allocates none.
    targets = torch.empty(N, dtype=torch.int32, device="cuda")
    counts = torch.empty(N, dtype=torch.int32, device="cuda")
    offsets = torch.empty(N, dtype=torch.int32, device="cuda")
    sorted_ = torch.empty(N, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    calls = 0
    for frame in range(3):
        p.render(scenes.cornell_camera(frame, W, H))
        if frame == 0:
            continue  # no temporal history yet, so no splats
        ref_targets = p.get_buffer("splat_targets")
        ref_counts = p.get_buffer("cell_counters")
        ref_offsets = p.get_buffer("cell_offsets")
        ref_sorted = p.get_buffer("sorted_splats")
        assert ref_sorted.size > N // 2, "the frame should splat most pixels"
        targets.copy_(torch.from_numpy(ref_targets.view(np.int32)))
        sorted_.fill_(-1)
        status = lib.rs_build_cell_lists_static(targets.data_ptr(), N, N, counts.data_ptr(), offsets.data_ptr(),
                                                sorted_.data_ptr(), C.c_void_p(stream))
        assert status == 0, lib.rs_last_error_string().decode()
        torch.cuda.synchronize()
        calls += 1
        np.testing.assert_array_equal(counts.cpu().numpy().view(np.uint32), ref_counts, err_msg=f"counts, call {calls}")
        np.testing.assert_array_equal(offsets.cpu().numpy().view(np.uint32), ref_offsets, err_msg=f"offsets, call {calls}")
        got = sorted_.cpu().numpy().view(np.uint32)
        np.testing.assert_array_equal(got[: ref_sorted.size], ref_sorted, err_msg=f"sorted splats, call {calls}")
    assert calls == 2
    p.close()


@pytest.mark.gpu
@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_static_cell_lists_fewer_cells_than_splats_and_crowded_cells(rs):
    """Targets at and beyond the cell count (numCells, numCells + 5, 0xffffffff) mean "no cell";
    fewer cells than splats, and one cell holding most splats (the work per splat stays bounded).
    Counts, offsets and the listed splats against numpy, on two calls in a row."""
    import torch

    torch.cuda.set_device(0)
    lib = rs.load_library()
    rng = np.random.default_rng(5)
    n, cells = 300_000, 4_000
    t = rng.integers(0, cells, n).astype(np.uint32)
    t[rng.random(n) < 0.6] = 17               # a crowded cell
    t[::7] = cells
    t[::11] = cells + 5
    t[::13] = 0xFFFFFFFF
    valid = t < cells
    ref_counts = np.bincount(t[valid], minlength=cells).astype(np.uint32)
    ref_offsets = np.concatenate([[0], np.cumsum(ref_counts)[:-1]]).astype(np.uint32)
    ref_sorted = np.argsort(np.where(valid, t, cells), kind="stable")[: int(valid.sum())].astype(np.uint32)
    targets = torch.from_numpy(t.view(np.int32)).cuda()
    counts = torch.empty(cells, dtype=torch.int32, device="cuda")
    offsets = torch.empty(cells, dtype=torch.int32, device="cuda")
    sorted_ = torch.empty(n, dtype=torch.int32, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        sorted_.fill_(-1)
        status = lib.rs_build_cell_lists_static(targets.data_ptr(), n, cells, counts.data_ptr(), offsets.data_ptr(),
                                                sorted_.data_ptr(), C.c_void_p(stream))
        assert status == 0, lib.rs_last_error_string().decode()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(counts.cpu().numpy().view(np.uint32), ref_counts, err_msg=f"counts, call {call}")
        np.testing.assert_array_equal(offsets.cpu().numpy().view(np.uint32), ref_offsets, err_msg=f"offsets, call {call}")
        np.testing.assert_array_equal(sorted_.cpu().numpy().view(np.uint32)[: ref_sorted.size], ref_sorted, err_msg=f"sorted, call {call}")
