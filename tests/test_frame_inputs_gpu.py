"""The pass's two frame inputs, `mvec` and `vbuffer` (ReservoirSplatting.cpp:64-72), supplied by the
caller through rs_frame_desc: the pass reads them in place of its own primary hits and motion
vectors (GatherTemporalResampling.rt.slang:79 and SpatialResampling.rt.slang:80 read the
vbuffer for the depth-of-field split; the gathers and scatter read the motion vectors)."""
import numpy as np
import pytest

import parity as P

pytestmark = pytest.mark.gpu


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


PROPS = [
    ("GatherOnly-Fast-DoF", {"temporalReuse": "GatherOnly", "gatherOption": "Fast", "maxSurfaceBounces": 1,
                             "enableSpatialResampling": True, "neighborCount": 3}),
    ("ScatterBackup-Clamped-DoF", {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 2,
                                   "enableSpatialResampling": True, "neighborCount": 2}),
]


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("name,props", PROPS, ids=[p[0] for p in PROPS])
def test_caller_vbuffer_and_mvec_reproduce_the_pass(rs, scenes, name, props):
    """A second pass fed the first pass's own primary hits and motion vectors through rs_frame_desc
    (so it launches no primary-hit kernel) renders the same reservoirs and colour bit for bit."""
    import torch
    W, H = 48, 40
    a = rs.ReservoirSplatting(props, W, H)
    b = rs.ReservoirSplatting(props, W, H)
    sc = scenes.cornell_box(0)
    a.set_scene(sc)
    b.set_scene(sc)
    vb = torch.empty((H, W, 4), dtype=torch.int32, device="cuda")
    mv = torch.empty((H, W, 2), dtype=torch.float32, device="cuda")
    for f in range(5):
        cam = scenes.cornell_camera(f, W, H)
        cam.aperture_radius = 0.02
        img_a = a.render(cam)
        launches_a = a.last_launch_count()
        vb.copy_(torch.from_numpy(a.get_buffer("vbuffer").view(np.int32).reshape(H, W, 4)))
        mv.copy_(torch.from_numpy(a.get_buffer("mvec").reshape(H, W, 2)))
        torch.cuda.synchronize()
        img_b = b.render(cam, mvec_ptr=mv.data_ptr(), vbuffer_ptr=vb.data_ptr())
        assert b.last_launch_count() == launches_a - 1, "the pass still launched its primary-hit kernel"
        np.testing.assert_array_equal(img_b, img_a, err_msg=f"frame {f}")
        np.testing.assert_array_equal(b.get_buffer("curr_reservoirs").view(np.uint32), a.get_buffer("curr_reservoirs").view(np.uint32))
        np.testing.assert_array_equal(b.get_buffer("curr_reconnection"), a.get_buffer("curr_reconnection"))
    a.close()
    b.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_caller_vbuffer_is_read(rs, scenes):
    """A vbuffer of misses (a valid input: an empty G-buffer) changes the depth-of-field split of
    the gather and spatial shifts, so the image differs from the pass's own; motion vectors of zero
    likewise change the backup gather.  Both inputs are read, not ignored."""
    import torch
    W, H = 40, 32
    props = PROPS[0][1]
    sc = scenes.cornell_box(0)
    base = rs.ReservoirSplatting(props, W, H)
    fed = rs.ReservoirSplatting(props, W, H)
    base.set_scene(sc)
    fed.set_scene(sc)
    misses = torch.zeros((H, W, 4), dtype=torch.int32, device="cuda")
    diff = 0
    for f in range(4):
        cam = scenes.cornell_camera(f, W, H)
        cam.aperture_radius = 0.05
        x = base.render(cam)
        y = fed.render(cam, vbuffer_ptr=misses.data_ptr())
        assert np.isfinite(y).all()
        diff += int((x != y).any())
    assert diff > 0, "a vbuffer of misses changed nothing: the caller's vbuffer is not read"
    # motion vectors: zero motion for a moving camera changes the gathered sample
    base2 = rs.ReservoirSplatting(PROPS[1][1], W, H)
    fed2 = rs.ReservoirSplatting(PROPS[1][1], W, H)
    base2.set_scene(sc)
    fed2.set_scene(sc)
    zero = torch.zeros((H, W, 2), dtype=torch.float32, device="cuda")
    diff = 0
    for f in range(4):
        cam = scenes.cornell_camera(3 * f, W, H)
        x = base2.render(cam)
        y = fed2.render(cam, mvec_ptr=zero.data_ptr())
        diff += int((x != y).any())
    assert diff > 0, "zero motion vectors changed nothing: the caller's mvec is not read"
    for p in (base, fed, base2, fed2):
        p.close()
