"""Host colour outputs with one frame of latency (rs_set_host_output_latency 1): each frame's copy to
host memory runs on the pass's copy stream while the next frame renders, so a frame's image is in
its host buffer once the next rs_execute (or rs_wait_host_output) returns.  The images must be the
synchronous ones bit for bit, frame by frame, with and without a device output beside them."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


PROPS = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 2, "enableSpatialResampling": True}


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("with_device_output", [False, True])
def test_pipelined_host_output_matches_synchronous(rs, scenes, with_device_output):
    import torch
    W, H, F = 64, 48, 6
    sc = scenes.cornell_box(0)
    p = rs.ReservoirSplatting(PROPS, W, H)
    p.set_scene(sc)
    stream = torch.cuda.Stream()
    sync = [p.render(scenes.cornell_camera(f, W, H), stream=stream.cuda_stream) for f in range(F)]
    p.reset()
    p.set_host_output_latency(1)
    dev = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
    outs = [torch.empty((H, W, 4), dtype=torch.float32, pin_memory=True).numpy() for _ in range(F)]
    for f in range(F):
        p.execute(scenes.cornell_camera(f, W, H), color_host=outs[f], stream=stream.cuda_stream,
                  color_ptr=dev.data_ptr() if with_device_output else None)
        if f > 0:
            np.testing.assert_array_equal(outs[f - 1], sync[f - 1], err_msg=f"frame {f - 1}")
    p.wait_host_output()
    np.testing.assert_array_equal(outs[F - 1], sync[F - 1], err_msg="last frame")
    if with_device_output:
        stream.synchronize()
        np.testing.assert_array_equal(dev.cpu().numpy(), sync[F - 1])
    # back to synchronous output: the next frame's image is on the host when the call returns
    p.set_host_output_latency(0)
    p.reset()
    np.testing.assert_array_equal(p.render(scenes.cornell_camera(0, W, H), stream=stream.cuda_stream), sync[0])
    p.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_host_output_latency_is_zero_or_one(rs):
    p = rs.ReservoirSplatting({}, 16, 16)
    with pytest.raises(rs.RsError):
        p.set_host_output_latency(2)
    p.wait_host_output()  # nothing in flight
    p.close()
