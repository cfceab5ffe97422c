"""A recorded camera path replayed through the pass: the reset flag on the first frame of the loop
and the freeze frame, which keeps the previous frame's history (rs_freeze) while it holds."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_replay_with_a_freeze_frame(rs, scenes, tmp_path):
    import reservoir_splatting_b200.camera_path as CP
    W, H = 96, 64
    path = tmp_path / "cameras.txt"
    with CP.CameraPathRecorder(path) as rec:
        for f in range(5):
            rec.record_camera(scenes.cornell_camera(f, W, H))
    template = scenes.cornell_camera(0, W, H)
    p = rs.ReservoirSplatting({"temporalReuse": "ScatterBackup", "maxSurfaceBounces": 2}, W, H)
    p.set_scene(scenes.cornell_box(0))
    r = CP.CameraPathReplayer.load(path, freeze_frame_id=2)
    out = np.empty((H, W, 4), np.float32)
    steps, history = [], []
    for _ in range(5):
        steps.append(CP.replay_frame(p, r, template, color_host=out))
        history.append(p.get_buffer("prev_reservoirs").copy())
    assert [(s.frame, s.frozen) for s in steps] == [(0, False), (1, False), (2, True), (2, True), (2, True)]
    assert steps[0].should_reset and not steps[1].should_reset
    # frozen frames read the same previous-frame history and leave it as it was
    np.testing.assert_array_equal(history[2].view(np.uint32), history[3].view(np.uint32))
    np.testing.assert_array_equal(history[3].view(np.uint32), history[4].view(np.uint32))
    r.unfreeze()
    nxt = CP.replay_frame(p, r, template, color_host=out)
    assert (nxt.frame, nxt.frozen) == (3, False)
    assert np.isfinite(out).all()
    p.close()
