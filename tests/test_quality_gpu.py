"""Image error against an FP64 ground truth (the quality half of the frame-rate metric).

The ground truth is the FP64 mean of many frames of the pass with temporal and spatial reuse off:
each is the initial-candidate estimate alone, an unbiased one-path-per-pixel estimate with its own
seed.  Resampled frames (ScatterBackup with spatial reuse, after a few frames of history) must sit
closer to it than one-path path tracing, and their mean must agree with it (no visible bias).
"""
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
@pytest.mark.parametrize("mode", ["ScatterBackup", "GatherOnly"])
def test_resampling_beats_path_tracing_against_fp64_ground_truth(rs, scenes, mode):
    import torch
    W = H = 64
    sc = scenes.cornell_box(0)
    cam = scenes.cornell_camera(0, W, H)
    gt_pass = rs.ReservoirSplatting({"enableTemporalResampling": False, "enableSpatialResampling": False, "maxSurfaceBounces": 2}, W, H)
    gt_pass.set_scene(sc)
    col = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
    acc = torch.zeros((H, W, 3), dtype=torch.float64, device="cuda")
    spp = 2048
    one = None
    for k in range(spp):
        gt_pass.execute(cam, color_ptr=col.data_ptr())
        acc += col[..., :3].double()
        if k == 0:
            one = col[..., :3].double().clone()
    gt = acc / spp
    p = rs.ReservoirSplatting({"temporalReuse": mode, "gatherOption": "Clamped", "enableSpatialResampling": True, "maxSurfaceBounces": 2}, W, H)
    p.set_scene(sc)
    errs, means = [], []
    for f in range(24):
        p.execute(cam, color_ptr=col.data_ptr())
        if f >= 8:
            img = col[..., :3].double()
            errs.append(float(((img - gt) ** 2).mean()))
            means.append(float(img.mean()))
    torch.cuda.synchronize()
    mse_pt = float(((one - gt) ** 2).mean())
    mse_rs = float(np.mean(errs))
    assert mse_rs < 0.5 * mse_pt, (mse_rs, mse_pt)
    assert abs(np.mean(means) - float(gt.mean())) < 0.03 * float(gt.mean())
    gt_pass.close()
    p.close()
