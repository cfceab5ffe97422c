"""Degenerate scenes against the oracle: no emitters (a black image, no light samples) and no
triangles at all (every ray misses), in three temporal modes; and a frame before any scene is set,
which must fail with RS_NOT_READY instead of touching the GPU."""
import numpy as np
import pytest

from test_parity_gpu import run_pair

pytestmark = pytest.mark.gpu


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


MODES = [{"temporalReuse": "ScatterBackup"}, {"temporalReuse": "GatherOnly", "gatherOption": "Robust"},
         {"temporalReuse": "MultiScatter", "numTimePartitions": 2}]


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("props", MODES, ids=["ScatterBackup", "GatherOnly-Robust", "MultiScatter"])
@pytest.mark.parametrize("kind", ["no_emitters", "no_triangles"])
def test_degenerate_scene(rs, oracle_mod, scenes, props, kind):
    sc = scenes.cornell_box(0)
    if kind == "no_emitters":
        mats = sc.materials.copy()
        mats[:, 4:7] = 0.0
        sc = scenes.Scene(sc.positions, sc.material_ids, mats, "cornell_dark")
    else:
        sc = scenes.Scene(np.zeros((0, 9), np.float32), np.zeros(0, np.uint32), sc.materials[:1].copy(), "empty")
    shutter = 0.04 if props["temporalReuse"] == "MultiScatter" else 0.0
    _, img = run_pair(rs, oracle_mod, sc, scenes.cornell_camera, dict(props, maxSurfaceBounces=2, enableSpatialResampling=True),
                      frames=3, width=32, height=24, shutter=shutter)
    assert np.isfinite(img).all()
    assert (img[..., :3] == 0).all()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_frame_before_a_scene_is_not_ready(rs, scenes):
    p = rs.ReservoirSplatting({}, 16, 16)
    with pytest.raises(rs.RsError, match="RS_NOT_READY"):
        p.render(scenes.cornell_camera(0, 16, 16))
    p.close()
