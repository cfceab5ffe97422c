"""setProperties / getProperties on a live pass (ReservoirSplatting.cpp:182-190, :303-344): a later
property dict changes only the keys it names, the outputSize selection stays relative to the
default size, and a pass created from get_properties() renders the same frames bit for bit."""
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
def test_set_properties_keeps_what_it_does_not_name(rs, scenes):
    W, H = 64, 48
    p = rs.ReservoirSplatting({"temporalReuse": "ScatterBackup", "gatherOption": "Robust", "maxSurfaceBounces": 2, "fixedSeed": 5,
                               "outputSize": "Half"}, W, H)
    assert (p.width, p.height) == (W // 2, H // 2)
    p.set_properties({"enableSpatialResampling": False, "misHeuristic": "PowerTwo"})
    assert (p.width, p.height) == (W // 2, H // 2)
    got = p.get_properties()
    assert got["temporalReuse"] == "ScatterBackup" and got["gatherOption"] == "Robust" and got["fixedSeed"] == 5
    assert got["enableSpatialResampling"] is False and got["misHeuristic"] == "PowerTwo" and got["outputSize"] == "Half"
    assert got["maxSurfaceBounces"] == 2 and got["maxDiffuseBounces"] == 2

    q = rs.ReservoirSplatting(got, W, H)
    sc = scenes.cornell_box(0)
    p.set_scene(sc)
    q.set_scene(sc)
    for f in range(4):
        cam = scenes.cornell_camera(f, p.width, p.height)
        np.testing.assert_array_equal(p.render(cam), q.render(cam), err_msg=f"frame {f}")
    p.set_properties({"outputSize": "Default"})
    assert (p.width, p.height) == (W, H) and p.get_properties()["gatherOption"] == "Robust"
    p.close()
    q.close()
