"""Schedule-independence of the frame and the ray-count build.

The pass runs independent shift kernels on side streams joined by events (ScatterBackup's four
shift chains, the two directions of spatial reuse); with stage timing on, the same kernels run in
order on one stream.  Both schedules must give the same bits.  The ray-count library (the same
sources built with RS_RAY_STATS) must count one closest-hit query per pixel for the primary hits and
give the same counts for the same frame."""
import importlib.util
import json
import subprocess
import sys
import textwrap
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parents[1]
PKG_DIR = ROOT / "reservoir-splatting_b200"


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def _scene(scenes):
    return scenes.terrain_spheres(seed=3, grid=96, spheres=40, subdiv=2, lights=12, extent=30.0, height=3.0)


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("props", [
    {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "enableSpatialResampling": True},
    {"temporalReuse": "ScatterBackup", "gatherOption": "Fast", "scatterBackupMISOption": "Pairwise", "enableSpatialResampling": True},
], ids=["clamped-balance", "fast-pairwise"])
def test_side_streams_match_serial_order(rs, scenes, props):
    import torch
    W, H = 384, 256
    sc = _scene(scenes)
    forked = rs.ReservoirSplatting(dict(props, maxSurfaceBounces=2), W, H)
    serial = rs.ReservoirSplatting(dict(props, maxSurfaceBounces=2), W, H)
    forked.set_scene(sc)
    serial.set_scene(sc)
    serial.enable_stage_timing(True)
    stream = torch.cuda.Stream()
    out = torch.empty((H, W, 4), device="cuda")
    for f in range(6):
        cam = scenes.orbit_camera(f, W, H, radius=25.0, height_above=9.0)
        forked.execute(cam, color_ptr=out.data_ptr(), stream=stream.cuda_stream)
        stream.synchronize()
        a = out.cpu().numpy().copy()
        b = serial.render(cam)
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32), err_msg=f"frame {f} colour")
        np.testing.assert_array_equal(forked.get_buffer("curr_reservoirs").view(np.uint32),
                                      serial.get_buffer("curr_reservoirs").view(np.uint32), err_msg=f"frame {f} reservoirs")
    assert forked.stage_rays() == {}  # the default library counts nothing
    forked.close()
    serial.close()


_COUNT = textwrap.dedent("""
    import importlib.util, json, sys
    from pathlib import Path
    pkg = Path(sys.argv[1])
    spec = importlib.util.spec_from_file_location("reservoir_splatting_b200", pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    rs = importlib.util.module_from_spec(spec); sys.modules["reservoir_splatting_b200"] = rs; spec.loader.exec_module(rs)
    rs.LIB_PATH = Path(sys.argv[2])
    import reservoir_splatting_b200.scenes as S
    W, H = 256, 160
    sc = S.terrain_spheres(seed=3, grid=96, spheres=40, subdiv=2, lights=12, extent=30.0, height=3.0)
    out = []
    for rep in range(2):
        p = rs.ReservoirSplatting({"temporalReuse": "ScatterBackup", "scatterBackupMISOption": "Balance", "maxSurfaceBounces": 2,
                                    "enableSpatialResampling": True}, W, H)
        p.set_scene(sc)
        for f in range(3):
            p.render(S.orbit_camera(f, W, H, radius=25.0, height_above=9.0))
        p.enable_stage_timing(True)
        p.render(S.orbit_camera(3, W, H, radius=25.0, height_above=9.0))
        out.append(p.stage_rays())
        p.close()
    print(json.dumps(out))
""")


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_ray_count_build(tmp_path):
    spec = importlib.util.spec_from_file_location("rs_build", PKG_DIR / "build.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    lib = b.build_ray_stats()
    script = tmp_path / "count.py"
    script.write_text(_COUNT)
    res = subprocess.run([sys.executable, str(script), str(PKG_DIR), str(lib)], check=True, capture_output=True, text=True)
    first, second = json.loads(res.stdout.strip().splitlines()[-1])
    assert first == second  # the same frame makes the same queries
    npix = 256 * 160
    assert first["vbuffer"] == [npix, 0]  # one primary closest-hit query per pixel
    c, v = first["initialCandidates"]
    assert c >= npix and v > 0  # the path tracer's primary ray per pixel, then bounces and shadow rays
    assert first["sbCombine"] == [0, 0] and first["spatialCombine"] == [0, 0]  # combines trace nothing
    for k in ("sbCurrScatter", "sbBackupScatter", "sbSplatScatter"):
        assert first[k][0] == 0 and first[k][1] > 0, k  # scatter shifts: visibility only
