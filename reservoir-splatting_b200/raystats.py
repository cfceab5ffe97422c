"""Ray queries per stage of a frame, and query rates: the traversal workload behind the stage times.

    python reservoir-splatting_b200/raystats.py [--width 1920 --height 1080] [--mode ScatterBackup]

Renders the benchmark scene (seeded terrain + icospheres, 3.08M triangles, orbiting camera) with
two libraries in two processes: the one built with ray counters (build.py build_ray_stats) gives
the closest-hit and visibility queries of every stage, the default one the stage times (CUDA
events with stage timing on).  Prints one markdown row per stage: queries, queries per pixel and
queries per second.  Needs a CUDA device and nvcc (the counting library is built on first use).
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import subprocess
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent
MODES = {
    "ScatterBackup": {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "scatterBackupMISOption": "Balance"},
    "ScatterOnly": {"temporalReuse": "ScatterOnly"},
    "GatherClamped": {"temporalReuse": "GatherOnly", "gatherOption": "Clamped"},
    "GatherRobust": {"temporalReuse": "GatherOnly", "gatherOption": "Robust"},
}
SCENE_ARGS = dict(seed=1, grid=512, spheres=500, subdiv=4, lights=64)


def _load(lib: Path):
    spec = importlib.util.spec_from_file_location("reservoir_splatting_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    rs = importlib.util.module_from_spec(spec)
    sys.modules["reservoir_splatting_b200"] = rs
    spec.loader.exec_module(rs)
    rs.LIB_PATH = lib
    return rs


def _measure(lib: Path, mode: str, W: int, H: int, frames: int) -> dict:
    """Stage times and ray counts averaged over `frames` stage-timed frames after 4 warm-up frames."""
    rs = _load(lib)
    import torch
    import reservoir_splatting_b200.scenes as S
    p = rs.ReservoirSplatting(dict(MODES[mode], maxSurfaceBounces=2, enableSpatialResampling=True), W, H)
    p.set_scene(S.terrain_spheres(**SCENE_ARGS))
    color = torch.empty((H, W, 4), device="cuda")
    for f in range(4):
        p.execute(S.orbit_camera(f, W, H), color_ptr=color.data_ptr())
    p.enable_stage_timing(True)
    ms, rays = {}, {}
    for f in range(4, 4 + frames):
        p.execute(S.orbit_camera(f, W, H), color_ptr=color.data_ptr())
        for k, v in p.stage_times().items():
            ms[k] = ms.get(k, 0.0) + v / frames
        for k, (c, v) in p.stage_rays().items():
            a = rays.setdefault(k, [0.0, 0.0])
            a[0] += c / frames
            a[1] += v / frames
    p.close()
    return {"ms": ms, "rays": rays}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--mode", default="ScatterBackup", choices=sorted(MODES))
    ap.add_argument("--frames", type=int, default=5)
    ap.add_argument("--inner", choices=["counts", "times"], help=argparse.SUPPRESS)
    a = ap.parse_args()
    spec = importlib.util.spec_from_file_location("rs_build", PKG_DIR / "build.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    if a.inner:
        lib = b.LIB_RAY_STATS if a.inner == "counts" else b.LIB
        print(json.dumps(_measure(lib, a.mode, a.width, a.height, a.frames)))
        return
    b.build_ray_stats()
    b.build()
    runs = {}
    for inner in ("counts", "times"):
        out = subprocess.run([sys.executable, __file__, "--inner", inner, "--mode", a.mode, "--width", str(a.width),
                              "--height", str(a.height), "--frames", str(a.frames)], check=True, capture_output=True, text=True)
        runs[inner] = json.loads(out.stdout.strip().splitlines()[-1])
    rays, ms = runs["counts"]["rays"], runs["times"]["ms"]
    npix = a.width * a.height
    print(f"| stage | closest-hit | visibility | queries / pixel | ms | G queries / s |")
    print("|---|---:|---:|---:|---:|---:|")
    tc = tv = tms = 0.0
    for k, t in ms.items():
        c, v = rays.get(k, (0.0, 0.0))
        if c + v == 0:
            continue
        tc, tv, tms = tc + c, tv + v, tms + t
        print(f"| {k} | {c:,.0f} | {v:,.0f} | {(c + v) / npix:.2f} | {t:.3f} | {(c + v) / t / 1e6:.2f} |")
    print(f"| all traversal stages | {tc:,.0f} | {tv:,.0f} | {(tc + tv) / npix:.2f} | {tms:.3f} | {(tc + tv) / tms / 1e6:.2f} |")
    print(f"frame: {sum(ms.values()):.3f} ms of stages (stage timing serialises the side streams)")


if __name__ == "__main__":
    main()
