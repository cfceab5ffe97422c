"""Benchmark of the Reservoir Splatting per-frame path (one step = one rendered frame).

Workload: the seeded terrain + icospheres scene (512 x 512 fBm heightfield, 500
icospheres at subdivision 4, 64 emissive triangles: 3.08M triangles flattened),
1920 x 1080, ScatterBackup with the Clamped gather and Balance MIS, path length 4
(maxSurfaceBounces = 2), spatial reuse on (the reference default), camera orbiting
0.5 degrees per frame.  `value` is frames/s on the device (whole job over N GPUs,
replicas: each rank renders its own instance); `e2e` is the same through the public
API with the colour image copied to pinned host memory every frame.

--impl reference times the reference algorithm's CPU restatement (oracle/) on all
host cores on a bounded sample (a 1/16-area crop-resolution render of the same
scene and camera path), scaled to 1080p frames/s.  The reference's own GPU path is
Slang on D3D12/Vulkan and cannot run on this machine.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG_DIR = ROOT / "reservoir-splatting_b200"
W_FULL, H_FULL = 1920, 1080
PROPS = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "scatterBackupMISOption": "Balance",
         "maxSurfaceBounces": 2, "enableSpatialResampling": True}
SCENE_ARGS = dict(seed=1, grid=512, spheres=500, subdiv=4, lights=64)
METRIC = "1080p frames/s (ScatterBackup, matched MSE); batched vs plain; bwd/fwd ratio"


def _package():
    if "reservoir_splatting_b200" in sys.modules:
        return sys.modules["reservoir_splatting_b200"]
    spec = importlib.util.spec_from_file_location("reservoir_splatting_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["reservoir_splatting_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def _peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("RS_CLOCKS_CSV", "/tmp/rs_clocks_%d.csv" % os.getpid()))

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def build_scene(scale: float = 1.0):
    _package()
    import reservoir_splatting_b200.scenes as S
    return S.terrain_spheres(**SCENE_ARGS)


def camera(frame, w, h):
    _package()
    import reservoir_splatting_b200.scenes as S
    return S.orbit_camera(frame, w, h)


# Algorithmic HBM bytes per pixel of each stage (R = 32 B reservoir record, C = 112 B reconnection
# record, T = 48 B triangle record, S = 5 x 16 B stored shift).
R, C_REC, T, S_SHIFT = 32, 112, 48, 80
STAGE_BYTES_PER_PIXEL = {
    # write the candidate reservoir and record; read ~3 hit triangles
    "initialCandidates": R + C_REC + 3 * T,
    # read curr/backup reservoirs, m terms, one splat (sorted index, reservoir, terms), 4 confidences,
    # mvec, the selected record and shift (about half the pixels); write reservoir, record (half), colour
    "sbCombine": 2 * R + 8 + 16 + 8 + 8 + (4 + R + 32) + 4 * 16 + 8 + (C_REC + S_SHIFT) // 2 + R + C_REC // 2 + 16,
    "vbuffer": 16 + 8 + T,
    "reproject": 16 + 8 + 16 + T + 4 + 4,
    "sortCells": 4 * 8,
}
STAGE_KERNEL = {"initialCandidates": "k_candidates_direct", "sbCombine": "k_sb_combine", "sbBackupScatter": "k_sb_backup_scatter",
                "spatialNeighbor": "k_sp_neighbor", "sortCells": "k_rsort_scatter"}


def measured_traffic():
    """DRAM bytes per launch from the committed ncu capture (profiles/ncu_traffic_1080p.txt)."""
    out = {}
    p = ROOT / "profiles" / "ncu_traffic_1080p.txt"
    if p.exists():
        for line in p.read_text().splitlines():
            if line and not line.startswith("#"):
                k, v = line.split()
                out[k] = int(v)
    return out


def roofline_entry(stage, stage_ms, W, H, peak, peak_kind, traffic):
    per_px = STAGE_BYTES_PER_PIXEL.get(stage, R + C_REC)
    alg = per_px * W * H
    ms = stage_ms[stage]
    achieved = alg / (ms / 1e3) / 1e9
    return {"bound": "hbm", "kernel": STAGE_KERNEL.get(stage, stage), "achieved": round(achieved, 2), "peak": peak,
            "unit": "GB/s", "frac": round(achieved / peak, 5), "traffic": traffic.get(STAGE_KERNEL.get(stage, ""), None),
            "algorithmic_bytes_per_pixel": per_px, "launch_ms": round(ms, 4), "peak_source": peak_kind + " (MEASURED_PEAKS hbm_gbs)"}


def rank_frame_offset(rank: int) -> int:
    """Replicas: each rank renders its own instance (the same scene, its own camera-path phase)."""
    return 97 * rank


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """The job time is the slowest rank's device time."""
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_ours(args):
    import torch
    rs = _package()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    else:
        torch.cuda.set_device(0)
    dev = torch.device("cuda", torch.cuda.current_device())
    scene = build_scene()
    W, H = W_FULL, H_FULL
    p = rs.ReservoirSplatting(PROPS, W, H)
    p.set_scene(scene)
    stream = torch.cuda.Stream()
    color = torch.empty((H, W, 4), dtype=torch.float32, device=dev)
    frame = 0

    def step(color_ptr=None, color_host=None):
        nonlocal frame
        p.execute(camera(frame + rank_frame_offset(rank), W, H), color_ptr=color_ptr, color_host=color_host, stream=stream.cuda_stream)
        frame += 1

    with torch.cuda.stream(stream):
        for _ in range(args.warmup):
            step(color.data_ptr())
    torch.cuda.synchronize()
    launches = 0
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    start, stop = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            start.record(stream)
            for _ in range(args.steps):
                step(color.data_ptr())
                launches += p.last_launch_count()
            stop.record(stream)
        torch.cuda.synchronize()
    ms = start.elapsed_time(stop)
    clocks = clk.summary()
    ms_max = max_over_ranks(ms, dist, dev)
    if dist:
        dist.barrier()
    value = world * args.steps / (ms_max / 1e3)

    # per-stage device times on the launching stream (CUDA events inside the pass)
    p.enable_stage_timing(True)
    stage_ms = {}
    with torch.cuda.stream(stream):
        for _ in range(3):
            step(color.data_ptr())
            for k, v in p.stage_times().items():
                stage_ms[k] = stage_ms.get(k, 0.0) + v / 3.0
    p.enable_stage_timing(False)
    torch.cuda.synchronize()

    # end to end through the public API, colour copied to pinned host memory every frame, over the
    # same frames as `value`: the pass restarts (rs_reset: frame count and seed), renders the same
    # warm-up frames and then the same timed frames, so both numbers time identical work
    # (once with rs_execute returning after each copy, once with one frame of latency: each frame's
    # copy overlaps the next frame's kernels and the last one is awaited inside the timed region)
    host = torch.empty((H, W, 4), dtype=torch.float32, pin_memory=True)
    host_np = host.numpy()

    def host_output_run(latency):
        nonlocal frame
        p.set_host_output_latency(latency)
        p.reset()
        frame = 0
        with torch.cuda.stream(stream):
            for _ in range(args.warmup):
                step(color.data_ptr())
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for _ in range(args.steps):
                step(None, host_np)
            p.wait_host_output()
            e1.record(stream)
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1), dist, dev)

    e2e_sync_ms = host_output_run(0)
    e2e_ms = host_output_run(1)
    p.set_host_output_latency(0)
    e2e_value = world * args.steps / (e2e_ms / 1e3)
    e2e_sync_value = world * args.steps / (e2e_sync_ms / 1e3)

    quality = None
    if rank == 0 and not args.no_quality:
        with torch.cuda.stream(stream):
            cams = [camera(f + rank_frame_offset(rank), W, H) for f in range(frame)]
            quality = measure_quality(args, torch, rs, scene, cams, torch.from_numpy(host_np), PROPS, W, H, stream)

    peak, peak_kind = _peaks()
    traffic = measured_traffic()
    dom = max(stage_ms, key=stage_ms.get) if stage_ms else "initialCandidates"
    roofline = roofline_entry(dom, stage_ms, W, H, peak, peak_kind, traffic)
    roofline["note"] = ("the dominant kernel is BVH-traversal latency bound (ncu: DRAM 9.9% of peak, its writes mostly evicted local frames; "
                        "46% issue active, 9.0 of 32 lanes); the frame's bandwidth-bound kernel is reported in hbm_kernel")
    if "sbCombine" in stage_ms:
        roofline["hbm_kernel"] = roofline_entry("sbCombine", stage_ms, W, H, peak, peak_kind, traffic)
    roofline["stage_ms"] = {k: round(v, 4) for k, v in stage_ms.items()}
    p.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 3), "unit": "frames/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": bench_config(scene.num_triangles, world, args),
            "e2e": {"value": round(e2e_value, 3), "unit": "frames/s", "h2d_bytes_per_step": int(C_frame_bytes()),
                    "d2h_bytes_per_step": int(W * H * 16), "host_output_latency_frames": 1,
                    "synchronous_value": round(e2e_sync_value, 3),
                    "how": "rs_execute with the colour copied to pinned host memory every frame; value: one frame of latency "
                           "(frame k's copy overlaps frame k+1, the last copy awaited before the end event); synchronous_value: "
                           "each call returns with its image on the host"},
            "gpu_launches": int(launches),
            "roofline": roofline,
            "clocks": clocks,
        }
        if quality is not None:
            line["quality"] = quality
        if world == 1 and not args.no_modes:
            line["modes"] = run_modes(args, torch, rs, scene, stream)
        if world == 1 and not args.no_batched:
            line["batched"] = run_batched(args, torch, rs, stream, dev)
            # beyond the configuration: all instances small (320 x 240, 10k-100k triangles), where one
            # instance's launches do not fill the GPU and batching has launches and idle SMs to save
            line["batched_small"] = run_batched(
                args, torch, rs, stream, dev, with_quality=False,
                insts=batch_instances(args.batch_instances, seed=12, resolutions=[(320, 240)], tri_range=(10_000, 100_000)),
                how="; an added workload, not the configuration: every instance 320 x 240 with 10k-100k triangles")
        if world == 1 and not args.no_motion_blur:
            line["motion_blur"] = run_motion_blur(args, torch, rs, stream)
        if world == 1 and not args.no_adjoint:
            line["adjoint"] = run_adjoint(args, torch, rs, stream)
        if world == 1 and not args.no_cpu_baseline:
            cb = cpu_baseline(args, quiet=True)
            cb.pop("triangles", None)
            line["cpu_baseline"] = cb
        print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def measure_quality(args, torch, rs, scene, cams, image, props, W, H, stream, before_frame=None, spp=None, setup=None):
    """Error of a rendered frame against an FP64 ground truth of the same frame.

    `cams` are the cameras of frames 0..f; `image` (float32 [H, W, 4], host or device) is frame f of
    the measured pass.  The ground-truth pass (same options with temporal and spatial reuse off, so
    each frame is the initial-candidate estimate alone: an unbiased one-path-per-pixel estimate)
    renders frames 0..f-1 to fill the same camera-keyframe ring (the shutter interpolates between
    those cameras), is frozen at frame f and accumulates `spp` renders of it in FP64, each with its
    own seed.  `before_frame(pass, f)` moves the geometry of frame f (moving scenes); `setup(pass)`
    adds what the scene lacks (an environment map).  The first
    accumulated render is also reported as the one-path path-tracing baseline; the ground truth's own
    noise (variance of the mean) is about mse_1spp / spp."""
    spp = spp or args.gt_spp
    gprops = dict(props, enableTemporalResampling=False, enableSpatialResampling=False)
    gt_pass = rs.ReservoirSplatting(gprops, W, H)
    gt_pass.set_scene(scene)
    if setup:
        setup(gt_pass)
    col = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
    acc = torch.zeros((H, W, 3), dtype=torch.float64, device="cuda")
    for f, c in enumerate(cams[:-1]):
        if before_frame:
            before_frame(gt_pass, f)
        gt_pass.execute(c, color_ptr=col.data_ptr(), stream=stream.cuda_stream)
    if before_frame:
        before_frame(gt_pass, len(cams) - 1)
    gt_pass.freeze(True)
    one = None
    for k in range(spp):
        gt_pass.execute(cams[-1], color_ptr=col.data_ptr(), stream=stream.cuda_stream)
        acc += col[..., :3].double()
        if k == 0:
            one = col[..., :3].double().clone()
    torch.cuda.synchronize()
    gt = acc / spp
    img = image[..., :3].to(device="cuda", dtype=torch.float64)
    mse = float(((img - gt) ** 2).mean())
    mse1 = float(((one - gt) ** 2).mean())
    rel = lambda a: float((((a - gt) ** 2) / (gt ** 2 + 1e-2)).mean())
    gt_pass.close()
    return {"mse_vs_fp64_gt": mse, "relmse_vs_fp64_gt": rel(img), "mse_1spp_path_tracing": mse1, "relmse_1spp_path_tracing": rel(one),
            "mse_ratio_1spp_over_restir": round(mse1 / mse, 3) if mse > 0 else None, "gt_spp": spp,
            "gt_noise_mse_estimate": mse1 / spp, "gt_mean_radiance": float(gt.mean()), "frame": len(cams) - 1,
            "how": "the frame vs the FP64 mean of gt_spp independent candidate-only renders of the same frame (same cameras, "
                   "keyframe ring and geometry; ground-truth pass frozen at that frame)"}


BATCH_RESOLUTIONS = [(320, 240), (640, 480), (1280, 720), (1920, 1080)]


MODE_PROPS = {
    "GatherOnly-Clamped": {"temporalReuse": "GatherOnly", "gatherOption": "Clamped"},
    "GatherOnly-Robust": {"temporalReuse": "GatherOnly", "gatherOption": "Robust"},
    "ScatterOnly": {"temporalReuse": "ScatterOnly"},
    "ScatterBackup-Fast-Pairwise": {"temporalReuse": "ScatterBackup", "gatherOption": "Fast", "scatterBackupMISOption": "Pairwise"},
    "MultiScatter-P4-shutter-1/24": {"temporalReuse": "MultiScatter", "numTimePartitions": 4, "artificialFrameTime": 1.0 / 48.0},
}
MODE_SHUTTER = {"MultiScatter-P4-shutter-1/24": 1.0 / 24.0}
# modes rendered under the seeded sky environment map as well as the scene's emissive triangles
MODE_ENV = {"ScatterBackup-Clamped-Balance+sky": {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped"}}


def run_modes(args, torch, rs, scene, stream):
    """The other temporal modes on the benchmark scene and camera path at 1080p (path length 4,
    spatial reuse on): device frames/s from CUDA events over `args.mode_frames` frames after 4
    warm-up frames, each mode in its own pass."""
    W, H = W_FULL, H_FULL
    color = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")
    out = {}
    sky = None
    for name, props in list(MODE_PROPS.items()) + list(MODE_ENV.items()):
        p = rs.ReservoirSplatting(dict(props, maxSurfaceBounces=2, enableSpatialResampling=True), W, H)
        p.set_scene(scene)
        if name in MODE_ENV:
            import reservoir_splatting_b200.scenes as S
            sky = sky if sky is not None else S.sky_env_map(1024, 512, seed=0)
            p.set_env_map(sky)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

        def cam(f):
            c = camera(f, W, H)
            c.shutter_speed = MODE_SHUTTER.get(name, 0.0)
            return c

        with torch.cuda.stream(stream):
            for f in range(4):
                p.execute(cam(f), color_ptr=color.data_ptr(), stream=stream.cuda_stream)
            a.record(stream)
            for f in range(4, 4 + args.mode_frames):
                p.execute(cam(f), color_ptr=color.data_ptr(), stream=stream.cuda_stream)
            b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b) / args.mode_frames
        out[name] = {"frames_per_s": round(1000.0 / ms, 3), "ms_per_frame": round(ms, 4)}
        if not args.no_quality:
            q = measure_quality(args, torch, rs, scene, [cam(f) for f in range(4 + args.mode_frames)], color,
                                dict(props, maxSurfaceBounces=2), W, H, stream, spp=args.mode_gt_spp,
                                setup=(lambda gp: gp.set_env_map(sky)) if name in MODE_ENV else None)
            out[name].update({k: q[k] for k in ("mse_vs_fp64_gt", "mse_1spp_path_tracing", "mse_ratio_1spp_over_restir",
                                                "gt_noise_mse_estimate", "gt_spp")})
        p.close()
    out["how"] = (f"1920x1080, the benchmark scene and orbit, path length 4, spatial reuse on; {args.mode_frames} frames "
                  "after 4 warm-up frames per mode, CUDA events on the launching stream; MSE of each mode's last frame against "
                  f"an FP64 ground truth of {args.mode_gt_spp} candidate-only renders of that frame; MultiScatter with shutter 1/24 s and "
                  "artificial frame time 1/48 s on the static scene; '+sky' adds a seeded 1024x512 sky environment light (NEE picks "
                  "sky or emissive triangles with probability 1/2 each)")
    return out


def batch_instances(count: int, seed: int = 11, resolutions=None, tri_range=(10_000, 500_000)):
    """Seeded batched workload: resolutions uniform over `resolutions` (BATCH_RESOLUTIONS), triangles
    uniform over `tri_range` (10k-500k) each from the same generator at subdivision 4 (about 60%
    terrain, the rest icospheres of 5,120 triangles, at least one)."""
    resolutions = resolutions or BATCH_RESOLUTIONS
    _package()
    import reservoir_splatting_b200.scenes as S
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        w, h = resolutions[int(rng.integers(0, len(resolutions)))]
        target = int(rng.uniform(*tri_range))
        grid = max(8, int((0.6 * target / 2) ** 0.5))
        spheres = max(1, int(0.4 * target / 5120))
        sc = S.terrain_spheres(seed=1000 + i, grid=grid, spheres=spheres, subdiv=4, lights=16)
        out.append((sc, w, h, i))
    return out


# ray queries per pixel of a ScatterBackup frame at path length 4 with spatial reuse (counted by the
# ray-counting build on the benchmark scene: profiles/rays_1080p.md)
QUERIES_PER_PIXEL = 12.48


def run_batched(args, torch, rs, stream, dev, insts=None, with_quality=True, how=""):
    """Config "batched": 64 seeded scene/camera instances of uneven resolution, ScatterBackup, 16 timed
    frames, in three forms over the same frames (every pass restarts its history before each form):
    plain (rs_execute per instance back to back on one stream), per-member graph branches
    (rs_batch_execute, flatten off) and the flattened form (rs_batch_execute: one persistent launch
    per stage over all instances of a resolution, tile widths and grid forms from rs_batch_tune).
    The autotuner (Batch.tune, then Batch.choose_form on four warm-up frames) picks the form;
    `batched_instance_frames_per_s` is the picked form's timed rate.  The three render
    identical images (checked here on every instance's last frame), so their MSE is matched by
    construction; the MSE of the smallest and largest instance against an FP64 ground truth is
    reported as well."""
    insts = insts or batch_instances(args.batch_instances)
    passes = [rs.ReservoirSplatting(PROPS, w, h) for _, w, h, _ in insts]
    for (sc, _, _, _), a in zip(insts, passes):
        a.set_scene(sc)
    outs = [torch.empty((h, w, 4), dtype=torch.float32, device=dev) for _, w, h, _ in insts]
    cams = lambda f: [camera(f + 13 * i, w, h) for _, w, h, i in insts]
    ev = lambda: torch.cuda.Event(enable_timing=True)
    branch = rs.Batch(passes, flatten=False)
    flat = rs.Batch(passes, flatten=True)
    warm, frames = max(6, args.batch_warmup), args.batch_frames
    choice = {}

    def plain_frame(f):
        for p, c, o in zip(passes, cams(f), outs):
            p.execute(c, color_ptr=o.data_ptr(), stream=stream.cuda_stream)

    def run_form(name, frame_fn, tune=False):
        for p in passes:
            p.reset()
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            for f in range(warm):
                if tune and f == 1:
                    # the autotuner: stage tiles and grid forms on frame 1, then the batch form on
                    # frames 2-5 (alternating), before the forced flattened timing
                    flat.tune(cams(f), [o.data_ptr() for o in outs], stream=stream.cuda_stream)
                    choice.update(flat.choose_form([cams(g) for g in range(2, 6)], [o.data_ptr() for o in outs],
                                                   stream=stream.cuda_stream))
                    flat.set_flatten(True)
                elif not (tune and 2 <= f < 6):
                    frame_fn(f)
            torch.cuda.synchronize()
            a, b = ev(), ev()
            a.record(stream)
            for f in range(warm, warm + frames):
                frame_fn(f)
            b.record(stream)
        torch.cuda.synchronize()
        last = [o.clone() for o in outs]
        return a.elapsed_time(b), last

    ms_plain, img_plain = run_form("plain", plain_frame)
    ms_branch, img_branch = run_form("branch", lambda f: branch.execute(cams(f), [o.data_ptr() for o in outs], stream=stream.cuda_stream))
    ms_flat, img_flat = run_form("flat", lambda f: flat.execute(cams(f), [o.data_ptr() for o in outs], stream=stream.cuda_stream), tune=True)
    identical = all(bool(torch.equal(x, y)) and bool(torch.equal(x, z)) for x, y, z in zip(img_plain, img_branch, img_flat))
    flattened = flat.last_flattened()
    n = len(insts)
    pixels = sum(w * h for _, w, h, _ in insts)
    tris = [sc.num_triangles for sc, _, _, _ in insts]
    rate = lambda ms: n * frames / (ms / 1e3)
    qps = lambda ms: QUERIES_PER_PIXEL * pixels * frames / (ms / 1e3) / 1e9
    tuning = flat.tuning()
    launch_count = flat.launch_count()
    branch.close()
    flat.close()
    for p in passes:
        p.close()
    quality = {}
    if with_quality and not args.no_quality:  # the ground-truth passes need the batch's pass slots back
        order = sorted(range(n), key=lambda i: insts[i][1] * insts[i][2])
        for k in (order[0], order[-1]):
            sc, w, h, i = insts[k]
            q = measure_quality(args, torch, rs, sc, [camera(f + 13 * i, w, h) for f in range(warm + frames)], img_flat[k], PROPS, w, h,
                                stream, spp=args.mode_gt_spp)
            quality[f"instance{k}_{w}x{h}"] = {kk: q[kk] for kk in ("mse_vs_fp64_gt", "mse_1spp_path_tracing", "gt_spp")}
    res = {"instances": n, "frames": frames, "warmup_frames": warm, "pixels_per_batch_frame": pixels,
           "resolutions": {f"{w}x{h}": sum(1 for _, ww, hh, _ in insts if (ww, hh) == (w, h)) for w, h in sorted({(w, h) for _, w, h, _ in insts})},
           "triangles_min": min(tris), "triangles_max": max(tris),
           "plain_instance_frames_per_s": round(rate(ms_plain), 3),
           "branch_graph_instance_frames_per_s": round(rate(ms_branch), 3),
           "flattened_instance_frames_per_s": round(rate(ms_flat), 3),
           "autotuned_form": "flattened" if choice.get("flatten") else "branch graph",
           "batched_instance_frames_per_s": round(rate(ms_flat if choice.get("flatten") else ms_branch), 3),
           "speedup": round(ms_plain / (ms_flat if choice.get("flatten") else ms_branch), 4),
           "speedup_flattened": round(ms_plain / ms_flat, 4), "speedup_branch_graph": round(ms_plain / ms_branch, 4),
           "form_choice_ms": {k: round(v, 3) for k, v in choice.items() if k != "flatten"},
           "flattened": flattened, "images_identical_across_forms": identical,
           "g_queries_per_s": {"plain": round(qps(ms_plain), 3), "branch_graph": round(qps(ms_branch), 3), "flattened": round(qps(ms_flat), 3)},
           "graph_launch_kernels": launch_count,
           "tuning": [e for e in tuning if e["width"] > 0 and e["stage"] in ("candidates", "reproject", "sbCurrScatter", "sbBackupGather",
                                                                                 "spatialCentral")]
                     + [e for e in tuning if e["width"] == 0],
           "quality": quality,
           "how": "16 timed frames after warm-up per form on the same passes restarted before each form; flattened = one launch per "
                  "stage over a work queue of all 64 instances (persistent kb_* kernels), tiles/grid forms from rs_batch_tune on the last "
                  "warm-up frame; queries/s = 12.48 ray queries per pixel (counted for this mode) x pixels / time" + how}
    return res


MB_PROPS = {"temporalReuse": "MultiScatter", "numTimePartitions": 4, "artificialFrameTime": 1.0 / 48.0,
            "scatterBackupMISOption": "Balance", "maxSurfaceBounces": 2, "enableSpatialResampling": True}
MB_FRAMES = 30


def run_motion_blur(args, torch, rs, stream):
    """Motion blur and depth of field: 1920 x 1080, the seeded terrain-and-spheres generator scaled to
    3.84M triangles (800 x 800 heightfield, 500 icospheres at subdivision 4, 64 emissive triangles)
    with 200 spheres moving linearly at U[0, 0.05] units per frame, shutter 1/24 s, simulated frame
    time 1/48 s, aperture radius 0.02, MultiSplatting with 4 shutter partitions, 30 frames.  Each
    frame moves the spheres on the device (rs_update_geometry: refit, previous-frame motion vectors)
    and renders; device time over the 30 frames after 3 untimed ones."""
    import reservoir_splatting_b200.scenes as S
    sc = S.motion_blur_scene()
    motion = S.SphereMotion(sc, moving=200, max_speed=0.05, seed=4)
    W, H = W_FULL, H_FULL
    p = rs.ReservoirSplatting(MB_PROPS, W, H)
    p.set_scene(sc)
    base = torch.from_numpy(motion.base).cuda()
    vel = torch.from_numpy(np.tile(motion.tri_velocity, (1, 3))).cuda()
    pos = torch.empty_like(base)
    color = torch.empty((H, W, 4), dtype=torch.float32, device="cuda")

    def frame(f):
        cam = camera(f, W, H)
        cam.shutter_speed = 1.0 / 24.0
        cam.aperture_radius = 0.02
        torch.add(base, vel, alpha=float(f), out=pos)
        p.update_geometry(pos, stream.cuda_stream)
        p.execute(cam, color_ptr=color.data_ptr(), stream=stream.cuda_stream)

    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        for f in range(3):
            frame(f)
        a.record(stream)
        for f in range(3, 3 + MB_FRAMES):
            frame(f)
        b.record(stream)
    torch.cuda.synchronize()
    ms = a.elapsed_time(b) / MB_FRAMES
    p.close()
    quality = {}
    if not args.no_quality:
        def cam_of(f):
            c = camera(f, W, H)
            c.shutter_speed = 1.0 / 24.0
            c.aperture_radius = 0.02
            return c

        def move(gp, f):
            torch.add(base, vel, alpha=float(f), out=pos)
            gp.update_geometry(pos, stream.cuda_stream)

        q = measure_quality(args, torch, rs, sc, [cam_of(f) for f in range(3 + MB_FRAMES)], color, MB_PROPS, W, H, stream,
                            before_frame=move, spp=args.mode_gt_spp)
        quality = {k: q[k] for k in ("mse_vs_fp64_gt", "mse_1spp_path_tracing", "mse_ratio_1spp_over_restir", "gt_noise_mse_estimate", "gt_spp")}
    return {"frames_per_s": round(1000.0 / ms, 3), "ms_per_frame": round(ms, 4), "frames": MB_FRAMES, "resolution": [W, H],
            "triangles": sc.num_triangles, "moving_spheres": 200, "time_partitions": 4, **quality,
            "how": "per frame: sphere positions on the device, rs_update_geometry (refit, previous positions), rs_execute; "
                   "camera orbiting 0.5 deg/frame with shutter 1/24 s and aperture 0.02"}


ADJ_RES = 512
ADJ_FRAMES = 8
ADJ_PROPS = {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "scatterBackupMISOption": "Balance",
             "maxSurfaceBounces": 2, "enableSpatialResampling": True}


def run_adjoint(args, torch, rs, stream):
    """Differentiation workload: 512 x 512, the seeded 199k-triangle scene with 32 metal-rough
    materials and 8 emitters, ScatterBackup with paths of up to four vertices (maxSurfaceBounces 2,
    the headline path length) over 8 frames of a translating camera, L2 loss against a
    target rendered with parameters perturbed by N(0, 0.05).  Forward = the 8 frames plus one
    reservoir checkpoint per frame; backward = rs_backward for each frame (path replay).  Device
    time of each, CUDA events on the launching stream, after one untimed sequence."""
    import reservoir_splatting_b200.scenes as S
    import reservoir_splatting_b200.adjoint as adj
    sc = S.inverse_scene()
    renderer = adj.Renderer(sc, ADJ_PROPS, ADJ_RES, ADJ_RES)
    cams = [S.translate_camera(f, ADJ_RES, ADJ_RES) for f in range(ADJ_FRAMES)]
    theta = renderer.params()
    rng = np.random.default_rng(7)
    pert = theta.clone()
    pert[:, :7] += torch.from_numpy(rng.normal(0.0, 0.05, (len(pert), 7)).astype(np.float32))
    emissive = theta[:, 4:7].amax(1) > 0
    pert[~emissive, 4:7] = 0.0
    pert[emissive, :4] = theta[emissive, :4]
    pert[:, :3] = pert[:, :3].clamp(0.0, 1.0)
    pert[:, 3] = pert[:, 3].clamp(0.1, 1.0)
    pert[:, 7] = theta[:, 7]
    ev = lambda: torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        renderer.apply(pert)
        target, _ = renderer.render(cams, keep_checkpoints=False)
        renderer.apply(theta)
        fwd_ms = bwd_ms = 0.0
        reps = max(1, args.adjoint_reps)
        for rep in range(reps + 1):
            a, b, c = ev(), ev(), ev()
            a.record(stream)
            images, ckpts = renderer.render(cams)
            b.record(stream)
            gimg = 2.0 * (images - target)
            gimg[..., 3] = 0.0
            b2 = ev()
            b2.record(stream)
            grad = renderer.backward(gimg, ckpts)
            c.record(stream)
            torch.cuda.synchronize()
            if rep > 0:  # the first sequence is the warm-up
                fwd_ms += a.elapsed_time(b)
                bwd_ms += b2.elapsed_time(c)
        stats = renderer.pass_.backward_stats()
        loss = float(((images - target)[..., :3] ** 2).sum().item())
    fwd = fwd_ms / reps / ADJ_FRAMES
    bwd = bwd_ms / reps / ADJ_FRAMES
    renderer.pass_.close()
    return {"resolution": [ADJ_RES, ADJ_RES], "frames": ADJ_FRAMES, "triangles": sc.num_triangles,
            "materials": int(sc.info["materials"]), "emitters": int(sc.info["emitters"]),
            "params": int(sc.info["materials"]) * 4 + int(sc.info["emitters"]) * 3,
            "fwd_ms_per_frame": round(fwd, 4), "bwd_ms_per_frame": round(bwd, 4), "bwd_over_fwd": round(bwd / fwd, 4),
            "loss": loss, "grad_norm": float(grad.norm().item()),
            "replayed_paths": int(stats[0]), "suffixes_held_fixed": int(stats[1]), "emitter_not_found": int(stats[2]),
            "how": "fwd: rs_execute x 8 frames + rs_checkpoint (144 B/pixel) per frame; bwd: rs_backward per frame "
                   "from its checkpoint; the gradient check against FP64 central differences is in the tests"}


def bench_config(triangles, world, args):
    """The workload both arms report (the GPU arm and --impl reference print the same dict)."""
    w, h = W_FULL // 4, H_FULL // 4
    return {"workload": "terrain512+500 icospheres(subdiv4)+64 emissive tris = %d tris, 1920x1080, ScatterBackup/Clamped/Balance, "
                        "path length 4, spatial reuse on, orbit 0.5 deg/frame; CPU sample: %d temporal frames at %dx%d, scaled x16"
                        % (triangles, max(1, args.cpu_frames), w, h),
            "resolution": [W_FULL, H_FULL], "triangles": triangles, "parallelism": "replicas" if world > 1 else "single",
            "l2": "per-frame working set (3 x 144 B/pixel reservoir sets + 348 MB BVH) exceeds the 126 MB L2"}


def C_frame_bytes():
    import ctypes
    rs = _package()
    return ctypes.sizeof(rs.abi.RsFrameDesc)


def cpu_baseline(args, quiet=False):
    """The oracle on all host cores on a 480 x 270 render (1/16 of the 1080p pixels) of the same
    scene and camera path; the frame time is scaled by 16 to 1080p frames/s."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle as O
    threads = os.cpu_count() or 1
    O.set_threads(threads)
    scene = build_scene()
    w, h = W_FULL // 4, H_FULL // 4
    p = O.OraclePass(PROPS, w, h)
    t0 = time.time()
    p.set_scene(scene)
    setup = time.time() - t0
    p.execute(camera(0, w, h))  # frame 0 (no temporal history)
    frames = max(1, args.cpu_frames)
    t0 = time.time()
    for f in range(1, 1 + frames):
        p.execute(camera(f, w, h))
    dt = (time.time() - t0) / frames
    scale = (W_FULL * H_FULL) / (w * h)
    return {"value": round(1.0 / (dt * scale), 5), "unit": "frames/s", "cores": threads, "kind": "port",
            "sample": f"{frames} temporal frame(s) at {w}x{h} (1/{scale:.0f} of 1080p), scaled by {scale:.0f}; scene setup {setup:.1f}s excluded",
            "triangles": scene.num_triangles}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    cb = cpu_baseline(args)
    line = {"metric": METRIC, "value": cb["value"], "unit": "frames/s", "n_gpus": int(os.environ.get("WORLD_SIZE", "1")),
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "impl": "reference",
            "dtype": "f32", "data": "synthetic (seeded procedural scene)",
            "config": bench_config(cb.pop("triangles"), int(os.environ.get("WORLD_SIZE", "1")), args),
            "cpu_baseline": cb, "e2e": {"value": cb["value"], "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference GPU path is Slang on D3D12/Vulkan DXR: unavailable on this box; timed: the CPU restatement of its algorithm"}
    print(json.dumps(line), flush=True)


RAY_STATS_MODES = {
    "ScatterBackup": {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "scatterBackupMISOption": "Balance"},
    "ScatterOnly": {"temporalReuse": "ScatterOnly"},
    "GatherClamped": {"temporalReuse": "GatherOnly", "gatherOption": "Clamped"},
    "GatherRobust": {"temporalReuse": "GatherOnly", "gatherOption": "Robust"},
}


def _ray_stats_inner(lib_kind: str, mode: str, frames: int):
    """One process of --ray-stats: stage times (default library) or ray counts (the library built
    with -DRS_RAY_STATS), averaged over `frames` stage-timed 1080p frames after 4 warm-up frames."""
    spec = importlib.util.spec_from_file_location("rs_build", PKG_DIR / "build.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    rs = _package()
    rs.LIB_PATH = b.LIB_RAY_STATS if lib_kind == "counts" else b.LIB
    import torch
    W, H = W_FULL, H_FULL
    p = rs.ReservoirSplatting(dict(RAY_STATS_MODES[mode], maxSurfaceBounces=2, enableSpatialResampling=True), W, H)
    p.set_scene(build_scene())
    color = torch.empty((H, W, 4), device="cuda")
    for f in range(4):
        p.execute(camera(f, W, H), color_ptr=color.data_ptr())
    p.enable_stage_timing(True)
    ms, rays = {}, {}
    for f in range(4, 4 + frames):
        p.execute(camera(f, W, H), color_ptr=color.data_ptr())
        for k, v in p.stage_times().items():
            ms[k] = ms.get(k, 0.0) + v / frames
        for k, (c, v) in p.stage_rays().items():
            a = rays.setdefault(k, [0.0, 0.0])
            a[0] += c / frames
            a[1] += v / frames
    p.close()
    print(json.dumps({"ms": ms, "rays": rays}))


def run_ray_stats(args):
    """Ray queries per stage and query rates (markdown table): counts from the counting library,
    times from the default one, each in its own process."""
    spec = importlib.util.spec_from_file_location("rs_build", PKG_DIR / "build.py")
    b = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(b)
    b.build_ray_stats()
    b.build()
    runs = {}
    for inner in ("counts", "times"):
        out = subprocess.run([sys.executable, __file__, "--ray-stats", args.ray_stats, "--ray-stats-inner", inner,
                              "--mode-frames", str(args.mode_frames)], check=True, capture_output=True, text=True)
        runs[inner] = json.loads(out.stdout.strip().splitlines()[-1])
    rays, ms = runs["counts"]["rays"], runs["times"]["ms"]
    npix = W_FULL * H_FULL
    print("| stage | closest-hit | visibility | queries / pixel | ms | G queries / s |")
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cpu-frames", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-instances", type=int, default=64)
    ap.add_argument("--batch-frames", type=int, default=16)
    ap.add_argument("--batch-warmup", type=int, default=2)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-quality", action="store_true")
    ap.add_argument("--no-motion-blur", action="store_true")
    ap.add_argument("--no-modes", action="store_true")
    ap.add_argument("--mode-frames", type=int, default=10)
    ap.add_argument("--gt-spp", type=int, default=4096)
    ap.add_argument("--mode-gt-spp", type=int, default=1024)
    ap.add_argument("--adjoint-reps", type=int, default=3)
    ap.add_argument("--ray-stats", choices=sorted(RAY_STATS_MODES),
                    help="print ray queries per stage of a 1080p frame in this mode instead of the bench line")
    ap.add_argument("--ray-stats-inner", choices=["counts", "times"], help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.ray_stats and args.ray_stats_inner:
        _ray_stats_inner(args.ray_stats_inner, args.ray_stats, args.mode_frames)
    elif args.ray_stats:
        run_ray_stats(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
