"""B200 Reservoir Splatting: Python host mirror of the reference render pass.

`ReservoirSplatting` follows the Python surface of the reference pass
(``createPass("ReservoirSplatting", props)``, ``reset()``, ``useFixedSeed``,
``fixedSeed``; ReservoirSplatting.cpp:142-156, scripts/ReservoirSplatting.py)
and drives the CUDA library ``lib/librs_b200.so`` through its C ABI
(include/rs_b200.h).  There is no CPU fallback: without the built library the
constructor raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import abi
from .abi import BUF, BUFFER_LAYOUT

PACKAGE_DIR = Path(__file__).resolve().parent
# RS_B200_LIB selects another build of the library (a variant built elsewhere for comparison)
LIB_PATH = Path(os.environ["RS_B200_LIB"]) if os.environ.get("RS_B200_LIB") else PACKAGE_DIR / "lib" / "librs_b200.so"

_lib = None


class RsError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{abi.STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


def load_library():
    """Loads the CUDA library (raises when it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(f"CUDA library missing: {LIB_PATH} (run __graft_entry__.build())")
    lib = C.CDLL(str(LIB_PATH))
    lib.rs_default_options.argtypes = [C.POINTER(abi.RsOptions)]
    lib.rs_default_options.restype = None
    lib.rs_create.argtypes = [C.POINTER(abi.RsOptions), C.POINTER(C.c_void_p)]
    lib.rs_destroy.argtypes = [C.c_void_p]
    lib.rs_set_options.argtypes = [C.c_void_p, C.POINTER(abi.RsOptions)]
    lib.rs_set_scene.argtypes = [C.c_void_p, C.POINTER(abi.RsSceneDesc)]
    lib.rs_set_env_map.argtypes = [C.c_void_p, C.POINTER(abi.RsEnvMap)]
    lib.rs_set_analytic_lights.argtypes = [C.c_void_p, C.POINTER(abi.RsAnalyticLight), C.c_uint32]
    lib.rs_execute.argtypes = [C.c_void_p, C.POINTER(abi.RsFrameDesc), C.c_void_p]
    lib.rs_reset.argtypes = [C.c_void_p]
    lib.rs_set_host_output_latency.argtypes = [C.c_void_p, C.c_uint32]
    lib.rs_wait_host_output.argtypes = [C.c_void_p]
    lib.rs_set_seed.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32]
    lib.rs_freeze.argtypes = [C.c_void_p, C.c_uint32]
    lib.rs_get_buffer.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.POINTER(C.c_size_t)]
    lib.rs_set_buffer.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
    lib.rs_enable_stage_timing.argtypes = [C.c_void_p, C.c_uint32]
    lib.rs_get_stage_times.argtypes = [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_uint32), C.c_char_p, C.c_size_t]
    lib.rs_debug_stage_rays.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]
    lib.rs_set_bvh_builder.argtypes = [C.c_void_p, C.c_uint32]
    lib.rs_tonemap_default_options.argtypes = [C.POINTER(abi.RsTonemapOptions)]
    lib.rs_tonemap_default_options.restype = None
    lib.rs_tonemap_workspace_bytes.argtypes = []
    lib.rs_tonemap_workspace_bytes.restype = C.c_size_t
    lib.rs_tonemap.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.POINTER(abi.RsTonemapOptions), C.c_void_p, C.c_void_p, C.c_void_p]
    lib.rs_tonemap_color_transform.argtypes = [C.POINTER(abi.RsTonemapOptions), C.c_void_p]
    lib.rs_last_launch_count.argtypes = [C.c_void_p]
    lib.rs_last_launch_count.restype = C.c_uint32
    lib.rs_last_error_string.restype = C.c_char_p
    lib.rs_debug_keep_candidates.argtypes = [C.c_void_p, C.c_uint32]
    lib.rs_batch_create.argtypes = [C.POINTER(C.c_void_p), C.c_uint32, C.POINTER(C.c_void_p)]
    lib.rs_batch_execute.argtypes = [C.c_void_p, C.POINTER(abi.RsFrameDesc), C.c_void_p]
    lib.rs_batch_destroy.argtypes = [C.c_void_p]
    lib.rs_batch_launch_count.argtypes = [C.c_void_p]
    lib.rs_batch_launch_count.restype = C.c_uint32
    lib.rs_batch_last_flattened.argtypes = [C.c_void_p]
    lib.rs_batch_last_flattened.restype = C.c_uint32
    lib.rs_batch_set_flatten.argtypes = [C.c_void_p, C.c_uint32]
    lib.rs_batch_tune.argtypes = [C.c_void_p, C.POINTER(abi.RsFrameDesc), C.c_void_p]
    lib.rs_batch_get_tuning.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_uint32)]
    lib.rs_batch_set_tuning.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
    lib.rs_set_materials.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
    lib.rs_checkpoint_bytes.argtypes = [C.c_void_p, C.POINTER(C.c_size_t)]
    lib.rs_checkpoint.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.rs_backward.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.rs_backward_stats.argtypes = [C.c_void_p, C.c_void_p]
    lib.rs_update_geometry.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
    lib.rs_debug_trace_rays.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.rs_debug_bvh_shape.argtypes = [C.c_void_p, C.c_void_p]
    lib.rs_build_cell_lists_static.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.rs_debug_sort_keys64.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
    lib.rs_debug_sort_keys32.argtypes = [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p]
    lib.rs_debug_scan.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p]
    for name in ("rs_create", "rs_destroy", "rs_set_options", "rs_set_scene", "rs_set_env_map", "rs_execute", "rs_reset", "rs_set_seed",
                 "rs_freeze", "rs_get_buffer", "rs_set_buffer", "rs_enable_stage_timing", "rs_get_stage_times",
                 "rs_debug_keep_candidates", "rs_batch_create", "rs_batch_execute", "rs_batch_destroy",
                 "rs_build_cell_lists_static", "rs_set_materials", "rs_checkpoint_bytes", "rs_checkpoint", "rs_backward",
                 "rs_backward_stats", "rs_debug_trace_rays", "rs_debug_bvh_shape", "rs_debug_stage_rays", "rs_tonemap", "rs_tonemap_color_transform",
                 "rs_set_bvh_builder", "rs_debug_sort_keys64", "rs_debug_sort_keys32", "rs_debug_scan",
                 "rs_batch_set_flatten", "rs_batch_tune", "rs_batch_get_tuning", "rs_batch_set_tuning",
                 "rs_update_geometry"):
        getattr(lib, name).restype = C.c_int
    _lib = lib
    return lib


def _check(status: int):
    if status != abi.RS_OK:
        raise RsError(status, load_library().rs_last_error_string().decode())


class ReservoirSplatting:
    """One instance of the pass (ReservoirSplatting.h:48-279) on the current CUDA device."""

    def __init__(self, props: dict | None = None, width: int = 1920, height: int = 1080):
        lib = load_library()
        self._lib = lib
        self.options = abi.options_from_properties(props, width, height)
        h = C.c_void_p()
        _check(lib.rs_create(C.byref(self.options), C.byref(h)))
        self._h = h
        self.width, self.height = self.options.frameWidth, self.options.frameHeight
        # the render graph's default size, which outputSize selections are relative to
        self._default_size = (width, height)
        self._output_size = abi.output_size_selection(props)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rs_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- reference-facing API
    def set_properties(self, props: dict, width: int | None = None, height: int | None = None):
        """setProperties (ReservoirSplatting.cpp:182-190): the options not named keep their values,
        and so does the outputSize selection, which is relative to the default size (the
        constructor's, unless width/height are given)."""
        default = (width or self._default_size[0], height or self._default_size[1])
        props = dict(props)
        if "outputSize" not in props:
            props["outputSize"] = self._output_size[0]
            props.setdefault("fixedOutputSize", self._output_size[1])
        options = abi.options_from_properties(props, *default, base=self.options)
        _check(self._lib.rs_set_options(self._h, C.byref(options)))
        self.options, self._default_size, self._output_size = options, default, abi.output_size_selection(props)
        self.width, self.height = self.options.frameWidth, self.options.frameHeight

    def get_properties(self) -> dict:
        """getProperties (ReservoirSplatting.cpp:303-344), followed by the ReSTIR keys; passing the
        dict back to set_properties restores these options."""
        return abi.properties_from_options(self.options, *self._output_size)

    def set_scene(self, scene):
        desc, keep = abi.scene_struct(scene)
        _check(self._lib.rs_set_scene(self._h, C.byref(desc)))
        del keep

    def set_env_map(self, texels, intensity: float = 1.0, tint=(1.0, 1.0, 1.0), rotation=(0.0, 0.0, 0.0)):
        """Environment light from a lat-long map float [H, W, 3|4] (None removes it); see rs_set_env_map."""
        desc, keep = abi.env_map_struct(texels, intensity, tint, rotation)
        _check(self._lib.rs_set_env_map(self._h, C.byref(desc)))
        del keep

    def set_analytic_lights(self, lights):
        """The scene's analytic lights, a list of dicts (abi.analytic_lights_array); see rs_set_analytic_lights."""
        lights = list(lights or [])
        _check(self._lib.rs_set_analytic_lights(self._h, abi.analytic_lights_array(lights), len(lights)))

    def reset(self):
        _check(self._lib.rs_reset(self._h))

    @property
    def useFixedSeed(self) -> bool:
        return bool(self.options.useFixedSeed)

    @useFixedSeed.setter
    def useFixedSeed(self, value: bool):
        self.options.useFixedSeed = 1 if value else 0
        _check(self._lib.rs_set_seed(self._h, self.options.useFixedSeed, self.options.fixedSeed))

    @property
    def fixedSeed(self) -> int:
        return int(self.options.fixedSeed)

    @fixedSeed.setter
    def fixedSeed(self, value: int):
        self.options.fixedSeed = int(value)
        _check(self._lib.rs_set_seed(self._h, self.options.useFixedSeed, self.options.fixedSeed))

    def freeze(self, frozen: bool = True):
        _check(self._lib.rs_freeze(self._h, 1 if frozen else 0))

    def execute(self, camera, color_ptr: int | None = None, color_host: np.ndarray | None = None, stream: int = 0,
                mvec_ptr: int | None = None, vbuffer_ptr: int | None = None, should_reset: bool = False):
        """Renders one frame.  `color_ptr` is a device float4[W*H]; or pass `color_host` (float32 [H, W, 4]).
        `mvec_ptr` / `vbuffer_ptr` are the optional device inputs (float2 / uint4 per pixel)."""
        f = abi.RsFrameDesc()
        f.camera = abi.camera_struct(camera)
        f.mvec = mvec_ptr or None
        f.vbuffer = vbuffer_ptr or None
        f.color = color_ptr or None
        if color_host is not None:
            assert color_host.dtype == np.float32 and color_host.flags.c_contiguous and color_host.size == 4 * self.width * self.height
            f.colorHost = color_host.ctypes.data
        else:
            f.colorHost = None
        f.sceneShouldReset = 1 if should_reset else 0
        _check(self._lib.rs_execute(self._h, C.byref(f), C.c_void_p(stream)))

    def set_host_output_latency(self, frames: int):
        """0: execute(color_host=...) returns with the image on the host; 1: the copy overlaps the
        next frame and completes when the next execute or wait_host_output returns."""
        _check(self._lib.rs_set_host_output_latency(self._h, int(frames)))

    def wait_host_output(self):
        """Completes the host copy in flight (latency 1) and raises on that frame's device fault."""
        _check(self._lib.rs_wait_host_output(self._h))

    def render(self, camera, **kw) -> np.ndarray:
        out = np.empty((self.height, self.width, 4), np.float32)
        self.execute(camera, color_host=out, **kw)
        return out

    # ---- buffers (parity / checkpoint)
    def get_buffer(self, name: str) -> np.ndarray:
        n = C.c_size_t(0)
        _check(self._lib.rs_get_buffer(self._h, BUF[name], None, C.byref(n)))
        dtype, width = BUFFER_LAYOUT[name]
        out = np.empty(n.value // 4, dtype)
        if n.value:
            _check(self._lib.rs_get_buffer(self._h, BUF[name], out.ctypes.data, C.byref(n)))
        return out.reshape(-1, width) if width > 1 else out

    def set_buffer(self, name: str, data: np.ndarray):
        data = np.ascontiguousarray(data)
        _check(self._lib.rs_set_buffer(self._h, BUF[name], data.ctypes.data, data.nbytes))

    def keep_candidates(self, keep: bool = True):
        _check(self._lib.rs_debug_keep_candidates(self._h, 1 if keep else 0))

    def enable_stage_timing(self, enable: bool = True):
        _check(self._lib.rs_enable_stage_timing(self._h, 1 if enable else 0))

    def stage_rays(self) -> dict:
        """{stage: (closest-hit queries, visibility queries)} of the last stage-timed frame; empty unless
        the library was built with ray counting (build.py build_ray_stats)."""
        cnt = C.c_uint32(64)
        rays = np.zeros(128, np.uint64)
        _check(self._lib.rs_debug_stage_rays(self._h, rays.ctypes.data, C.byref(cnt)))
        names = list(self.stage_times().keys())
        return {names[i]: (int(rays[2 * i]), int(rays[2 * i + 1])) for i in range(min(cnt.value, len(names)))}

    def stage_times(self) -> dict:
        cnt = C.c_uint32(64)
        ms = (C.c_float * 64)()
        names = C.create_string_buffer(4096)
        _check(self._lib.rs_get_stage_times(self._h, ms, C.byref(cnt), names, 4096))
        labels = names.raw.split(b"\0")[: cnt.value]
        out = {}
        for k, v in zip(labels, ms[: cnt.value]):
            out[k.decode()] = out.get(k.decode(), 0.0) + float(v)
        return out

    def last_launch_count(self) -> int:
        return int(self._lib.rs_last_launch_count(self._h))

    # ---- path-replay adjoint (no reference counterpart)
    def set_materials(self, materials: np.ndarray):
        """Replaces the scene's material records (n x 16 float32, the rs_material layout)."""
        m = np.ascontiguousarray(materials, np.float32)
        _check(self._lib.rs_set_materials(self._h, m.ctypes.data, len(m)))

    def checkpoint_bytes(self) -> int:
        n = C.c_size_t(0)
        _check(self._lib.rs_checkpoint_bytes(self._h, C.byref(n)))
        return int(n.value)

    def checkpoint(self, dst_ptr: int, stream: int = 0):
        """Copies the last frame's final reservoirs to device memory at dst_ptr."""
        _check(self._lib.rs_checkpoint(self._h, C.c_void_p(dst_ptr), C.c_void_p(stream)))

    def backward(self, grad_color_ptr: int, grad_materials_ptr: int, checkpoint_ptr: int | None = None, stream: int = 0):
        """gradMaterials (device, n x 8 float32) += d loss / d parameters for d loss / d colour."""
        _check(self._lib.rs_backward(self._h, C.c_void_p(checkpoint_ptr) if checkpoint_ptr else None,
                                     C.c_void_p(grad_color_ptr), C.c_void_p(grad_materials_ptr), C.c_void_p(stream)))

    # ---- moving geometry
    def update_geometry(self, positions, stream: int = 0):
        """Moves the triangles for the next frame: positions is a host array (n x 9 float32) or a
        CUDA tensor of the same shape."""
        if hasattr(positions, "data_ptr"):
            assert positions.is_cuda and positions.dtype.itemsize == 4 and positions.is_contiguous()
            _check(self._lib.rs_update_geometry(self._h, C.c_void_p(positions.data_ptr()), positions.numel() // 9, 1, C.c_void_p(stream)))
        else:
            q = np.ascontiguousarray(positions, np.float32).reshape(-1, 9)
            _check(self._lib.rs_update_geometry(self._h, q.ctypes.data, len(q), 0, C.c_void_p(stream)))

    # ---- ray-query diagnostics
    def trace_rays(self, rays: np.ndarray):
        """Closest hits of rays (n x 8 float32: origin, direction, tMin, tMax): prim, tuv, counts."""
        r = np.ascontiguousarray(rays, np.float32).reshape(-1, 8)
        n = len(r)
        prim = np.empty(n, np.int32)
        tuv = np.empty((n, 3), np.float32)
        counts = np.empty((n, 2), np.uint32)
        _check(self._lib.rs_debug_trace_rays(self._h, r.ctypes.data, n, prim.ctypes.data, tuv.ctypes.data, counts.ctypes.data))
        return prim, tuv, counts

    def set_bvh_builder(self, builder: str):
        """Binary-tree builder of the next set_scene: "PLOC" (default) or "LBVH" (Karras radix tree)."""
        _check(self._lib.rs_set_bvh_builder(self._h, {"PLOC": 0, "LBVH": 1}[builder]))

    def bvh_shape(self) -> dict:
        out = np.zeros(6, np.float64)
        _check(self._lib.rs_debug_bvh_shape(self._h, out.ctypes.data))
        return dict(zip(["nodes", "depth", "internal_children", "leaf_children", "leaf_triangles", "sah_cost"], out.tolist()))

    def backward_stats(self) -> np.ndarray:
        """Counters since the last read: replayed, suffixes held fixed (not replayable), emitter not found, value mismatch."""
        out = np.zeros(4, np.uint64)
        _check(self._lib.rs_backward_stats(self._h, out.ctypes.data))
        return out


class Batch:
    """Renders one frame of several passes with one CUDA graph launch (rs_batch_execute).

    Members in the same ScatterBackup/Clamped configuration run the flattened form (one persistent
    launch per stage over all members); `flatten=False` forces one graph branch per member.
    `tuning_cache` names a JSON file of stage tile widths and grid forms: read when the batch is made,
    written by `tune()`, keyed by the GPU name so that another GPU model tunes again."""

    def __init__(self, passes, flatten: bool = True, tuning_cache: str | None = None):
        self._lib = load_library()
        self.passes = list(passes)
        arr = (C.c_void_p * len(self.passes))(*[p._h.value for p in self.passes])
        h = C.c_void_p()
        _check(self._lib.rs_batch_create(arr, len(self.passes), C.byref(h)))
        self._h = h
        self.flatten = flatten
        _check(self._lib.rs_batch_set_flatten(self._h, 1 if flatten else 0))
        self.tuning_cache = tuning_cache
        if tuning_cache:
            self._load_tuning()

    def _frames(self, cameras, color_ptrs, should_reset=False):
        frames = (abi.RsFrameDesc * len(self.passes))()
        for f, cam, ptr in zip(frames, cameras, color_ptrs):
            f.camera = abi.camera_struct(cam)
            f.color = ptr
            f.sceneShouldReset = 1 if should_reset else 0
        return frames

    def execute(self, cameras, color_ptrs, stream: int = 0, should_reset: bool = False):
        _check(self._lib.rs_batch_execute(self._h, self._frames(cameras, color_ptrs, should_reset), C.c_void_p(stream)))

    def tune(self, cameras, color_ptrs, stream: int = 0) -> list:
        """Renders one frame while timing every stage's tile widths and grid forms (rs_batch_tune),
        keeps the fastest and, with a tuning cache, writes it."""
        _check(self._lib.rs_batch_tune(self._h, self._frames(cameras, color_ptrs), C.c_void_p(stream)))
        entries = self.tuning()
        if self.tuning_cache:
            self._save_tuning(entries)
        return entries

    def choose_form(self, camera_frames, color_ptrs, stream: int = 0) -> dict:
        """Renders the frames of `camera_frames` (a list of per-member camera lists, an even number of
        frames) alternately in the flattened form and as per-member graph branches, times each on the
        device, and keeps the faster form (stored with the tuning cache).  Both forms render the same
        images, so the choice changes only the speed."""
        import torch
        times = {True: 0.0, False: 0.0}
        for k, cams in enumerate(camera_frames):
            form = k % 2 == 0
            _check(self._lib.rs_batch_set_flatten(self._h, 1 if form else 0))
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s = torch.cuda.ExternalStream(stream) if stream else torch.cuda.current_stream()
            a.record(s)
            self.execute(cams, color_ptrs, stream)
            b.record(s)
            torch.cuda.synchronize()
            times[form] += a.elapsed_time(b)
        self.flatten = times[True] <= times[False]
        _check(self._lib.rs_batch_set_flatten(self._h, 1 if self.flatten else 0))
        if self.tuning_cache:
            self._save_tuning(self.tuning())
        return {"flattened_ms": times[True], "branches_ms": times[False], "flatten": self.flatten}

    def tuning(self) -> list:
        n = C.c_uint32(0)
        _check(self._lib.rs_batch_get_tuning(self._h, None, C.byref(n)))
        arr = (abi.RsBatchTuningEntry * n.value)()
        _check(self._lib.rs_batch_get_tuning(self._h, arr, C.byref(n)))
        return [{"stage": abi.BATCH_STAGES[e.stage], "width": e.width, "height": e.height, "tile": e.tile, "grid": e.grid,
                 "ms": round(float(e.ms), 4)} for e in arr]

    def set_tuning(self, entries: list):
        arr = (abi.RsBatchTuningEntry * len(entries))()
        for a, e in zip(arr, entries):
            a.stage = abi.BATCH_STAGES.index(e["stage"])
            a.width, a.height = int(e["width"]), int(e["height"])
            a.tile, a.grid, a.ms = int(e["tile"]), int(e["grid"]), float(e.get("ms", 0.0))
        _check(self._lib.rs_batch_set_tuning(self._h, arr, len(entries)))

    @staticmethod
    def _gpu_key() -> str:
        try:
            import torch
            return torch.cuda.get_device_name()
        except Exception:
            return "unknown"

    def _load_tuning(self):
        import json
        from pathlib import Path
        path = Path(self.tuning_cache)
        if path.exists():
            data = json.loads(path.read_text()).get(self._gpu_key())
            if data:
                self.set_tuning(data["entries"])
                self.flatten = bool(data.get("flatten", self.flatten))
                _check(self._lib.rs_batch_set_flatten(self._h, 1 if self.flatten else 0))

    def _save_tuning(self, entries):
        import json
        from pathlib import Path
        path = Path(self.tuning_cache)
        data = json.loads(path.read_text()) if path.exists() else {}
        data[self._gpu_key()] = {"entries": entries, "flatten": self.flatten}
        path.write_text(json.dumps(data, indent=1))

    def set_flatten(self, enable: bool):
        self.flatten = bool(enable)
        _check(self._lib.rs_batch_set_flatten(self._h, 1 if enable else 0))

    def last_flattened(self) -> bool:
        return bool(self._lib.rs_batch_last_flattened(self._h))

    def launch_count(self) -> int:
        return int(self._lib.rs_batch_launch_count(self._h))

    def close(self):
        if getattr(self, "_h", None):
            self._lib.rs_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def createPass(name: str, props: dict | None = None, width: int = 1920, height: int = 1080) -> ReservoirSplatting:
    """Falcor-style factory: createPass("ReservoirSplatting", {...})."""
    if name != "ReservoirSplatting":
        raise ValueError(f"unknown pass {name!r}")
    return ReservoirSplatting(props, width, height)
