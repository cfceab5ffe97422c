"""ctypes wrapper of the CPU oracle (oracle/rs_oracle.cpp).

TEST INFRASTRUCTURE: used by tests/, the smoke check and the bench's CPU-baseline
leg only.  It mirrors the buffer names and layouts of the CUDA pass so a parity
test compares the same arrays.
"""
from __future__ import annotations

import ctypes as C
import importlib.util
import os
import subprocess
import sys
from pathlib import Path

import numpy as np

ORACLE_DIR = Path(__file__).resolve().parent
ORACLE_SO = ORACLE_DIR / "_build" / "librs_oracle.so"
PKG_DIR = ORACLE_DIR.parent / "reservoir-splatting_b200"


def _abi():
    name = "reservoir_splatting_b200.abi"
    if name in sys.modules:
        return sys.modules[name]
    if "reservoir_splatting_b200" not in sys.modules:
        spec = importlib.util.spec_from_file_location("reservoir_splatting_b200", PKG_DIR / "__init__.py",
                                                      submodule_search_locations=[str(PKG_DIR)])
        mod = importlib.util.module_from_spec(spec)
        sys.modules["reservoir_splatting_b200"] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def build(force: bool = False) -> Path:
    """Compiles the oracle with the host compiler (no contraction, IEEE float)."""
    src = ORACLE_DIR / "rs_oracle.cpp"
    deps = [src] + sorted((PKG_DIR / "csrc" / "core").glob("*.h")) + [ORACLE_DIR.parent / "include" / "rs_b200.h"]
    if not force and ORACLE_SO.exists() and ORACLE_SO.stat().st_mtime >= max(d.stat().st_mtime for d in deps):
        return ORACLE_SO
    ORACLE_SO.parent.mkdir(exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O2", "-fopenmp", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
           "-o", str(ORACLE_SO), str(src)]
    subprocess.run(cmd, check=True)
    return ORACLE_SO


_lib = None


def load():
    global _lib
    if _lib is not None:
        return _lib
    build()
    lib = C.CDLL(str(ORACLE_SO))
    a = _abi()
    lib.ro_create.argtypes = [C.POINTER(a.RsOptions)]
    lib.ro_create.restype = C.c_void_p
    lib.ro_destroy.argtypes = [C.c_void_p]
    lib.ro_set_threads.argtypes = [C.c_int]
    lib.ro_set_threads.restype = C.c_int
    lib.ro_set_scene.argtypes = [C.c_void_p, C.POINTER(a.RsSceneDesc)]
    lib.ro_set_env_map.argtypes = [C.c_void_p, C.POINTER(a.RsEnvMap)]
    lib.ro_set_analytic_lights.argtypes = [C.c_void_p, C.POINTER(a.RsAnalyticLight), C.c_uint32]
    lib.ro_get_env_importance.argtypes = [C.c_void_p, C.c_void_p]
    lib.ro_env_debug.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p]
    lib.ro_execute.argtypes = [C.c_void_p, C.POINTER(a.RsFrameDesc), C.c_void_p, C.c_void_p]
    lib.ro_freeze.argtypes = [C.c_void_p, C.c_int]
    lib.ro_reset.argtypes = [C.c_void_p]
    lib.ro_get_buffer.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
    lib.ro_get_buffer.restype = C.c_long
    lib.ro_set_buffer.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_size_t]
    lib.ro_frame_count.argtypes = [C.c_void_p]
    lib.ro_frame_count.restype = C.c_uint32
    lib.ro_set_materials.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
    lib.ro_update_geometry.argtypes = [C.c_void_p, C.c_void_p, C.c_uint32]
    lib.ro_backward.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ro_replay_loss.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32]
    lib.ro_replay_loss.restype = C.c_double
    lib.ro_test_bsdf_grad.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_uint32, C.c_void_p, C.c_void_p]
    _lib = lib
    return lib


def set_threads(n: int) -> int:
    return load().ro_set_threads(n)


class OraclePass:
    """CPU restatement of one ReservoirSplatting pass instance."""

    def __init__(self, props: dict | None = None, width: int = 256, height: int = 256, options=None):
        self._lib = load()
        a = _abi()
        self._abi = a
        self.options = options if options is not None else a.options_from_properties(props, width, height)
        self.width, self.height = self.options.frameWidth, self.options.frameHeight
        self._h = self._lib.ro_create(C.byref(self.options))

    def __del__(self):
        try:
            if self._h:
                self._lib.ro_destroy(self._h)
                self._h = None
        except Exception:
            pass

    def set_scene(self, scene):
        desc, keep = self._abi.scene_struct(scene)
        st = self._lib.ro_set_scene(self._h, C.byref(desc))
        if st != 0:
            raise RuntimeError(f"oracle set_scene failed: {st}")

    def set_env_map(self, texels, intensity: float = 1.0, tint=(1.0, 1.0, 1.0), rotation=(0.0, 0.0, 0.0)):
        desc, keep = self._abi.env_map_struct(texels, intensity, tint, rotation)
        st = self._lib.ro_set_env_map(self._h, C.byref(desc))
        del keep
        if st != 0:
            raise RuntimeError(f"oracle set_env_map failed: {st}")

    def set_analytic_lights(self, lights):
        lights = list(lights or [])
        st = self._lib.ro_set_analytic_lights(self._h, self._abi.analytic_lights_array(lights), len(lights))
        if st != 0:
            raise RuntimeError(f"oracle set_analytic_lights failed: {st}")

    def env_importance(self) -> np.ndarray:
        """The importance mips (512^2 .. 1 texels back to back)."""
        out = np.empty(349525, np.float32)
        st = self._lib.ro_get_env_importance(self._h, out.ctypes.data)
        if st != 0:
            raise RuntimeError("no env map set")
        return out

    def env_samples(self, rnd: np.ndarray) -> np.ndarray:
        """[n, 11]: sampled dir.xyz, pdf, Le.xyz, then evalPdf(dir) and eval(dir).xyz, for rnd [n, 2]."""
        rnd = np.ascontiguousarray(rnd, np.float32)
        out = np.empty((len(rnd), 11), np.float32)
        st = self._lib.ro_env_debug(self._h, rnd.ctypes.data, len(rnd), out.ctypes.data)
        if st != 0:
            raise RuntimeError("no env map set")
        return out

    def execute(self, camera, mvec: np.ndarray | None = None, should_reset: bool = False) -> np.ndarray:
        f = self._abi.RsFrameDesc()
        f.camera = self._abi.camera_struct(camera)
        f.sceneShouldReset = 1 if should_reset else 0
        out = np.empty((self.height, self.width, 4), np.float32)
        mp = None
        if mvec is not None:
            mvec = np.ascontiguousarray(mvec, np.float32)
            mp = mvec.ctypes.data
        st = self._lib.ro_execute(self._h, C.byref(f), mp, out.ctypes.data)
        if st != 0:
            raise RuntimeError(f"oracle execute failed: {st}")
        return out

    def freeze(self, frozen: bool = True):
        self._lib.ro_freeze(self._h, 1 if frozen else 0)

    def reset(self):
        self._lib.ro_reset(self._h)

    def get_buffer(self, name: str) -> np.ndarray:
        bid = self._abi.BUF[name]
        n = self._lib.ro_get_buffer(self._h, bid, None, 0)
        if n < 0:
            raise KeyError(name)
        dtype, width = self._abi.BUFFER_LAYOUT[name]
        out = np.empty(n // 4, dtype)
        if n:
            self._lib.ro_get_buffer(self._h, bid, out.ctypes.data, n)
        return out.reshape(-1, width) if width > 1 else out

    def set_buffer(self, name: str, data: np.ndarray):
        data = np.ascontiguousarray(data)
        st = self._lib.ro_set_buffer(self._h, self._abi.BUF[name], data.ctypes.data, data.nbytes)
        if st != 0:
            raise RuntimeError(f"oracle set_buffer failed: {st}")

    def update_geometry(self, positions: np.ndarray):
        """Moves the triangles (n x 9 float32) for the next frame."""
        q = np.ascontiguousarray(positions, np.float32).reshape(-1, 9)
        st = self._lib.ro_update_geometry(self._h, q.ctypes.data, len(q))
        if st != 0:
            raise RuntimeError(f"oracle update_geometry failed: {st}")

    # ---- path-replay adjoint (checker of rs_backward)
    def set_materials(self, materials: np.ndarray):
        m = np.ascontiguousarray(materials, np.float32)
        st = self._lib.ro_set_materials(self._h, m.ctypes.data, len(m))
        if st != 0:
            raise RuntimeError(f"oracle set_materials failed: {st}")

    def backward(self, grad_color: np.ndarray, num_materials: int):
        """Analytic replay gradient of the last frame: (num_materials x 8 float64, stats[4])."""
        g = np.ascontiguousarray(grad_color, np.float32).reshape(-1, 4)
        out = np.zeros((num_materials, 8), np.float64)
        stats = np.zeros(4, np.uint64)
        st = self._lib.ro_backward(self._h, g.ctypes.data, out.ctypes.data, stats.ctypes.data)
        if st != 0:
            raise RuntimeError(f"oracle backward failed: {st}")
        return out, stats

    def replay_loss(self, target: np.ndarray, params: np.ndarray) -> float:
        """FP64 replay loss of the last frame at `params` (materials x 8 float64: baseColor.xyz,
        roughness, emissive.xyz, metallic); the detached terms stay at the pass's materials."""
        t = np.ascontiguousarray(target, np.float32).reshape(-1, 4)
        q = np.ascontiguousarray(params, np.float64)
        return float(self._lib.ro_replay_loss(self._h, t.ctypes.data, q.ctypes.data, len(q)))


def bsdf_grad(material, wi, wo, lobe_mask: int = 0, specular=None):
    """(value, dBase, dRough) in FP32, the FP64 value and dMetal in FP32, for the BSDF derivative
    check.  material:
    baseColor.xyz, roughness, metallic, ior; with `specular` (a colour) the material is spec-gloss
    and material[3] its glossiness."""
    lib = load()
    m = np.zeros(10, np.float32)
    m[:len(material)] = material
    if specular is not None:
        m[6] = 1.0
        m[7:10] = specular
    a, b = np.asarray(wi, np.float32), np.asarray(wo, np.float32)
    out = np.zeros(12, np.float32)
    vd = np.zeros(3, np.float64)
    lib.ro_test_bsdf_grad(m.ctypes.data, a.ctypes.data, b.ctypes.data, lobe_mask, out.ctypes.data, vd.ctypes.data)
    return out[0:3], out[3:6], out[6:9], vd, out[9:12]
