"""Builds the sm_100a CUDA library lib/librs_b200.so with nvcc (in-tree, no JIT cache).

Flags that the parity contract depends on: -fmad=false (no contraction on the
device), -prec-div=true -prec-sqrt=true (IEEE division and square root) and
-ffp-contract=off for the host compiler, so host and device round identically.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "lib" / "librs_b200.so"
SOURCES = ["kernels.cu", "pass.cu", "bvh_build.cu", "bvh_debug.cu", "cells_static.cu", "frame_output.cu", "radix_sort.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-fmad=false", "-prec-div=true", "-prec-sqrt=true",
         "-Xcompiler", "-fPIC,-ffp-contract=off,-fvisibility=hidden", "-shared"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _deps():
    return [CSRC / s for s in SOURCES] + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + \
        sorted((CSRC / "core").glob("*.h")) + [PKG.parent / "include" / "rs_b200.h"]


def build(force: bool = False, verbose: bool = False, lib: Path = LIB, defines=()) -> Path:
    """Compiles every source to an object in parallel (they are separate translation units either
    way: no relocatable device code), then links the shared library."""
    if not force and lib.exists() and lib.stat().st_mtime >= max(p.stat().st_mtime for p in _deps()):
        return lib
    lib.parent.mkdir(exist_ok=True)
    objdir = lib.parent / ("_obj_" + lib.stem)
    objdir.mkdir(exist_ok=True)
    compile_flags = [f for f in FLAGS if f != "-shared"]
    procs = []
    for src in SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        cmd = [nvcc()] + ARCH + compile_flags + [f"-D{d}" for d in defines] + ["-c", "-o", str(obj), str(CSRC / src)]
        if verbose:
            print(" ".join(cmd))
        procs.append((subprocess.Popen(cmd, cwd=str(CSRC)), obj))
    failed = [p.args for p, _ in procs if p.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    cmd = [nvcc()] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-o", str(lib)] + [str(o) for _, o in procs]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True, cwd=str(CSRC))
    return lib


# The same library with ray-query counters (RS_RAY_STATS): for workload measurement only, the
# counting atomics and per-stage synchronisation make it slower.
LIB_RAY_STATS = PKG / "lib" / "librs_b200_raystats.so"


def build_ray_stats(force: bool = False, verbose: bool = False) -> Path:
    return build(force, verbose, LIB_RAY_STATS, ("RS_RAY_STATS",))


if __name__ == "__main__":
    print(build(force=True, verbose=True))
