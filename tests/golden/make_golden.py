"""Generates the committed golden vectors in this directory.

* rng_kat.json: known-answer vectors of the per-pixel random streams, computed by
  the pure-Python restatement below (TEA, Morton interleave, the 32-bit LCG of
  Utils/Sampling/Pseudorandom/LCG.slang:50-56 with A = 1664525, C = 1013904223 -
  the constants the reference's PseudorandomTests.cpp pins - and PCG32).  The C++
  core is tested against these, so the vectors are independent of it.
* cornell_*.npz: oracle outputs (reservoirs, reconnection records, splat cell
  lists, colour) of the seeded Cornell box for fixed options; a regression pin of
  the oracle itself (any change to them must be explained).

Run from the repository root:  python tests/golden/make_golden.py
"""
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
M32 = 0xFFFFFFFF


def interleave_32bit(x, y):
    def spread(v):
        v &= 0xFFFF
        v = (v | (v << 8)) & 0x00FF00FF
        v = (v | (v << 4)) & 0x0F0F0F0F
        v = (v | (v << 2)) & 0x33333333
        v = (v | (v << 1)) & 0x55555555
        return v
    return spread(x) | (spread(y) << 1)


def tea16(v0, v1):
    s = 0
    for _ in range(16):
        s = (s + 0x9E3779B9) & M32
        v0 = (v0 + ((((v1 << 4) & M32) + 0xA341316C) ^ ((v1 + s) & M32) ^ ((v1 >> 5) + 0xC8013EA4))) & M32
        v1 = (v1 + ((((v0 << 4) & M32) + 0xAD90777D) ^ ((v0 + s) & M32) ^ ((v0 >> 5) + 0x7E95761E))) & M32
    return v0, v1


def tiny_uniform(px, py, seed, n):
    state = tea16(interleave_32bit(px, py), seed)[0]
    out = []
    for _ in range(n):
        state = (1664525 * state + 1013904223) & M32
        out.append(state)
    return out


def pcg32(px, py, seed, n):
    M64 = (1 << 64) - 1
    mult, inc = 6364136223846793005, 1442695040888963407
    v0, v1 = tea16(interleave_32bit(px, py), seed)
    init = (v0 << 32) | v1
    state = 0
    state = (state * mult + inc) & M64
    state = (state + init) & M64
    state = (state * mult + inc) & M64
    out = []
    for _ in range(n):
        old = state
        state = (old * mult + inc) & M64
        xs = (((old >> 18) ^ old) >> 27) & M32
        rot = old >> 59
        out.append(((xs >> rot) | (xs << ((32 - rot) & 31))) & M32)
    return out


CASES = [(0, 0, 0), (1, 0, 8), (255, 17, 1234), (1919, 1079, 8 * 61 + 6), (4095, 4095, 0xDEADBEEF)]


def make_rng():
    data = {"cases": []}
    for px, py, seed in CASES:
        data["cases"].append({"pixel": [px, py], "seed": seed, "interleave": interleave_32bit(px, py),
                              "tea": list(tea16(interleave_32bit(px, py), seed)),
                              "tiny_uniform": tiny_uniform(px, py, seed, 16), "pcg32": pcg32(px, py, seed, 16)})
    (HERE / "rng_kat.json").write_text(json.dumps(data, indent=1))


GOLDEN_RUNS = {
    "cornell_scatteronly": {"temporalReuse": "ScatterOnly", "maxSurfaceBounces": 1, "enableSpatialResampling": True},
    "cornell_scatterbackup": {"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "maxSurfaceBounces": 2,
                              "enableSpatialResampling": True},
}
GOLDEN_SIZE = 32
GOLDEN_FRAMES = 4


def run_oracle(props, frames=GOLDEN_FRAMES, size=GOLDEN_SIZE):
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle
    oracle._abi()
    import reservoir_splatting_b200.scenes as S
    p = oracle.OraclePass(props, size, size)
    p.set_scene(S.cornell_box(0))
    for f in range(frames):
        img = p.execute(S.cornell_camera(f, size, size))
    return {"color": img, "reservoirs": p.get_buffer("curr_reservoirs"), "reconnection": p.get_buffer("curr_reconnection"),
            "cell_counters": p.get_buffer("cell_counters"), "sorted_splats": p.get_buffer("sorted_splats")}


def make_oracle_golden():
    for name, props in GOLDEN_RUNS.items():
        np.savez_compressed(HERE / f"{name}.npz", **run_oracle(props))


if __name__ == "__main__":
    make_rng()
    make_oracle_golden()
    print("golden vectors written to", HERE)
