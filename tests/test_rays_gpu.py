"""The CUDA ray-query layer (PLOC binary tree for closest hits, 4-wide tree for visibility) against the
oracle's median-split tree, ray by ray through rs_debug_trace_rays: the closest hit is the (t, scene
index) minimum over all triangles the exact test accepts, so both trees must return the same
triangle and the same t, u, v bits, whatever their topology.  The oracle tree itself is checked
against brute force in test_oracle_cpu.py."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def _rays(scene, rng, n):
    tri = np.asarray(scene.positions, np.float32).reshape(-1, 3, 3)
    lo, hi = tri.reshape(-1, 3).min(0), tri.reshape(-1, 3).max(0)
    out = []
    # random rays from outside and inside the scene box
    o = rng.uniform(lo - 2.0, hi + 2.0, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    out.append(np.concatenate([o, d / np.linalg.norm(d, axis=1, keepdims=True), np.zeros((n, 1)), np.full((n, 1), 1e30)], 1))
    # axis-parallel directions (zero components) and negative zeros
    k = n // 4
    o = rng.uniform(lo, hi, (k, 3)).astype(np.float32)
    axes = np.eye(3, dtype=np.float32)[rng.integers(0, 3, k)] * rng.choice([-1.0, 1.0], (k, 1)).astype(np.float32)
    axes[axes == 0] = rng.choice([0.0, -0.0], int((axes == 0).sum())).astype(np.float32)
    out.append(np.concatenate([o, axes, np.zeros((k, 1)), np.full((k, 1), 1e30)], 1))
    # rays aimed exactly at vertices and edge midpoints of random triangles
    t = tri[rng.integers(0, len(tri), k)]
    tgt = np.where(rng.random((k, 1)) < 0.5, t[:, 0], 0.5 * (t[:, 0] + t[:, 1]))
    o = rng.uniform(lo - 1.0, hi + 1.0, (k, 3)).astype(np.float32)
    d = tgt - o
    out.append(np.concatenate([o, d / np.linalg.norm(d, axis=1, keepdims=True), np.zeros((k, 1)), np.full((k, 1), 1e30)], 1))
    # rays leaving triangle centroids along the normal and along the surface, with bounded t
    t = tri[rng.integers(0, len(tri), k)]
    c = t.mean(1)
    nrm = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True) + 1e-30
    tang = (t[:, 1] - t[:, 0]) / (np.linalg.norm(t[:, 1] - t[:, 0], axis=1, keepdims=True) + 1e-30)
    d = np.where(rng.random((k, 1)) < 0.5, nrm, tang)
    out.append(np.concatenate([c, d, np.full((k, 1), 1e-4), rng.uniform(0.1, 50.0, (k, 1))], 1))
    return np.ascontiguousarray(np.concatenate(out).astype(np.float32))


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("which", ["cornell", "terrain"])
@pytest.mark.parametrize("builder", ["PLOC", "LBVH"])
def test_closest_hits_match_the_oracle_tree(rs, oracle_mod, scenes, which, builder):
    sc = scenes.cornell_box(0) if which == "cornell" else scenes.terrain_spheres(seed=9, grid=64, spheres=20, subdiv=2, lights=8,
                                                                                   extent=30.0, height=3.0)
    p = rs.ReservoirSplatting({"maxSurfaceBounces": 1}, 16, 16)
    p.set_bvh_builder(builder)
    p.set_scene(sc)
    ora = oracle_mod.OraclePass({"maxSurfaceBounces": 1}, 16, 16)
    ora.set_scene(sc)
    lib = oracle_mod.load()
    lib.ro_test_closest.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ro_test_closest.restype = C.c_int
    rays = _rays(sc, np.random.default_rng(3), 4000)
    prim, tuv, counts = p.trace_rays(rays)
    assert (prim >= 0).sum() > len(rays) // 4
    for i in range(len(rays)):
        tv = np.zeros(3, np.float32)
        q = np.ascontiguousarray(rays[i])
        op = lib.ro_test_closest(ora._h, q.ctypes.data, tv.ctypes.data)
        assert op == prim[i], (i, rays[i], op, prim[i])
        if op >= 0:
            np.testing.assert_array_equal(tv, tuv[i], err_msg=f"ray {i}")
    shape = p.bvh_shape()
    assert shape["leaf_triangles"] == sc.num_triangles
    p.close()


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_nan_rays_miss_without_traversal(rs, oracle_mod, scenes):
    """A NaN in the origin, direction or interval (a NaN camera time makes such rays) hits nothing
    and visits no node, on the GPU and in the oracle alike."""
    sc = scenes.terrain_spheres(seed=9, grid=64, spheres=20, subdiv=2, lights=8, extent=30.0, height=3.0)
    p = rs.ReservoirSplatting({"maxSurfaceBounces": 1}, 16, 16)
    p.set_scene(sc)
    ora = oracle_mod.OraclePass({"maxSurfaceBounces": 1}, 16, 16)
    ora.set_scene(sc)
    lib = oracle_mod.load()
    lib.ro_test_closest.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ro_test_closest.restype = C.c_int
    base = np.array([0.0, 10.0, 0.0, 0.0, -1.0, 0.0, 0.0, 1e30], np.float32)  # straight down onto the terrain
    rays = np.tile(base, (9, 1))
    for k in range(8):
        rays[k + 1, k] = np.nan
    prim, tuv, counts = p.trace_rays(rays)
    assert prim[0] >= 0 and counts[0, 0] > 0
    assert (prim[1:] == -1).all() and (counts[1:] == 0).all()
    for i in range(1, len(rays)):
        tv = np.zeros(3, np.float32)
        assert lib.ro_test_closest(ora._h, np.ascontiguousarray(rays[i]).ctypes.data, tv.ctypes.data) == -1
    p.close()
