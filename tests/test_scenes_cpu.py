"""Seeded procedural scenes: sizes, determinism and emitter orientation."""
import numpy as np


def _normals(pos):
    p0, p1, p2 = pos[:, 0:3], pos[:, 3:6], pos[:, 6:9]
    n = np.cross(p1 - p0, p2 - p0)
    return n / np.linalg.norm(n, axis=1, keepdims=True)


def test_cornell_box_layout(scenes):
    sc = scenes.cornell_box(0)
    assert sc.num_triangles == 36
    mats = sc.materials
    light = np.nonzero(mats[:, 4:7].sum(1) > 0)[0]
    assert len(light) == 1
    lt = sc.positions[sc.material_ids == light[0]]
    assert len(lt) == 2
    np.testing.assert_allclose(_normals(lt), [[0, -1, 0], [0, -1, 0]], atol=1e-6)
    np.testing.assert_allclose(mats[light[0], 4:7], [17, 12, 4])
    area = 0.5 * np.linalg.norm(np.cross(lt[:, 3:6] - lt[:, 0:3], lt[:, 6:9] - lt[:, 0:3]), axis=1).sum()
    assert area == np.float32(0.0625)


def test_terrain_scene_counts_and_determinism(scenes):
    a = scenes.terrain_spheres(seed=5, grid=32, spheres=6, subdiv=2, lights=5)
    b = scenes.terrain_spheres(seed=5, grid=32, spheres=6, subdiv=2, lights=5)
    assert a.num_triangles == 2 * 31 * 31 + 6 * 20 * 4 ** 2 + 5
    np.testing.assert_array_equal(a.positions, b.positions)
    np.testing.assert_array_equal(a.materials, b.materials)
    c = scenes.terrain_spheres(seed=6, grid=32, spheres=6, subdiv=2, lights=5)
    assert not np.array_equal(a.positions, c.positions)
    lights = np.nonzero(a.materials[:, 4:7].sum(1) > 0)[0]
    em = a.positions[np.isin(a.material_ids, lights)]
    assert len(em) == 5 and (_normals(em)[:, 1] < -0.99).all()
    rough = a.materials[1:7, 3]
    assert ((rough >= 0.1) & (rough <= 0.8)).all()


def test_headline_scene_size(scenes):
    info = scenes.terrain_spheres(seed=1, grid=512, spheres=500, subdiv=4, lights=64).info
    assert info["terrain_triangles"] == 2 * 511 * 511
    assert info["sphere_triangles_each"] == 20 * 4 ** 4
    assert info["triangles"] == 522242 + 500 * 5120 + 64


def test_camera_paths(scenes):
    c0, c1 = scenes.cornell_camera(0, 64, 64), scenes.cornell_camera(1, 64, 64)
    assert c1.position[0] - c0.position[0] == np.float64(0.01) or abs(c1.position[0] - c0.position[0] - 0.01) < 1e-12
    o0, o1 = scenes.orbit_camera(0, 64, 64), scenes.orbit_camera(1, 64, 64)
    a0 = np.degrees(np.arctan2(o0.position[2], o0.position[0]))
    a1 = np.degrees(np.arctan2(o1.position[2], o1.position[0]))
    assert abs((a1 - a0) - 0.5) < 1e-9
