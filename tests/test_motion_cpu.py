"""Moving geometry on the CPU oracle: motion vectors read the previous frame's positions
(Scene::getPrevPosW, VBufferRT.slang:84) while everything else reads the current ones."""
import numpy as np


PROPS = {"temporalReuse": "ScatterBackup", "maxSurfaceBounces": 1, "enableSpatialResampling": False}


def _translated(cam, dx):
    import dataclasses
    return dataclasses.replace(cam, position=(cam.position[0] + dx, cam.position[1], cam.position[2]),
                               target=(cam.target[0] + dx, cam.target[1], cam.target[2]))


def test_unmoved_update_changes_nothing(oracle_mod, scenes):
    sc = scenes.cornell_box(0)
    a = oracle_mod.OraclePass(PROPS, 24, 24); a.set_scene(sc)
    b = oracle_mod.OraclePass(PROPS, 24, 24); b.set_scene(sc)
    for f in range(3):
        cam = scenes.cornell_camera(f, 24, 24)
        b.update_geometry(sc.positions)
        np.testing.assert_array_equal(a.execute(cam), b.execute(cam))
        np.testing.assert_array_equal(a.get_buffer("mvec"), b.get_buffer("mvec"))


def test_geometry_moving_with_the_camera_has_no_motion(oracle_mod, scenes):
    """Scene and camera translated together: every surface point keeps its screen position, so
    the motion vectors vanish; the camera alone moving gives the ordinary camera motion."""
    sc = scenes.cornell_box(0)
    cam0 = scenes.cornell_camera(0, 32, 32)
    p = oracle_mod.OraclePass(PROPS, 32, 32)
    p.set_scene(sc)
    p.execute(cam0)
    shift = np.tile(np.array([0.05, 0.0, 0.0], np.float32), 3)
    p.update_geometry(sc.positions + shift)
    p.execute(_translated(cam0, 0.05))
    mv = p.get_buffer("mvec")
    hit = p.get_buffer("vbuffer")[:, 0] != 0
    assert hit.sum() > 100
    assert np.abs(mv[hit]).max() < 1e-4
    q = oracle_mod.OraclePass(PROPS, 32, 32)
    q.set_scene(sc)
    q.execute(cam0)
    q.execute(_translated(cam0, 0.05))
    mq = q.get_buffer("mvec")
    assert np.abs(mq[hit]).max() > 1e-3


def test_sphere_motion_moves_only_the_chosen_spheres(scenes):
    sc = scenes.terrain_spheres(seed=2, grid=16, spheres=6, subdiv=1, lights=2, extent=20.0, height=2.0)
    m = scenes.SphereMotion(sc, moving=3, max_speed=0.05, seed=1)
    d = m.positions(10) - m.positions(0)
    moved = np.abs(d).max(1) > 0
    per = sc.info["sphere_triangles_each"]
    assert moved.sum() <= 3 * per and moved.sum() > 0
    assert not moved[: sc.info["terrain_triangles"]].any()
    assert np.abs(d[:, 1::3]).max() == 0.0  # motion in the ground plane
    assert np.linalg.norm(d[moved][:, :3], axis=1).max() <= 0.5 + 1e-5
