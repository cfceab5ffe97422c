"""OBJ/MTL import with the material mapping of the reference's Assimp importer
(AssimpImporter.cpp:66-73, 845-935): spec-gloss materials, Phong exponent to glossiness,
`.doublesided` names, fan triangulation and negative indices."""
import math

import numpy as np
import pytest


def _u32(x):
    return int(np.float32(x).view(np.uint32))


def test_obj_faces_and_materials(rs, tmp_path):
    import reservoir_splatting_b200.importers as I
    (tmp_path / "s.mtl").write_text(
        "newmtl red\nKd 0.65 0.05 0.05\nKs 0.04 0.04 0.04\nNs 100\nNi 1.4\n\n"
        "newmtl lamp.doublesided\nKd 0 0 0\nKe 17 12 4\n# comment\n")
    (tmp_path / "s.obj").write_text(
        "mtllib s.mtl\n"
        "v 0 0 0\nv 1 0 0\nv 1 1 0\nv 0 1 0\nvt 0 0\nvn 0 0 1\n"
        "f 1 2 3\n"                      # before usemtl: default material
        "usemtl red\n"
        "f 1/1/1 2/1/1 3/1/1 4/1/1\n"    # quad -> two triangles (fan)
        "usemtl lamp.doublesided\n"
        "v 0 0 1\nv 1 0 1\nv 0 1 1\n"
        "f -3//1 -2//1 -1//1\n")
    sc = I.load_obj(tmp_path / "s.obj")
    assert sc.num_triangles == 4
    np.testing.assert_array_equal(sc.material_ids, [0, 1, 1, 2])
    np.testing.assert_array_equal(sc.positions[1], [0, 0, 0, 1, 0, 0, 1, 1, 0])
    np.testing.assert_array_equal(sc.positions[2], [0, 0, 0, 1, 1, 0, 0, 1, 0])
    np.testing.assert_array_equal(sc.positions[3], [0, 0, 1, 1, 0, 1, 0, 1, 1])
    red, lamp = sc.materials[1], sc.materials[2]
    np.testing.assert_allclose(red[0:3], [0.65, 0.05, 0.05])
    np.testing.assert_allclose(red[10:13], [0.04, 0.04, 0.04])
    gloss = np.float32(1) - np.float32(min(1.0, math.sqrt(2.0 / 102.0)))
    assert abs(red[3] - gloss) < 1e-6 and abs(red[8] - 1.4) < 1e-6
    assert _u32(red[9]) == 2             # spec-gloss, single sided
    assert _u32(lamp[9]) == 3            # spec-gloss, double sided
    np.testing.assert_allclose(lamp[4:7], [17, 12, 4])
    assert _u32(sc.materials[0][9]) == 2 and sc.materials[0][3] == 0.0  # default: grey, glossiness 0


def test_spec_power_to_roughness(rs):
    import reservoir_splatting_b200.importers as I
    assert I.spec_power_to_roughness(0.0) == 1.0
    assert abs(I.spec_power_to_roughness(98.0) - math.sqrt(0.02)) < 1e-7
    assert I.spec_power_to_roughness(-1.5) == 1.0  # clamped


def test_obj_round_trip_of_a_generated_scene(rs, scenes, tmp_path):
    import reservoir_splatting_b200.importers as I
    sc = scenes.cornell_box(0)
    I.save_obj(sc, tmp_path / "cb.obj", ["white", "red", "green", "light"],
               {"white": {"Kd": (0.73, 0.73, 0.73)}, "red": {"Kd": (0.65, 0.05, 0.05)}, "green": {"Kd": (0.12, 0.45, 0.15)},
                "light": {"Kd": (0, 0, 0), "Ke": (17, 12, 4)}})
    back = I.load_obj(tmp_path / "cb.obj")
    np.testing.assert_array_equal(back.positions, sc.positions)
    np.testing.assert_array_equal(back.material_ids, sc.material_ids)
    np.testing.assert_array_equal(back.materials[:, 0:3], sc.materials[:, 0:3])
    np.testing.assert_array_equal(back.materials[:, 4:7], sc.materials[:, 4:7])


def test_empty_obj_is_rejected(rs, tmp_path):
    import reservoir_splatting_b200.importers as I
    (tmp_path / "e.obj").write_text("v 0 0 0\n")
    with pytest.raises(ValueError):
        I.load_obj(tmp_path / "e.obj")
