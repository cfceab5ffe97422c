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


PBRT_SCENE = """# a small PBRT v4 scene
LookAt 0 1 -5   0 1 0   0 1 0
Camera "perspective" "float fov" [ 40 ]
Film "rgb" "integer xresolution" [64] "integer yresolution" [48] "string filename" "x.exr"
WorldBegin
LightSource "infinite" "rgb L" [0.2 0.3 0.5] "float scale" 2
MakeNamedMaterial "floor" "string type" "diffuse" "rgb reflectance" [0.7 0.6 0.5]
AttributeBegin
  NamedMaterial "floor"
  Shape "trianglemesh" "point3 P" [-5 0 -5  5 0 -5  5 0 5  -5 0 5] "integer indices" [0 1 2 0 2 3]
AttributeEnd
AttributeBegin
  AreaLightSource "diffuse" "rgb L" [4 4 3] "float scale" 2
  Translate 0 3 0
  Shape "bilinearmesh" "point3 P" [-1 0 -1  1 0 -1  -1 0 1  1 0 1]
AttributeEnd
AttributeBegin
  Material "conductor" "rgb eta" [0.2 0.9 1.1] "rgb k" [3.9 2.4 2.2] "float roughness" 0.08
  Translate 1 1 0
  Shape "sphere" "float radius" 0.5
AttributeEnd
ObjectBegin "quad"
  Material "coateddiffuse" "rgb reflectance" [0.2 0.8 0.2] "float roughness" 0.1
  Shape "plymesh" "string filename" "quad.ply"
ObjectEnd
AttributeBegin
  Translate -1 0.5 0
  ObjectInstance "quad"
AttributeEnd
AttributeBegin
  Translate -2 0.5 0
  Rotate 90 0 1 0
  ObjectInstance "quad"
AttributeEnd
Include "more.pbrt"
"""


def _write_pbrt(tmp_path, binary_ply=False):
    (tmp_path / "scene.pbrt").write_text(PBRT_SCENE)
    (tmp_path / "more.pbrt").write_text('Material "dielectric" "float eta" 1.33\nShape "trianglemesh" "point3 P" [0 0 1 1 0 1 0 1 1]\n')
    verts = np.array([[0, 0, 0], [0.5, 0, 0], [0.5, 0.5, 0], [0, 0.5, 0]], np.float32)
    if binary_ply:
        head = ("ply\nformat binary_little_endian 1.0\nelement vertex 4\nproperty float x\nproperty float y\nproperty float z\n"
                "element face 1\nproperty list uchar int vertex_indices\nend_header\n").encode()
        body = verts.tobytes() + bytes([4]) + np.array([0, 1, 2, 3], "<i4").tobytes()
        (tmp_path / "quad.ply").write_bytes(head + body)
    else:
        (tmp_path / "quad.ply").write_text("ply\nformat ascii 1.0\nelement vertex 4\nproperty float x\nproperty float y\nproperty float z\n"
                                          "element face 1\nproperty list uchar int vertex_indices\nend_header\n"
                                          + "\n".join(" ".join(str(float(c)) for c in v) for v in verts) + "\n4 0 1 2 3\n")
    return tmp_path / "scene.pbrt"


@pytest.mark.parametrize("binary_ply", [False, True])
def test_pbrt_scene(rs, tmp_path, binary_ply):
    import reservoir_splatting_b200.importers as I
    sc = I.load_pbrt(_write_pbrt(tmp_path, binary_ply))
    # floor 2 + light quad 2 + icosphere 1280 + two instanced PLY quads 2 x 2 + included triangle 1
    assert sc.positions.shape == (1289, 9) and sc.material_ids.shape == (1289,)
    m = sc.materials
    floor, light, metal, coated, glass = (m[sc.material_ids[i]] for i in (0, 2, 4, 1284, 1288))
    assert np.allclose(floor[:3], [0.7, 0.6, 0.5]) and floor[3] == 1.0 and floor[7] == 0.0
    assert np.allclose(light[4:7], [8, 8, 6]) and np.allclose(light[:3], 0.5)
    eta, k = np.array([0.2, 0.9, 1.1]), np.array([3.9, 2.4, 2.2])
    assert np.allclose(metal[:3], ((eta - 1) ** 2 + k ** 2) / ((eta + 1) ** 2 + k ** 2), rtol=1e-6) and metal[7] == 1.0
    # getRoughness as written: sqrt(u + v), then the StandardMaterial takes its square root
    assert abs(metal[3] - np.sqrt(np.sqrt(0.16))) < 1e-6 and abs(coated[3] - np.sqrt(np.sqrt(0.2))) < 1e-6
    assert abs(glass[8] - 1.33) < 1e-6 and np.allclose(glass[:3], 0.0)
    # the light quad is moved up by 3, the rotated instance lies in the x = -2 plane
    assert np.allclose(sc.positions[2:4, 1::3], 3.0)
    inst = sc.positions[1286:1288].reshape(-1, 3)
    assert np.allclose(inst[:, 0], -2.0, atol=1e-6) and inst[:, 1].min() >= 0.5 - 1e-6
    cam = sc.info["camera"]
    assert np.allclose(cam["position"], [0, 1, -5]) and np.allclose(cam["target"], [0, 1, -4]) and cam["fovDegrees"] == 40.0
    assert sc.info["env"].shape[2] == 3 and np.allclose(sc.info["env"][0, 0], [0.4, 0.6, 1.0])
    c = I.pbrt_camera(sc, 64, 48)
    assert abs(2 * np.degrees(np.arctan(0.5 * c.frame_height / c.focal_length)) - 40.0) < 1e-9


def test_pbrt_rejects_what_it_does_not_convert(rs, tmp_path):
    import reservoir_splatting_b200.importers as I
    for body in ('Shape "disk"', 'Material "measured"\nShape "sphere"',
                 'LightSource "infinite" "string filename" "sky.exr"'):
        p = tmp_path / "bad.pbrt"
        p.write_text("WorldBegin\n" + body + "\n")
        with pytest.raises(ValueError):
            I.load_pbrt(p)


def test_pbrt_lights(rs, tmp_path):
    """createLight (PBRTImporter.cpp:643-700): a distant light becomes a directional analytic light
    (L * scale * illuminance, direction = transformed to - from); point and spot lights are skipped
    with a warning, as the reference importer does."""
    import reservoir_splatting_b200.importers as I
    p = tmp_path / "lights.pbrt"
    p.write_text('WorldBegin\nAttributeBegin\nRotate 90 0 0 1\n'
                 'LightSource "distant" "rgb L" [1 2 3] "float scale" 2 "float illuminance" 1.5 "point3 from" [0 0 0] "point3 to" [1 0 0]\n'
                 'AttributeEnd\nLightSource "point" "rgb I" [1 1 1]\nLightSource "spot" "rgb I" [1 1 1]\n'
                 'Shape "trianglemesh" "point3 P" [0 0 0 1 0 0 0 1 0]\n')
    with pytest.warns(UserWarning, match="not supported"):
        sc = I.load_pbrt(p)
    (L,) = sc.info["lights"]
    assert L["type"] == "directional" and np.allclose(L["intensity"], [3, 6, 9])
    assert np.allclose(L["direction"], [0, 1, 0], atol=1e-12)  # +x rotated by 90 degrees about z
    m = tmp_path / "lights.xml"
    m.write_text('<scene version="3.0.0"><emitter type="point"/><shape type="rectangle"/></scene>')
    with pytest.warns(UserWarning, match="not supported"):
        I.load_mitsuba(m)


MITSUBA_SCENE = """<scene version="3.0.0">
  <default name="spp" value="16"/>
  <default name="wall" value="0.6"/>
  <sensor type="perspective">
    <float name="fov" value="35"/>
    <transform name="to_world"><lookat origin="0, 1, -6" target="0, 1, 0" up="0, 1, 0"/></transform>
  </sensor>
  <emitter type="constant"><rgb name="radiance" value="0.1, 0.2, 0.3"/></emitter>
  <bsdf type="twosided" id="white"><bsdf type="diffuse"><rgb name="reflectance" value="$wall"/></bsdf></bsdf>
  <shape type="rectangle">
    <transform name="to_world"><scale value="4"/><rotate x="1" angle="90"/></transform>
    <ref id="white"/>
  </shape>
  <shape type="rectangle">
    <transform name="to_world"><rotate x="1" angle="90"/><translate y="3"/></transform>
    <emitter type="area"><rgb name="radiance" value="5, 4, 3"/></emitter>
  </shape>
  <shape type="cube">
    <transform name="to_world"><scale value="0.5"/><translate x="1" y="0.5"/></transform>
    <bsdf type="roughconductor"><rgb name="eta" value="0.2, 0.9, 1.1"/><rgb name="k" value="3.9, 2.4, 2.2"/><float name="alpha" value="0.2"/></bsdf>
  </shape>
  <shape type="sphere">
    <point name="center" value="-1, 0.5, 0"/><float name="radius" value="0.4"/>
    <bsdf type="roughplastic"><rgb name="diffuse_reflectance" value="0.1, 0.3, 0.8"/><float name="alpha" value="0.3"/><string name="int_ior" value="bk7"/></bsdf>
  </shape>
  <shape type="obj"><string name="filename" value="tri.obj"/><bsdf type="dielectric"><float name="int_ior" value="1.33"/></bsdf></shape>
</scene>
"""


def _write_mitsuba(tmp_path):
    (tmp_path / "scene.xml").write_text(MITSUBA_SCENE)
    (tmp_path / "tri.obj").write_text("v 0 0 2\nv 1 0 2\nv 0 1 2\nf 1 2 3\n")
    return tmp_path / "scene.xml"


def test_mitsuba_scene(rs, tmp_path):
    import reservoir_splatting_b200.importers as I
    sc = I.load_mitsuba(_write_mitsuba(tmp_path))
    # floor 2 + light 2 + cube 12 + icosphere 1280 + obj 1
    assert sc.positions.shape == (1297, 9)
    m = sc.materials[sc.material_ids]
    floor, light, cube, ball, glass = m[0], m[2], m[4], m[16], m[1296]
    assert np.allclose(floor[:3], 0.6) and floor[3] == 1.0
    # rectangle rotated about x by 90 degrees, scaled by 4: it lies in y = 0 with x, z in [-4, 4]
    assert np.allclose(sc.positions[0:2, 1::3], 0.0, atol=1e-6) and np.abs(sc.positions[0:2, 0::3]).max() == 4.0
    assert np.allclose(light[4:7], [5, 4, 3]) and np.allclose(sc.positions[2:4, 1::3], 3.0, atol=1e-6)
    eta, k = np.array([0.2, 0.9, 1.1]), np.array([3.9, 2.4, 2.2])
    assert np.allclose(cube[:3], ((eta - 1) ** 2 + k ** 2) / ((eta + 1) ** 2 + k ** 2), rtol=1e-6)
    assert cube[7] == 1.0 and abs(cube[3] - np.sqrt(0.2)) < 1e-6
    cube_pts = sc.positions[4:16].reshape(-1, 3)
    assert np.allclose(cube_pts.min(0), [0.5, 0.0, -0.5]) and np.allclose(cube_pts.max(0), [1.5, 1.0, 0.5])
    assert np.allclose(ball[:3], [0.1, 0.3, 0.8]) and abs(ball[3] - np.sqrt(0.3)) < 1e-6 and abs(ball[8] - 1.5046 / 1.00028) < 1e-5
    assert abs(glass[8] - 1.33 / 1.00028) < 1e-5
    cam = sc.info["camera"]
    assert np.allclose(cam["position"], [0, 1, -6]) and np.allclose(cam["target"], [0, 1, -5]) and cam["fovDegrees"] == 35.0
    assert np.allclose(sc.info["env"][0, 0], [0.1, 0.2, 0.3])


def test_mitsuba_rejects_what_it_does_not_convert(rs, tmp_path):
    import reservoir_splatting_b200.importers as I
    for body in ('<shape type="disk"/>', '<emitter type="envmap"><string name="filename" value="sky.exr"/></emitter>',
                 '<shape type="cube"><bsdf type="hair"/></shape>'):
        p = tmp_path / "bad.xml"
        p.write_text(f'<scene version="3.0.0">{body}</scene>')
        with pytest.raises(ValueError):
            I.load_mitsuba(p)


PYSCENE = """
white = StandardMaterial('white')
white.baseColor = float4(0.7, 0.7, 0.7, 1.0)
white.roughness = 0.8
light = StandardMaterial('light')
light.emissiveColor = float3(1.0, 0.9, 0.8)
light.emissiveFactor = 10.0
metal = Material('metal')
metal.specularParams = float4(0.0, 0.3, 1.0, 0.0)
plain = StandardMaterial('plain')

floor = sceneBuilder.addTriangleMesh(TriangleMesh.createQuad(), white)
lamp = sceneBuilder.addTriangleMesh(TriangleMesh.createQuad(float2(0.25)), light)
box = sceneBuilder.addTriangleMesh(TriangleMesh.createCube(float3(0.3)), metal)
ball = sceneBuilder.addTriangleMesh(TriangleMesh.createSphere(0.2, 16, 8), plain)
disk = sceneBuilder.addTriangleMesh(TriangleMesh.createDisk(0.5, 12), white)

t = Transform(); t.scaling = float3(2.0, 1.0, 2.0)
sceneBuilder.addMeshInstance(sceneBuilder.addNode('floor', t), floor)
t = Transform(); t.translation = float3(0.0, 1.0, 0.0); t.rotationEulerDeg = float3(180.0, 0.0, 0.0)
sceneBuilder.addMeshInstance(sceneBuilder.addNode('lamp', t), lamp)
g = Transform(); g.translation = float3(0.0, 0.0, -0.5)
root = sceneBuilder.addNode('group', g)
t = Transform(); t.translation = float3(0.3, 0.15, 0.0)
sceneBuilder.addMeshInstance(sceneBuilder.addNode('box', t, root), box)
t = Transform(); t.translation = float3(-0.3, 0.2, 0.0); t.scaling = float3(-1.0, 1.0, 1.0)
sceneBuilder.addMeshInstance(sceneBuilder.addNode('ball', t, root), ball)
t = Transform(); t.lookAt(float3(0.0, 0.5, 0.9), float3(1.0, 0.5, 0.9), float3(0.0, 1.0, 0.0))
sceneBuilder.addMeshInstance(sceneBuilder.addNode('wall', t), disk)

spot = PointLight('spot')
spot.position = float3(0.0, 0.9, 0.0)
spot.openingAngle = 0.6
spot.intensity = float3(2.0, 2.0, 2.0)
sceneBuilder.addLight(spot)
sun = DistantLight('sun')
sun.direction = float3(0.2, -1.0, 0.1)
sceneBuilder.addLight(sun)
off = DirectionalLight('off')
off.active = False
sceneBuilder.addLight(off)

camera = Camera()
camera.position = float3(0.0, 0.5, 2.5)
camera.target = float3(0.0, 0.4, 0.0)
camera.focalLength = 30.0
sceneBuilder.addCamera(camera)
"""


def test_pyscene_scene(rs, tmp_path):
    """A Falcor Python scene (PythonImporter): TriangleMesh generators with Falcor's layouts, node
    hierarchies, Transform (T x R x S, Euler degrees, lookAt), a mirrored instance, StandardMaterial
    parameters and defaults, analytic lights and the camera."""
    import reservoir_splatting_b200.importers as I
    p = tmp_path / "room.pyscene"
    p.write_text(PYSCENE)
    sc = I.load_pyscene(p)
    # quad 2 + quad 2 + cube 12 + sphere 16 x 8 x 2 + disk 12
    assert sc.positions.shape == (2 + 2 + 12 + 256 + 12, 9)
    t = sc.positions.reshape(-1, 3, 3).astype(np.float64)
    n = np.cross(t[:, 1] - t[:, 0], t[:, 2] - t[:, 0])
    assert np.all(n[0:2, 1] > 0) and np.all(n[2:4, 1] < 0)  # createQuad faces +y; the lamp is turned over
    assert np.allclose(np.abs(t[0:2, :, [0, 2]]).max(), 1.0)  # scaled by 2 in x and z
    assert np.allclose(t[2:4, :, 1], 1.0)
    box = t[4:16].reshape(-1, 3)
    assert np.allclose(box.min(0), [0.15, 0.0, -0.65]) and np.allclose(box.max(0), [0.45, 0.3, -0.35])  # parent and child
    cb = box.mean(0)
    assert np.all(np.einsum("ij,ij->i", n[4:16], t[4:16].mean(1) - cb) > 0)  # the cube's faces point out
    ball = t[16:272]
    centre = np.array([-0.3, 0.2, -0.5])
    assert np.allclose(np.linalg.norm(ball.reshape(-1, 3) - centre, axis=1), 0.2, atol=1e-6)
    outward = np.einsum("ij,ij->i", n[16:272], ball.mean(1) - centre)
    big = np.linalg.norm(n[16:272], axis=1) > 1e-9
    # the sphere's own winding faces outward; mirroring keeps it outward (Falcor flips the normal of
    # a mirrored instance)
    assert np.all(outward[big] > 0) or np.all(outward[big] < 0)
    p2 = tmp_path / "room2.pyscene"
    p2.write_text(PYSCENE.replace("t.scaling = float3(-1.0, 1.0, 1.0)", ""))
    n2 = (lambda tt: np.cross(tt[:, 1] - tt[:, 0], tt[:, 2] - tt[:, 0]))(I.load_pyscene(p2).positions.reshape(-1, 3, 3).astype(np.float64))
    out2 = np.einsum("ij,ij->i", n2[16:272], I.load_pyscene(p2).positions.reshape(-1, 3, 3)[16:272].mean(1) - centre)
    assert np.all(np.sign(outward[big]) == np.sign(out2[big]))
    disk = t[272:]
    # lookAt toward +x: columns (right, up, -dir) = (+z, +y, -x), so the disk stays level at y = 0.5
    # and its first rim vertex, object (r, 0, 0), lands at position + r * right
    assert np.allclose(disk[:, :, 1], 0.5, atol=1e-6) and np.all(n[272:, 1] > 0)
    assert np.allclose(disk[0, 1], [0.0, 0.5, 1.4], atol=1e-6)
    m = sc.materials
    white, light, metal, plain = m[0], m[1], m[2], m[3]
    assert np.allclose(white[:3], 0.7) and abs(white[3] - 0.8) < 1e-6
    assert np.allclose(light[4:7], [10.0, 9.0, 8.0]) and np.allclose(metal[[3, 7]], [0.3, 1.0])
    assert np.allclose(plain[:3], 1.0) and plain[3] == 0.0 and abs(plain[8] - 1.5) < 1e-6  # BasicMaterial defaults
    lights = sc.info["lights"]
    assert [l["type"] for l in lights] == ["point", "distant"]  # the inactive light is dropped
    assert lights[0]["openingAngle"] == 0.6 and np.allclose(lights[1]["direction"], [0.2, -1.0, 0.1])
    assert abs(lights[1]["angle"] - 0.5 * 0.53 * np.pi / 180.0) < 1e-9
    cam = I.pyscene_camera(sc, 64, 48)
    assert cam.focal_length == 30.0 and cam.frame_height == 24.0 and np.allclose(cam.position, [0.0, 0.5, 2.5])


def test_pyscene_rejects_what_it_does_not_convert(rs, tmp_path):
    import reservoir_splatting_b200.importers as I
    for body in ("g = SDFGrid.createSBS()", "sceneBuilder.envMap = EnvMap('sky.exr')",
                 "m = StandardMaterial('t')\nm.loadTexture(0, 'albedo.png')",
                 "m = StandardMaterial('t')\nsceneBuilder.addTriangleMesh(TriangleMesh.createFromFile('mesh.fbx'), m)",
                 "x = 1"):
        p = tmp_path / "bad.pyscene"
        p.write_text(body + "\n")
        with pytest.raises(ValueError):
            I.load_pyscene(p)


def _rgbe(img):
    """float [H, W, 3] -> RGBE bytes (mantissa = c * 2^(136 - e), the exponent of the largest channel)."""
    mx = img.max(-1)
    e = np.where(mx > 1e-32, np.floor(np.log2(np.maximum(mx, 1e-32))) + 1 + 128, 0).astype(np.int32)
    m = np.where(e[..., None] > 0, img * np.ldexp(1.0, 136 - e)[..., None], 0)
    return np.concatenate([np.clip(np.floor(m), 0, 255), e[..., None]], -1).astype(np.uint8)


def _write_hdr(path, img, rle):
    h, w = img.shape[:2]
    px = _rgbe(img)
    out = bytearray(b"#?RADIANCE\nFORMAT=32-bit_rle_rgbe\n\n" + f"-Y {h} +X {w}\n".encode())
    for y in range(h):
        if not rle:
            out += px[y].tobytes()
            continue
        out += bytes([2, 2, w >> 8, w & 255])
        for c in range(4):
            row, x = px[y, :, c], 0
            while x < w:
                n = 1
                while x + n < w and n < 127 and row[x + n] == row[x]:
                    n += 1
                if n >= 3:
                    out += bytes([128 + n, row[x]])
                else:
                    n = min(128, w - x)
                    out += bytes([n]) + row[x:x + n].tobytes()
                x += n
    path.write_bytes(bytes(out))
    e = px[..., 3].astype(np.int32)
    return np.where(e[..., None] > 0, px[..., :3] * np.ldexp(1.0, e - 136)[..., None], 0.0).astype(np.float32)


@pytest.mark.parametrize("rle", [False, True], ids=["flat", "rle"])
def test_hdr_and_pfm_environment_images(rs, tmp_path, rle):
    import reservoir_splatting_b200.importers as I
    rng = np.random.default_rng(1)
    img = (rng.uniform(0, 4, (6, 40, 3)) ** 2).astype(np.float32)
    img[2] = 1.5  # long runs of one value
    img[3, :5] = 0.0
    want = _write_hdr(tmp_path / "sky.hdr", img, rle)
    got = I.read_env_image(tmp_path / "sky.hdr")
    assert got.shape == (6, 40, 3) and np.array_equal(got, want)
    assert np.all(np.abs(got - img) <= img.max(-1, keepdims=True) / 64)  # 8-bit mantissas on the largest channel's exponent
    for scale, dt in ((-1.0, "<f4"), (1.0, ">f4")):
        body = np.ascontiguousarray(img[::-1]).astype(dt).tobytes()  # rows bottom to top
        (tmp_path / "sky.pfm").write_bytes(f"PF\n40 6\n{scale}\n".encode() + body)
        assert np.array_equal(I.read_env_image(tmp_path / "sky.pfm"), img)
    with pytest.raises(ValueError):
        I.read_env_image(tmp_path / "sky.exr")


def test_environment_maps_from_mitsuba_and_pyscene(rs, tmp_path):
    """Mitsuba envmap (MitsubaImporter.cpp:686-701: intensity = scale, rotation = the XYZ Euler angles
    of to_world x flipZ) and a pyscene EnvMap (rotation, intensity, tint)."""
    import reservoir_splatting_b200.importers as I
    img = np.full((4, 8, 3), 0.5, np.float32)
    _write_hdr(tmp_path / "sky.hdr", img, False)
    (tmp_path / "env.xml").write_text('<scene version="3.0.0"><emitter type="envmap"><string name="filename" value="sky.hdr"/>'
                                      '<float name="scale" value="2.5"/></emitter><shape type="rectangle"/></scene>')
    sc = I.load_mitsuba(tmp_path / "env.xml")
    assert np.allclose(sc.info["env"], 0.5) and sc.info["env_params"]["intensity"] == 2.5
    # identity to_world: flipZ alone, whose XYZ Euler angles are (-180, 0, -180) degrees
    assert np.allclose(sc.info["env_params"]["rotation"], (-180.0, 0.0, -180.0))
    (tmp_path / "env.pyscene").write_text("e = EnvMap('sky.hdr')\ne.intensity = 3.0\ne.rotation = float3(0, 90, 0)\n"
                                          "e.tint = float3(1, 0.5, 0.25)\nsceneBuilder.envMap = e\n"
                                          "sceneBuilder.addMeshInstance(sceneBuilder.addNode('q'), "
                                          "sceneBuilder.addTriangleMesh(TriangleMesh.createQuad(), StandardMaterial('m')))\n")
    sc = I.load_pyscene(tmp_path / "env.pyscene")
    assert sc.info["env"].shape == (4, 8, 3)
    assert sc.info["env_params"] == {"intensity": 3.0, "tint": (1.0, 0.5, 0.25), "rotation": (0.0, 90.0, 0.0)}


def _oct_to_dir(u, v):
    """Inverse equal-area octahedral map (Clarberg 2008), float64: unit square -> unit directions."""
    px, py = 2 * u - 1, 2 * v - 1
    d = 1 - (np.abs(px) + np.abs(py))
    r = 1 - np.abs(d)
    phi = np.where(r > 0, ((np.abs(py) - np.abs(px)) / np.where(r > 0, r, 1) + 1) * np.pi / 4, 0)
    f = r * np.sqrt(np.maximum(2 - r * r, 0))
    return np.stack([f * np.sign(px) * np.abs(np.cos(phi)), f * np.sign(py) * np.abs(np.sin(phi)), np.sign(d) * (1 - r * r)], -1)


def test_equal_area_octahedral_map_to_latlong(rs):
    """EnvMapConverter: the lat-long texel at direction w holds the octahedral map's value at w."""
    import reservoir_splatting_b200.importers as I
    n = 256
    c = (np.arange(n) + 0.5) / n
    dirs = _oct_to_dir(c[None, :], c[:, None])  # row y, column x
    f = lambda d: np.stack([1.5 + d[..., 0], 1.5 + d[..., 1], 1.5 + d[..., 2]], -1)
    ll = I.equal_area_oct_to_latlong(f(dirs).astype(np.float32))
    assert ll.shape == (n, 2 * n, 3)
    u = (np.arange(2 * n) + 0.5) / (2 * n)
    v = (np.arange(n) + 0.5) / n
    phi, th = np.pi * (2 * u[None, :] - 1), np.pi * v[:, None]
    w = np.stack([np.sin(th) * np.sin(phi), np.cos(th) * np.ones_like(phi), -np.sin(th) * np.cos(phi)], -1)
    err = np.abs(ll - f(w))
    assert np.median(err) < 2e-3 and np.quantile(err, 0.99) < 2e-2  # bilinear, apart from the map's folds


def test_pbrt_image_infinite_light(rs, tmp_path):
    import reservoir_splatting_b200.importers as I
    n = 32
    img = np.full((n, n, 3), 0.25, np.float32)
    (tmp_path / "sky.pfm").write_bytes(f"PF\n{n} {n}\n-1.0\n".encode() + img.astype("<f4").tobytes())
    p = tmp_path / "s.pbrt"
    p.write_text('WorldBegin\nAttributeBegin\nRotate 30 0 1 0\nLightSource "infinite" "string filename" "sky.pfm" "float scale" 4\n'
                 'AttributeEnd\nShape "trianglemesh" "point3 P" [0 0 0 1 0 0 0 1 0]\n')
    sc = I.load_pbrt(p)
    assert sc.info["env"].shape == (n, 2 * n, 3) and np.allclose(sc.info["env"], 0.25)
    ep = sc.info["env_params"]
    # Rotate 30 about +y: extractEulerAngleXYZ gives (0, 30, 0) degrees
    assert ep["intensity"] == 4.0 and np.allclose(ep["rotation"], (0.0, 30.0, 0.0), atol=1e-9), ep
