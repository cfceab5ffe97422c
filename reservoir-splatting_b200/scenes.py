"""Seeded procedural scenes and camera paths for the Reservoir Splatting pass.

The reference renders Falcor scene files (``media/test_scenes/cornell_box.pyscene``
and the like, ``README.md:17``); those are not part of its repository, so the
workloads here are generated from a seed with the shapes, sizes and value
ranges of the benchmark configurations:

* ``cornell_box``: a Cornell-style room (5 walls, two boxes rotated +-18 degrees,
  a 0.25 x 0.25 ceiling light of radiance (17, 12, 4)), 36 triangles.
* ``terrain_spheres``: an fBm heightfield terrain plus instanced icospheres with
  per-object GGX roughness and albedo, and small emissive triangles above the
  terrain.

Every scene is a flattened world-space triangle soup (``positions`` float32
[T, 9], ``material_ids`` uint32 [T]) plus a material table (float32 [M, 16] in
the ``rs_material`` layout).  Materials are Falcor StandardMaterial metal-rough
parameters: base colour, roughness, metallic, emissive radiance, IoR.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

MATERIAL_FLOATS = 16
DOUBLE_SIDED = 1
SPEC_GLOSS = 2


def material(base=(0.73, 0.73, 0.73), roughness=1.0, emissive=(0.0, 0.0, 0.0), metallic=0.0, ior=1.5, double_sided=True):
    """Metal-rough StandardMaterial parameters in the rs_material layout."""
    m = np.zeros(MATERIAL_FLOATS, np.float32)
    m[0:3] = base
    m[3] = roughness
    m[4:7] = emissive
    m[7] = metallic
    m[8] = ior
    m[9] = np.frombuffer(np.uint32(DOUBLE_SIDED if double_sided else 0).tobytes(), np.float32)[0]
    return m


def spec_gloss_material(diffuse=(0.73, 0.73, 0.73), specular=(0.0, 0.0, 0.0), glossiness=0.0, emissive=(0.0, 0.0, 0.0), ior=1.5,
                        double_sided=False):
    """Spec-gloss StandardMaterial parameters (ShadingModel::SpecGloss): the roughness slot holds the
    glossiness, metallic is derived from the two colours when the material is shaded."""
    m = np.zeros(MATERIAL_FLOATS, np.float32)
    m[0:3] = diffuse
    m[3] = glossiness
    m[4:7] = emissive
    m[8] = ior
    m[9] = np.frombuffer(np.uint32(SPEC_GLOSS | (DOUBLE_SIDED if double_sided else 0)).tobytes(), np.float32)[0]
    m[10:13] = specular
    return m


@dataclasses.dataclass
class Scene:
    positions: np.ndarray      # float32 [T, 9]
    material_ids: np.ndarray   # uint32 [T]
    materials: np.ndarray      # float32 [M, 16]
    name: str = ""
    info: dict = dataclasses.field(default_factory=dict)

    @property
    def num_triangles(self) -> int:
        return int(self.positions.shape[0])


@dataclasses.dataclass
class Camera:
    position: tuple
    target: tuple
    up: tuple = (0.0, 1.0, 0.0)
    focal_length: float = 35.0
    frame_height: float = 24.0
    aspect_ratio: float = 1.0
    focal_distance: float = 10000.0
    aperture_radius: float = 0.0
    shutter_speed: float = 0.0
    near_z: float = 0.1
    far_z: float = 1000.0


def _quad(p0, p1, p2, p3):
    """Two triangles (p0, p1, p2), (p0, p2, p3); normal = (p1 - p0) x (p2 - p0)."""
    return [np.concatenate([p0, p1, p2]), np.concatenate([p0, p2, p3])]


def _box(center, size, angle_deg):
    """Axis-aligned box rotated about +Y, outward winding; 12 triangles."""
    cx, cy, cz = center
    sx, sy, sz = size
    a = math.radians(angle_deg)
    c, s = math.cos(a), math.sin(a)

    def P(x, y, z):
        x, z = x * sx / 2, z * sz / 2
        return np.array([cx + c * x + s * z, cy + y * sy, cz - s * x + c * z], np.float32)

    v = {k: P(*k) for k in [(-1, 0, -1), (1, 0, -1), (1, 0, 1), (-1, 0, 1), (-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1)]}
    t = []
    t += _quad(v[(-1, 1, -1)], v[(-1, 1, 1)], v[(1, 1, 1)], v[(1, 1, -1)])        # top (+y)
    t += _quad(v[(-1, 0, -1)], v[(1, 0, -1)], v[(1, 0, 1)], v[(-1, 0, 1)])        # bottom (-y)
    t += _quad(v[(-1, 0, 1)], v[(1, 0, 1)], v[(1, 1, 1)], v[(-1, 1, 1)])          # +z
    t += _quad(v[(1, 0, -1)], v[(-1, 0, -1)], v[(-1, 1, -1)], v[(1, 1, -1)])      # -z
    t += _quad(v[(1, 0, 1)], v[(1, 0, -1)], v[(1, 1, -1)], v[(1, 1, 1)])          # +x
    t += _quad(v[(-1, 0, -1)], v[(-1, 0, 1)], v[(-1, 1, 1)], v[(-1, 1, -1)])      # -x
    return t


def cornell_box(seed: int = 0) -> Scene:
    """Cornell-style unit room: 36 triangles, one 0.25 x 0.25 ceiling light."""
    rng = np.random.default_rng(seed)
    jitter = float(rng.uniform(-1e-3, 1e-3))  # the seed only nudges the boxes
    mats = np.stack([
        material((0.73, 0.73, 0.73)),             # 0 white
        material((0.65, 0.05, 0.05)),             # 1 red
        material((0.12, 0.45, 0.15)),             # 2 green
        material((0.0, 0.0, 0.0), emissive=(17.0, 12.0, 4.0), double_sided=False),  # 3 light
    ])
    P = lambda *a: np.array(a, np.float32)
    tris, mid = [], []

    def add(ts, m):
        tris.extend(ts)
        mid.extend([m] * len(ts))

    add(_quad(P(0, 0, 0), P(0, 0, 1), P(1, 0, 1), P(1, 0, 0)), 0)   # floor, +y
    add(_quad(P(0, 1, 0), P(1, 1, 0), P(1, 1, 1), P(0, 1, 1)), 0)   # ceiling, -y
    add(_quad(P(0, 0, 0), P(1, 0, 0), P(1, 1, 0), P(0, 1, 0)), 0)   # back wall, +z
    add(_quad(P(0, 0, 0), P(0, 1, 0), P(0, 1, 1), P(0, 0, 1)), 1)   # left wall (red), +x
    add(_quad(P(1, 0, 0), P(1, 0, 1), P(1, 1, 1), P(1, 1, 0)), 2)   # right wall (green), -x
    add(_box((0.33 + jitter, 0.0, 0.62), (0.3, 0.3, 0.3), 18.0), 0)
    add(_box((0.66, 0.0, 0.36 + jitter), (0.3, 0.6, 0.3), -18.0), 0)
    y = 0.999
    add(_quad(P(0.375, y, 0.375), P(0.625, y, 0.375), P(0.625, y, 0.625), P(0.375, y, 0.625)), 3)  # faces -y
    pos = np.stack(tris).astype(np.float32)
    return Scene(pos, np.array(mid, np.uint32), mats.astype(np.float32), "cornell_box",
                 {"triangles": len(pos), "emissive_triangles": 2})


def cornell_camera(frame: int, width: int, height: int) -> Camera:
    """Pinhole camera translating +x by 0.01 units per frame."""
    fov_y = math.radians(40.0)
    f = 0.5 * 24.0 / math.tan(0.5 * fov_y)
    x = 0.5 + 0.01 * frame
    return Camera((x, 0.5, 2.2), (x, 0.5, 0.0), focal_length=f, aspect_ratio=width / height)


def _icosphere(subdiv: int) -> np.ndarray:
    t = (1.0 + 5 ** 0.5) / 2.0
    v = [(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
         (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)]
    f = [(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6),
         (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7),
         (9, 8, 1)]
    V = np.array(v, np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    T = V[np.array(f)]  # [F, 3, 3]
    for _ in range(subdiv):
        a, b, c = T[:, 0], T[:, 1], T[:, 2]
        ab, bc, ca = a + b, b + c, c + a
        ab /= np.linalg.norm(ab, axis=1, keepdims=True)
        bc /= np.linalg.norm(bc, axis=1, keepdims=True)
        ca /= np.linalg.norm(ca, axis=1, keepdims=True)
        T = np.concatenate([np.stack([a, ab, ca], 1), np.stack([ab, b, bc], 1), np.stack([ca, bc, c], 1),
                            np.stack([ab, bc, ca], 1)])
    return T  # outward winding


def _fbm(n: int, rng: np.random.Generator, octaves: int = 6) -> np.ndarray:
    """Value-noise fBm on an n x n grid in [0, 1]."""
    h = np.zeros((n, n), np.float64)
    amp, total = 1.0, 0.0
    for o in range(octaves):
        cells = 4 * (2 ** o)
        g = rng.random((cells + 2, cells + 2))
        x = np.linspace(0, cells, n, endpoint=False)
        i = x.astype(np.int64)
        fr = x - i
        s = fr * fr * (3 - 2 * fr)
        g00 = g[i][:, i]
        g10 = g[i + 1][:, i]
        g01 = g[i][:, i + 1]
        g11 = g[i + 1][:, i + 1]
        sy = s[:, None]
        sx = s[None, :]
        h += amp * ((g00 * (1 - sx) + g01 * sx) * (1 - sy) + (g10 * (1 - sx) + g11 * sx) * sy)
        total += amp
        amp *= 0.5
    return h / total


def terrain_spheres(seed: int = 1, grid: int = 512, spheres: int = 500, subdiv: int = 4, lights: int = 64,
                    extent: float = 100.0, height: float = 10.0) -> Scene:
    """fBm terrain (grid x grid vertices) + `spheres` icospheres + `lights` emissive triangles."""
    rng = np.random.default_rng(seed)
    hmap = _fbm(grid, rng) * height
    xs = np.linspace(-extent / 2, extent / 2, grid)
    X, Z = np.meshgrid(xs, xs)
    P = np.stack([X, hmap, Z], -1)
    a, b, c, d = P[:-1, :-1], P[:-1, 1:], P[1:, 1:], P[1:, :-1]
    # winding so that (p1 - p0) x (p2 - p0) points up
    t1 = np.stack([a, c, b], 2).reshape(-1, 9)
    t2 = np.stack([a, d, c], 2).reshape(-1, 9)
    terrain = np.concatenate([t1, t2]).astype(np.float32)
    mats = [material((0.45, 0.42, 0.38), roughness=0.9)]
    mids = [np.zeros(len(terrain), np.uint32)]
    blocks = [terrain]
    ico = _icosphere(subdiv)
    for s in range(spheres):
        r = rng.uniform(0.2, 1.5)
        px, pz = rng.uniform(-0.45 * extent, 0.45 * extent, 2)
        gi = int((px + extent / 2) / extent * (grid - 1))
        gj = int((pz + extent / 2) / extent * (grid - 1))
        py = hmap[min(max(gj, 0), grid - 1), min(max(gi, 0), grid - 1)] + r * 0.8
        tri = (ico * r + np.array([px, py, pz])).reshape(-1, 9).astype(np.float32)
        mats.append(material(tuple(rng.uniform(0.2, 0.9, 3)), roughness=float(rng.uniform(0.1, 0.8))))
        blocks.append(tri)
        mids.append(np.full(len(tri), len(mats) - 1, np.uint32))
    for l in range(lights):
        cx, cz = rng.uniform(-0.45 * extent, 0.45 * extent, 2)
        cy = height + rng.uniform(4.0, 12.0)
        s = rng.uniform(1.0, 3.0)
        le = tuple(rng.uniform(5.0, 50.0, 3))
        p0 = (cx - s, cy, cz - s)
        p1 = (cx + s, cy, cz - s)
        p2 = (cx, cy, cz + s)
        blocks.append(np.array([p0 + p1 + p2], np.float32))   # (p1-p0)x(p2-p0) points down
        mats.append(material((0.0, 0.0, 0.0), emissive=le, double_sided=False))
        mids.append(np.array([len(mats) - 1], np.uint32))
    pos = np.concatenate(blocks).astype(np.float32)
    info = {"triangles": int(len(pos)), "terrain_triangles": int(len(terrain)),
            "sphere_triangles_each": int(len(ico)), "spheres": spheres, "emissive_triangles": lights}
    return Scene(pos, np.concatenate(mids), np.stack(mats).astype(np.float32), "terrain_spheres", info)


class SphereMotion:
    """Linear motion of some of terrain_spheres' icospheres: sphere s moves by velocity[s] per frame
    (uniform direction in the ground plane, speed U[0, max_speed]).  positions(frame) gives the
    scene's triangle soup (n x 9 float32) at that frame, for ReservoirSplatting.update_geometry."""

    def __init__(self, scene: Scene, moving: int = 200, max_speed: float = 0.05, seed: int = 0):
        info = scene.info
        self.base = np.ascontiguousarray(scene.positions, np.float32).reshape(-1, 9).copy()
        first = info["terrain_triangles"]
        per = info["sphere_triangles_each"]
        rng = np.random.default_rng(seed)
        moving = min(moving, info["spheres"])
        self.spheres = np.sort(rng.choice(info["spheres"], moving, replace=False))
        ang = rng.uniform(0.0, 2.0 * math.pi, moving)
        speed = rng.uniform(0.0, max_speed, moving)
        self.velocity = np.stack([speed * np.cos(ang), np.zeros(moving), speed * np.sin(ang)], 1).astype(np.float32)
        self.ranges = [(first + int(k) * per, per) for k in self.spheres]
        self.tri_velocity = np.zeros((len(self.base), 3), np.float32)
        for (a, n), v in zip(self.ranges, self.velocity):
            self.tri_velocity[a:a + n] = v

    def positions(self, frame: int) -> np.ndarray:
        return self.base + np.tile(self.tri_velocity * np.float32(frame), (1, 3))


def motion_blur_scene(seed: int = 3, grid: int = 800, spheres: int = 500, subdiv: int = 4, lights: int = 64):
    """terrain_spheres scaled to about 4M triangles (800 x 800 heightfield: 1.28M, 500 icospheres at
    subdivision 4: 2.56M, 64 emissive triangles)."""
    return terrain_spheres(seed=seed, grid=grid, spheres=spheres, subdiv=subdiv, lights=lights)


def inverse_scene(seed: int = 5, grid: int = 300, spheres: int = 16, subdiv: int = 3, materials: int = 32,
                  emitters: int = 8, extent: float = 60.0, height: float = 6.0) -> Scene:
    """Scene for differentiation: fBm terrain + icospheres sharing `materials` metal-rough materials
    (albedo U[0.2, 0.9] per channel, roughness U[0.1, 0.8], half of them with metallic U[0, 1]) and
    `emitters` emissive quads, each with its own material (radiance U[5, 50] per channel).
    The defaults give 199,298 triangles."""
    rng = np.random.default_rng(seed)
    hmap = _fbm(grid, rng) * height
    xs = np.linspace(-extent / 2, extent / 2, grid)
    X, Z = np.meshgrid(xs, xs)
    P = np.stack([X, hmap, Z], -1)
    a, b, c, d = P[:-1, :-1], P[:-1, 1:], P[1:, 1:], P[1:, :-1]
    t1 = np.stack([a, c, b], 2).reshape(-1, 9)
    t2 = np.stack([a, d, c], 2).reshape(-1, 9)
    terrain = np.concatenate([t1, t2]).astype(np.float32)
    mats = []
    for m in range(materials):
        metallic = float(rng.uniform(0.0, 1.0)) if m % 2 else 0.0
        mats.append(material(tuple(rng.uniform(0.2, 0.9, 3)), roughness=float(rng.uniform(0.1, 0.8)), metallic=metallic))
    # terrain in bands of the first four materials, spheres over the rest
    band = np.clip(((terrain[:, 0] + extent / 2) / extent * 4).astype(np.int64), 0, 3)
    blocks, mids = [terrain], [band.astype(np.uint32)]
    ico = _icosphere(subdiv)
    for s in range(spheres):
        r = rng.uniform(0.8, 3.0)
        px, pz = rng.uniform(-0.4 * extent, 0.4 * extent, 2)
        gi = int((px + extent / 2) / extent * (grid - 1))
        gj = int((pz + extent / 2) / extent * (grid - 1))
        py = hmap[min(max(gj, 0), grid - 1), min(max(gi, 0), grid - 1)] + r * 0.8
        tri = (ico * r + np.array([px, py, pz])).reshape(-1, 9).astype(np.float32)
        blocks.append(tri)
        mids.append(np.full(len(tri), 4 + s % (materials - 4), np.uint32))
    for e in range(emitters):
        cx, cz = rng.uniform(-0.4 * extent, 0.4 * extent, 2)
        cy = height + rng.uniform(6.0, 14.0)
        s = rng.uniform(1.5, 3.5)
        p0, p1, p2, p3 = (cx - s, cy, cz - s), (cx + s, cy, cz - s), (cx + s, cy, cz + s), (cx - s, cy, cz + s)
        blocks.append(np.array([p0 + p1 + p2, p0 + p2 + p3], np.float32))  # normals point down
        mats.append(material((0.0, 0.0, 0.0), emissive=tuple(rng.uniform(5.0, 50.0, 3)), double_sided=False))
        mids.append(np.full(2, len(mats) - 1, np.uint32))
    pos = np.concatenate(blocks).astype(np.float32)
    info = {"triangles": int(len(pos)), "materials": materials, "emitters": emitters}
    return Scene(pos, np.concatenate(mids), np.stack(mats).astype(np.float32), "inverse_scene", info)


def orbit_camera(frame: int, width: int, height: int, degrees_per_frame: float = 0.5, radius: float = 60.0,
                 height_above: float = 22.0, fov_y_deg: float = 45.0) -> Camera:
    """Camera orbiting the scene centre at `degrees_per_frame`."""
    a = math.radians(30.0 + degrees_per_frame * frame)
    f = 0.5 * 24.0 / math.tan(0.5 * math.radians(fov_y_deg))
    return Camera((radius * math.cos(a), height_above, radius * math.sin(a)), (0.0, 2.0, 0.0), focal_length=f,
                  aspect_ratio=width / height, far_z=10000.0)


def translate_camera(frame: int, width: int, height: int, step: float = 0.05) -> Camera:
    f = 0.5 * 24.0 / math.tan(0.5 * math.radians(45.0))
    return Camera((-20.0 + step * frame, 18.0, 40.0), (-20.0 + step * frame, 2.0, 0.0), focal_length=f,
                  aspect_ratio=width / height, far_z=10000.0)


def sky_env_map(width: int = 256, height: int = 128, seed: int = 0, sun_dir=(0.4, 0.6, -0.5), sun_radiance: float = 40.0,
                sun_radius_deg: float = 6.0) -> np.ndarray:
    """A seeded lat-long sky float32 [height, width, 3] in the layout rs_set_env_map reads (row 0 at
    the top, u = 0.5 looking along -z): a blue-to-white gradient above the horizon, dim ground below,
    a bright sun disc around `sun_dir`, and a little seeded per-texel noise so the importance map is
    not smooth."""
    rng = np.random.default_rng(seed)
    v = (np.arange(height, dtype=np.float64) + 0.5) / height
    u = (np.arange(width, dtype=np.float64) + 0.5) / width
    theta = np.pi * v[:, None]                     # 0 = up
    phi = np.pi * (2.0 * u[None, :] - 1.0)
    d = np.stack([np.sin(theta) * np.sin(phi), np.cos(theta) * np.ones_like(phi), -np.sin(theta) * np.cos(phi)], -1)
    up = d[..., 1]
    sky = np.where(up[..., None] > 0, np.array([0.35, 0.55, 1.0]) * (1 - up[..., None]) + np.array([1.0, 1.0, 1.0]) * up[..., None],
                   np.array([0.18, 0.16, 0.14]))
    s = np.asarray(sun_dir, np.float64)
    s = s / np.linalg.norm(s)
    cosang = np.clip(d @ s, -1.0, 1.0)
    sun = (cosang > math.cos(math.radians(sun_radius_deg)))[..., None] * sun_radiance * np.array([1.0, 0.9, 0.75])
    img = sky + sun + rng.uniform(0.0, 0.05, (height, width, 3))
    return img.astype(np.float32)
