"""The analytic light layer of the shared core (csrc/core/analytic_lights.h) against float64 numpy
restatements written from Falcor's formulas: the host-side light data of Scene/Lights/Light.cpp
(spot cone cosine, distant-light rotation, area-light transform, inverse transpose and surface
area) and the per-type samples of Rendering/Lights/LightHelpers.slang:67-284.  Plus the property
that pins the area lights' solid-angle pdf independently: the mean of 1/pdf over uniform samples
is the solid angle the light's front side subtends (Van Oosterom and Strackee's triangle formula)."""
import ctypes as C
import math

import numpy as np
import pytest

REL = 2e-5  # float32 core against float64


@pytest.fixture(scope="module")
def hook(oracle_mod, rs):
    lib = oracle_mod.load()
    lib.ro_test_analytic.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    lib.ro_test_analytic.restype = C.c_int
    abi = rs.abi

    def run(light: dict, x, u=(0.5, 0.5)):
        arr = abi.analytic_lights_array([light])
        pos = np.asarray(x, np.float32)
        uu = np.asarray(u, np.float32)
        out = np.zeros(40, np.float32)
        ok = lib.ro_test_analytic(C.addressof(arr), pos.ctypes.data, uu.ctypes.data, out.ctypes.data)
        if not ok:
            return None
        return {"ok": out[0] != 0, "posW": out[1:4], "normalW": out[4:7], "dir": out[7:10], "distance": out[10], "Li": out[11:14],
                "pdf": out[14], "cosOpening": out[15], "penumbra": out[16], "cosSubtended": out[17], "area": out[18],
                "M": out[19:31].reshape(3, 4), "MIT": out[31:40].reshape(3, 3)}
    return run


def close(a, b, rel=REL, abs_=1e-6):
    a = np.asarray(a, np.float64); b = np.asarray(b, np.float64)
    return np.all(np.abs(a - b) <= abs_ + rel * np.maximum(np.abs(a), np.abs(b)))


def smoothstep(a, b, x):
    t = min(max((x - a) / (b - a), 0.0), 1.0)
    return t * t * (3.0 - 2.0 * t)


def area_matrix(rng):
    """A random object-to-world transform (rotation, translation) and scaling."""
    q, _ = np.linalg.qr(rng.normal(size=(3, 3)))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    T = np.eye(4)
    T[:3, :3] = q
    T[:3, 3] = rng.uniform(-2, 2, 3)
    return T, rng.uniform(0.3, 1.5, 3)


def test_point_and_spot_lights(hook):
    rng = np.random.default_rng(1)
    for _ in range(200):
        d = rng.normal(size=3)
        light = {"type": "point", "intensity": rng.uniform(0.5, 4, 3), "position": rng.uniform(-3, 3, 3), "direction": d,
                 "openingAngle": rng.uniform(0.2, 3.3), "penumbraAngle": rng.uniform(0.0, 0.6)}
        x = rng.uniform(-3, 3, 3)
        r = hook(light, x)
        open_ = min(max(light["openingAngle"], 0.0), math.pi)
        pen = min(max(light["penumbraAngle"], 0.0), open_)
        assert close(r["cosOpening"], math.cos(np.float32(open_)), 1e-6)
        dirW = d / np.linalg.norm(d)
        to = np.asarray(light["position"], np.float64) - x
        d2 = max(to @ to, 1e-9)
        dist = math.sqrt(d2)
        w = to / dist
        cos_t = -(w @ dirW)
        if cos_t < math.cos(open_) - 1e-5 or (pen > 0 and abs(open_ - math.acos(min(1.0, cos_t))) < 1e-4):
            continue  # on the cone's edge the float32 and float64 decisions may differ
        fall = 0.0 if cos_t < math.cos(open_) else (smoothstep(0.0, pen, open_ - math.acos(min(1.0, cos_t))) if pen > 0 else 1.0)
        assert r["ok"] and r["pdf"] == 0.0
        assert close(r["distance"], dist) and close(r["dir"], w, 1e-5, 1e-6)
        assert close(r["Li"], np.asarray(light["intensity"]) * fall / d2, 1e-4, 1e-7), (r["Li"], fall)


def test_directional_light(hook):
    d = np.array([0.3, -1.0, 0.2])
    r = hook({"type": "directional", "intensity": (1.0, 2.0, 3.0), "direction": d}, (0.0, 0.0, 0.0))
    w = d / np.linalg.norm(d)
    assert r["ok"] and r["pdf"] == 0.0 and r["distance"] == np.float32(3.4028234663852886e38)
    assert close(r["dir"], -w) and close(r["Li"], (1.0, 2.0, 3.0))
    assert hook({"type": "directional", "direction": (0.0, 0.0, 0.0)}, (0, 0, 0)) is None  # zero direction rejected


def test_distant_light_cone(hook):
    rng = np.random.default_rng(2)
    for _ in range(30):
        d = rng.normal(size=3)
        ang = rng.uniform(0.01, 0.5)
        light = {"type": "distant", "intensity": (2.0, 2.0, 2.0), "direction": d, "angle": ang}
        w = -d / np.linalg.norm(d)
        # the rotation takes +z onto -dirW (Light.cpp DistantLight::update)
        r0 = hook(light, (0, 0, 0), (1.0, 0.3))  # z = 1: the cone's axis
        assert close(r0["dir"], w, 1e-5, 1e-6)
        assert close(r0["M"][:, :3] @ np.array([0.0, 0.0, 1.0]), w, 1e-5, 1e-6)
        assert close(r0["M"][:, :3] @ r0["M"][:, :3].T, np.eye(3), 1e-5, 1e-6)
        assert close(r0["cosSubtended"], math.cos(np.float32(ang)), 1e-6)
        for u in rng.uniform(0, 1, (20, 2)):
            r = hook(light, (0, 0, 0), u)
            z = u[0] * (1 - r0["cosSubtended"]) + r0["cosSubtended"]
            assert r["dir"] @ w >= z - 2e-5
            assert close(r["pdf"], 1.0 / (2 * math.pi * (1 - float(r0["cosSubtended"]))), 1e-4)
            assert close(r["normalW"], -r["dir"]) and close(r["Li"], (2.0, 2.0, 2.0))


@pytest.mark.parametrize("kind", ["rect", "disc", "sphere"])
def test_area_light_samples(hook, kind):
    rng = np.random.default_rng({"rect": 3, "disc": 4, "sphere": 5}[kind])
    for _ in range(40):
        T, sc = area_matrix(rng)
        if kind == "sphere":
            sc = np.full(3, sc[0])
        light = {"type": kind, "intensity": rng.uniform(0.5, 3, 3), "transform": T, "scaling": sc}
        M = T[:3, :3] * sc[None, :]
        MIT = np.linalg.inv(M).T
        x = rng.uniform(-4, 4, 3)
        u = rng.uniform(0, 1, 2)
        r = hook(light, x, u)
        assert close(r["M"][:, :3], M, 1e-6, 1e-6) and close(r["M"][:, 3], T[:3, 3], 1e-6, 1e-6)
        assert close(r["MIT"], MIT, 1e-5, 1e-6)
        rx, ry, rz = np.linalg.norm(M, axis=0)
        area = {"rect": 4 * rx * ry, "disc": math.pi * rx * ry,
                "sphere": 4 * math.pi * ((rx * ry) ** 1.6 + (ry * rz) ** 1.6 + (rx * rz) ** 1.6 / 3.0) ** (1 / 1.6)}[kind]
        assert close(r["area"], area, 1e-5)
        if kind == "rect":
            p, n = np.array([2 * u[0] - 1, 2 * u[1] - 1, 0.0]), np.array([0.0, 0.0, 1.0])
        elif kind == "disc":
            rr, ph = math.sqrt(u[0]), 2 * math.pi * u[1]
            p, n = np.array([rr * math.cos(ph), rr * math.sin(ph), 0.0]), np.array([0.0, 0.0, 1.0])
        else:
            ph, ct = 2 * math.pi * u[1], 1 - 2 * u[0]
            st = math.sqrt(max(0.0, 1 - ct * ct))
            p = np.array([st * math.cos(ph), st * math.sin(ph), ct]); n = p
        pw = M @ p + T[:3, 3]
        nw = MIT @ n
        nw /= np.linalg.norm(nw)
        to = pw - x
        d2 = max(to @ to, 1e-9)
        w = to / math.sqrt(d2)
        cos_t = nw @ -w
        assert close(r["posW"], pw, 1e-5, 1e-5) and close(r["normalW"], nw, 1e-4, 1e-5)
        if abs(cos_t) < 1e-4:
            continue
        assert r["ok"] == (cos_t > 0)
        if cos_t > 0:
            assert close(r["pdf"], d2 / (cos_t * area), 1e-3) and close(r["Li"], light["intensity"] * area * cos_t / d2, 1e-3)


def _solid_angle_triangle(a, b, c):
    """Van Oosterom and Strackee (1983): solid angle of triangle abc seen from the origin."""
    la, lb, lc = np.linalg.norm(a), np.linalg.norm(b), np.linalg.norm(c)
    num = a @ np.cross(b, c)
    den = la * lb * lc + (a @ b) * lc + (a @ c) * lb + (b @ c) * la
    return abs(2.0 * math.atan2(num, den))


def test_rect_light_pdf_integrates_to_its_solid_angle(hook):
    """E[1/pdf] over uniform (u1, u2) = the solid angle of the rect's front side."""
    rng = np.random.default_rng(6)
    T, sc = area_matrix(rng)
    M = T[:3, :3] * sc[None, :]
    normal = np.linalg.inv(M).T @ np.array([0, 0, 1.0])
    normal /= np.linalg.norm(normal)
    x = T[:3, 3] + 1.7 * normal + 0.4 * M[:, 0]  # in front of the light
    light = {"type": "rect", "transform": T, "scaling": sc}
    n = 96
    acc = 0.0
    for i in range(n):
        for j in range(n):
            r = hook(light, x, ((i + 0.5) / n, (j + 0.5) / n))
            if r["ok"]:
                acc += 1.0 / float(r["pdf"])
    est = acc / (n * n)
    corners = [M @ np.array(c) + T[:3, 3] - x for c in ((-1, -1, 0), (1, -1, 0), (1, 1, 0), (-1, 1, 0))]
    omega = _solid_angle_triangle(corners[0], corners[1], corners[2]) + _solid_angle_triangle(corners[0], corners[2], corners[3])
    assert abs(est - omega) < 2e-3 * omega, (est, omega)
