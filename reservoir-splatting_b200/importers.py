"""Scene import: Wavefront OBJ (+ MTL) into the pass's triangle soup and StandardMaterial parameters.

The reference loads OBJ files through its Assimp importer, which makes spec-gloss StandardMaterials
from the MTL parameters (Source/plugins/importers/AssimpImporter/AssimpImporter.cpp:66-73, 845-935):

* ``Kd`` -> diffuse (base) colour, ``Ks`` -> specular colour, ``Ke`` -> emitted radiance,
  ``Ni`` -> index of refraction;
* ``Ns`` (Phong exponent) -> glossiness 1 - clamp(sqrt(2 / (Ns + 2)), 0, 1);
* a material name with a ``.doublesided`` token is double sided.

Faces are fan-triangulated polygons (``f`` with ``v``, ``v/vt``, ``v//vn`` or ``v/vt/vn`` corners,
negative indices counting back from the last vertex).  Textures, normals and texture coordinates are
not used (the pass shades with face normals), so ``map_*``, ``vt`` and ``vn`` are ignored, as are
groups, objects and smoothing.  Faces before any ``usemtl`` get a grey diffuse material.
"""
from __future__ import annotations

import math
import warnings
from pathlib import Path

import numpy as np

from .scenes import Scene, material, spec_gloss_material


def spec_power_to_roughness(ns: float) -> float:
    """AssimpImporter.cpp:66-73 (in float32, as the importer computes it)."""
    r = np.float32(math.sqrt(np.float32(2.0) / (np.float32(ns) + np.float32(2.0))))
    return float(np.clip(r, np.float32(0.0), np.float32(1.0)))


def _floats(tokens, n, default=0.0):
    vals = [float(t) for t in tokens[:n]]
    return tuple(vals + [default] * (n - len(vals)))


def parse_mtl(path) -> dict:
    """name -> dict of the MTL parameters the importer uses."""
    mats, cur = {}, None
    for raw in Path(path).read_text().splitlines():
        t = raw.split("#", 1)[0].split()
        if not t:
            continue
        key, args = t[0], t[1:]
        if key == "newmtl":
            cur = mats.setdefault(" ".join(args), {})
        elif cur is None:
            continue
        elif key in ("Kd", "Ks", "Ke"):
            cur[key] = _floats(args, 3) if len(args) >= 3 else (float(args[0]),) * 3
        elif key in ("Ns", "Ni"):
            cur[key] = float(args[0])
    return mats


def _material_params(name: str, mtl: dict) -> np.ndarray:
    gloss = 0.0
    if "Ns" in mtl:
        gloss = float(np.float32(1.0) - np.float32(spec_power_to_roughness(mtl["Ns"])))
    double_sided = "doublesided" in [tok.lower() for tok in name.split(".")[1:]]
    return spec_gloss_material(diffuse=mtl.get("Kd", (0.0, 0.0, 0.0)), specular=mtl.get("Ks", (0.0, 0.0, 0.0)), glossiness=gloss,
                               emissive=mtl.get("Ke", (0.0, 0.0, 0.0)), ior=mtl.get("Ni", 1.5), double_sided=double_sided)


def load_obj(path) -> Scene:
    path = Path(path)
    verts, tris, mids = [], [], []
    library, names, index = {}, [], {}
    current = None

    def material_index(name):
        if name not in index:
            index[name] = len(names)
            names.append(name)
        return index[name]

    for raw in path.read_text().splitlines():
        t = raw.split("#", 1)[0].split()
        if not t:
            continue
        key, args = t[0], t[1:]
        if key == "v":
            verts.append(_floats(args, 3))
        elif key == "mtllib":
            for lib in args:
                p = path.parent / lib
                if p.exists():
                    library.update(parse_mtl(p))
        elif key == "usemtl":
            current = " ".join(args)
        elif key == "f":
            corners = []
            for c in args:
                i = int(c.split("/")[0])
                corners.append(i - 1 if i > 0 else len(verts) + i)
            if len(corners) < 3:
                continue
            m = material_index(current)
            for k in range(1, len(corners) - 1):
                tris.append(verts[corners[0]] + verts[corners[k]] + verts[corners[k + 1]])
                mids.append(m)
    if not tris:
        raise ValueError(f"{path}: no faces")
    mats = []
    for name in names:
        if name is None:
            mats.append(spec_gloss_material(diffuse=(0.6, 0.6, 0.6)))
        else:
            mats.append(_material_params(name, library.get(name, {})))
    return Scene(np.asarray(tris, np.float32), np.asarray(mids, np.uint32), np.stack(mats).astype(np.float32), path.stem,
                 {"triangles": len(tris), "materials": names})


def save_obj(scene: Scene, path, material_names=None, mtl_params=None):
    """Writes a scene's triangles as an OBJ (one vertex triple per triangle) and, when `mtl_params`
    (name -> {"Kd": .., "Ks": .., "Ke": .., "Ns": .., "Ni": ..}) is given, an MTL beside it."""
    path = Path(path)
    names = material_names or [f"m{i}" for i in range(len(scene.materials))]
    lines = []
    if mtl_params:
        lines.append(f"mtllib {path.stem}.mtl")
        mtl = []
        for n in names:
            mtl.append(f"newmtl {n}")
            for k, v in mtl_params.get(n, {}).items():
                mtl.append(f"{k} " + (" ".join(repr(float(x)) for x in v) if isinstance(v, (tuple, list)) else repr(float(v))))
        path.with_suffix(".mtl").write_text("\n".join(mtl) + "\n")
    cur = None
    for t, m in zip(scene.positions, scene.material_ids):
        if names[m] != cur:
            cur = names[m]
            lines.append(f"usemtl {cur}")
        for k in range(3):
            lines.append("v " + " ".join(repr(float(x)) for x in t[3 * k:3 * k + 3]))
        lines.append("f -3 -2 -1")
    path.write_text("\n".join(lines) + "\n")


# ---------------------------------------------------------------------------------------- PBRT v4
# A subset of the reference's PBRT importer (Source/plugins/importers/PBRTImporter: Parser.cpp for
# the syntax, PBRTImporter.cpp for the conversion to StandardMaterials, the path without PBRT
# materials):
#   * the transform stack (Identity, Translate, Scale, Rotate, LookAt, ConcatTransform, Transform,
#     AttributeBegin/End, ReverseOrientation), Camera "perspective", WorldBegin, Include/Import,
#     ObjectBegin/End/ObjectInstance (flattened);
#   * Shape "trianglemesh", "bilinearmesh", "sphere" (tessellated) and "plymesh" (ascii or binary
#     little-endian PLY, polygons fan-triangulated);
#   * materials by the StandardMaterial mapping of PBRTImporter.cpp:992-1175: diffuse (base =
#     reflectance, roughness 1), coateddiffuse (roughness sqrt of the scalar roughness), conductor and
#     coatedconductor (metallic, base = the Fresnel reflectance at normal incidence of eta, k or the
#     given reflectance), dielectric (IoR eta; the pass has no transmission lobe, so only its
#     reflection remains); the scalar roughness is getRoughness (:424-462) as written: float2(u + v),
#     square-rooted when remaproughness, and getScalarRoughness averages the two equal components;
#   * AreaLightSource "diffuse" (L * scale emitted by the shapes that follow, twosided);
#   * LightSource "infinite" with a constant "rgb L" (an environment map of that radiance), or with an
#     equal-area octahedral image (.hdr / .pfm here) converted to lat-long as the reference's
#     EnvMapConverter does, with intensity = scale and the light transform's XYZ Euler rotation;
#   * LightSource "distant" as a directional analytic light (createLight, PBRTImporter.cpp:676-699:
#     intensity L * scale, times illuminance when it is positive; direction the transformed
#     to - from); "point", "spot", "goniometric" and "projection" lights are skipped with a warning,
#     as the reference importer does.
# Textures, named spectra other than the defaults, .exr images, curves, disks and
# cylinders are not read.

_PBRT_COPPER_F0 = (0.955, 0.638, 0.538)  # RGB normal-incidence reflectance used for the default conductor (metal-Cu)


def _pbrt_tokens(text: str):
    i, n = 0, len(text)
    while i < n:
        c = text[i]
        if c.isspace():
            i += 1
        elif c == "#":
            while i < n and text[i] != "\n":
                i += 1
        elif c in "[]":
            yield c
            i += 1
        elif c == '"':
            j = text.index('"', i + 1)
            yield text[i:j + 1]
            i = j + 1
        else:
            j = i
            while j < n and not text[j].isspace() and text[j] not in '[]"#':
                j += 1
            yield text[i:j]
            i = j


def _pbrt_value(tok: str):
    if tok.startswith('"'):
        return tok[1:-1]
    if tok in ("true", "false"):
        return tok == "true"
    return float(tok)


class _PbrtReader:
    def __init__(self, tokens):
        self.toks = list(tokens)
        self.i = 0

    def more(self):
        return self.i < len(self.toks)

    def next(self):
        t = self.toks[self.i]
        self.i += 1
        return t

    def peek(self):
        return self.toks[self.i] if self.more() else None

    def numbers(self, k):
        out = []
        if self.peek() == "[":
            self.next()
            while self.peek() != "]":
                out.append(float(self.next()))
            self.next()
        else:
            for _ in range(k):
                out.append(float(self.next()))
        return out

    def params(self):
        """The "type name" value lists after a directive's positional arguments."""
        ps = {}
        while self.more() and self.peek().startswith('"'):
            decl = self.next()[1:-1].split()
            if len(decl) != 2:
                self.i -= 1
                break
            ptype, pname = decl
            if self.peek() == "[":
                self.next()
                vals = []
                while self.peek() != "]":
                    vals.append(_pbrt_value(self.next()))
                self.next()
            else:
                vals = [_pbrt_value(self.next())]
            ps[pname] = (ptype, vals)
        return ps


def _rotate(deg, axis):
    a = np.asarray(axis, np.float64)
    a = a / np.linalg.norm(a)
    s, c = math.sin(math.radians(deg)), math.cos(math.radians(deg))
    x, y, z = a
    m = np.eye(4)
    m[:3, :3] = [[x * x + (1 - x * x) * c, x * y * (1 - c) - z * s, x * z * (1 - c) + y * s],
                 [x * y * (1 - c) + z * s, y * y + (1 - y * y) * c, y * z * (1 - c) - x * s],
                 [x * z * (1 - c) - y * s, y * z * (1 - c) + x * s, z * z + (1 - z * z) * c]]
    return m


def _look_at(eye, look, up):
    """World-to-camera matrix of PBRT's LookAt (camera looks down +z, y up)."""
    eye, look, up = (np.asarray(v, np.float64) for v in (eye, look, up))
    d = look - eye
    d = d / np.linalg.norm(d)
    right = np.cross(up / np.linalg.norm(up), d)
    right = right / np.linalg.norm(right)
    new_up = np.cross(d, right)
    cam_to_world = np.eye(4)
    cam_to_world[:3, 0], cam_to_world[:3, 1], cam_to_world[:3, 2], cam_to_world[:3, 3] = right, new_up, d, eye
    return np.linalg.inv(cam_to_world)


def _read_ply(path: Path):
    """Vertex positions [V, 3] and polygon index lists of an ascii or binary little-endian PLY."""
    data = path.read_bytes()
    end = data.index(b"end_header") + len(b"end_header")
    while data[end:end + 1] in (b"\r", b"\n"):
        end += 1
        if data[end - 1:end] == b"\n":
            break
    header = data[:end].decode("ascii").splitlines()
    fmt = next(l.split()[1] for l in header if l.startswith("format"))
    elements, cur = [], None
    for l in header:
        t = l.split()
        if t and t[0] == "element":
            cur = {"name": t[1], "count": int(t[2]), "props": []}
            elements.append(cur)
        elif t and t[0] == "property":
            cur["props"].append(t[1:])
    np_t = {"char": "i1", "int8": "i1", "uchar": "u1", "uint8": "u1", "short": "i2", "int16": "i2", "ushort": "u2", "uint16": "u2",
            "int": "i4", "int32": "i4", "uint": "u4", "uint32": "u4", "float": "f4", "float32": "f4", "double": "f8", "float64": "f8"}
    verts, faces = None, []
    if fmt == "ascii":
        lines = data[end:].decode("ascii").split("\n")
        li = 0
        for el in elements:
            rows = []
            for _ in range(el["count"]):
                while not lines[li].strip():
                    li += 1
                rows.append(lines[li].split())
                li += 1
            if el["name"] == "vertex":
                names = [p[-1] for p in el["props"]]
                idx = [names.index(k) for k in ("x", "y", "z")]
                verts = np.array([[float(r[j]) for j in idx] for r in rows], np.float64)
            elif el["name"] == "face":
                faces = [[int(v) for v in r[1:1 + int(r[0])]] for r in rows]
        return verts, faces
    if fmt != "binary_little_endian":
        raise ValueError(f"{path}: PLY format {fmt} is not read")
    off = end
    for el in elements:
        if all(p[0] != "list" for p in el["props"]):
            dt = np.dtype([(p[1], "<" + np_t[p[0]]) for p in el["props"]])
            arr = np.frombuffer(data, dt, el["count"], off)
            off += dt.itemsize * el["count"]
            if el["name"] == "vertex":
                verts = np.stack([arr["x"], arr["y"], arr["z"]], -1).astype(np.float64)
        else:
            rows = []
            for _ in range(el["count"]):
                row = []
                for p in el["props"]:
                    if p[0] == "list":
                        ct, it = np.dtype("<" + np_t[p[1]]), np.dtype("<" + np_t[p[2]])
                        k = int(np.frombuffer(data, ct, 1, off)[0])
                        off += ct.itemsize
                        row.append(np.frombuffer(data, it, k, off).tolist())
                        off += it.itemsize * k
                    else:
                        off += np.dtype(np_t[p[0]]).itemsize
                rows.append(row)
            if el["name"] == "face":
                faces = [r[0] for r in rows]
    return verts, faces


def _pbrt_rgb(ps, name, default):
    if name not in ps:
        return tuple(default)
    ptype, vals = ps[name]
    if ptype == "rgb":
        return tuple(float(v) for v in vals[:3])
    if ptype == "float":
        return (float(vals[0]),) * 3
    return tuple(default)  # named or sampled spectra are not converted


def _pbrt_float(ps, name, default):
    return float(ps[name][1][0]) if name in ps else float(default)


def _pbrt_scalar_roughness(ps, prefix=""):
    """getRoughness + getScalarRoughness (PBRTImporter.cpp:424-479), as written."""
    r = _pbrt_float(ps, prefix + "roughness", 0.0)
    u = _pbrt_float(ps, prefix + "uroughness", r)
    v = _pbrt_float(ps, prefix + "vroughness", r)
    both = u + v
    if ps.get("remaproughness", ("bool", [True]))[1][0]:
        both = math.sqrt(both)
    return 0.5 * (both + both)


def _conductor_f0(ps, prefix=""):
    """getConductorSpecularAlbedo (PBRTImporter.cpp:496-587): the conductor Fresnel at normal
    incidence, from rgb eta and k or directly from a reflectance."""
    if prefix + "reflectance" in ps:
        return _pbrt_rgb(ps, prefix + "reflectance", (0.0, 0.0, 0.0))
    if ps.get(prefix + "eta", ("", []))[0] == "rgb" and ps.get(prefix + "k", ("", []))[0] == "rgb":
        eta, k = _pbrt_rgb(ps, prefix + "eta", (1, 1, 1)), _pbrt_rgb(ps, prefix + "k", (0, 0, 0))
        return tuple(((e - 1) ** 2 + kk ** 2) / ((e + 1) ** 2 + kk ** 2) for e, kk in zip(eta, k))
    return _PBRT_COPPER_F0


def _pbrt_material(mtype, ps):
    """(base, roughness, metallic, ior) of the StandardMaterial the reference makes."""
    if mtype in ("diffuse", "", "interface"):
        return _pbrt_rgb(ps, "reflectance", (0.5, 0.5, 0.5)), 1.0, 0.0, 1.5
    if mtype == "coateddiffuse":
        return _pbrt_rgb(ps, "reflectance", (0.5, 0.5, 0.5)), math.sqrt(_pbrt_scalar_roughness(ps)), 0.0, 1.5
    if mtype == "conductor":
        return _conductor_f0(ps), math.sqrt(_pbrt_scalar_roughness(ps)), 1.0, 1.5
    if mtype == "coatedconductor":
        return _conductor_f0(ps, "conductor."), math.sqrt(_pbrt_scalar_roughness(ps, "conductor.")), 1.0, 1.5
    if mtype in ("dielectric", "thindielectric"):
        eta = _pbrt_float(ps, "eta", 1.5)
        return (0.0, 0.0, 0.0), math.sqrt(_pbrt_scalar_roughness(ps)), 0.0, eta
    raise ValueError(f"PBRT material {mtype!r} is not converted")


def load_pbrt(path) -> Scene:
    """A PBRT v4 scene file as the pass's triangle soup; info holds "camera" (position, target, up,
    fovDegrees), "env" (an [h, w, 3] radiance map for rs_set_env_map) and "lights" (analytic lights
    for rs_set_analytic_lights) when the file has them."""
    path = Path(path)
    tris, mids, mat_rows, mat_index = [], [], [], {}
    state = {"ctm": np.eye(4), "material": ("diffuse", {}), "area": None, "reverse": False}
    stack, named, objects = [], {}, {}
    current_object = None
    camera, env, env_params = None, None, None
    lights = []

    def material_id(mat, area):
        mtype, ps = mat
        base, rough, metal, ior = _pbrt_material(mtype, ps)
        emissive = (0.0, 0.0, 0.0)
        two = True
        if area is not None:
            L = _pbrt_rgb(area, "L", (1.0, 1.0, 1.0))
            scale = _pbrt_float(area, "scale", 1.0)
            emissive = tuple(c * scale for c in L)
            two = bool(area.get("twosided", ("bool", [False]))[1][0])
        key = (base, rough, metal, ior, emissive, two)
        if key not in mat_index:
            mat_index[key] = len(mat_rows)
            mat_rows.append(material(base=base, roughness=rough, emissive=emissive, metallic=metal, ior=ior, double_sided=two))
        return mat_index[key]

    def emit(points, faces, xform, mid, reverse):
        p = np.c_[np.asarray(points, np.float64), np.ones(len(points))] @ xform.T
        p = p[:, :3] / p[:, 3:4]
        flip = reverse ^ (np.linalg.det(xform[:3, :3]) < 0)
        for f in faces:
            for k in range(1, len(f) - 1):
                a, b, c = (f[0], f[k + 1], f[k]) if flip else (f[0], f[k], f[k + 1])
                tris.append(np.concatenate([p[a], p[b], p[c]]))
                mids.append(mid)

    def shape(stype, ps, base_dir):
        if stype == "trianglemesh":
            P = np.asarray(ps["P"][1], np.float64).reshape(-1, 3)
            idx = ps["indices"][1] if "indices" in ps else list(range(len(P)))
            faces = np.asarray(idx, np.int64).reshape(-1, 3).tolist()
        elif stype == "bilinearmesh":
            P = np.asarray(ps["P"][1], np.float64).reshape(-1, 3)
            idx = ps["indices"][1] if "indices" in ps else list(range(len(P)))
            faces = [[q[0], q[1], q[3], q[2]] for q in np.asarray(idx, np.int64).reshape(-1, 4).tolist()]
        elif stype == "sphere":
            from .scenes import _icosphere
            ico = _icosphere(3).reshape(-1, 3) * _pbrt_float(ps, "radius", 1.0)
            P, faces = ico, np.arange(len(ico)).reshape(-1, 3).tolist()
        elif stype == "plymesh":
            P, faces = _read_ply(base_dir / ps["filename"][1][0])
        else:
            raise ValueError(f"PBRT shape {stype!r} is not converted")
        return P, faces

    def parse(file_path: Path):
        nonlocal camera, env, env_params, current_object
        r = _PbrtReader(_pbrt_tokens(file_path.read_text()))
        base_dir = file_path.parent
        while r.more():
            d = r.next()
            if d == "Identity":
                state["ctm"] = np.eye(4)
            elif d == "Translate":
                t = np.eye(4)
                t[:3, 3] = r.numbers(3)
                state["ctm"] = state["ctm"] @ t
            elif d == "Scale":
                state["ctm"] = state["ctm"] @ np.diag(r.numbers(3) + [1.0])
            elif d == "Rotate":
                v = r.numbers(4)
                state["ctm"] = state["ctm"] @ _rotate(v[0], v[1:])
            elif d == "LookAt":
                v = r.numbers(9)
                state["ctm"] = state["ctm"] @ _look_at(v[0:3], v[3:6], v[6:9])
            elif d in ("ConcatTransform", "Transform"):
                m = np.asarray(r.numbers(16), np.float64).reshape(4, 4).T  # column-major in the file
                state["ctm"] = (state["ctm"] @ m) if d == "ConcatTransform" else m
            elif d == "Camera":
                ctype = r.next()[1:-1]
                ps = r.params()
                c2w = np.linalg.inv(state["ctm"])
                pos = c2w @ [0, 0, 0, 1]
                tgt = c2w @ [0, 0, 1, 1]
                up = c2w @ [0, 1, 0, 0]
                camera = {"type": ctype, "position": tuple(float(x) for x in pos[:3]), "target": tuple(float(x) for x in tgt[:3]),
                          "up": tuple(float(x) for x in up[:3]), "fovDegrees": _pbrt_float(ps, "fov", 90.0)}
            elif d == "WorldBegin":
                state["ctm"] = np.eye(4)
            elif d == "AttributeBegin":
                stack.append(dict(state))
            elif d == "AttributeEnd":
                state.update(stack.pop())
            elif d == "ReverseOrientation":
                state["reverse"] = not state["reverse"]
            elif d == "Material":
                mtype = r.next()[1:-1]
                state["material"] = (mtype, r.params())
            elif d == "MakeNamedMaterial":
                name = r.next()[1:-1]
                ps = r.params()
                named[name] = (ps.pop("type", ("string", ["diffuse"]))[1][0], ps)
            elif d == "NamedMaterial":
                state["material"] = named[r.next()[1:-1]]
            elif d == "AreaLightSource":
                atype = r.next()[1:-1]
                ps = r.params()
                if atype != "diffuse":
                    raise ValueError(f"PBRT area light {atype!r} is not converted")
                state["area"] = ps
            elif d == "LightSource":
                ltype = r.next()[1:-1]
                ps = r.params()
                if ltype == "infinite":
                    if "filename" in ps and "L" in ps:
                        raise ValueError("PBRT infinite light: both L and filename")
                    if "filename" in ps:
                        # createLight (PBRTImporter.cpp:722-737): the equal-area octahedral image to
                        # lat-long, intensity = scale, rotation = XYZ Euler angles of the light's transform
                        env = equal_area_oct_to_latlong(read_env_image(file_path.parent / ps["filename"][1][0]))
                        env_params = {"intensity": _pbrt_float(ps, "scale", 1.0), "tint": (1.0, 1.0, 1.0),
                                      "rotation": _euler_xyz_degrees(state["ctm"])}
                    else:
                        L = np.asarray(_pbrt_rgb(ps, "L", (1.0, 1.0, 1.0)), np.float32) * _pbrt_float(ps, "scale", 1.0)
                        env = np.broadcast_to(L, (8, 16, 3)).astype(np.float32).copy()
                elif ltype == "distant":
                    I = np.asarray(_pbrt_rgb(ps, "L", (1.0, 1.0, 1.0)), np.float64) * _pbrt_float(ps, "scale", 1.0)
                    illum = _pbrt_float(ps, "illuminance", -1.0)
                    if illum > 0.0:
                        I = I * illum
                    fr = np.asarray(ps["from"][1][:3], np.float64) if "from" in ps else np.zeros(3)
                    to = np.asarray(ps["to"][1][:3], np.float64) if "to" in ps else np.array([0.0, 0.0, 1.0])
                    d = state["ctm"][:3, :3] @ (to - fr)
                    lights.append({"type": "directional", "intensity": tuple(I), "direction": tuple(d / np.linalg.norm(d))})
                else:
                    warnings.warn(f"PBRT light type {ltype!r} is currently not supported and ignored")
            elif d == "Shape":
                stype = r.next()[1:-1]
                ps = r.params()
                P, faces = shape(stype, ps, base_dir)
                mid = material_id(state["material"], state["area"])
                if current_object is not None:
                    objects[current_object].append((P, faces, state["ctm"].copy(), mid, state["reverse"]))
                else:
                    emit(P, faces, state["ctm"], mid, state["reverse"])
            elif d == "ObjectBegin":
                current_object = r.next()[1:-1]
                objects[current_object] = []
                stack.append(dict(state))
            elif d == "ObjectEnd":
                current_object = None
                state.update(stack.pop())
            elif d == "ObjectInstance":
                for P, faces, xf, mid, rev in objects[r.next()[1:-1]]:
                    emit(P, faces, state["ctm"] @ xf, mid, rev)
            elif d in ("Include", "Import"):
                parse(base_dir / r.next()[1:-1])
            elif d in ("Film", "Sampler", "Integrator", "PixelFilter", "Accelerator", "ColorSpace", "Option", "Texture",
                       "CoordinateSystem", "CoordSysTransform", "MakeNamedMedium", "MediumInterface", "Attribute",
                       "TransformBegin", "TransformEnd", "ActiveTransform", "TransformTimes", "WorldEnd"):
                if d == "TransformBegin":
                    stack.append(dict(state))
                elif d == "TransformEnd":
                    state.update(stack.pop())
                elif d == "Texture":
                    r.next(); r.next(); r.next()
                    r.params()
                elif d in ("CoordinateSystem", "CoordSysTransform", "ActiveTransform", "MediumInterface"):
                    r.next()
                    if d == "MediumInterface" and r.more() and r.peek().startswith('"') and len(r.peek().split()) == 1:
                        r.next()
                elif d == "TransformTimes":
                    r.numbers(2)
                elif d in ("MakeNamedMedium",):
                    r.next(); r.params()
                elif d in ("Option", "Attribute"):
                    r.next()
                    r.params()
                elif d != "WorldEnd":
                    if r.more() and r.peek().startswith('"') and len(r.peek()[1:-1].split()) == 1:
                        r.next()
                    r.params()
            else:
                raise ValueError(f"{file_path}: PBRT directive {d!r} is not read")

    parse(path)
    if not tris:
        raise ValueError(f"{path}: no shapes")
    info = {"triangles": len(tris), "materials": len(mat_rows)}
    if camera:
        info["camera"] = camera
    if env is not None:
        info["env"] = env
    if lights:
        info["lights"] = lights
    if env_params is not None:
        info["env_params"] = env_params
    return Scene(np.asarray(tris, np.float32), np.asarray(mids, np.uint32), np.stack(mat_rows).astype(np.float32), path.stem, info)


def pbrt_camera(scene: Scene, width: int, height: int):
    """The pass camera of a load_pbrt scene: its LookAt, with the field of view taken across the
    shorter image side (PBRT's "fov"), on a 24 mm film height."""
    from .scenes import Camera
    c = scene.info["camera"]
    half = math.radians(c["fovDegrees"]) * 0.5
    frame_height = 24.0
    if width < height:  # fov spans the width: convert to the vertical extent
        half = math.atan(math.tan(half) * height / width)
    return Camera(position=c["position"], target=c["target"], up=c["up"], focal_length=0.5 * frame_height / math.tan(half),
                  frame_height=frame_height, aspect_ratio=width / height)


# ---------------------------------------------------------------------------------------- Mitsuba
# A subset of the reference's Mitsuba importer (Source/plugins/importers/MitsubaImporter/
# MitsubaImporter.cpp:249-400 BSDFs, :468-530 shapes, :668-700 emitters), mapped to the one
# StandardMaterial model the pass has: diffuse (reflectance, roughness 1), plastic / roughplastic
# (diffuse_reflectance, IoR int_ior / ext_ior, roughness sqrt(alpha) for the rough one), conductor /
# roughconductor (metallic, base = the normal-incidence Fresnel reflectance of rgb eta, k; copper
# without them; roughness sqrt(alpha)), dielectric / roughdielectric / thindielectric (IoR only: no
# transmission lobe), twosided (its nested BSDF); shapes obj, ply, rectangle, cube, sphere; area
# emitters nested in shapes, constant emitters as an env map, envmap emitters from .hdr / .pfm images
# (point, spot, projector and directional
# emitters are skipped with a warning: the reference importer converts none of them); a perspective sensor.  <default> and
# $name substitution, refs by id, and to_world transforms (translate, scale, rotate, matrix, lookat).
# Image environment maps, textures and other plugins are rejected with a message.

_MITSUBA_IOR = {"vacuum": 1.0, "air": 1.00028, "water": 1.333, "acetone": 1.36, "ethanol": 1.361, "glycerol": 1.4729,
                "bk7": 1.5046, "polypropylene": 1.49, "acrylic glass": 1.49, "pet": 1.575, "diamond": 2.419,
                "fused quartz": 1.458, "sapphire": 1.77}


def _mi_floats(text):
    return [float(v) for v in text.replace(",", " ").split()]


def _mi_transform(el):
    m = np.eye(4)
    for op in el:
        a = op.attrib
        if op.tag == "translate":
            t = np.eye(4)
            t[:3, 3] = [float(a.get(k, 0.0)) for k in "xyz"] if "value" not in a else _mi_floats(a["value"])
            m = t @ m
        elif op.tag == "scale":
            if "value" in a:
                v = _mi_floats(a["value"])
                v = v * 3 if len(v) == 1 else v
            else:
                v = [float(a.get(k, 1.0)) for k in "xyz"]
            m = np.diag(v + [1.0]) @ m
        elif op.tag == "rotate":
            axis = [float(a.get(k, 0.0)) for k in "xyz"] if "value" not in a else _mi_floats(a["value"])
            m = _rotate(float(a["angle"]), axis) @ m
        elif op.tag == "matrix":
            m = np.asarray(_mi_floats(a["value"]), np.float64).reshape(4, 4) @ m
        elif op.tag == "lookat":
            m = np.linalg.inv(_look_at(_mi_floats(a["origin"]), _mi_floats(a["target"]), _mi_floats(a.get("up", "0 1 0")))) @ m
        else:
            raise ValueError(f"Mitsuba transform {op.tag!r} is not read")
    return m


def load_mitsuba(path) -> Scene:
    """A Mitsuba 3 scene XML as the pass's triangle soup; info holds "camera" and "env" like load_pbrt,
    and "env_params" (intensity, tint, rotation for rs_set_env_map) with an envmap emitter."""
    import xml.etree.ElementTree as ET
    path = Path(path)
    text = path.read_text()
    root = ET.fromstring(text)
    defaults = {d.attrib["name"]: d.attrib["value"] for d in root.iter("default")}

    def sub(v):
        for k, d in defaults.items():
            v = v.replace("$" + k, d)
        return v
    for el in root.iter():
        for k, v in list(el.attrib.items()):
            el.attrib[k] = sub(v)
    ids = {el.attrib["id"]: el for el in root.iter() if "id" in el.attrib and el.tag != "ref"}

    def props(el):
        out = {}
        for c in el:
            n = c.attrib.get("name")
            if c.tag in ("float", "integer"):
                out[n] = float(c.attrib["value"])
            elif c.tag in ("rgb", "spectrum", "color"):
                v = _mi_floats(c.attrib["value"])
                out[n] = tuple(v * 3 if len(v) == 1 else v[:3])
            elif c.tag in ("string", "boolean"):
                out[n] = c.attrib["value"]
            elif c.tag == "transform":
                out[n] = _mi_transform(c)
        return out

    def ior(p, name, default):
        v = p.get(name, default)
        return _MITSUBA_IOR[v.lower()] if isinstance(v, str) else float(v)

    def bsdf(el):
        if el.tag == "ref":
            el = ids[el.attrib["id"]]
        t, p = el.attrib["type"], props(el)
        if t == "twosided":
            inner = [c for c in el if c.tag in ("bsdf", "ref")]
            return bsdf(inner[0])
        if t == "diffuse":
            return p.get("reflectance", (0.5,) * 3), 1.0, 0.0, 1.5
        if t in ("plastic", "roughplastic"):
            rough = math.sqrt(p.get("alpha", 0.1)) if t == "roughplastic" else 0.0
            return p.get("diffuse_reflectance", (0.5,) * 3), rough, 0.0, ior(p, "int_ior", "polypropylene") / ior(p, "ext_ior", "air")
        if t in ("conductor", "roughconductor"):
            if "eta" in p and "k" in p:
                f0 = tuple(((e - 1) ** 2 + k ** 2) / ((e + 1) ** 2 + k ** 2) for e, k in zip(p["eta"], p["k"]))
            else:
                f0 = _PBRT_COPPER_F0
            rough = math.sqrt(p.get("alpha", 0.1)) if t == "roughconductor" else 0.0
            return f0, rough, 1.0, 1.5
        if t in ("dielectric", "roughdielectric", "thindielectric"):
            rough = math.sqrt(p.get("alpha", 0.1)) if t == "roughdielectric" else 0.0
            return (0.0, 0.0, 0.0), rough, 0.0, ior(p, "int_ior", "bk7") / ior(p, "ext_ior", "air")
        raise ValueError(f"Mitsuba BSDF {t!r} is not converted")

    tris, mids, rows, index = [], [], [], {}
    camera, env, env_params = None, None, None

    def material_id(mat, emission):
        base, rough, metal, eta = mat
        key = (tuple(base), rough, metal, eta, tuple(emission))
        if key not in index:
            index[key] = len(rows)
            rows.append(material(base=base, roughness=rough, emissive=emission, metallic=metal, ior=eta, double_sided=True))
        return index[key]

    cube_faces = [[0, 2, 3, 1], [4, 5, 7, 6], [0, 1, 5, 4], [2, 6, 7, 3], [0, 4, 6, 2], [1, 3, 7, 5]]
    cube_verts = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float64)
    for el in root:
        if el.tag == "sensor":
            p = props(el)
            c2w = p.get("to_world", np.eye(4))
            pos, tgt, up = c2w @ [0, 0, 0, 1], c2w @ [0, 0, 1, 1], c2w @ [0, 1, 0, 0]
            camera = {"type": el.attrib["type"], "position": tuple(float(x) for x in pos[:3]), "target": tuple(float(x) for x in tgt[:3]),
                      "up": tuple(float(x) for x in up[:3]), "fovDegrees": float(p.get("fov", 45.0))}
        elif el.tag == "emitter":
            t, p = el.attrib["type"], props(el)
            if t == "constant":
                env = np.broadcast_to(np.asarray(p.get("radiance", (1.0,) * 3), np.float32), (8, 16, 3)).astype(np.float32).copy()
            elif t == "envmap":
                # MitsubaImporter.cpp:686-701: the image, intensity = scale, and the rotation as the XYZ
                # Euler angles (extractEulerAngleXYZ, MatrixMath.h:331-342) of to_world x flipZ
                env = read_env_image(path.parent / str(p["filename"]))
                m = np.asarray(p.get("to_world", np.eye(4)), np.float64) @ np.diag([1.0, 1.0, -1.0, 1.0])
                t1 = math.atan2(m[1][2], m[2][2])
                t2 = math.atan2(-m[0][2], math.sqrt(m[0][0] * m[0][0] + m[0][1] * m[0][1]))
                s1, c1 = math.sin(t1), math.cos(t1)
                t3 = math.atan2(s1 * m[2][0] - c1 * m[1][0], c1 * m[1][1] - s1 * m[2][1])
                env_params = {"intensity": float(p.get("scale", 1.0)), "tint": (1.0, 1.0, 1.0),
                              "rotation": tuple(math.degrees(-a) for a in (t1, t2, t3))}
            elif t in ("point", "spot", "projector", "directional", "directionalarea"):
                # MitsubaImporter.cpp:703-721 converts none of these (unsupportedType, a warning)
                warnings.warn(f"Mitsuba emitter type {t!r} is not supported")
            else:
                raise ValueError(f"Mitsuba emitter {t!r} is not converted (area emitters belong inside shapes)")
        elif el.tag == "shape":
            t, p = el.attrib["type"], props(el)
            xform = p.get("to_world", np.eye(4))
            mat = (0.5, 0.5, 0.5), 1.0, 0.0, 1.5
            emission = (0.0, 0.0, 0.0)
            for c in el:
                if c.tag in ("bsdf", "ref") and (c.tag == "bsdf" or ids[c.attrib["id"]].tag == "bsdf"):
                    mat = bsdf(c)
                elif c.tag == "emitter" and c.attrib["type"] == "area":
                    emission = props(c).get("radiance", (1.0,) * 3)
            if t == "obj":
                s = load_obj(path.parent / p["filename"])
                P, faces = s.positions.reshape(-1, 3).astype(np.float64), np.arange(len(s.positions) * 3).reshape(-1, 3).tolist()
            elif t == "ply":
                P, faces = _read_ply(path.parent / p["filename"])
            elif t == "rectangle":
                P, faces = np.array([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0]], np.float64), [[0, 1, 2, 3]]
            elif t == "cube":
                P, faces = cube_verts, cube_faces
            elif t == "sphere":
                from .scenes import _icosphere
                center = np.asarray(_mi_floats(el.find("point[@name='center']").attrib["value"])
                                    if el.find("point[@name='center']") is not None else [0, 0, 0], np.float64)
                P = _icosphere(3).reshape(-1, 3).astype(np.float64) * float(p.get("radius", 1.0)) + center
                faces = np.arange(len(P)).reshape(-1, 3).tolist()
            else:
                raise ValueError(f"Mitsuba shape {t!r} is not converted")
            mid = material_id(mat, emission)
            hp = np.c_[np.asarray(P, np.float64), np.ones(len(P))] @ xform.T
            hp = hp[:, :3] / hp[:, 3:4]
            flip = np.linalg.det(xform[:3, :3]) < 0
            for f in faces:
                for k in range(1, len(f) - 1):
                    a, b, c = (f[0], f[k + 1], f[k]) if flip else (f[0], f[k], f[k + 1])
                    tris.append(np.concatenate([hp[a], hp[b], hp[c]]))
                    mids.append(mid)
    if not tris:
        raise ValueError(f"{path}: no shapes")
    info = {"triangles": len(tris), "materials": len(rows)}
    if camera:
        info["camera"] = camera
    if env is not None:
        info["env"] = env
    if env_params is not None:
        info["env_params"] = env_params
    return Scene(np.asarray(tris, np.float32), np.asarray(mids, np.uint32), np.stack(rows).astype(np.float32), path.stem, info)


# ---------------------------------------------------------------- Falcor Python scenes (.pyscene)
# The reference's PythonImporter (Source/plugins/importers/PythonImporter/PythonImporter.cpp) runs a
# .pyscene file as a Python script with `sceneBuilder` and Falcor's scene classes in scope.  This
# runs it with stand-ins for the classes the pass renders, with the semantics of their Falcor
# definitions:
#   * float2 / float3 / float4 (one argument broadcasts);
#   * Transform (Scene/Transform.cpp): translation, scaling, rotationEuler (radians, the quaternion
#     of Utils/Math/QuaternionMath.h:398-409) or rotationEulerDeg, lookAt(position, target, up);
#     matrix = T x R x S (the default ScaleRotateTranslate order);
#   * TriangleMesh (Scene/TriangleMesh.cpp:58-194): createQuad, createDisk, createCube, createSphere
#     with their vertex and index layouts, createFromFile for OBJ files, and addVertex / addTriangle;
#   * StandardMaterial (alias Material; Scene/Material/BasicMaterial.cpp, StandardMaterial.cpp):
#     baseColor, roughness, metallic, specularParams (occlusion, roughness, metallic; or specular
#     colour and glossiness with ShadingModel.SpecGloss), emissiveColor x emissiveFactor,
#     indexOfRefraction, doubleSided; defaults baseColor 1, roughness 0, metallic 0, IoR 1.5,
#     single-sided;
#   * Camera (Scene/Camera/Camera.cpp:426-440, CameraData.slang defaults);
#   * PointLight, DirectionalLight, DistantLight, RectLight, DiscLight, SphereLight (Scene/Lights/
#     Light.cpp:404-440) as analytic lights (info["lights"], for rs_set_analytic_lights);
#   * EnvMap (Scene/Lights/EnvMap.cpp:140-157) from .hdr or .pfm images, with rotation, intensity and
#     tint (info["env"], info["env_params"], for rs_set_env_map);
#   * sceneBuilder: addTriangleMesh, addMaterial, getMaterial, addNode (with parents), addMeshInstance,
#     addLight, getLight, addCamera, envMap.
# Meshes are flattened to world space per instance; the winding is flipped when the mesh's front face
# is clockwise or the instance transform mirrors, as Falcor flips the face normal then.  Textures,
# environment images other than .hdr / .pfm, SDF grids, volumes, curves and animations raise ValueError.

def _pys_vec(n):
    def make(*a):
        if len(a) == 1 and not isinstance(a[0], (int, float)):
            a = tuple(a[0])
        if len(a) == 1:
            a = a * n
        if len(a) != n:
            raise ValueError(f"float{n} takes 1 or {n} values")
        return tuple(float(x) for x in a)
    return make


class _PysTransform:
    def __init__(self):
        self.translation = (0.0, 0.0, 0.0)
        self.scaling = (1.0, 1.0, 1.0)
        self._R = np.eye(3)

    @property
    def rotationEuler(self):
        raise AttributeError("reading rotationEuler is not supported")

    @rotationEuler.setter
    def rotationEuler(self, a):
        c, s = np.cos(np.asarray(a, np.float64) * 0.5), np.sin(np.asarray(a, np.float64) * 0.5)
        x = s[0] * c[1] * c[2] - c[0] * s[1] * s[2]
        y = c[0] * s[1] * c[2] + s[0] * c[1] * s[2]
        z = c[0] * c[1] * s[2] - s[0] * s[1] * c[2]
        w = c[0] * c[1] * c[2] + s[0] * s[1] * s[2]
        self._R = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y)],
                            [2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x)],
                            [2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)]])

    @property
    def rotationEulerDeg(self):
        raise AttributeError("reading rotationEulerDeg is not supported")

    @rotationEulerDeg.setter
    def rotationEulerDeg(self, a):
        self.rotationEuler = tuple(math.radians(float(v)) for v in a)

    def lookAt(self, position, target, up):
        # Transform::lookAt: translation = position; rotation columns (right, up', -dir), right handed
        self.translation = tuple(float(v) for v in position)
        d = np.asarray(target, np.float64) - np.asarray(position, np.float64)
        d /= np.linalg.norm(d)
        zc = -d
        right = np.cross(np.asarray(up, np.float64), zc)
        right /= np.linalg.norm(right)
        self._R = np.stack([right, np.cross(zc, right), zc], axis=1)

    @property
    def matrix(self):
        M = np.eye(4)
        M[:3, :3] = self._R @ np.diag(np.asarray(self.scaling, np.float64))
        M[:3, 3] = self.translation
        return M


class _PysMesh:
    def __init__(self, positions=None, indices=None, front_face_cw=False):
        self.positions = [] if positions is None else [tuple(map(float, p)) for p in positions]
        self.indices = [] if indices is None else [int(i) for i in indices]
        self.frontFaceCW = bool(front_face_cw)
        self.name = ""

    def addVertex(self, position, normal=None, texCoord=None):
        self.positions.append(tuple(float(v) for v in position))
        return len(self.positions) - 1

    def addTriangle(self, i0, i1, i2):
        self.indices += [int(i0), int(i1), int(i2)]

    @staticmethod
    def createQuad(size=(1.0, 1.0)):
        hx, hy = 0.5 * float(size[0]), 0.5 * float(size[1])
        return _PysMesh([(-hx, 0, -hy), (hx, 0, -hy), (-hx, 0, hy), (hx, 0, hy)], [2, 1, 0, 1, 2, 3], float(size[0]) * float(size[1]) < 0)

    @staticmethod
    def createDisk(radius=1.0, segments=32):
        P, I = [(0.0, 0.0, 0.0)], []
        for i in range(segments):
            phi = np.float32(i) / np.float32(segments) * np.float32(2.0 * math.pi)
            P.append((math.cos(phi) * radius, 0.0, -math.sin(phi) * radius))
            I += [0, i + 1, (i + 1) % segments + 1]
        return _PysMesh(P, I)

    @staticmethod
    def createCube(size=(1.0, 1.0, 1.0)):
        faces = [[(-.5, -.5, -.5), (-.5, -.5, .5), (.5, -.5, .5), (.5, -.5, -.5)], [(-.5, .5, .5), (-.5, .5, -.5), (.5, .5, -.5), (.5, .5, .5)],
                 [(-.5, .5, -.5), (-.5, -.5, -.5), (.5, -.5, -.5), (.5, .5, -.5)], [(.5, .5, .5), (.5, -.5, .5), (-.5, -.5, .5), (-.5, .5, .5)],
                 [(-.5, .5, .5), (-.5, -.5, .5), (-.5, -.5, -.5), (-.5, .5, -.5)], [(.5, .5, -.5), (.5, -.5, -.5), (.5, -.5, .5), (.5, .5, .5)]]
        s = np.asarray(size, np.float64)
        P, I = [], []
        for f in faces:
            b = len(P)
            I += [b, b + 2, b + 1, b, b + 3, b + 2]
            P += [tuple(np.asarray(v) * s) for v in f]
        return _PysMesh(P, I, float(s[0] * s[1] * s[2]) < 0)

    @staticmethod
    def createSphere(radius=1.0, segmentsU=32, segmentsV=32):
        P, I = [], []
        for v in range(segmentsV + 1):
            for u in range(segmentsU + 1):
                th, ph = u / segmentsU * 2 * math.pi, v / segmentsV * math.pi
                P.append((math.cos(th) * math.sin(ph) * radius, math.cos(ph) * radius, math.sin(th) * math.sin(ph) * radius))
        for v in range(segmentsV):
            for u in range(segmentsU):
                i0, i1 = v * (segmentsU + 1) + u, v * (segmentsU + 1) + (u + 1) % (segmentsU + 1)
                i2, i3 = (v + 1) * (segmentsU + 1) + u, (v + 1) * (segmentsU + 1) + (u + 1) % (segmentsU + 1)
                I += [i0, i1, i2, i2, i1, i3]
        return _PysMesh(P, I)


class _PysMaterial:
    def __init__(self, name="", model=0):
        self.name = name
        self.model = int(model)  # 0 MetalRough, 1 SpecGloss (ShadingModel)
        self.baseColor = (1.0, 1.0, 1.0, 1.0)
        self.specularParams = (0.0, 0.0, 0.0, 0.0)
        self.emissiveColor = (0.0, 0.0, 0.0)
        self.emissiveFactor = 1.0
        self.indexOfRefraction = 1.5
        self.doubleSided = False
        self.specularTransmission = 0.0
        self.diffuseTransmission = 0.0
        self.thinSurface = False

    roughness = property(lambda self: self.specularParams[1],
                         lambda self, v: setattr(self, "specularParams", (self.specularParams[0], float(v)) + tuple(self.specularParams[2:])))
    metallic = property(lambda self: self.specularParams[2],
                        lambda self, v: setattr(self, "specularParams", tuple(self.specularParams[:2]) + (float(v), self.specularParams[3])))

    def loadTexture(self, *a, **k):
        raise ValueError("pyscene: textures are not read")

    load_texture = setTexture = loadTexture

    def row(self):
        if self.specularTransmission > 0 or self.diffuseTransmission > 0:
            warnings.warn(f"pyscene material {self.name!r}: transmission is not built; the pass shades it opaque")
        em = tuple(float(c) * float(self.emissiveFactor) for c in self.emissiveColor[:3])
        base = tuple(float(c) for c in self.baseColor[:3])
        if self.model == 1:
            return spec_gloss_material(base, tuple(self.specularParams[:3]), float(self.specularParams[3]), em, float(self.indexOfRefraction),
                                       bool(self.doubleSided))
        return material(base, float(self.specularParams[1]), em, float(self.specularParams[2]), float(self.indexOfRefraction), bool(self.doubleSided))


class _PysCamera:
    def __init__(self, name=""):
        self.name = name
        self.position, self.target, self.up = (0.0, 0.0, 0.0), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0)
        self.focalLength, self.frameHeight, self.aspectRatio = 21.0, 24.0, 1.7777777
        self.focalDistance, self.apertureRadius, self.shutterSpeed = 10000.0, 0.0, 0.0
        self.nearPlane, self.farPlane = 0.1, 1000.0


class _PysLight:
    kind = "point"

    def __init__(self, name=""):
        self.name = name
        self.intensity = (1.0, 1.0, 1.0)
        self.active = True
        self.position = (0.0, 0.0, 0.0)
        self.direction = (0.0, -1.0, 0.0)  # LightData.dirW's default
        self.openingAngle = math.pi
        self.penumbraAngle = 0.0
        self.angle = 0.5 * 0.53 * math.pi / 180.0  # DistantLight's default: about the sun's half-angle
        self.transform = None
        self.scaling = (1.0, 1.0, 1.0)

    def desc(self):
        d = {"type": self.kind, "intensity": tuple(float(v) for v in self.intensity)}
        if self.kind in ("point", "directional", "distant"):
            d["direction"] = tuple(float(v) for v in self.direction)
        if self.kind == "point":
            d.update(position=tuple(float(v) for v in self.position), openingAngle=float(self.openingAngle),
                     penumbraAngle=float(self.penumbraAngle))
        if self.kind == "distant":
            d["angle"] = float(self.angle)
        if self.kind in ("rect", "disc", "sphere"):
            T = self.transform
            d["transform"] = np.eye(4) if T is None else (T.matrix if isinstance(T, _PysTransform) else np.asarray(T, np.float64))
            d["scaling"] = tuple(float(v) for v in self.scaling)
        return d


class _PysEnvMap:
    """EnvMap (Scene/Lights/EnvMap.cpp:140-157): a lat-long image with rotation (degrees), intensity
    and tint; read from .hdr or .pfm files here."""
    base_dir = Path(".")

    def __init__(self, path):
        p = Path(path)
        self.path = str(p)
        self.texels = read_env_image(p if p.is_absolute() else self.base_dir / p)
        self.rotation = (0.0, 0.0, 0.0)
        self.intensity = 1.0
        self.tint = (1.0, 1.0, 1.0)

    @classmethod
    def createFromFile(cls, path):
        return cls(path)


def _pys_light_class(kind):
    return type(f"_Pys_{kind}", (_PysLight,), {"kind": kind})


def _pys_unsupported(what):
    def f(*a, **k):
        raise ValueError(f"pyscene: {what} is not supported by the pass")
    return f


class _PysSceneBuilder:
    def __init__(self, base_dir):
        self.base_dir = base_dir
        self.meshes, self.nodes, self.instances = [], [], []
        self.materials, self.lights, self.cameras = [], [], []
        self.env = None

    def addMaterial(self, m):
        if m not in self.materials:
            self.materials.append(m)
        return m

    def getMaterial(self, name):
        return next((m for m in self.materials if m.name == name), None)

    def addTriangleMesh(self, triangleMesh, material, isAnimated=False):
        self.addMaterial(material)
        self.meshes.append((triangleMesh, material))
        return len(self.meshes) - 1

    def addNode(self, name, transform=None, parent=None):
        M = np.eye(4) if transform is None else (transform.matrix if isinstance(transform, _PysTransform) else np.asarray(transform, np.float64))
        if parent is not None and parent >= 0:
            M = self.nodes[parent] @ M
        self.nodes.append(M)
        return len(self.nodes) - 1

    def addMeshInstance(self, nodeID, meshID):
        self.instances.append((nodeID, meshID))

    def addLight(self, light):
        self.lights.append(light)
        return len(self.lights) - 1

    def getLight(self, name):
        return next((l for l in self.lights if l.name == name), None)

    def addCamera(self, camera):
        self.cameras.append(camera)
        return len(self.cameras) - 1

    @property
    def envMap(self):
        return self.env

    @envMap.setter
    def envMap(self, value):
        self.env = value

    addSDFGrid = addSDFGridInstance = property(lambda self: _pys_unsupported("an SDF grid"))
    addGridVolume = addVolume = property(lambda self: _pys_unsupported("a grid volume"))
    addCustomPrimitive = property(lambda self: _pys_unsupported("a custom primitive"))
    addAnimation = property(lambda self: _pys_unsupported("an animation"))
    addCurve = property(lambda self: _pys_unsupported("a curve"))


def load_pyscene(path) -> Scene:
    """A Falcor .pyscene file as the pass's triangle soup; info holds "camera" (the first camera the
    script adds, as Camera keyword arguments for pyscene_camera), "lights" (its analytic lights) and
    "env" / "env_params" (its environment map and the map's intensity, tint and rotation).
    The file runs as a Python script, as it does in Falcor: load only scene files you trust."""
    path = Path(path)
    sb = _PysSceneBuilder(path.parent)

    def mesh_from_file(p, *a, **k):
        p = Path(p)
        p = p if p.is_absolute() else path.parent / p
        if p.suffix.lower() != ".obj":
            raise ValueError(f"pyscene: TriangleMesh.createFromFile reads OBJ files here, not {p.suffix}")
        s = load_obj(p)
        return _PysMesh(s.positions.reshape(-1, 3), list(range(len(s.positions) * 3)))

    mesh_class = type("TriangleMesh", (_PysMesh,), {"createFromFile": staticmethod(mesh_from_file)})
    ns = {
        "sceneBuilder": sb, "float2": _pys_vec(2), "float3": _pys_vec(3), "float4": _pys_vec(4), "Transform": _PysTransform,
        "TriangleMesh": mesh_class, "StandardMaterial": _PysMaterial, "Material": _PysMaterial,
        "ShadingModel": type("ShadingModel", (), {"MetalRough": 0, "SpecGloss": 1}), "Camera": _PysCamera,
        "PointLight": _pys_light_class("point"), "DirectionalLight": _pys_light_class("directional"),
        "DistantLight": _pys_light_class("distant"), "RectLight": _pys_light_class("rect"), "DiscLight": _pys_light_class("disc"),
        "SphereLight": _pys_light_class("sphere"), "EnvMap": type("EnvMap", (_PysEnvMap,), {"base_dir": path.parent}),
        "SDFGrid": type("SDFGrid", (), {"__getattr__": lambda self, n: _pys_unsupported("an SDF grid")}),
        "__file__": str(path), "__name__": "__pyscene__",
    }
    for n in ("createSBS", "createNDGrid", "createSVS", "createSVO"):
        setattr(ns["SDFGrid"], n, staticmethod(_pys_unsupported("an SDF grid")))
    exec(compile(path.read_text(), str(path), "exec"), ns)
    rows = [m.row() for m in sb.materials]
    tris, mids = [], []
    for node, mesh_id in sb.instances:
        mesh, mat = sb.meshes[mesh_id]
        M = sb.nodes[node]
        P = np.asarray(mesh.positions, np.float64).reshape(-1, 3)
        W = P @ M[:3, :3].T + M[:3, 3]
        flip = mesh.frontFaceCW != (np.linalg.det(M[:3, :3]) < 0)
        I = np.asarray(mesh.indices, np.int64).reshape(-1, 3)
        for a, b, c in I:
            tris.append(np.concatenate([W[a], W[c], W[b]]) if flip else np.concatenate([W[a], W[b], W[c]]))
            mids.append(sb.materials.index(mat))
    if not tris:
        raise ValueError(f"{path}: no triangle mesh instances")
    info = {"triangles": len(tris), "materials": len(rows)}
    if sb.cameras:
        c = sb.cameras[0]
        info["camera"] = {"position": tuple(c.position), "target": tuple(c.target), "up": tuple(c.up), "focal_length": float(c.focalLength),
                          "frame_height": float(c.frameHeight), "aspect_ratio": float(c.aspectRatio), "focal_distance": float(c.focalDistance),
                          "aperture_radius": float(c.apertureRadius), "shutter_speed": float(c.shutterSpeed), "near_z": float(c.nearPlane),
                          "far_z": float(c.farPlane)}
    lights = [l.desc() for l in sb.lights if getattr(l, "active", True)]
    if lights:
        info["lights"] = lights
    if sb.env is not None:
        info["env"] = sb.env.texels
        info["env_params"] = {"intensity": float(sb.env.intensity), "tint": tuple(float(v) for v in sb.env.tint),
                              "rotation": tuple(float(v) for v in sb.env.rotation)}
    return Scene(np.asarray(tris, np.float32), np.asarray(mids, np.uint32), np.stack(rows).astype(np.float32), path.stem, info)


def pyscene_camera(scene: Scene, width: int, height: int):
    """The pass camera of a load_pyscene scene (its first camera) at the image's aspect ratio."""
    from .scenes import Camera
    c = dict(scene.info["camera"])
    c["aspect_ratio"] = width / height
    return Camera(**c)


# ---------------------------------------------------------------- HDR images for environment maps
# Latitude-longitude environment maps from Radiance .hdr (RGBE, flat or run-length encoded
# scanlines) and Portable Float Map .pfm files, as float32 [H, W, 3] with row 0 at the top (the
# layout rs_set_env_map reads).  OpenEXR and other formats are not decoded.

def _read_hdr(path: Path) -> np.ndarray:
    data = path.read_bytes()
    pos = 0

    def line():
        nonlocal pos
        end = data.index(b"\n", pos)
        s = data[pos:end].decode("ascii", "replace")
        pos = end + 1
        return s

    if not line().startswith("#?"):
        raise ValueError(f"{path}: not a Radiance HDR file")
    while True:
        s = line()
        if s == "":
            break
        if s.startswith("FORMAT=") and s != "FORMAT=32-bit_rle_rgbe":
            raise ValueError(f"{path}: {s} is not read (only 32-bit_rle_rgbe)")
    res = line().split()
    if len(res) != 4 or res[0] != "-Y" or res[2] != "+X":
        raise ValueError(f"{path}: resolution line {' '.join(res)!r} is not read (only -Y H +X W)")
    h, w = int(res[1]), int(res[3])
    rgbe = np.zeros((h, w, 4), np.uint8)
    buf = np.frombuffer(data, np.uint8)
    for y in range(h):
        if 8 <= w < 32768 and buf[pos] == 2 and buf[pos + 1] == 2 and (int(buf[pos + 2]) << 8 | int(buf[pos + 3])) == w:
            pos += 4
            for c in range(4):  # each channel run-length encoded on its own
                x = 0
                while x < w:
                    n = int(buf[pos]); pos += 1
                    if n > 128:
                        n -= 128
                        rgbe[y, x:x + n, c] = buf[pos]; pos += 1
                    else:
                        rgbe[y, x:x + n, c] = buf[pos:pos + n]; pos += n
                    x += n
        else:
            rgbe[y] = buf[pos:pos + 4 * w].reshape(w, 4)
            pos += 4 * w
    e = rgbe[..., 3].astype(np.int32)
    scale = np.where(e > 0, np.ldexp(1.0, e - 136), 0.0).astype(np.float32)
    return rgbe[..., :3].astype(np.float32) * scale[..., None]


def _read_pfm(path: Path) -> np.ndarray:
    data = path.read_bytes()
    parts, pos = [], 0
    while len(parts) < 4:  # "PF" | "Pf", width, height, scale (negative: little endian)
        while data[pos:pos + 1].isspace():
            pos += 1
        end = pos
        while not data[end:end + 1].isspace():
            end += 1
        parts.append(data[pos:end].decode("ascii"))
        pos = end
    pos += 1
    kind, w, h, scale = parts[0], int(parts[1]), int(parts[2]), float(parts[3])
    if kind not in ("PF", "Pf"):
        raise ValueError(f"{path}: not a PFM file")
    ch = 3 if kind == "PF" else 1
    img = np.frombuffer(data, "<f4" if scale < 0 else ">f4", count=w * h * ch, offset=pos).reshape(h, w, ch)
    img = img[::-1].astype(np.float32)  # PFM rows run bottom to top
    return np.repeat(img, 3, axis=2) if ch == 1 else img


def read_env_image(path) -> np.ndarray:
    """A lat-long environment image (.hdr or .pfm) as float32 [H, W, 3], row 0 at the top."""
    path = Path(path)
    ext = path.suffix.lower()
    if ext == ".hdr":
        return _read_hdr(path)
    if ext == ".pfm":
        return _read_pfm(path)
    raise ValueError(f"{path}: environment images are read from .hdr or .pfm files, not {ext}")


def _euler_xyz_degrees(m) -> tuple:
    """extractEulerAngleXYZ (Utils/Math/MatrixMath.h:331-342) of a row-major matrix, in degrees."""
    t1 = math.atan2(m[1][2], m[2][2])
    t2 = math.atan2(-m[0][2], math.sqrt(m[0][0] * m[0][0] + m[0][1] * m[0][1]))
    s1, c1 = math.sin(t1), math.cos(t1)
    t3 = math.atan2(s1 * m[2][0] - c1 * m[1][0], c1 * m[1][1] - s1 * m[2][1])
    return tuple(math.degrees(-a) for a in (t1, t2, t3))


def equal_area_oct_to_latlong(img: np.ndarray) -> np.ndarray:
    """EnvMapConverter (PBRTImporter/EnvMapConverter.cs.slang, .h): a square equal-area octahedral map
    [N, N, 3] to a lat-long map [N, 2N, 3]: per output texel centre its direction
    (latlong_map_to_world, MathHelpers.slang:128-137), that direction's equal-area octahedral
    coordinates (ndir_to_oct_equal_area_unorm, :213-230), and a bilinear, clamp-to-edge fetch."""
    n = img.shape[0]
    if img.shape[1] != n:
        raise ValueError("an equal-area octahedral map is square")
    h, w = n, 2 * n
    u = (np.arange(w, dtype=np.float64) + 0.5) / w
    v = (np.arange(h, dtype=np.float64) + 0.5) / h
    phi = math.pi * (2.0 * u[None, :] - 1.0)
    theta = math.pi * v[:, None]
    dx, dy, dz = np.sin(theta) * np.sin(phi), np.cos(theta) * np.ones_like(phi), -np.sin(theta) * np.cos(phi)
    r = np.sqrt(1.0 - np.abs(dz))
    ang = np.arctan2(np.abs(dy), np.abs(dx))
    py = r * ang * (2.0 / math.pi)
    px = r - py
    lower = dz < 0.0
    px, py = np.where(lower, 1.0 - py, px), np.where(lower, 1.0 - px, py)
    px, py = px * np.sign(dx), py * np.sign(dy)
    ou, ov = px * 0.5 + 0.5, py * 0.5 + 0.5
    fx, fy = ou * n - 0.5, ov * n - 0.5
    x0, y0 = np.floor(fx).astype(np.int64), np.floor(fy).astype(np.int64)
    ax, ay = (fx - x0)[..., None], (fy - y0)[..., None]
    cl = lambda i: np.clip(i, 0, n - 1)
    src = img.astype(np.float64)
    top = src[cl(y0), cl(x0)] * (1 - ax) + src[cl(y0), cl(x0 + 1)] * ax
    bot = src[cl(y0 + 1), cl(x0)] * (1 - ax) + src[cl(y0 + 1), cl(x0 + 1)] * ax
    return (top * (1 - ay) + bot * ay).astype(np.float32)
