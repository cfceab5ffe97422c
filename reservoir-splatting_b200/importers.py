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
from pathlib import Path

import numpy as np

from .scenes import Scene, spec_gloss_material


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
