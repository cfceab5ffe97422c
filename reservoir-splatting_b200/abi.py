"""ctypes mirror of include/rs_b200.h and the property parsing of the reference pass.

`options_from_properties` accepts the property dictionary a Falcor render-graph
script passes to ``createPass("ReservoirSplatting", {...})``
(scripts/ReservoirSplatting.py:13-21, keys of ReservoirSplatting.cpp:99-131),
including the enum values by name ("ScatterBackup", "Clamped", "Pairwise", ...).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

RS_OK, RS_INVALID_ARG, RS_OOM, RS_CUDA_ERROR, RS_DEVICE_FAULT, RS_NOT_READY = range(6)
STATUS_NAMES = {0: "RS_OK", 1: "RS_INVALID_ARG", 2: "RS_OOM", 3: "RS_CUDA_ERROR", 4: "RS_DEVICE_FAULT", 5: "RS_NOT_READY"}

TEMPORAL_REUSE = {"GatherOnly": 0, "ScatterOnly": 1, "ScatterBackup": 2, "MultiScatter": 3}
GATHER_MECHANISM = {"Fast": 0, "Clamped": 1, "Robust": 2}
SCATTER_BACKUP_MIS = {"Balance": 0, "Pairwise": 1}
MIS_HEURISTIC = {"Balance": 0, "PowerTwo": 1, "PowerExp": 2}
EMISSIVE_SAMPLER = {"Uniform": 0, "LightBVH": 1, "Power": 2}
SAMPLE_GENERATOR = {"TinyUniform": 0, "PCG32": 2}

BUF = {
    "curr_reservoirs": 0, "curr_reconnection": 1, "prev_reservoirs": 2, "prev_reconnection": 3,
    "cell_counters": 4, "cell_offsets": 5, "sorted_splats": 6, "floating_coords": 7, "mvec": 8, "vbuffer": 9,
    "splat_targets": 10, "candidate_reservoirs": 11, "candidate_reconnection": 12,
    "backup_reservoirs": 13, "backup_reconnection": 14, "env_importance": 15,
}


class RsOptions(C.Structure):
    _fields_ = [
        ("samplesPerPixel", C.c_uint32), ("maxSurfaceBounces", C.c_uint32), ("maxDiffuseBounces", C.c_uint32),
        ("maxSpecularBounces", C.c_uint32), ("maxTransmissionBounces", C.c_uint32), ("sampleGenerator", C.c_uint32),
        ("useFixedSeed", C.c_uint32), ("fixedSeed", C.c_uint32), ("useRussianRoulette", C.c_uint32),
        ("misHeuristic", C.c_uint32), ("misPowerExponent", C.c_float), ("disableCaustics", C.c_uint32),
        ("specularRoughnessThreshold", C.c_float), ("enableTemporalResampling", C.c_uint32),
        ("enableSpatialResampling", C.c_uint32), ("temporalReuse", C.c_uint32), ("scatterBackupMISOption", C.c_uint32),
        ("gatherOption", C.c_uint32), ("numTimePartitions", C.c_uint32), ("useConfidenceWeightsTemporally", C.c_uint32),
        ("numSpatialIterations", C.c_uint32), ("spatialGatherRadius", C.c_float), ("neighborCount", C.c_uint32),
        ("useConfidenceWeightsSpatially", C.c_uint32), ("artificialFrameTime", C.c_float), ("frameWidth", C.c_uint32),
        ("frameHeight", C.c_uint32), ("emissiveSampler", C.c_uint32),
    ]


class RsEnvMap(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("texels", C.c_void_p), ("intensity", C.c_float),
                ("tint", C.c_float * 3), ("rotation", C.c_float * 3)]


class RsAnalyticLight(C.Structure):
    _fields_ = [("type", C.c_uint32), ("intensity", C.c_float * 3), ("position", C.c_float * 3), ("direction", C.c_float * 3),
                ("openingAngle", C.c_float), ("penumbraAngle", C.c_float), ("angle", C.c_float), ("transform", C.c_float * 16),
                ("scaling", C.c_float * 3)]


LIGHT_TYPE = {"point": 0, "directional": 1, "distant": 2, "rect": 3, "disc": 4, "sphere": 5}


def analytic_lights_array(lights) -> C.Array:
    """rs_analytic_light[] from dicts with the keys of Falcor's light classes (Scene/Lights/Light.h):
    "type" (point, directional, distant, rect, disc, sphere), "intensity", "position", "direction",
    "openingAngle", "penumbraAngle", "angle", "transform" (4x4 object-to-world) and "scaling"."""
    lights = list(lights or [])
    arr = (RsAnalyticLight * max(1, len(lights)))()
    for i, d in enumerate(lights):
        L = arr[i]
        t = d.get("type", "point")
        if t not in LIGHT_TYPE:
            raise ValueError(f"unknown analytic light type {t!r}")
        L.type = LIGHT_TYPE[t]
        L.intensity[:] = [float(v) for v in d.get("intensity", (1.0, 1.0, 1.0))]
        L.position[:] = [float(v) for v in d.get("position", (0.0, 0.0, 0.0))]
        L.direction[:] = [float(v) for v in d.get("direction", (0.0, -1.0, 0.0))]
        L.openingAngle = float(d.get("openingAngle", np.pi))
        L.penumbraAngle = float(d.get("penumbraAngle", 0.0))
        L.angle = float(d.get("angle", 0.5 * np.pi / 180.0))
        L.transform[:] = [float(v) for v in np.asarray(d.get("transform", np.eye(4)), np.float64).reshape(16)]
        L.scaling[:] = [float(v) for v in d.get("scaling", (1.0, 1.0, 1.0))]
    return arr


def env_map_struct(texels, intensity=1.0, tint=(1.0, 1.0, 1.0), rotation=(0.0, 0.0, 0.0)) -> tuple[RsEnvMap, np.ndarray | None]:
    """Descriptor of a lat-long map given as float [H, W, 3] or [H, W, 4] (row 0 at the top), and the
    RGBA array it points into (keep it alive during the call).  None removes the map."""
    e = RsEnvMap()
    if texels is None:
        return e, None
    t = np.asarray(texels, np.float32)
    if t.ndim != 3 or t.shape[2] not in (3, 4):
        raise ValueError("env map texels must be [H, W, 3] or [H, W, 4]")
    rgba = np.zeros((t.shape[0], t.shape[1], 4), np.float32)
    rgba[..., :t.shape[2]] = t
    rgba = np.ascontiguousarray(rgba)
    e.width, e.height, e.texels = t.shape[1], t.shape[0], rgba.ctypes.data
    e.intensity = float(intensity)
    e.tint[:] = [float(v) for v in tint]
    e.rotation[:] = [float(v) for v in rotation]
    return e, rgba


class RsSceneDesc(C.Structure):
    _fields_ = [("numTriangles", C.c_uint32), ("positions", C.c_void_p), ("materialIds", C.c_void_p),
                ("numMaterials", C.c_uint32), ("materials", C.c_void_p)]


class RsCamera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("target", C.c_float * 3), ("up", C.c_float * 3),
                ("focalLength", C.c_float), ("frameHeight", C.c_float), ("aspectRatio", C.c_float),
                ("focalDistance", C.c_float), ("apertureRadius", C.c_float), ("shutterSpeed", C.c_float),
                ("nearZ", C.c_float), ("farZ", C.c_float)]


class RsFrameDesc(C.Structure):
    _fields_ = [("camera", RsCamera), ("mvec", C.c_void_p), ("vbuffer", C.c_void_p), ("color", C.c_void_p),
                ("colorHost", C.c_void_p), ("sceneShouldReset", C.c_uint32)]


TONEMAP_OPERATOR = {"Linear": 0, "Reinhard": 1, "ReinhardModified": 2, "HejiHableAlu": 3, "HableUc2": 4, "Aces": 5}


class RsBatchTuningEntry(C.Structure):
    _fields_ = [("stage", C.c_uint32), ("width", C.c_uint32), ("height", C.c_uint32), ("tile", C.c_uint32), ("grid", C.c_uint32),
                ("ms", C.c_float)]


# rs_batch_tuning_entry.stage
BATCH_STAGES = ["candidates", "sbCurrScatter", "sbCurrGather", "sbBackupGather", "sbBackupScatter", "sbSplatScatter", "sbSplatGather",
                "spatialCentral", "spatialNeighbor", "vbuffer", "reproject", "sbCombine", "spatialCombine"]


class RsTonemapOptions(C.Structure):
    _fields_ = [("op", C.c_uint32), ("exposureCompensation", C.c_float), ("autoExposure", C.c_uint32), ("filmSpeed", C.c_float),
                ("fNumber", C.c_float), ("shutter", C.c_float), ("clamp", C.c_uint32), ("whiteMaxLuminance", C.c_float),
                ("whiteScale", C.c_float), ("whiteBalance", C.c_uint32), ("whitePoint", C.c_float)]


def default_options(width: int = 1920, height: int = 1080) -> RsOptions:
    """ReservoirSplatting.h:124-184 defaults (the C library's rs_default_options, restated for CPU-only use)."""
    o = RsOptions()
    o.samplesPerPixel = 1
    o.maxSurfaceBounces = o.maxDiffuseBounces = o.maxSpecularBounces = o.maxTransmissionBounces = 9
    o.sampleGenerator = 0
    o.useFixedSeed = 0
    o.fixedSeed = 1
    o.useRussianRoulette = 1
    o.misHeuristic = 0
    o.misPowerExponent = 2.0
    o.disableCaustics = 0
    o.specularRoughnessThreshold = 0.25
    o.enableTemporalResampling = 1
    o.enableSpatialResampling = 1
    o.temporalReuse = TEMPORAL_REUSE["GatherOnly"]
    o.scatterBackupMISOption = 0
    o.gatherOption = GATHER_MECHANISM["Fast"]
    o.numTimePartitions = 2
    o.useConfidenceWeightsTemporally = 1
    o.numSpatialIterations = 1
    o.spatialGatherRadius = 30.0
    o.neighborCount = 1
    o.useConfidenceWeightsSpatially = 1
    o.artificialFrameTime = 1.0 / 60.0
    o.frameWidth = width
    o.frameHeight = height
    o.emissiveSampler = EMISSIVE_SAMPLER["Power"]
    return o


_ENUMS = {"temporalReuse": TEMPORAL_REUSE, "gatherOption": GATHER_MECHANISM, "scatterBackupMISOption": SCATTER_BACKUP_MIS,
          "hybridMISOption": SCATTER_BACKUP_MIS, "misHeuristic": MIS_HEURISTIC, "sampleGenerator": SAMPLE_GENERATOR}
_ALIASES = {"hybridMISOption": "scatterBackupMISOption"}


# Properties of ReservoirSplatting.cpp:99-131 that change nothing this build renders: alpha testing
# (the scenes carry no alpha textures), shading-normal adjustment (shading uses face normals), nested
# dielectrics and lights inside them (materials are opaque), texture LOD (no textures) and the
# internal colour format (declared by the reference, read by none of its shaders).  They are
# accepted so that a render-graph script runs unchanged.
_NO_EFFECT = {"useAlphaTest", "adjustShadingNormals", "maxNestedMaterials", "useLightsInDielectricVolumes", "primaryLodMode",
              "lodBias", "colorFormat", "lightBVHOptions"}
# RenderPassHelpers::IOSize of the outputSize property: the frame size relative to the default
# (the createPass width and height), or fixedOutputSize.
_IO_SIZE = {"Default": 1.0, "Full": 1.0, "Half": 0.5, "Quarter": 0.25, "Double": 2.0}


def options_from_properties(props: dict | None, width: int, height: int, base: RsOptions | None = None) -> RsOptions:
    """parseProperties (ReservoirSplatting.cpp:192-261) for a createPass() property dict: keys not
    given keep their values in `base` (the defaults without one); width and height are the default
    frame size that outputSize selects from."""
    o = default_options(width, height)
    if base is not None:
        C.memmove(C.byref(o), C.byref(base), C.sizeof(RsOptions))
        o.frameWidth, o.frameHeight = width, height
    props = dict(props or {})
    names = {f for f, _ in RsOptions._fields_}
    size = props.get("outputSize")
    if isinstance(size, str):
        if size == "Fixed":
            fixed = props.get("fixedOutputSize", (512, 512))
            o.frameWidth, o.frameHeight = int(fixed[0]), int(fixed[1])
        elif size in _IO_SIZE:
            o.frameWidth, o.frameHeight = max(1, int(width * _IO_SIZE[size])), max(1, int(height * _IO_SIZE[size]))
        else:
            raise ValueError(f"unknown value {size!r} for property 'outputSize'")
    for key, value in props.items():
        if key in _NO_EFFECT or key == "fixedOutputSize" or (key == "outputSize" and isinstance(value, str)):
            continue
        if key == "emissiveSampler":
            v = EMISSIVE_SAMPLER.get(value, value) if isinstance(value, str) else int(value)
            if isinstance(v, str):
                raise ValueError(f"unknown value {value!r} for property 'emissiveSampler'")
            if v not in (0, 2):
                raise ValueError("emissiveSampler: the Uniform and Power samplers are built (LightBVH is not)")
            o.emissiveSampler = v
            continue
        field = _ALIASES.get(key, key)
        if key in _ENUMS and isinstance(value, str):
            if value not in _ENUMS[key]:
                raise ValueError(f"unknown value {value!r} for property {key!r}")
            value = _ENUMS[key][value]
        if key == "fixedSeed":
            o.fixedSeed = int(value)
            o.useFixedSeed = 1
            continue
        if key == "outputSize":
            o.frameWidth, o.frameHeight = int(value[0]), int(value[1])
            continue
        if field not in names:
            raise KeyError(f"Unknown property '{key}' in ReservoirSplatting properties.")
        setattr(o, field, type(getattr(o, field))(value))
    # maxSurfaceBounces initialises the per-type limits that are not given explicitly (:236-247)
    if "maxSurfaceBounces" in props:
        for k in ("maxDiffuseBounces", "maxSpecularBounces", "maxTransmissionBounces"):
            if k not in props:
                setattr(o, k, o.maxSurfaceBounces)
    else:
        o.maxSurfaceBounces = max(o.maxDiffuseBounces, o.maxSpecularBounces, o.maxTransmissionBounces)
    o.maxSurfaceBounces = max(o.maxSurfaceBounces, o.maxDiffuseBounces, o.maxSpecularBounces, o.maxTransmissionBounces)
    return o


def _enum_name(table: dict, value: int) -> str | int:
    return next((k for k, v in table.items() if v == value), int(value))


def properties_from_options(o: RsOptions, output_size="Default", fixed_output_size=(512, 512)) -> dict:
    """getProperties (ReservoirSplatting.cpp:303-344): the scripting keys in the reference's order,
    fixedSeed only when a fixed seed is set, fixedOutputSize only with outputSize "Fixed", and the
    keys that change nothing here at the values this build renders with.  The reference leaves the
    ReSTIR keys (:125-130) out of its dict; they follow here, with the further ReSTIR parameters of
    the options struct, so that options_from_properties(properties_from_options(o)) gives o back."""
    p = {"samplesPerPixel": int(o.samplesPerPixel), "maxSurfaceBounces": int(o.maxSurfaceBounces),
         "maxDiffuseBounces": int(o.maxDiffuseBounces), "maxSpecularBounces": int(o.maxSpecularBounces),
         "maxTransmissionBounces": int(o.maxTransmissionBounces),
         "sampleGenerator": _enum_name(SAMPLE_GENERATOR, o.sampleGenerator)}
    if o.useFixedSeed:
        p["fixedSeed"] = int(o.fixedSeed)
    p.update({"useRussianRoulette": bool(o.useRussianRoulette), "misHeuristic": _enum_name(MIS_HEURISTIC, o.misHeuristic),
              "misPowerExponent": float(o.misPowerExponent), "emissiveSampler": _enum_name(EMISSIVE_SAMPLER, o.emissiveSampler),
              "useAlphaTest": True, "adjustShadingNormals": False, "maxNestedMaterials": 2,
              "useLightsInDielectricVolumes": False, "disableCaustics": bool(o.disableCaustics),
              "specularRoughnessThreshold": float(o.specularRoughnessThreshold), "primaryLodMode": "Mip0", "lodBias": 0.0,
              "outputSize": output_size})
    if output_size == "Fixed":
        p["fixedOutputSize"] = (int(fixed_output_size[0]), int(fixed_output_size[1]))
    p["colorFormat"] = "LogLuvHDR"
    p.update({"enableTemporalResampling": bool(o.enableTemporalResampling),
              "enableSpatialResampling": bool(o.enableSpatialResampling),
              "temporalReuse": _enum_name(TEMPORAL_REUSE, o.temporalReuse),
              "scatterBackupMISOption": _enum_name(SCATTER_BACKUP_MIS, o.scatterBackupMISOption),
              "gatherOption": _enum_name(GATHER_MECHANISM, o.gatherOption), "numTimePartitions": int(o.numTimePartitions),
              "useConfidenceWeightsTemporally": int(o.useConfidenceWeightsTemporally),
              "numSpatialIterations": int(o.numSpatialIterations), "spatialGatherRadius": float(o.spatialGatherRadius),
              "neighborCount": int(o.neighborCount), "useConfidenceWeightsSpatially": int(o.useConfidenceWeightsSpatially),
              "artificialFrameTime": float(o.artificialFrameTime)})
    return p


def output_size_selection(props: dict | None) -> tuple:
    """The outputSize selection and fixedOutputSize a property dict makes (ReservoirSplatting.cpp:223-225);
    a (width, height) pair given as outputSize counts as a fixed size."""
    props = props or {}
    size = props.get("outputSize", "Default")
    if isinstance(size, str):
        return size, tuple(props.get("fixedOutputSize", (512, 512)))
    return "Fixed", (int(size[0]), int(size[1]))


def camera_struct(cam) -> RsCamera:
    c = RsCamera()
    c.position[:] = [float(v) for v in cam.position]
    c.target[:] = [float(v) for v in cam.target]
    c.up[:] = [float(v) for v in cam.up]
    c.focalLength = cam.focal_length
    c.frameHeight = cam.frame_height
    c.aspectRatio = cam.aspect_ratio
    c.focalDistance = cam.focal_distance
    c.apertureRadius = cam.aperture_radius
    c.shutterSpeed = cam.shutter_speed
    c.nearZ = cam.near_z
    c.farZ = cam.far_z
    return c


def scene_struct(scene) -> tuple[RsSceneDesc, tuple]:
    """Returns the descriptor and the arrays it points into (keep them alive during the call)."""
    pos = np.ascontiguousarray(scene.positions, np.float32)
    mid = np.ascontiguousarray(scene.material_ids, np.uint32)
    mats = np.ascontiguousarray(scene.materials, np.float32)
    d = RsSceneDesc()
    d.numTriangles = pos.shape[0]
    d.positions = pos.ctypes.data
    d.materialIds = mid.ctypes.data
    d.numMaterials = mats.shape[0]
    d.materials = mats.ctypes.data
    return d, (pos, mid, mats)


BUFFER_LAYOUT = {
    "curr_reservoirs": (np.float32, 8), "prev_reservoirs": (np.float32, 8), "candidate_reservoirs": (np.float32, 8),
    "backup_reservoirs": (np.float32, 8),
    "curr_reconnection": (np.uint32, 28), "prev_reconnection": (np.uint32, 28), "candidate_reconnection": (np.uint32, 28),
    "backup_reconnection": (np.uint32, 28), "env_importance": (np.float32, 1),
    "cell_counters": (np.uint32, 1), "cell_offsets": (np.uint32, 1), "sorted_splats": (np.uint32, 1),
    "splat_targets": (np.uint32, 1), "floating_coords": (np.float32, 2), "mvec": (np.float32, 2), "vbuffer": (np.uint32, 4),
}
