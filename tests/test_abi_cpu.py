"""The C ABI library loads without a GPU, exports every symbol include/rs_b200.h declares, and
its host-side option handling follows the reference pass (no device work is started here)."""
import ctypes as C
import re
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "rs_b200.h"


def declared_symbols():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"RS_API\s+[\w\s\*]+?\b(rs_\w+)\s*\(", text)))


def test_header_declares_the_pass_interface():
    syms = declared_symbols()
    for name in ("rs_create", "rs_destroy", "rs_set_options", "rs_set_scene", "rs_execute", "rs_reset",
                 "rs_set_seed", "rs_freeze", "rs_get_buffer", "rs_set_buffer", "rs_last_error_string"):
        assert name in syms


def test_library_exports_every_declared_symbol(rs):
    lib = rs.load_library()
    missing = [s for s in declared_symbols() if not hasattr(lib, s)]
    assert not missing, missing


def test_default_options_match_reference_defaults(rs):
    lib = rs.load_library()
    o = rs.abi.RsOptions()
    lib.rs_default_options(C.byref(o))
    ref = rs.abi.default_options(1920, 1080)
    for name, _ in rs.abi.RsOptions._fields_:
        assert getattr(o, name) == pytest.approx(getattr(ref, name)), name
    # ReservoirSplatting.h:124-184
    assert o.samplesPerPixel == 1 and o.maxSurfaceBounces == 9 and o.temporalReuse == 0 and o.gatherOption == 0
    assert o.enableSpatialResampling == 1 and o.neighborCount == 1 and o.spatialGatherRadius == 30.0
    assert o.numTimePartitions == 2 and o.artificialFrameTime == pytest.approx(1 / 60)


def test_properties_parse_like_the_render_graph_script(rs):
    # scripts/ReservoirSplatting.py:13-21
    props = {"samplesPerPixel": 1, "enableTemporalResampling": True, "enableSpatialResampling": True,
             "temporalReuse": "ScatterOnly", "numTimePartitions": 2, "hybridMISOption": "Balance", "gatherOption": "Fast"}
    o = rs.abi.options_from_properties(props, 640, 480)
    assert o.temporalReuse == 1 and o.scatterBackupMISOption == 0 and o.gatherOption == 0
    o = rs.abi.options_from_properties({"maxSurfaceBounces": 3}, 64, 64)
    assert (o.maxDiffuseBounces, o.maxSpecularBounces, o.maxTransmissionBounces) == (3, 3, 3)
    o = rs.abi.options_from_properties({"maxDiffuseBounces": 4, "maxSpecularBounces": 2}, 64, 64)
    assert o.maxSurfaceBounces == 9  # max of the per-type limits (the transmission default is 9)
    o = rs.abi.options_from_properties({"fixedSeed": 7}, 64, 64)
    assert o.useFixedSeed == 1 and o.fixedSeed == 7
    with pytest.raises(KeyError):
        rs.abi.options_from_properties({"noSuchKey": 1}, 64, 64)
    with pytest.raises(ValueError):
        rs.abi.options_from_properties({"temporalReuse": "Sideways"}, 64, 64)


def test_every_reference_property_key_is_accepted(rs):
    # every scripting key of ReservoirSplatting.cpp:99-131, with the reference's default values
    props = {"samplesPerPixel": 1, "maxSurfaceBounces": 3, "maxDiffuseBounces": 3, "maxSpecularBounces": 3,
             "maxTransmissionBounces": 10, "sampleGenerator": "TinyUniform", "fixedSeed": 1, "useRussianRoulette": False,
             "misHeuristic": "Balance", "misPowerExponent": 2.0, "emissiveSampler": "Power", "lightBVHOptions": {},
             "useAlphaTest": True, "adjustShadingNormals": False, "maxNestedMaterials": 2,
             "useLightsInDielectricVolumes": False, "disableCaustics": False, "specularRoughnessThreshold": 0.25,
             "primaryLodMode": "Mip0", "lodBias": 0.0, "outputSize": "Default", "fixedOutputSize": (512, 512),
             "colorFormat": "LogLuvHDR", "enableTemporalResampling": True, "enableSpatialResampling": True,
             "temporalReuse": "ScatterBackup", "scatterBackupMISOption": "Pairwise", "gatherOption": "Clamped",
             "numTimePartitions": 2}
    o = rs.abi.options_from_properties(props, 320, 240)
    assert (o.frameWidth, o.frameHeight) == (320, 240) and o.temporalReuse == 2 and o.gatherOption == 1
    assert o.scatterBackupMISOption == 1 and o.maxTransmissionBounces == 10 and o.useFixedSeed == 1
    o = rs.abi.options_from_properties({"outputSize": "Half"}, 320, 240)
    assert (o.frameWidth, o.frameHeight) == (160, 120)
    o = rs.abi.options_from_properties({"outputSize": "Fixed", "fixedOutputSize": (96, 64)}, 320, 240)
    assert (o.frameWidth, o.frameHeight) == (96, 64)
    assert rs.abi.options_from_properties({"emissiveSampler": "Uniform"}, 64, 64).emissiveSampler == 0
    assert o.emissiveSampler == 2  # Power, the default (EmissiveLightSamplerType::Power)
    with pytest.raises(ValueError):
        rs.abi.options_from_properties({"emissiveSampler": "LightBVH"}, 64, 64)
    with pytest.raises(ValueError):
        rs.abi.options_from_properties({"outputSize": "Triple"}, 64, 64)


@pytest.mark.parametrize("bad", [{"samplesPerPixel": 0}, {"samplesPerPixel": 17}, {"numTimePartitions": 9},
                                 {"maxDiffuseBounces": 300}, {"specularRoughnessThreshold": 2.0},
                                 {"misHeuristic": "PowerExp", "misPowerExponent": 0.0},
                                 {"misHeuristic": "PowerExp", "misPowerExponent": 11.0}])
def test_invalid_options_are_rejected_before_any_device_work(rs, bad):
    lib = rs.load_library()
    o = rs.abi.options_from_properties(bad, 64, 64)
    h = C.c_void_p()
    st = lib.rs_create(C.byref(o), C.byref(h))
    assert st == rs.abi.RS_INVALID_ARG
    assert lib.rs_last_error_string()


def test_light_bvh_sampler_is_rejected(rs):
    lib = rs.load_library()
    o = rs.abi.default_options(64, 64)
    o.emissiveSampler = 1  # EmissiveLightSamplerType::LightBVH, not built
    h = C.c_void_p()
    assert lib.rs_create(C.byref(o), C.byref(h)) == rs.abi.RS_INVALID_ARG
    assert b"LightBVH" in lib.rs_last_error_string()


def test_oversized_frame_is_rejected(rs):
    lib = rs.load_library()
    o = rs.abi.options_from_properties({}, 4097, 16)
    h = C.c_void_p()
    assert lib.rs_create(C.byref(o), C.byref(h)) == rs.abi.RS_INVALID_ARG
    assert b"4096" in lib.rs_last_error_string()


def test_null_arguments_return_errors(rs):
    lib = rs.load_library()
    assert lib.rs_destroy(None) == rs.abi.RS_INVALID_ARG
    assert lib.rs_execute(None, None, None) == rs.abi.RS_INVALID_ARG
    assert lib.rs_last_launch_count(None) == 0


def test_missing_library_fails_loudly(rs, tmp_path, monkeypatch):
    monkeypatch.setattr(rs, "_lib", None)
    monkeypatch.setattr(rs, "LIB_PATH", tmp_path / "librs_b200.so")
    with pytest.raises(RuntimeError, match="CUDA library missing"):
        rs.ReservoirSplatting({}, 16, 16)


def _fields(o):
    return {name: getattr(o, name) for name, _ in o._fields_}


@pytest.mark.parametrize("props", [{}, {"fixedSeed": 9, "misHeuristic": "PowerExp", "misPowerExponent": 3.5, "emissiveSampler": "Uniform",
                                        "temporalReuse": "MultiScatter", "numTimePartitions": 4, "gatherOption": "Robust",
                                        "maxDiffuseBounces": 2, "maxSpecularBounces": 5, "maxTransmissionBounces": 1,
                                        "neighborCount": 3, "spatialGatherRadius": 12.5, "disableCaustics": True},
                                   {"outputSize": "Fixed", "fixedOutputSize": (96, 64), "samplesPerPixel": 4, "maxSurfaceBounces": 2},
                                   {"outputSize": "Half", "enableTemporalResampling": False, "scatterBackupMISOption": "Pairwise"}])
def test_get_properties_round_trips(rs, props):
    """properties_from_options is getProperties (ReservoirSplatting.cpp:303-344): parsing its dict
    gives the same options back, and the reference's keys come first, in its order."""
    o = rs.abi.options_from_properties(props, 320, 240)
    got = rs.abi.properties_from_options(o, *rs.abi.output_size_selection(props))
    assert _fields(rs.abi.options_from_properties(got, 320, 240)) == _fields(o)
    keys = list(got)
    assert keys[:5] == ["samplesPerPixel", "maxSurfaceBounces", "maxDiffuseBounces", "maxSpecularBounces", "maxTransmissionBounces"]
    assert ("fixedSeed" in got) == bool(o.useFixedSeed) and ("fixedOutputSize" in got) == (got["outputSize"] == "Fixed")
    assert keys.index("colorFormat") < keys.index("enableTemporalResampling")
    assert "lightBVHOptions" not in got


def test_properties_given_later_keep_the_others(rs):
    """setProperties parses only the keys it is given (ReservoirSplatting.cpp:192-261): the others
    keep their values; maxSurfaceBounces resets the per-type limits not named beside it (:236-241)."""
    base = rs.abi.options_from_properties({"temporalReuse": "ScatterBackup", "gatherOption": "Clamped", "fixedSeed": 3,
                                           "maxDiffuseBounces": 2, "maxSpecularBounces": 4}, 64, 64)
    o = rs.abi.options_from_properties({"enableSpatialResampling": False}, 64, 64, base=base)
    assert o.temporalReuse == 2 and o.gatherOption == 1 and o.useFixedSeed == 1 and o.fixedSeed == 3
    assert o.enableSpatialResampling == 0 and (o.maxDiffuseBounces, o.maxSpecularBounces, o.maxSurfaceBounces) == (2, 4, 9)
    o = rs.abi.options_from_properties({"maxSurfaceBounces": 3, "maxSpecularBounces": 1}, 64, 64, base=base)
    assert (o.maxSurfaceBounces, o.maxDiffuseBounces, o.maxSpecularBounces, o.maxTransmissionBounces) == (3, 3, 1, 3)
    o = rs.abi.options_from_properties({"outputSize": "Quarter"}, 64, 64, base=base)
    assert (o.frameWidth, o.frameHeight) == (16, 16) and o.temporalReuse == 2
