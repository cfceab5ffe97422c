"""Frame files of the FrameDumper mirror: the PAM header of FrameDumper.cpp:156-157 byte for byte,
texels in row order, and an 8-bit RGBA PNG that decodes to the same texels."""
import struct
import zlib

import numpy as np
import pytest


def test_pam_header_and_round_trip(rs, tmp_path):
    import reservoir_splatting_b200.frame_output as FO
    img = np.random.default_rng(0).integers(0, 256, (5, 7, 4), dtype=np.uint8)
    p = tmp_path / "frame.00000.pam"
    FO.write_pam(p, img)
    data = p.read_bytes()
    header = b"P7\nWIDTH 7\nHEIGHT 5\nDEPTH 4\nMAXVAL 255\nTUPLTYPE RGB_ALPHA\nENDHDR\n"
    assert data[:len(header)] == header and len(data) == len(header) + img.size
    np.testing.assert_array_equal(FO.read_pam(p), img)


def test_png_decodes_to_the_texels(rs, tmp_path):
    import reservoir_splatting_b200.frame_output as FO
    img = np.random.default_rng(1).integers(0, 256, (9, 6, 4), dtype=np.uint8)
    p = tmp_path / "frame.00000.png"
    FO.write_png(p, img)
    data = p.read_bytes()
    assert data[:8] == b"\x89PNG\r\n\x1a\n"
    pos, idat, ihdr = 8, b"", None
    while pos < len(data):
        n = struct.unpack(">I", data[pos:pos + 4])[0]
        tag, payload = data[pos + 4:pos + 8], data[pos + 8:pos + 8 + n]
        assert struct.unpack(">I", data[pos + 8 + n:pos + 12 + n])[0] == zlib.crc32(tag + payload) & 0xffffffff
        if tag == b"IHDR":
            ihdr = struct.unpack(">IIBBBBB", payload)
        elif tag == b"IDAT":
            idat += payload
        pos += 12 + n
    assert ihdr == (6, 9, 8, 6, 0, 0, 0)
    raw = np.frombuffer(zlib.decompress(idat), np.uint8).reshape(9, 1 + 6 * 4)
    assert (raw[:, 0] == 0).all()
    np.testing.assert_array_equal(raw[:, 1:].reshape(9, 6, 4), img)


def test_tonemap_options_by_name(rs):
    import reservoir_splatting_b200.abi as abi
    assert abi.TONEMAP_OPERATOR == {"Linear": 0, "Reinhard": 1, "ReinhardModified": 2, "HejiHableAlu": 3, "HableUc2": 4, "Aces": 5}


def test_tonemap_rejects_bad_arguments_before_device_work(rs):
    """rs_tonemap validates its arguments before any device work (callable without a GPU)."""
    import ctypes as C
    import reservoir_splatting_b200.frame_output as FO
    lib = rs.load_library()
    o = FO.tonemap_options()
    fake = C.c_void_p(0x1000)  # never dereferenced: every call below fails validation
    assert lib.rs_tonemap(None, 4, 4, C.byref(o), fake, None, None) == rs.abi.RS_INVALID_ARG
    assert lib.rs_tonemap(fake, 4, 4, None, fake, None, None) == rs.abi.RS_INVALID_ARG
    assert lib.rs_tonemap(fake, 4, 4, C.byref(o), None, None, None) == rs.abi.RS_INVALID_ARG
    bad = FO.tonemap_options(op=6 - 1)
    bad.op = 6
    assert lib.rs_tonemap(fake, 4, 4, C.byref(bad), fake, None, None) == rs.abi.RS_INVALID_ARG
    assert lib.rs_tonemap(fake, 4, 4, C.byref(FO.tonemap_options(fNumber=0.0)), fake, None, None) == rs.abi.RS_INVALID_ARG
    assert lib.rs_tonemap(fake, 4, 4, C.byref(FO.tonemap_options(autoExposure=1)), fake, None, None) == rs.abi.RS_INVALID_ARG
    assert lib.rs_tonemap(fake, 0, 4, C.byref(o), fake, None, None) == rs.abi.RS_OK  # nothing to do
    assert lib.rs_tonemap_workspace_bytes() >= 8


def _xyz_of_kelvin(T):
    """Kang et al. 2002 blackbody chromaticity (xy) as XYZ with Y = 1, restated for the check."""
    t = float(T)
    if T < 4000:
        x = -0.2661239e9 / t**3 - 0.2343580e6 / t**2 + 0.8776956e3 / t + 0.179910
    else:
        x = -3.0258469e9 / t**3 + 2.1070379e6 / t**2 + 0.2226347e3 / t + 0.240390
    if T < 2222:
        y = -1.1063814 * x**3 - 1.34811020 * x**2 + 2.18555832 * x - 0.20219683
    elif T < 4000:
        y = -0.9549476 * x**3 - 1.37418593 * x**2 + 2.09137015 * x - 0.16748867
    else:
        y = 3.0817580 * x**3 - 5.87338670 * x**2 + 3.75112997 * x - 0.37001483
    return np.array([x / y, 1.0, (1 - x - y) / y])


RGB_TO_XYZ = np.array([[0.4123907992659595, 0.3575843393838780, 0.1804807884018343],
                       [0.2126390058715104, 0.7151686787677559, 0.0721923153607337],
                       [0.0193308187155918, 0.1191947797946259, 0.9505321522496608]])


def test_white_balance_transform(rs):
    """The colour grading transform of rs_tonemap (ToneMapper.cpp:530-550 with ColorUtils.h:209-226):
    the exposure scale alone without white balance, the identity at 6500 K, and otherwise the matrix
    that maps the white point's blackbody colour to the 6500 K one (von Kries in CAT02 LMS)."""
    import reservoir_splatting_b200.frame_output as FO
    o = FO.tonemap_options(exposureCompensation=1.0, filmSpeed=200.0, fNumber=2.0, shutter=0.5)
    scale = 2.0 * (0.01 * 200.0) / (0.5 * 2.0 * 2.0)
    assert np.allclose(FO.color_transform(o), np.eye(3) * scale, rtol=1e-6)
    o = FO.tonemap_options(whiteBalance=1, whitePoint=6500.0, exposureCompensation=0.0)
    assert np.allclose(FO.color_transform(o), np.eye(3), atol=1e-6)
    xyz_to_rgb = np.linalg.inv(RGB_TO_XYZ)
    for kelvin in (1905.0, 2500.0, 3800.0, 5000.0, 9000.0, 25000.0):
        o = FO.tonemap_options(whiteBalance=1, whitePoint=kelvin, exposureCompensation=0.0)
        m = FO.color_transform(o).astype(np.float64)
        src = xyz_to_rgb @ _xyz_of_kelvin(kelvin)
        dst = xyz_to_rgb @ _xyz_of_kelvin(6500.0)
        assert np.allclose(m @ src, dst, rtol=1e-5, atol=1e-6), kelvin
    for bad in (1000.0, 30000.0, float("nan")):
        with pytest.raises(ValueError):
            FO.color_transform(FO.tonemap_options(whiteBalance=1, whitePoint=bad))
