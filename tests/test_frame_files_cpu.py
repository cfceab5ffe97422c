"""Frame files of the FrameDumper mirror: the PAM header of FrameDumper.cpp:156-157 byte for byte,
texels in row order, and an 8-bit RGBA PNG that decodes to the same texels."""
import struct
import zlib

import numpy as np


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
