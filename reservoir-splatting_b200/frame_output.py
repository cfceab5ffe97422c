"""Frame output after the pass: tone mapping and frame files, the ToneMapper and FrameDumper passes
the reference's render graphs end with.

`tonemap` runs the library's rs_tonemap kernel (ToneMapper operators, exposure, auto exposure and
clamp, then the FrameDumper blit's 8-bit sRGB conversion) on a device colour buffer.  `FrameDumper`
writes one file per frame as the reference pass does (FrameDumper.cpp:131-158):
``<dir>/<base>.<frame:05d>.pam`` (P7, RGB_ALPHA, MAXVAL 255) or ``.png``.
"""
from __future__ import annotations

import ctypes as C
import struct
import zlib
from pathlib import Path

import numpy as np

from . import abi


def tonemap_options(**kw) -> abi.RsTonemapOptions:
    """ToneMapper properties by name (``op`` may be an operator name such as "Aces"); the rest of the
    fields keep the pass defaults (ToneMapper.h:131-156)."""
    from . import load_library
    o = abi.RsTonemapOptions()
    load_library().rs_tonemap_default_options(C.byref(o))
    for k, v in kw.items():
        if k in ("op", "operator"):
            v = abi.TONEMAP_OPERATOR[v] if isinstance(v, str) else int(v)
            k = "op"
        if not hasattr(o, k):
            raise KeyError(f"unknown tone mapper option {k!r}")
        setattr(o, k, type(getattr(o, k))(v))
    return o


def color_transform(options: abi.RsTonemapOptions) -> "np.ndarray":
    """The 3x3 colour transform rs_tonemap applies (white balance times exposure), float32 [3, 3]."""
    from . import load_library
    m = (C.c_float * 9)()
    st = load_library().rs_tonemap_color_transform(C.byref(options), m)
    if st != 0:
        raise ValueError("invalid tone mapper options")
    return np.array(m[:], np.float32).reshape(3, 3)


def tonemap(color, width: int, height: int, options: abi.RsTonemapOptions | None = None, out=None, stream: int = 0):
    """RGBA8 (uint8 [H, W, 4], CUDA) of a float4 [H, W, 4] CUDA colour tensor; `out` may be given."""
    import torch
    from . import _check, load_library
    lib = load_library()
    o = options or tonemap_options()
    if out is None:
        out = torch.empty((height, width, 4), dtype=torch.uint8, device=color.device)
    ws = torch.empty(int(lib.rs_tonemap_workspace_bytes()), dtype=torch.uint8, device=color.device) if o.autoExposure else None
    _check(lib.rs_tonemap(C.c_void_p(color.data_ptr()), width, height, C.byref(o), C.c_void_p(out.data_ptr()),
                          C.c_void_p(ws.data_ptr()) if ws is not None else None, C.c_void_p(stream)))
    return out


def write_pam(path, rgba8: np.ndarray):
    """P7 file with the FrameDumper header (FrameDumper.cpp:156-157) and the texels row by row."""
    rgba8 = np.ascontiguousarray(rgba8, np.uint8)
    h, w = rgba8.shape[:2]
    with open(path, "wb") as f:
        f.write(b"P7\nWIDTH %d\nHEIGHT %d\nDEPTH 4\nMAXVAL 255\nTUPLTYPE RGB_ALPHA\nENDHDR\n" % (w, h))
        f.write(rgba8.tobytes())


def read_pam(path) -> np.ndarray:
    data = Path(path).read_bytes()
    end = data.index(b"ENDHDR\n") + len(b"ENDHDR\n")
    fields = dict(line.split(b" ", 1) for line in data[:end].split(b"\n")[1:-2])
    w, h, d = int(fields[b"WIDTH"]), int(fields[b"HEIGHT"]), int(fields[b"DEPTH"])
    return np.frombuffer(data[end:end + w * h * d], np.uint8).reshape(h, w, d)


def write_png(path, rgba8: np.ndarray):
    """8-bit RGBA PNG (no filter, zlib)."""
    rgba8 = np.ascontiguousarray(rgba8, np.uint8)
    h, w = rgba8.shape[:2]
    raw = b"".join(b"\x00" + rgba8[y].tobytes() for y in range(h))

    def chunk(tag, payload):
        return struct.pack(">I", len(payload)) + tag + payload + struct.pack(">I", zlib.crc32(tag + payload) & 0xffffffff)

    with open(path, "wb") as f:
        f.write(b"\x89PNG\r\n\x1a\n")
        f.write(chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, 8, 6, 0, 0, 0)))
        f.write(chunk(b"IDAT", zlib.compress(raw, 6)))
        f.write(chunk(b"IEND", b""))


class FrameDumper:
    """Writes every frame it is given (FrameDumper pass: output directory, base name, start frame,
    PNG or PAM).  `dump` tone-maps a CUDA float4 colour tensor with `options` and writes the file;
    it returns the path."""

    def __init__(self, output_dir, base: str = "frame", start_frame: int = 0, png: bool = False,
                 options: abi.RsTonemapOptions | None = None):
        self.dir = Path(output_dir)
        self.dir.mkdir(parents=True, exist_ok=True)
        self.base, self.frame, self.png = base, int(start_frame), png
        self.options = options

    def path(self, frame: int) -> Path:
        return self.dir / f"{self.base}.{frame:05d}.{'png' if self.png else 'pam'}"

    def dump(self, color, width: int, height: int, stream: int = 0) -> Path:
        import torch
        rgba8 = tonemap(color, width, height, self.options, stream=stream)
        torch.cuda.synchronize()
        p = self.path(self.frame)
        (write_png if self.png else write_pam)(p, rgba8.cpu().numpy())
        self.frame += 1
        return p
