"""Frame output (rs_tonemap, FrameDumper) against a numpy restatement of the ToneMapper shader
(RenderPasses/ToneMapper/ToneMapping.ps.slang:45-173, ToneMapper.cpp:538-550) and the FrameDumper's
RGBA8 sRGB texels (FrameDumper.cpp:80-90): every operator, clamp on and off, manual and auto exposure,
and NaN, zero, negative and very large inputs.  The operators run in float32 as the shader does (so
overflow to inf and NaN behave alike); 8-bit texels may differ by one step where the powers and
exponentials of numpy and CUDA round to different sides of a level."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def lum(c):
    return c[..., 0] * 0.299 + c[..., 1] * 0.587 + c[..., 2] * 0.114


def uc2(x):
    A, B, C, D, E, F = 0.22, 0.3, 0.1, 0.2, 0.01, 0.3
    return ((x * (A * x + C * B) + D * E) / (x * (A * x + B) + D * F)) - (E / F)


def reference(color, op, clamp=True, auto=False, comp=0.0, film=100.0, fnum=1.0, shutter=1.0, wml=1.0, ws=11.2, matrix=None):
    f = np.float32
    c = color[..., :3].astype(f)
    with np.errstate(all="ignore"):
        if auto:
            # max(0.0001, NaN) is 0.0001 in the shader (and fmaxf): np.fmax, not np.maximum
            mean = np.mean(np.log2(np.fmax(f(1e-4), lum(color[..., :3].astype(f)))).astype(np.float64))
            c = c * f(0.042 / np.exp2(np.float32(mean)))
        scale = f(2.0 ** comp)
        if not auto:
            scale = scale * (f(0.01) * f(film)) / (f(shutter) * f(fnum) * f(fnum))
        if matrix is None:
            c = c * scale
        else:  # the colour grading transform (white balance times exposure), applied in float32
            m = matrix.astype(f)
            c = (c[..., 0:1] * m[:, 0] + c[..., 1:2] * m[:, 1] + c[..., 2:3] * m[:, 2]).astype(f)
        if op == "Reinhard":
            l = lum(c)[..., None]
            c = c * ((l / (l + 1)) / l)
        elif op == "ReinhardModified":
            l = lum(c)[..., None]
            c = c * ((l * (1 + l / (wml * wml)) * (1 + l)) / l)
        elif op == "HejiHableAlu":
            c = np.maximum(0.0, c - 0.004)
            c = (c * (6.2 * c + 0.5)) / (c * (6.2 * c + 1.7) + 0.06)
            c = np.power(c, 2.2)
        elif op == "HableUc2":
            c = uc2(f(2.0) * c) * (f(1.0) / uc2(f(ws)))
        elif op == "Aces":
            c = c * 0.6
            c = np.clip((c * (2.51 * c + 0.03)) / (c * (2.43 * c + 0.59) + 0.14), 0.0, 1.0)
        c = np.where(np.isnan(c), f(0.0), c).astype(f)
        if clamp:
            c = np.clip(c, f(0.0), f(1.0))
        x = np.clip(c, f(0.0), f(1.0)).astype(np.float64)
        e = np.where(x <= 0.0031308, 12.92 * x, 1.055 * np.power(x, 1 / 2.4) - 0.055)
    rgb = np.rint(e * 255.0)
    a = np.rint(np.clip(color[..., 3].astype(np.float64), 0.0, 1.0) * 255.0)
    return np.concatenate([rgb, a[..., None]], -1).astype(np.int32)


def _image(h=96, w=128, seed=1):
    rng = np.random.default_rng(seed)
    img = np.exp(rng.normal(-1.0, 2.0, (h, w, 4))).astype(np.float32)
    img[..., 3] = rng.uniform(-0.2, 1.2, (h, w))
    img[0, :8, :3] = [[0, 0, 0], [-1, 2, 3], [np.nan, 1, 1], [1e30, 1e30, 1e30], [1e-8, 0, 0], [0.5, 0.5, 0.5],
                      [100, 0.01, 1], [3, 3, 3]]
    return img


OPS = ["Linear", "Reinhard", "ReinhardModified", "HejiHableAlu", "HableUc2", "Aces"]


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("op", OPS)
@pytest.mark.parametrize("clamp,auto,comp", [(True, False, 0.0), (False, False, 1.5), (True, True, -0.5)])
def test_tonemap_matches_the_shader(rs, op, clamp, auto, comp):
    import torch
    import reservoir_splatting_b200.frame_output as FO
    img = _image()
    h, w = img.shape[:2]
    o = FO.tonemap_options(op=op, clamp=int(clamp), autoExposure=int(auto), exposureCompensation=comp, fNumber=1.4, shutter=2.0,
                           filmSpeed=200.0)
    out = FO.tonemap(torch.from_numpy(img).cuda(), w, h, o).cpu().numpy().astype(np.int32)
    ref = reference(img, op, clamp, auto, comp, film=200.0, fnum=1.4, shutter=2.0)
    diff = np.abs(out - ref)
    assert diff.max() <= 1, (op, np.argwhere(diff > 1)[:3].tolist())
    assert (diff > 0).mean() < 0.01


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
@pytest.mark.parametrize("kelvin", [2500.0, 6500.0, 12000.0])
def test_white_balance_matches_the_shader(rs, kelvin):
    """ToneMapping.ps.slang:157-158: the white balance matrix (times exposure) before the operator."""
    import torch
    import reservoir_splatting_b200.frame_output as FO
    img = _image(seed=3)
    img[0, :8, :3] = np.abs(img[0, :8, :3])  # keep the matrix product free of NaN and inf rows
    img[0, 3, :3] = 5.0
    h, w = img.shape[:2]
    o = FO.tonemap_options(op="Aces", whiteBalance=1, whitePoint=kelvin, exposureCompensation=0.5)
    m = FO.color_transform(o)
    out = FO.tonemap(torch.from_numpy(img).cuda(), w, h, o).cpu().numpy().astype(np.int32)
    ref = reference(img, "Aces", comp=0.5, matrix=m)
    diff = np.abs(out - ref)
    assert diff.max() <= 1
    assert (diff > 0).mean() < 0.01


@pytest.mark.skipif(not _cuda_ok(), reason="no CUDA device")
def test_frame_dumper_writes_the_tonemapped_frames(rs, scenes, tmp_path):
    import torch
    import reservoir_splatting_b200.frame_output as FO
    W, H = 96, 64
    p = rs.ReservoirSplatting({"temporalReuse": "ScatterBackup", "maxSurfaceBounces": 2}, W, H)
    p.set_scene(scenes.cornell_box(0))
    color = torch.empty((H, W, 4), device="cuda")
    dumper = FO.FrameDumper(tmp_path / "dump", base="frame", start_frame=7)
    paths = []
    for f in range(3):
        p.execute(scenes.cornell_camera(f, W, H), color_ptr=color.data_ptr())
        torch.cuda.synchronize()
        paths.append(dumper.dump(color, W, H))
        expected = FO.tonemap(color, W, H).cpu().numpy()
        np.testing.assert_array_equal(FO.read_pam(paths[-1]), expected)
    assert [q.name for q in paths] == ["frame.00007.pam", "frame.00008.pam", "frame.00009.pam"]
    head = paths[0].read_bytes()[:80]
    assert head.startswith(b"P7\nWIDTH 96\nHEIGHT 64\nDEPTH 4\nMAXVAL 255\nTUPLTYPE RGB_ALPHA\nENDHDR\n")
    p.close()
