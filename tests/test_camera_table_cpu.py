"""The frame table of the camera manager (core/camera.h) against orient_camera itself: the CUDA
kernels orient the camera from per-frame constants (keyframe forwards, the slerp axis and angle of
each keyframe pair, the film extents), which must give orient_camera's bits for every keyframe
ring and time.  The shared float core is compiled for the host here with the flags of the device
build (no contraction), and the two forms are compared bit for bit."""
import subprocess
from pathlib import Path

import pytest

CORE = Path(__file__).resolve().parents[1] / "reservoir-splatting_b200" / "csrc" / "core"

HARNESS = r"""
#include "camera.h"
#include <cstdio>
#include <cstdlib>
#include <cstring>
using namespace rs;
static uint32_t st = 12345u;
static float uni() { st = st * 1664525u + 1013904223u; return (float)(st >> 8) * (1.0f / 16777216.0f); }
static uint32_t bits(float x) { uint32_t u; memcpy(&u, &x, 4); return u; }
int main(int argc, char** argv)
{
    st = (uint32_t)atoi(argv[1]);
    long checked = 0, mismatched = 0;
    for (int ring = 0; ring < 200; ring++)
    {
        CameraManager cm;
        cm.artificialFrameTime = ring % 3 == 0 ? 1.f / 60.f : 1.f / (24.f + 40.f * uni());
        cm.keyframes = 2 + (uint32_t)(uni() * 14.f);
        const bool still = ring % 5 == 0;  // equal forwards: the angle < 0.001 branch
        for (uint32_t i = 0; i < cm.keyframes; i++)
        {
            float a = still ? 0.3f : 6.2831853f * uni(), r = 20.f + 60.f * uni();
            cm.positions[i] = mk3(r * cosf(a), 5.f + 20.f * uni(), r * sinf(a));
            cm.targets[i] = still ? cm.positions[i] + mk3(1.f, -0.2f, 0.5f) : mk3(uni() - 0.5f, 2.f * uni(), uni() - 0.5f);
        }
        CameraData cam;
        memset(&cam, 0, sizeof(cam));
        cam.focalLength = 20.f + 40.f * uni(); cam.frameHeight = 24.f; cam.aspectRatio = 16.f / 9.f;
        cam.focalDistance = 1.f + 10.f * uni();
        CameraTable T;
        for (uint32_t i = 0; i < cm.keyframes; i++) T.forward[i] = camera_table_forward(cm, (int)i);
        for (uint32_t i = 0; i < cm.keyframes; i++) camera_table_pair(cm, T.forward, (int)i, T.pairAxis[i], T.pairAngle[i]);
        camera_table_extents(cam, T.ulen, T.vlen);
        for (int k = 0; k < 400; k++)
        {
            uint32_t frame = (uint32_t)(uni() * 1000.f);
            float time = (k % 7 == 0) ? 0.f : uni() * cm.artificialFrameTime * (float)(cm.keyframes + 1) - 0.1f * cm.artificialFrameTime;
            CameraData a = cam, b = cam;
            orient_camera(cm, a, frame, time);
            orient_camera_table(cm, T, b, frame, time);
            const float* pa = &a.posW.x; const float* pb = &b.posW.x;
            for (int j = 0; j < 18; j++) { checked++; if (bits(pa[j]) != bits(pb[j])) mismatched++; }
            // the derived unit vectors and lengths, and that they are those of the basis
            const float* da = &a.unitU.x; const float* db = &b.unitU.x;
            for (int j = 0; j < 12; j++) { checked++; if (bits(da[j]) != bits(db[j])) mismatched++; }
            CameraData r = b;
            camera_set_derived(r);
            const float* dr = &r.unitU.x;
            for (int j = 0; j < 12; j++) { checked++; if (bits(dr[j]) != bits(db[j])) mismatched++; }
        }
    }
    printf("%ld %ld\n", checked, mismatched);
    return 0;
}
"""


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    d = tmp_path_factory.mktemp("camtable")
    src = d / "camtable.cpp"
    src.write_text(HARNESS)
    exe = d / "camtable"
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", f"-I{CORE}", str(src), "-o", str(exe)],
                   check=True)
    return exe


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_table_orientation_has_orient_camera_bits(harness, seed):
    out = subprocess.run([str(harness), str(seed)], check=True, capture_output=True, text=True).stdout.split()
    checked, mismatched = int(out[0]), int(out[1])
    assert checked == 200 * 400 * (18 + 24)
    assert mismatched == 0
