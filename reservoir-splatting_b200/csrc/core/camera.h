// Thin-lens camera and the pass's camera-keyframe manager.
//
//   Scene/Camera/Camera.cpp:179-185          U/V/W basis from pos/target/up, fovY, focal distance
//   Scene/Camera/Camera.slang:146-170        computeRayThinlensSubPixelRandom
//   RenderPasses/ReservoirSplatting/CameraManager.slang:50-113
//       angularLerp (quaternion slerp of the forward vector), recalculateCameraVectors,
//       orientCamera (camera at time t before "now" from a ring of keyframes)
//   Utils/Math/Quaternion.slang:38-59        qmul / rotate_vector / rotate_angle_axis
#pragma once
#include "geom.h"

namespace rs {

constexpr uint32_t kMaxCameraKeyframes = 16;

struct CameraData
{
    f3 posW, target, up;
    f3 cameraU, cameraV, cameraW;
    float focalLength;   // mm
    float frameHeight;   // mm
    float aspectRatio;   // width / height
    float focalDistance; // scene units
    float apertureRadius;
    float shutterSpeed;
    float nearZ, farZ;
    // derived from cameraU/V/W by camera_set_derived (normalize / length of each), kept with them
    // by every function that sets the basis
    f3 unitU, unitV, unitW;
    float lenU, lenV, lenW;
};

RS_HD void camera_set_derived(CameraData& c)
{
    c.unitU = normalize(c.cameraU); c.unitV = normalize(c.cameraV); c.unitW = normalize(c.cameraW);
    c.lenU = length(c.cameraU); c.lenV = length(c.cameraV); c.lenW = length(c.cameraW);
}

RS_HD float camera_fovY(const CameraData& c)
{
    return c.focalLength == 0.f ? 0.f : 2.f * f_atan(0.5f * c.frameHeight / c.focalLength);
}

// Camera.cpp:179-185
RS_HD void camera_update_basis(CameraData& c)
{
    float fovY = camera_fovY(c);
    c.cameraW = normalize(c.target - c.posW) * c.focalDistance;
    c.cameraU = normalize(cross(c.cameraW, c.up));
    c.cameraV = normalize(cross(c.cameraU, c.cameraW));
    const float ulen = c.focalDistance * f_tan(fovY * 0.5f) * c.aspectRatio;
    c.cameraU = c.cameraU * ulen;
    const float vlen = c.focalDistance * f_tan(fovY * 0.5f);
    c.cameraV = c.cameraV * vlen;
    camera_set_derived(c);
}

struct CameraManager
{
    float artificialFrameTime;
    uint32_t keyframes;
    f3 positions[kMaxCameraKeyframes];
    f3 targets[kMaxCameraKeyframes];
};

struct quat { float x, y, z, w; };
RS_HD quat qmul(quat q1, quat q2)
{
    f3 a = mk3(q1.x, q1.y, q1.z), b = mk3(q2.x, q2.y, q2.z);
    f3 v = b * q1.w + a * q2.w + cross(a, b);
    quat r; r.x = v.x; r.y = v.y; r.z = v.z; r.w = q1.w * q2.w - dot(a, b);
    return r;
}
RS_HD f3 rotate_vector(f3 v, quat r)
{
    quat rc; rc.x = r.x * -1.f; rc.y = r.y * -1.f; rc.z = r.z * -1.f; rc.w = r.w * 1.f;
    quat vq; vq.x = v.x; vq.y = v.y; vq.z = v.z; vq.w = 0.f;
    quat o = qmul(r, qmul(vq, rc));
    return mk3(o.x, o.y, o.z);
}
RS_HD quat rotate_angle_axis(float angle, f3 axis)
{
    float sn, cs;
    f_sincos(angle * 0.5f, sn, cs);
    quat q; q.x = axis.x * sn; q.y = axis.y * sn; q.z = axis.z * sn; q.w = cs;
    return q;
}

// CameraManager::angularLerp
RS_HD f3 angular_lerp(f3 prevForward, f3 currForward, float t)
{
    f3 axis = normalize(cross(currForward, prevForward));
    float angle = f_acos(dot(currForward, prevForward));
    if (angle < 0.001f) return currForward;
    quat q = rotate_angle_axis(angle * t, axis);
    return rotate_vector(currForward, q);
}

// CameraManager::recalculateCameraVectors
RS_HD void recalculate_camera_vectors(CameraData& c, f3 forward)
{
    c.cameraW = forward * c.focalDistance;
    c.cameraU = normalize(cross(c.cameraW, c.up));
    c.cameraV = normalize(cross(c.cameraU, c.cameraW));
    float fovY = camera_fovY(c);
    float ulen = c.focalDistance * f_tan(fovY * 0.5f) * c.aspectRatio;
    float vlen = c.focalDistance * f_tan(fovY * 0.5f);
    c.cameraU = c.cameraU * ulen;
    c.cameraV = c.cameraV * vlen;
    camera_set_derived(c);
}

// The keyframe pair and interpolation weight of CameraManager::orientCamera at `time`.
RS_HD void camera_keyframes_at(const CameraManager& cm, uint32_t frameCount, float time, int& first, int& second, float& t)
{
    const int K = (int)cm.keyframes;
    int currIndex = (int)(frameCount % cm.keyframes);
    int frameIndex = (int)f_floor(time / cm.artificialFrameTime);
    first = (currIndex - frameIndex - 1 + K) % K;
    if (first < 0) first += K; // times outside [0, shutter + frame time] stay in the ring
    second = (first + 1 + K) % K;
    t = (time - (float)frameIndex * cm.artificialFrameTime) / cm.artificialFrameTime;
}

// CameraManager::orientCamera: camera at `time` seconds before the current frame.
RS_HD void orient_camera(const CameraManager& cm, CameraData& c, uint32_t frameCount, float time)
{
    int firstCameraIndex, secondCameraIndex;
    float t;
    camera_keyframes_at(cm, frameCount, time, firstCameraIndex, secondCameraIndex, t);
    f3 firstPos = cm.positions[firstCameraIndex], firstTarget = cm.targets[firstCameraIndex];
    f3 secondPos = cm.positions[secondCameraIndex], secondTarget = cm.targets[secondCameraIndex];
    c.up = mk3(0.f, 1.f, 0.f);
    c.posW = lerp(secondPos, firstPos, t);
    f3 firstForward = normalize(firstTarget - firstPos);
    f3 secondForward = normalize(secondTarget - secondPos);
    f3 interpolatedForward = angular_lerp(firstForward, secondForward, t);
    recalculate_camera_vectors(c, interpolatedForward);
}

// The parts of orient_camera that depend only on the frame (its keyframes and camera): each
// keyframe's forward direction, the angular_lerp axis and angle of each keyframe pair
// (i, i + 1 mod K), and the film extents of recalculate_camera_vectors.  camera_table_* compute
// them with orient_camera's own operations, so orient_camera_table returns orient_camera's bits
// while evaluating per call only what depends on the time.
struct CameraTable
{
    f3 forward[kMaxCameraKeyframes];
    f3 pairAxis[kMaxCameraKeyframes];
    float pairAngle[kMaxCameraKeyframes];
    float ulen, vlen;
    // the oriented camera at the two times most queries use (the current frame, 0, and the
    // previous one, the artificial frame time, when the shutter is closed)
    float time[2];
    CameraData at[2];
};
RS_HD f3 camera_table_forward(const CameraManager& cm, int i) { return normalize(cm.targets[i] - cm.positions[i]); }
// Pair (i, i + 1 mod K) from the forwards: angular_lerp(prev = forward[i], curr = forward[i + 1]).
RS_HD void camera_table_pair(const CameraManager& cm, const f3* forward, int i, f3& axis, float& angle)
{
    const int K = (int)cm.keyframes;
    const f3 prevForward = forward[i], currForward = forward[(i + 1 + K) % K];
    axis = normalize(cross(currForward, prevForward));
    angle = f_acos(dot(currForward, prevForward));
}
RS_HD void camera_table_extents(const CameraData& c, float& ulen, float& vlen)
{
    float fovY = camera_fovY(c);
    ulen = c.focalDistance * f_tan(fovY * 0.5f) * c.aspectRatio;
    vlen = c.focalDistance * f_tan(fovY * 0.5f);
}
// orient_camera(cm, c, frameCount, time) for c = the frame's camera, from its table.
RS_HD void orient_camera_table(const CameraManager& cm, const CameraTable& T, CameraData& c, uint32_t frameCount, float time)
{
    int first, second;
    float t;
    camera_keyframes_at(cm, frameCount, time, first, second, t);
    c.up = mk3(0.f, 1.f, 0.f);
    c.posW = lerp(cm.positions[second], cm.positions[first], t);
    const f3 currForward = T.forward[second];
    const float angle = T.pairAngle[first];
    f3 forward = currForward;
    if (!(angle < 0.001f)) forward = rotate_vector(currForward, rotate_angle_axis(angle * t, T.pairAxis[first]));
    c.cameraW = forward * c.focalDistance;
    c.cameraU = normalize(cross(c.cameraW, c.up));
    c.cameraV = normalize(cross(c.cameraU, c.cameraW));
    c.cameraU = c.cameraU * T.ulen;
    c.cameraV = c.cameraV * T.vlen;
    camera_set_derived(c);
}

// Camera::computeRayThinlensSubPixelRandom
RS_HD Ray camera_ray_thinlens(const CameraData& c, uint32_t W, uint32_t H, f2 fractionalPixel, f2 lensSample)
{
    const float epsilon = 0.001f;
    fractionalPixel.x = f_clamp(fractionalPixel.x, epsilon, (float)W - epsilon);
    fractionalPixel.y = f_clamp(fractionalPixel.y, epsilon, (float)H - epsilon);
    f2 p = mk2(fractionalPixel.x / (float)W, fractionalPixel.y / (float)H);
    f2 ndc = mk2(2.f * p.x + -1.f, -2.f * p.y + 1.f);
    Ray ray;
    ray.origin = c.posW;
    ray.dir = c.cameraU * ndc.x + c.cameraV * ndc.y + c.cameraW;
    f3 rayTarget = ray.origin + ray.dir;
    ray.origin += (c.unitU * lensSample.x + c.unitV * lensSample.y) * c.apertureRadius;
    ray.dir = normalize(rayTarget - ray.origin);
    float invCos = 1.f / dot(c.unitW, ray.dir);
    ray.tMin = c.nearZ * invCos;
    ray.tMax = c.farZ * invCos;
    return ray;
}

// Lens point written as posW + aperture * (lens.x * U^ + lens.y * V^)
// (PathTracer.slang:218-220, 817-819).
RS_HD f3 camera_lens_point(const CameraData& c, f2 lensSample)
{
    return c.posW + (c.unitU * lensSample.x + c.unitV * lensSample.y) * c.apertureRadius;
}

// Lens point written as posW + ((aperture * lens.x) * U^ + (aperture * lens.y) * V^)
// (ShiftMapping.slang:114-116, 317-321; ReprojectTemporalSamples.rt.slang:92-95).
RS_HD f3 camera_lens_point_scaled(const CameraData& c, f2 lensSample)
{
    float lx = c.apertureRadius * lensSample.x, ly = c.apertureRadius * lensSample.y;
    return c.posW + (c.unitU * lx + c.unitV * ly);
}

} // namespace rs
