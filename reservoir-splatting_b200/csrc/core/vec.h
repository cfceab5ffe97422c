// Small vector types shared by the kernels and the host code.  Operation order
// is fixed (left to right), so host and device round identically.
// dot/cross/normalize/length follow the HLSL definitions used throughout the
// reference shaders; normalize(v) is written as v * (1 / sqrt(dot(v, v))).
#pragma once
#include "fmath.h"

namespace rs {

struct f2 { float x, y; };
struct f3 { float x, y, z; };
struct u2 { uint32_t x, y; };

RS_HD f2 mk2(float x, float y) { f2 r; r.x = x; r.y = y; return r; }
RS_HD f3 mk3(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
RS_HD f3 mk3(float s) { return mk3(s, s, s); }

RS_HD f2 operator+(f2 a, f2 b) { return mk2(a.x + b.x, a.y + b.y); }
RS_HD f2 operator-(f2 a, f2 b) { return mk2(a.x - b.x, a.y - b.y); }
RS_HD f2 operator*(f2 a, f2 b) { return mk2(a.x * b.x, a.y * b.y); }
RS_HD f2 operator/(f2 a, f2 b) { return mk2(a.x / b.x, a.y / b.y); }
RS_HD f2 operator*(f2 a, float s) { return mk2(a.x * s, a.y * s); }
RS_HD f2 operator*(float s, f2 a) { return mk2(s * a.x, s * a.y); }
RS_HD f2 operator/(f2 a, float s) { return mk2(a.x / s, a.y / s); }
RS_HD f2 operator+(f2 a, float s) { return mk2(a.x + s, a.y + s); }
RS_HD f2 operator-(f2 a, float s) { return mk2(a.x - s, a.y - s); }

RS_HD f3 operator+(f3 a, f3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
RS_HD f3 operator-(f3 a, f3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
RS_HD f3 operator*(f3 a, f3 b) { return mk3(a.x * b.x, a.y * b.y, a.z * b.z); }
RS_HD f3 operator/(f3 a, f3 b) { return mk3(a.x / b.x, a.y / b.y, a.z / b.z); }
RS_HD f3 operator*(f3 a, float s) { return mk3(a.x * s, a.y * s, a.z * s); }
RS_HD f3 operator*(float s, f3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
RS_HD f3 operator/(f3 a, float s) { return mk3(a.x / s, a.y / s, a.z / s); }
RS_HD f3 operator-(f3 a) { return mk3(-a.x, -a.y, -a.z); }
RS_HD f3& operator+=(f3& a, f3 b) { a = a + b; return a; }
RS_HD f3& operator*=(f3& a, f3 b) { a = a * b; return a; }
RS_HD f3& operator*=(f3& a, float s) { a = a * s; return a; }
RS_HD f3& operator/=(f3& a, float s) { a = a / s; return a; }

RS_HD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
RS_HD float dot(f2 a, f2 b) { return a.x * b.x + a.y * b.y; }
RS_HD f3 cross(f3 a, f3 b)
{
    return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
RS_HD float length(f3 a) { return f_sqrt(dot(a, a)); }
RS_HD float length(f2 a) { return f_sqrt(dot(a, a)); }
RS_HD f3 normalize(f3 a) { return a * (1.f / f_sqrt(dot(a, a))); }
RS_HD f3 lerp(f3 a, f3 b, float t) { return mk3(f_lerp(a.x, b.x, t), f_lerp(a.y, b.y, t), f_lerp(a.z, b.z, t)); }
RS_HD f3 abs3(f3 a) { return mk3(f_abs(a.x), f_abs(a.y), f_abs(a.z)); }
RS_HD bool any_gt0(f3 a) { return a.x > 0.f || a.y > 0.f || a.z > 0.f; }
RS_HD bool all_eq0(f3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
RS_HD float luminance(f3 c) { return c.x * 0.2126f + c.y * 0.7152f + c.z * 0.0722f; } // ColorHelpers.slang:45-49
RS_HD f2 floor2(f2 a) { return mk2(f_floor(a.x), f_floor(a.y)); }

} // namespace rs
