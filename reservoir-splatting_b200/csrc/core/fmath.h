// Scalar float semantics shared by the sm_100a kernels and the host code.
//
// Every function here is built only from IEEE-754 binary32 operations that are
// correctly rounded on both x86-64 (SSE, -ffp-contract=off) and sm_100a
// (-fmad=false -prec-div=true -prec-sqrt=true): + - * / sqrtf floorf rintf
// fabsf and comparisons.  The transcendental functions are written from their
// Taylor series after a Cody-Waite range reduction (constants derived from pi
// in this file's comments), so a host build and a device build of the same
// expression produce the same bits.  They are accurate to a few ulp over the
// argument ranges the renderer uses (|x| < 24 for sin/cos).
//
// Reference correspondence: these replace the Slang intrinsics sin/cos/acos/
// atan/tan/pow used by Utils/Math/MathHelpers.slang:269-277, 323-355,
// Utils/Math/Quaternion.slang:54-59, RenderPasses/ReservoirSplatting/
// CameraManager.slang:50-82 and Rendering/Materials/Fresnel.slang:42-51.
#pragma once
#include <stdint.h>
#include <string.h>
#include <math.h>

#if defined(__CUDACC__)
#define RS_HD __host__ __device__ __forceinline__
#define RS_HDI __host__ __device__ inline
#else
#define RS_HD inline
#define RS_HDI inline
#endif

namespace rs {

// pi and friends rounded to binary32 (bit patterns in the comments).
constexpr float kPi = 3.14159274101257324f;      // 0x40490fdb
constexpr float k1OverPi = 0.318309873342514038f; // 0x3ea2f983
constexpr float k2Pi = 6.28318548202514648f;     // 0x40c90fdb
constexpr float kPiOver2 = 1.57079637050628662f; // 0x3fc90fdb
constexpr float kPiOver4 = 0.785398185253143311f; // 0x3f490fdb
constexpr float kPiOver6 = 0.523598790168762207f; // 0x3f060a92
constexpr float kSqrt3 = 1.73205077648162842f;   // 0x3fddb3d7
constexpr float kFltMin = 1.17549435e-38f;       // FLT_MIN
constexpr float kRayTMax = 1e30f;                 // PathStates.slang:40

RS_HD uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
RS_HD float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
RS_HD int32_t f2i_bits(float f) { int32_t u; memcpy(&u, &f, 4); return u; }
RS_HD float i2f_bits(int32_t u) { float f; memcpy(&f, &u, 4); return f; }

RS_HD bool f_isnan(float x) { return x != x; }
RS_HD float f_min(float a, float b) { return (b < a) ? b : a; }  // HLSL min with non-NaN args
RS_HD float f_max(float a, float b) { return (a < b) ? b : a; }
RS_HD float f_abs(float x) { return fabsf(x); }
RS_HD float f_sqrt(float x) { return sqrtf(x); }
RS_HD float f_floor(float x) { return floorf(x); }
RS_HD float f_round(float x) { return rintf(x); }  // HLSL round(): nearest, ties to even
RS_HD float f_saturate(float x) { return f_min(f_max(x, 0.f), 1.f); }
RS_HD float f_clamp(float x, float lo, float hi) { return f_min(f_max(x, lo), hi); }
RS_HD float f_lerp(float a, float b, float t) { return a + t * (b - a); }
RS_HD float f_sign(float x) { return x > 0.f ? 1.f : (x < 0.f ? -1.f : 0.f); }

// Range reduction x = k * pi/2 + r with pi/2 = P1 + P2 + P3, P1 holding the
// top 20 significand bits of pi/2 so that k * P1 is exact for |k| < 16.
// P1 = 0x3fc90fd0, P2 = 0x35aa2217, P3 = 0xa967b967 (pi/2 - P1 - P2).
RS_HD float reduce_half_pi(float x, int& quadrant)
{
    const float kTwoOverPi = 0.636619746685028076f; // 0x3f22f983
    const float P1 = 1.57079505920410156f;
    const float P2 = 1.26759084650984730e-06f;
    const float P3 = -5.14531146367843560e-14f;
    float k = rintf(x * kTwoOverPi);
    quadrant = (int)k;
    float r = x - k * P1;
    r = r - k * P2;
    r = r - k * P3;
    return r;
}

// Taylor polynomials on |r| <= pi/4 (coefficients +-1/n!).
RS_HD float sin_poly(float r)
{
    float r2 = r * r;
    float p = -2.50521083854417188e-08f;             // -1/11!
    p = p * r2 + 2.75573192239858907e-06f;          //  1/9!
    p = p * r2 + -1.98412698412698413e-04f;         // -1/7!
    p = p * r2 + 8.33333333333333333e-03f;          //  1/5!
    p = p * r2 + -1.66666666666666667e-01f;         // -1/3!
    return r + r * (r2 * p);
}

RS_HD float cos_poly(float r)
{
    float r2 = r * r;
    float p = 2.08767569878680990e-09f;              //  1/12!
    p = p * r2 + -2.75573192239858907e-07f;         // -1/10!
    p = p * r2 + 2.48015873015873016e-05f;          //  1/8!
    p = p * r2 + -1.38888888888888889e-03f;         // -1/6!
    p = p * r2 + 4.16666666666666667e-02f;          //  1/4!
    p = p * r2 + -0.5f;                             // -1/2!
    return 1.f + r2 * p;
}

RS_HD void f_sincos(float x, float& s, float& c)
{
    int q;
    float r = reduce_half_pi(x, q);
    float sr = sin_poly(r), cr = cos_poly(r);
    switch (q & 3)
    {
    case 0: s = sr; c = cr; break;
    case 1: s = cr; c = -sr; break;
    case 2: s = -sr; c = -cr; break;
    default: s = -cr; c = sr; break;
    }
}
RS_HD float f_sin(float x) { float s, c; f_sincos(x, s, c); return s; }
RS_HD float f_cos(float x) { float s, c; f_sincos(x, s, c); return c; }
RS_HD float f_tan(float x) { float s, c; f_sincos(x, s, c); return s / c; }

// atan via atan(x) = pi/2 - atan(1/x) for |x| > 1 and
// atan(x) = pi/6 + atan((sqrt(3) x - 1) / (x + sqrt(3))) for x > tan(pi/12),
// then the Taylor series of atan on |t| <= tan(pi/12) = 0.2679.
RS_HD float f_atan(float x)
{
    float ax = fabsf(x);
    if (f_isnan(x)) return x;
    bool inv = ax > 1.f;
    if (inv) ax = 1.f / ax;
    bool red = ax > 0.267949194f;
    float t = red ? (ax * kSqrt3 - 1.f) / (ax + kSqrt3) : ax;
    float t2 = t * t;
    float p = 0.0666666666666666667f;   //  1/15
    p = p * t2 + -0.0769230769230769231f; // -1/13
    p = p * t2 + 0.0909090909090909091f;  //  1/11
    p = p * t2 + -0.111111111111111111f;  // -1/9
    p = p * t2 + 0.142857142857142857f;   //  1/7
    p = p * t2 + -0.2f;                   // -1/5
    p = p * t2 + 0.333333333333333333f;   //  1/3
    float a = t - t * (t2 * p);
    if (red) a = kPiOver6 + a;
    if (inv) a = kPiOver2 - a;
    return x < 0.f ? -a : a;
}

// acos(x) = atan(sqrt(1-x^2)/x) folded to [0, pi].  The argument is clamped to
// [-1, 1] first, so a dot product of unit vectors that rounds to 1 + ulp gives 0
// instead of NaN (a documented restatement choice: HLSL acos is undefined there).
RS_HD float f_acos(float x)
{
    if (f_isnan(x)) return x;
    x = f_clamp(x, -1.f, 1.f);
    float s = f_sqrt((1.f - x) * (1.f + x));
    if (x == 0.f) return kPiOver2;
    if (x > 0.f) return f_atan(s / x);
    return kPi - f_atan(s / -x);
}

// atan2 from atan of the quotient of magnitudes, placed in the quadrant of (x, y): (0, 0) gives 0,
// x = 0 gives +-pi/2, y = +-0 with x < 0 gives pi.
RS_HD float f_atan2(float y, float x)
{
    if (f_isnan(x) || f_isnan(y)) return x + y;
    if (x == 0.f) return y > 0.f ? kPiOver2 : (y < 0.f ? -kPiOver2 : 0.f);
    float a = f_atan(fabsf(y) / fabsf(x));
    if (x < 0.f) a = kPi - a;
    return y < 0.f ? -a : a;
}

// Integer powers written out as products (replaces pow(x, 3) / pow(x, 5)).
RS_HD float f_pow3(float x) { return x * x * x; }
RS_HD float f_pow5(float x) { float x2 = x * x; return x2 * x2 * x; }

// binary16 <-> binary32 (round to nearest even), written from the IEEE-754
// encodings; used for the alias-table thresholds (EmissivePowerSampler.cpp:154-160).
RS_HDI uint16_t f32_to_f16(float f)
{
    uint32_t x = f2u(f);
    uint32_t sign = (x >> 16) & 0x8000u;
    int32_t exp = (int32_t)((x >> 23) & 0xffu);
    uint32_t mant = x & 0x7fffffu;
    if (exp == 0xff) return (uint16_t)(sign | 0x7c00u | (mant ? 0x200u : 0u));
    int32_t e = exp - 127 + 15;
    if (e >= 0x1f) return (uint16_t)(sign | 0x7c00u);
    if (e <= 0)
    {
        if (e < -10) return (uint16_t)sign;
        mant |= 0x800000u;
        uint32_t shift = (uint32_t)(14 - e);
        uint32_t half = mant >> shift;
        uint32_t rem = mant & ((1u << shift) - 1u);
        uint32_t mid = 1u << (shift - 1u);
        if (rem > mid || (rem == mid && (half & 1u))) half++;
        return (uint16_t)(sign | half);
    }
    uint32_t half = sign | ((uint32_t)e << 10) | (mant >> 13);
    uint32_t rem = mant & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (half & 1u))) half++;
    return (uint16_t)half;
}

RS_HDI float f16_to_f32(uint16_t h)
{
    uint32_t sign = ((uint32_t)h & 0x8000u) << 16;
    uint32_t exp = ((uint32_t)h >> 10) & 0x1fu;
    uint32_t mant = (uint32_t)h & 0x3ffu;
    if (exp == 0)
    {
        if (mant == 0) return u2f(sign);
        float m = (float)mant * (1.f / 16777216.f); // mant * 2^-24
        return sign ? -m : m;
    }
    if (exp == 0x1f) return u2f(sign | 0x7f800000u | (mant << 13));
    return u2f(sign | ((exp + 112u) << 23) | (mant << 13));
}

// ---- x^e for the PowerExp MIS heuristic (PathTracer.slang:498-503), as 2^(e log2 x) in binary64
// (correctly rounded +, -, *, / on host and device, so both produce the same bits), rounded once to
// binary32.  log2: x = m 2^k with m in [sqrt(1/2), sqrt(2)), ln m = 2 atanh(s) = 2 (s + s^3/3 +
// s^5/5 + ...) with s = (m - 1) / (m + 1), |s| <= 0.172 (terms to s^23).  2^f for the fraction
// f in [-1/2, 1/2]: the Taylor series of exp(f ln 2) to its 17th power, then the power of two by
// the exponent bits.  About 1 ulp of binary32 over the MIS weights' range.
constexpr double kLn2D = 0.693147180559945309417232121458;
constexpr double kInvLn2D = 1.442695040888963407359924681002;

RS_HD uint64_t d2u(double d) { uint64_t u; memcpy(&u, &d, 8); return u; }
RS_HD double u2d(uint64_t u) { double d; memcpy(&d, &u, 8); return d; }

// log2 x for finite x > 0.
RS_HD double d_log2(double x)
{
    int k = 0;
    if (x < 2.2250738585072014e-308) { x = x * 18014398509481984.0; k = -54; } // subnormal: scale by 2^54
    uint64_t b = d2u(x);
    k += (int)((b >> 52) & 0x7ffu) - 1023;
    double m = u2d((b & 0x000fffffffffffffull) | 0x3ff0000000000000ull); // [1, 2)
    if (m > 1.4142135623730951) { m = m * 0.5; k += 1; }
    const double s = (m - 1.0) / (m + 1.0), s2 = s * s;
    double poly = 1.0 / 23.0;
    poly = poly * s2 + 1.0 / 21.0;
    poly = poly * s2 + 1.0 / 19.0;
    poly = poly * s2 + 1.0 / 17.0;
    poly = poly * s2 + 1.0 / 15.0;
    poly = poly * s2 + 1.0 / 13.0;
    poly = poly * s2 + 1.0 / 11.0;
    poly = poly * s2 + 1.0 / 9.0;
    poly = poly * s2 + 1.0 / 7.0;
    poly = poly * s2 + 1.0 / 5.0;
    poly = poly * s2 + 1.0 / 3.0;
    poly = poly * s2 + 1.0;
    return (double)k + (2.0 * s * poly) * kInvLn2D;
}

// 2^y for finite y (0 below 2^-1075, +inf above 2^1024).
RS_HD double d_exp2(double y)
{
    if (y < -1075.0) return 0.0;
    if (y >= 1024.0) return u2d(0x7ff0000000000000ull);
    const double n = floor(y + 0.5);
    const double t = (y - n) * kLn2D; // |t| <= ln2 / 2
    // 1 / n! for n = 1 .. 17 (the n = 0 term is added last)
    const double inv[17] = {1.0, 1.0 / 2.0, 1.0 / 6.0, 1.0 / 24.0, 1.0 / 120.0, 1.0 / 720.0, 1.0 / 5040.0, 1.0 / 40320.0,
                            1.0 / 362880.0, 1.0 / 3628800.0, 1.0 / 39916800.0, 1.0 / 479001600.0, 1.0 / 6227020800.0,
                            1.0 / 87178291200.0, 1.0 / 1307674368000.0, 1.0 / 20922789888000.0, 1.0 / 355687428096000.0};
    double r = inv[16];
#pragma unroll
    for (int i = 15; i >= 0; i--) r = r * t + inv[i];
    r = r * t + 1.0;
    int e = (int)n;
    // scale by 2^e in at most two exact steps (each factor a normal power of two)
    if (e > 1023) { r = r * u2d(0x7fe0000000000000ull); e -= 1023; }
    if (e < -1022) { r = r * u2d(0x0010000000000000ull); e += 1022; }
    return r * u2d((uint64_t)(e + 1023) << 52);
}

// x^e for x >= 0 and e > 0 (0 for x = 0; NaN for NaN or negative x, as pow gives).
RS_HD float f_pow_pos(float x, float e)
{
    if (x == 0.f) return 0.f;
    if (!(x > 0.f)) return u2f(0x7fc00000u);
    if (x == INFINITY) return x;
    return (float)d_exp2((double)e * d_log2((double)x));
}

} // namespace rs
