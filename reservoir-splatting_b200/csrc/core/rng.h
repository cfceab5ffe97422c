// Per-pixel random streams.
//
// TinyUniform (the reference pass default, ReservoirSplatting.h:134):
//   seed  = TEA(interleave_32bit(pixel), sampleNumber).x    TinyUniformSampleGenerator.slang:58-69
//   state = 1664525 * state + 1013904223                    LCG.slang:50-56
//   u     = (next >> 8) * 2^-24                              SampleGeneratorInterface.slang:50-56
// PCG32 (selectable): O'Neill's XSH-RR output over a 64-bit LCG, seeded from the
// same TEA hash (initstate = TEA.x << 32 | TEA.y, default increment).
// The generator is a value type: the shift mappings receive it by value
// (ShiftMapping.slang:90,183,301), so draws inside a shift do not advance the
// caller's stream.
#pragma once
#include "fmath.h"

namespace rs {

enum SampleGeneratorKind : uint32_t { kSgTinyUniform = 0, kSgPCG32 = 2 };

RS_HD uint32_t interleave_32bit(uint32_t vx, uint32_t vy) // BitTricks.slang:47-62
{
    uint32_t x = vx & 0x0000ffffu;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    uint32_t y = vy & 0x0000ffffu;
    y = (y | (y << 8)) & 0x00FF00FFu;
    y = (y | (y << 4)) & 0x0F0F0F0Fu;
    y = (y | (y << 2)) & 0x33333333u;
    y = (y | (y << 1)) & 0x55555555u;
    return x | (y << 1);
}

RS_HD void tea16(uint32_t& v0, uint32_t& v1) // HashUtils.slang:62-73, 16 rounds
{
    uint32_t sum = 0;
    const uint32_t delta = 0x9e3779b9u;
    for (int i = 0; i < 16; i++)
    {
        sum += delta;
        v0 += ((v1 << 4) + 0xa341316cu) ^ (v1 + sum) ^ ((v1 >> 5) + 0xc8013ea4u);
        v1 += ((v0 << 4) + 0xad90777du) ^ (v0 + sum) ^ ((v0 >> 5) + 0x7e95761eu);
    }
}

struct SampleGen
{
    uint64_t state;
    uint32_t kind;
};

RS_HD SampleGen sg_create(uint32_t px, uint32_t py, uint32_t seed, uint32_t kind)
{
    uint32_t v0 = interleave_32bit(px, py), v1 = seed;
    tea16(v0, v1);
    SampleGen sg;
    sg.kind = kind;
    if (kind == kSgPCG32)
    {
        const uint64_t inc = 1442695040888963407ull;
        uint64_t init = ((uint64_t)v0 << 32) | (uint64_t)v1;
        sg.state = 0;
        sg.state = sg.state * 6364136223846793005ull + inc;
        sg.state += init;
        sg.state = sg.state * 6364136223846793005ull + inc;
    }
    else
    {
        sg.state = v0;
    }
    return sg;
}

RS_HD uint32_t sg_next(SampleGen& sg)
{
    if (sg.kind == kSgPCG32)
    {
        uint64_t old = sg.state;
        sg.state = old * 6364136223846793005ull + 1442695040888963407ull;
        uint32_t xs = (uint32_t)(((old >> 18u) ^ old) >> 27u);
        uint32_t rot = (uint32_t)(old >> 59u);
        return (xs >> rot) | (xs << ((32u - rot) & 31u));
    }
    uint32_t s = (uint32_t)sg.state * 1664525u + 1013904223u;
    sg.state = s;
    return s;
}

RS_HD float sampleNext1D(SampleGen& sg) { return (float)(sg_next(sg) >> 8) * 5.9604644775390625e-08f; }

} // namespace rs
