// Shared helpers of the ffbp_b200 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ffbp {

constexpr float TWO_PI_F = 6.28318530717958647692f;
constexpr double TWO_PI = 6.28318530717958647692;
constexpr double C_LIGHT = 299792458.0;

// exp(2 pi i c) for a phase c in cycles already reduced to [-0.5, 0.5]: the hardware sine and cosine are accurate to
// about 4e-7 absolute on [-pi, pi], which is the whole range they are given here.
__device__ __forceinline__ float2 cis_reduced(float c)
{
    float s, co;
    __sincosf(TWO_PI_F * c, &s, &co);
    return make_float2(co, s);
}

// exp(2 pi i c) for any float32 phase in cycles (reduced first).
__device__ __forceinline__ float2 cis_cycles(float c)
{
    return cis_reduced(c - rintf(c));
}

// exp(2 pi i c) for a float64 phase in cycles: the reduction in float64, the sine and cosine in float32.
__device__ __forceinline__ float2 cis_cycles_d(double c)
{
    return cis_reduced((float)(c - rint(c)));
}

__device__ __forceinline__ float2 cmul(float2 a, float2 b)
{
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// Two float32 fused multiply-adds in one instruction (sm_100's packed FMA): (a.x b.x + c.x, a.y b.y + c.y), each
// rounded as fmaf rounds it.
__device__ __forceinline__ float2 ffma2(float2 a, float2 b, float2 c)
{
    float2 d;
    asm("{\n\t.reg .b64 pa, pb, pc, pd;\n\t"
        "mov.b64 pa, {%2, %3};\n\tmov.b64 pb, {%4, %5};\n\tmov.b64 pc, {%6, %7};\n\t"
        "fma.rn.f32x2 pd, pa, pb, pc;\n\tmov.b64 {%0, %1}, pd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(c.x), "f"(c.y));
    return d;
}

}  // namespace ffbp
