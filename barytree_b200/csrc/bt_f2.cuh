// bt_f2.cuh -- FP32 building blocks of the mixed-precision kernels
// (internal): single-instruction special functions and packed FP32 pairs.
#pragma once

namespace bt {

__device__ __forceinline__ float rsqrt_apx(float x)
{
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float ex2_apx(float x)
{
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// Packed FP32 pairs (sm_100 f32x2 instructions): one instruction applies the
// same operation to two FP32 values held in a 64-bit register pair, which
// halves the issue slots of the near-field arithmetic.  Flush-to-zero, like
// the files that include this (compiled with -ftz=true).
typedef unsigned long long f2_t;

__device__ __forceinline__ f2_t f2_make(float lo, float hi)
{
    f2_t r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void f2_split(f2_t v, float &lo, float &hi)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2_t f2_sub(f2_t a, f2_t b)
{
    f2_t r;
    asm("sub.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2_t f2_mul(f2_t a, f2_t b)
{
    f2_t r;
    asm("mul.rn.ftz.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ f2_t f2_fma(f2_t a, f2_t b, f2_t c)
{
    f2_t r;
    asm("fma.rn.ftz.f32x2 %0, %1, %2, %3;" : "=l"(r) : "l"(a), "l"(b), "l"(c));
    return r;
}

// f2_rsqrt_sw (below) for one value: the same operations, so the same
// result as either lane of the packed form.
__device__ __forceinline__ float rsqrt_sw(float x)
{
    float y = __uint_as_float(0x5f375a86u - (__float_as_uint(x) >> 1));
    float e = fmaf(x, y * y, -1.0f);
    y = fmaf(y * e, -0.5f, y);
    e = fmaf(x, y * y, -1.0f);
    return fmaf(y * e, fmaf(e, 0.375f, -0.5f), y);
}

// 1/sqrt(x) for a packed pair on the FP32 and integer pipes, for finite
// x > 0 (normal numbers): the bit-pattern estimate of C. Lomont ("Fast
// Inverse Square Root", 2003; constant 0x5f375a86, relative error below
// 3.5e-2), one Newton step y <- y - y e / 2 (error below 1.8e-3), then one
// third-order step y <- y (1 - e/2 + 3 e^2 / 8), each with e = x y^2 - 1;
// the last leaves (5/16)|e|^3 < 2e-8 relative plus the rounding of its
// operations, about the accuracy of the MUFU approximation.  Nine packed
// FP32 instructions and four integer ones; used where the MUFU is the
// busier pipe.
__device__ __forceinline__ f2_t f2_rsqrt_sw(f2_t x)
{
    float a, b;
    f2_split(x, a, b);
    f2_t y = f2_make(__uint_as_float(0x5f375a86u - (__float_as_uint(a) >> 1)),
                     __uint_as_float(0x5f375a86u - (__float_as_uint(b) >> 1)));
    const f2_t m1 = f2_make(-1.0f, -1.0f), c38 = f2_make(0.375f, 0.375f), mh = f2_make(-0.5f, -0.5f);
    f2_t e = f2_fma(x, f2_mul(y, y), m1);
    y = f2_fma(f2_mul(y, e), mh, y);
    e = f2_fma(x, f2_mul(y, y), m1);
    return f2_fma(f2_mul(y, e), f2_fma(e, c38, mh), y);
}

}  // namespace bt
