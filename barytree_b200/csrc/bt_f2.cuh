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

}  // namespace bt
