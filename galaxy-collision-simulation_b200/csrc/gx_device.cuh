// gx_device.cuh -- device helpers shared by the sm_100a kernels of the engine.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "precision.cuh"

namespace gx {

// ---------------------------------------------------------------------------------------
// FP64 reciprocal square root.  Seed: the hardware approximation rsqrt.approx.ftz.f64
// (relative error below 2^-20 measured on B200).  One Householder step of order 2 on the
// series (1 - e)^(-1/2) = 1 + e/2 + 3e^2/8 + O(e^3) with e = 1 - s*y^2 leaves a relative
// error of about (5/16) e^3 < 2^-57, i.e. at the level of the final rounding.
// 5 FP64 pipe operations after the MUFU seed.  s == 0 gives a non-finite result; callers
// with eps == 0 select it away.
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ double rsqrt_f64(double s) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(s));
    const double e = fma(-s, y * y, 1.0);
    const double p = fma(0.375, e, 0.5);
    return fma(y * e, p, y);
}

__device__ __forceinline__ float rsqrt_f32(float s) {
    float y;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(s));
    return y;
}

// ---------------------------------------------------------------------------------------
// Packed FP32 pairs (PTX .f32x2, sm_100+).  One instruction applies the operation to two
// FP32 lanes held in a 64-bit register pair: the same FP32-pipe work as two scalar
// instructions but one issue slot, which leaves issue bandwidth for the MUFU rsqrt and the
// shared-memory loads of the pair kernel.
// ---------------------------------------------------------------------------------------
typedef unsigned long long f2;

__device__ __forceinline__ f2 pk2(float lo, float hi) {
    f2 r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
    return r;
}
__device__ __forceinline__ void upk2(f2 v, float& lo, float& hi) {
    asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2 sub2(f2 a, f2 b) {
    f2 d;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 mul2(f2 a, f2 b) {
    f2 d;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
    return d;
}
__device__ __forceinline__ f2 fma2(f2 a, f2 b, f2 c) {
    f2 d;
    asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
    return d;
}

// 16-byte shared-memory load of two packed pairs (p must be 16-byte aligned shared memory).
__device__ __forceinline__ void lds_v2b64(const float* p, f2& a, f2& b) {
    const unsigned addr = (unsigned)__cvta_generic_to_shared(p);
    asm volatile("ld.shared.v2.b64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "r"(addr));
}

// Knuth's TwoSum: s + e == a + b exactly (round-to-nearest, no overflow).
__device__ __forceinline__ void two_sum(float a, float b, float& s, float& e) {
    s = __fadd_rn(a, b);
    const float bp = __fsub_rn(s, a);
    const float ap = __fsub_rn(s, bp);
    e = __fadd_rn(__fsub_rn(a, ap), __fsub_rn(b, bp));
}

// Compensated FP32 accumulator: value = hi + lo.
struct CompF {
    float hi, lo;
    __device__ __forceinline__ void init() { hi = 0.f; lo = 0.f; }
    __device__ __forceinline__ void add(float v) {
        float s, e;
        two_sum(hi, v, s, e);
        hi = s;
        lo = __fadd_rn(lo, e);
    }
    __device__ __forceinline__ double value() const { return (double)hi + (double)lo; }
};

// Reference-order FP64 helpers: no FMA contraction (the reference's x86-64 build has none).
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

// Warp reductions.
__device__ __forceinline__ double warp_min(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace gx
