// Packed single-precision pairs for sm_100a.
//
// Blackwell executes add / mul / fma on two FP32 values held in a register
// pair with one instruction (`__ffma2_rn` and friends, PTX `.f32x2`, sm_100
// and later); each half is rounded exactly as the scalar `.rn` operation
// would round it. The
// RK5 stage combinations apply the same coefficient to every state variable,
// so pairing the variables halves their instruction count; the coefficient
// pairs come from constant memory (one operand of the packed instruction).
#pragma once
#include <stdint.h>
#include <cuda_runtime.h>

namespace ngpu {

typedef float2 f2;   // x = first, y = second

__device__ __forceinline__ f2 f2_pack(float lo, float hi) { return make_float2(lo, hi); }
__device__ __forceinline__ float f2_lo(f2 v) { return v.x; }
__device__ __forceinline__ float f2_hi(f2 v) { return v.y; }
__device__ __forceinline__ void f2_unpack(f2 v, float &lo, float &hi) {
  lo = v.x;
  hi = v.y;
}
// the sm_100 paired intrinsics (one FP32x2 instruction each)
__device__ __forceinline__ f2 f2_fma(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }   // a * b + c
__device__ __forceinline__ f2 f2_mul(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 f2_add(f2 a, f2 b) { return __fadd2_rn(a, b); }

// 2^x and log2(x) of the special-function unit (PTX ex2.approx / lg2.approx,
// relative error of a few units in the last place, denormals flushed)
__device__ __forceinline__ float ex2_approx(float x) {
  float r;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float lg2_approx(float x) {
  float r;
  asm("lg2.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// e^x as 2^(x log2 e): the exponential of the mathematical identity, with
// the scaling folded into the caller's argument where it can be
constexpr float kLog2e = 1.4426950408889634f;

}  // namespace ngpu
