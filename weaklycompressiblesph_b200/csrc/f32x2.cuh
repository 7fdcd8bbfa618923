// Packed FP32x2 arithmetic of sm_100 (PTX add/sub/mul/fma .rn.f32x2).  Each
// lane of a packed operation rounds exactly like the scalar FP32 operation,
// so packed code reproduces scalar results bit for bit while issuing one
// instruction per two values.
#pragma once
#include <cstdint>

namespace wcsph {

typedef unsigned long long f2;  // two FP32 values in one 64-bit register pair: lo = .x, hi = .y

__device__ __forceinline__ f2 pk(float lo, float hi) {
  f2 r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ f2 dup(float v) { return pk(v, v); }
__device__ __forceinline__ float lo(f2 v) {
  float a, b;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
  return a;
}
__device__ __forceinline__ float hi(f2 v) {
  float a, b;
  asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
  return b;
}
__device__ __forceinline__ f2 add2(f2 a, f2 b) {
  f2 d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
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
// Per-lane helpers with no packed form.
__device__ __forceinline__ f2 max0_2(f2 a) { return pk(fmaxf(lo(a), 0.0f), fmaxf(hi(a), 0.0f)); }
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ f2 rcp2(f2 a) { return pk(rcp_approx(lo(a)), rcp_approx(hi(a))); }
__device__ __forceinline__ f2 rsqrt2(f2 a) { return pk(rsqrtf(lo(a)), rsqrtf(hi(a))); }

}  // namespace wcsph
