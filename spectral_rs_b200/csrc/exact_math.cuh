// Correctly rounded reciprocal and square root for arguments in [1, 2^126).
//
// The Boris push and the position update divide by and take square roots of
// quantities that are at least 1 (gamma = sqrt(1 + |p|^2/c^2), 1 + |u|^2/c^2,
// 1 + |b|^2).  On that domain the hardware approximations need none of the
// special-case handling of the full-range IEEE operations, and two fused
// multiply-add corrections give the correctly rounded result.  Method:
// P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Develop. 34(1), 1990 (Newton-Raphson
// refinement whose last step is a fused multiply-add on an exactly computed
// residual).  Outside the domain (and for NaN) the callers' guards fall back to
// the IEEE operations; tests/test_gpu_rounding.py checks every float of the
// domain against them.
#pragma once

namespace spx {

// 1/x rounded to nearest, x in [1, 2^126)
__device__ __forceinline__ float rcp_rn_ge1(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  float e = __fmaf_rn(-x, y, 1.0f);  // residual 1 - x y
  y = __fmaf_rn(y, e, y);            // one Newton step: within one ulp
  e = __fmaf_rn(-x, y, 1.0f);        // exact residual of the refined value
  return __fmaf_rn(y, e, y);         // correction, rounded once
}

// sqrt(x) rounded to nearest, x in [1, 2^126)
__device__ __forceinline__ float sqrt_rn_ge1(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  float g = __fmul_rn(x, y);           // ~ sqrt(x)
  float h = __fmul_rn(0.5f, y);        // ~ 1 / (2 sqrt(x))
  const float r = __fmaf_rn(-g, h, 0.5f);
  g = __fmaf_rn(g, r, g);
  h = __fmaf_rn(h, r, h);
  const float d = __fmaf_rn(-g, g, x);  // exact remainder x - g^2
  return __fmaf_rn(d, h, g);            // correction, rounded once
}

constexpr float kExactMathMax = 85070591730234615865843651857942052864.0f;  // 2^126

// IEEE-equal versions for any argument: the fast path on [1, 2^126), else the IEEE operation
__device__ __forceinline__ float rcp_exact(float x) {
  return (x >= 1.0f && x < kExactMathMax) ? rcp_rn_ge1(x) : __frcp_rn(x);
}
__device__ __forceinline__ float sqrt_exact(float x) {
  return (x >= 1.0f && x < kExactMathMax) ? sqrt_rn_ge1(x) : __fsqrt_rn(x);
}

}  // namespace spx
