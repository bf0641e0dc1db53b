// Device helpers for the output stage of the filters: the phase of a complex
// sum.
#pragma once

#include <cuda_runtime.h>

namespace dcl {

// atan2(y, x) in float within 6e-7 rad (about 2^-21) of the exact angle for
// finite arguments whose larger magnitude is a normal float (at least
// 2^-126), in about 20 instructions.
//
// Method: with a = min(|x|, |y|) / max(|x|, |y|) in [0, 1], atan(a) is
// approximated by a * P(a^2), P a degree-6 polynomial fitted to
// atan(sqrt(s)) / sqrt(s) on s in [0, 1] by the Remez exchange algorithm,
// minimising the absolute error of a * P(a^2) (2.5e-7 rad in exact
// arithmetic; the coefficients were computed for this library).  The octant
// is then restored: pi/2 - r where |y| > |x|, pi - r where x < 0, and the
// sign of y (its sign bit, so atan2(-0, x) = -0 or -pi as for atan2f).  x = y
// = 0 gives 0 (or pi for negative zero x, like atan2f); a NaN argument gives
// NaN; when both magnitudes are subnormal the quotient is taken against
// 2^-126 instead of the larger one, so the angle is not accurate there.  The
// quotient uses the approximate reciprocal (1 ulp), which adds at most
// 1.2e-7 rad.
__device__ __forceinline__ float atan2_fast(float y, float x) {
  const float ax = fabsf(x), ay = fabsf(y);
  const float mx = fmaxf(ax, ay), mn = fminf(ax, ay);
  float inv;
  // max(.., 2^-126) keeps the reciprocal finite for a zero or subnormal
  // larger magnitude (0 / 0 would be NaN; the quotient is then 0 for
  // x = y = 0) and leaves every normal one exact
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(inv) : "f"(fmaxf(mx, 1.17549435e-38f)));
  const float a = mn * inv;
  const float s = a * a;
  float p = 0.006811792962253094f;
  p = fmaf(p, s, -0.0336042195558548f);
  p = fmaf(p, s, 0.07962366938591003f);
  p = fmaf(p, s, -0.1323334276676178f);
  p = fmaf(p, s, 0.19807815551757812f);
  p = fmaf(p, s, -0.3331736922264099f);
  p = fmaf(p, s, 0.9999961256980896f);
  float r = a * p;
  if (ay > ax) r = 1.57079637f - r;
  if (__float_as_int(x) < 0) r = 3.14159274f - r;
  // x NaN or y NaN: fmax/fmin returned the other operand, so restore NaN
  if (x != x || y != y) r = x + y;
  return copysignf(r, y);
}

}  // namespace dcl
