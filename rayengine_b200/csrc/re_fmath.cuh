// Elementary functions with a fixed operation sequence, for the shaded SDF
// frame (sky, fog, tone curve, gamma, vignetting).  The library's exact
// paths avoid the CUDA math library's transcendentals so that the CPU
// checker, built with the same operation sequence, gives identical bits.
//
//   e^x:  Cody-Waite argument reduction x = n ln2 + r (|r| <= ln2 / 2) with
//         Cephes' two-constant split of ln 2 (ln2 = C1 + C2, C1 = 355/512
//         exactly, so n * C1 is exact for |n| < 2^15), then the Taylor
//         polynomial of e^r to r^7 in Horner form (truncation error below
//         6e-9 relative), scaled by 2^n through the exponent field.
//         Arguments are clamped to [-87, 88], so 2^n stays a normal number.
//   ln x: x = m 2^e with m in [sqrt(1/2), sqrt(2)); ln m = 2 atanh(s),
//         s = (m - 1) / (m + 1), by its series s + s^3/3 + ... + s^11/11
//         (|s| <= 0.1716, truncation error below 1e-10); ln x = e ln2 + ln m.
//   x^y:  e^(y ln x) for x > 0; 0 for x below the smallest normal float.
//
// Accuracy against the true functions: a few units in the last place over
// the arguments the frame uses (checked on the GPU against CUDA's expf,
// logf and powf).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace re {

constexpr float kLn2C1 = 0.693359375f;      // 355/512
constexpr float kLn2C2 = -2.12194440e-4f;   // ln 2 - 355/512
constexpr float kLog2e = 1.44269504088896341f;
constexpr float kLn2 = 0.693147180559945309f;
constexpr float kSqrtHalf = 0.707106781186547524f;

__device__ __forceinline__ float fm_exp(float x) {
  x = fminf(fmaxf(x, -87.0f), 88.0f);
  float n = rintf(x * kLog2e);
  float r = __fmaf_rn(-n, kLn2C1, x);
  r = __fmaf_rn(-n, kLn2C2, r);
  float p = 1.0f / 5040.0f;
  p = __fmaf_rn(p, r, 1.0f / 720.0f);
  p = __fmaf_rn(p, r, 1.0f / 120.0f);
  p = __fmaf_rn(p, r, 1.0f / 24.0f);
  p = __fmaf_rn(p, r, 1.0f / 6.0f);
  p = __fmaf_rn(p, r, 0.5f);
  p = __fmaf_rn(p, r, 1.0f);
  p = __fmaf_rn(p, r, 1.0f);
  return p * __int_as_float(((int)n + 127) << 23);
}

// x > 0, normal
__device__ __forceinline__ float fm_log(float x) {
  uint32_t b = __float_as_uint(x);
  int e = (int)((b >> 23) & 255u) - 127;
  float m = __uint_as_float((b & 0x007FFFFFu) | 0x3F800000u);  // [1, 2)
  if (m > 2.0f * kSqrtHalf) {
    m *= 0.5f;
    e += 1;
  }
  float s = (m - 1.0f) / (m + 1.0f);
  float z = s * s;
  float q = 1.0f / 11.0f;
  q = __fmaf_rn(q, z, 1.0f / 9.0f);
  q = __fmaf_rn(q, z, 1.0f / 7.0f);
  q = __fmaf_rn(q, z, 1.0f / 5.0f);
  q = __fmaf_rn(q, z, 1.0f / 3.0f);
  q = __fmaf_rn(q, z, 1.0f);
  float lnm = 2.0f * (s * q);
  return __fmaf_rn((float)e, kLn2, lnm);
}

__device__ __forceinline__ float fm_pow(float x, float y) {
  if (!(x >= 1.17549435e-38f)) return 0.0f;
  return fm_exp(y * fm_log(x));
}

}  // namespace re
