// Neural SDF surrogate of the volumetric terrain: shared definitions of the
// network used by the training kernels (SIMT FP32 with BF16-rounded weights
// and activations) and the tensor-core inference kernels (BF16 operands in
// shared memory, FP32 accumulators in tensor memory).
//
// Network: 3 -> 128 Fourier features -> 64 -> 64 -> 64 -> 64 -> 1, softplus
// after each hidden layer.  The reference has no learned component; this is
// new work that stands in for the fBm density (sdf_functions.cuh:147-206).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace re {
namespace nsdf {

constexpr int kIn = 128;      // padded feature width
constexpr int kHidden = 64;   // hidden width
constexpr int kChains = 2;    // frequency chains: base f0 and f0 * sqrt(2)
constexpr int kOctaves = 8;   // doublings per chain -> 16 log-spaced frequencies

// flat FP32 parameter vector: W1 (64x128, row = output), b1, W2..W4
// (64x64), b2..b4, w5 (64), b5
constexpr int OFF_W1 = 0;
constexpr int OFF_B1 = OFF_W1 + kHidden * kIn;
constexpr int OFF_W2 = OFF_B1 + kHidden;
constexpr int OFF_B2 = OFF_W2 + kHidden * kHidden;
constexpr int OFF_W3 = OFF_B2 + kHidden;
constexpr int OFF_B3 = OFF_W3 + kHidden * kHidden;
constexpr int OFF_W4 = OFF_B3 + kHidden;
constexpr int OFF_B4 = OFF_W4 + kHidden * kHidden;
constexpr int OFF_W5 = OFF_B4 + kHidden;
constexpr int OFF_B5 = OFF_W5 + kHidden;
constexpr int kNumParams = OFF_B5 + 1;

__host__ __device__ constexpr int w_off(int layer) {
  return layer == 0 ? OFF_W1 : layer == 1 ? OFF_W2 : layer == 2 ? OFF_W3 : OFF_W4;
}
__host__ __device__ constexpr int b_off(int layer) {
  return layer == 0 ? OFF_B1 : layer == 1 ? OFF_B2 : layer == 2 ? OFF_B3 : OFF_B4;
}

// Input transform: q = (p - center) * inv_half maps the training box to
// [-1, 1]^3; f0 is the lowest frequency in cycles per normalised unit.
struct InputMap {
  float center[3], inv_half[3];
  float f0;
};

__device__ __forceinline__ float bf16_round(float x) {
  return __bfloat162float(__float2bfloat16_rn(x));
}

// Features, in this order (index = chain*48 + octave*6 + 2*axis + {sin,cos}):
// sin/cos(2 pi f q) for f = f0 * 2^octave (chain 0) and f0 * sqrt2 * 2^octave
// (chain 1), then q.xyz at 96..98, zeros to 127.  Each chain evaluates one
// sin/cos pair per axis (argument reduced to [-0.5, 0.5] cycles) and doubles
// it with sin 2a = 2 sin a cos a, cos 2a = 1 - 2 sin^2 a.
__device__ __forceinline__ void chain_features(const InputMap& m, const float q[3], int chain,
                                               float out[48]) {
  float f = chain ? m.f0 * 1.41421356f : m.f0;
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    float arg = f * q[j];
    float r = arg - rintf(arg);
    float s, c;
    __sincosf(6.28318531f * r, &s, &c);
#pragma unroll
    for (int o = 0; o < kOctaves; ++o) {
      out[o * 6 + 2 * j] = s;
      out[o * 6 + 2 * j + 1] = c;
      float s2 = 2.0f * s * c;
      float c2 = __fmaf_rn(-2.0f * s, s, 1.0f);
      s = s2;
      c = c2;
    }
  }
}

__device__ __forceinline__ void normalise(const InputMap& m, float px, float py, float pz,
                                          float q[3]) {
  q[0] = (px - m.center[0]) * m.inv_half[0];
  q[1] = (py - m.center[1]) * m.inv_half[1];
  q[2] = (pz - m.center[2]) * m.inv_half[2];
}

// softplus(x) = max(x, 0) + log1p(exp(-|x|)), with log1p(u) on [0, 1]
// replaced by a degree-6 polynomial fitted to it (max error 2.6e-6): one
// special-function instruction (exp) and FMAs per activation.
__device__ __forceinline__ float lp_poly(float u) {
  float p = __fmaf_rn(u, -0.017806457f, 0.083866805f);
  p = __fmaf_rn(u, p, -0.19167475f);
  p = __fmaf_rn(u, p, 0.31643057f);
  p = __fmaf_rn(u, p, -0.49753284f);
  p = __fmaf_rn(u, p, 0.9998613f);
  return u * p;
}
__device__ __forceinline__ float lp_poly_deriv(float u) {
  float p = __fmaf_rn(u, 6.0f * -0.017806457f, 5.0f * 0.083866805f);
  p = __fmaf_rn(u, p, 4.0f * -0.19167475f);
  p = __fmaf_rn(u, p, 3.0f * 0.31643057f);
  p = __fmaf_rn(u, p, 2.0f * -0.49753284f);
  p = __fmaf_rn(u, p, 0.9998613f);
  return p;
}
__device__ __forceinline__ float softplus_approx(float x) {
  float u = __expf(-fabsf(x));
  return fmaxf(x, 0.0f) + lp_poly(u);
}
__device__ __forceinline__ float softplus_approx_deriv(float x) {
  float u = __expf(-fabsf(x));
  float g = u * lp_poly_deriv(u);
  return x > 0.0f ? 1.0f - g : g;
}

}  // namespace nsdf
}  // namespace re
