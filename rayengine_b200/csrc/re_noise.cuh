// Improved-Perlin noise and fBm on the device.
//
// Value part of eval() (RayEngine/src/cuda-src/sdf_functions.cuh:84-135):
// lattice cell from floor & 255, quintic fade (:57-60), 16-case gradient dot
// (:26-47) and the k0..k7 polynomial form of the trilinear blend.  The
// reference's hash (:77-81) reads a linearly filtered, normalised-float
// texture and cannot be reproduced; the lattice hash here is
// P[P[P[x] + y] + z] over RPerlinNoise's table (PerlinNoise.h:16-52), which
// the kernels keep in shared memory.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "re_math.cuh"

namespace re {

struct PermTable {
  uint8_t p[512];
};

// The table lives in shared memory in 16 interleaved copies: entry j of
// lane c is the word 16*j + (c & 15), so of a warp's 32 divergent lookups
// only lanes c and c + 16 can meet in a bank (when their entries have the
// same parity).  512 entries x 16 copies x 4 B = 32 KB; measured on B200 2 %
// faster on the SDF march than 32 conflict-free copies (64 KB), which allow
// one block per SM fewer.  Each
// word holds P[j] in bits 0-7 and the gradient case h = P[j] & 15 decoded
// for grad_dot in bits 28-31: bit 28 set when its first operand is y (else
// x), bit 29 when its second operand is y (else z), bit 30 when the second
// operand is negated and bit 31 when the first one is (so that negation is
// an XOR of the operand's sign bit with the word).  Bits 28-31 fall out of
// the interleaved table's 32-bit index arithmetic (Perm::word), so chained
// lookups use the word unmasked.
constexpr uint32_t kPermSmemBytes = 512 * 16 * 4;

__host__ __device__ __forceinline__ uint32_t perm_word(uint32_t p) {
  const uint32_t h = p & 15u;
  return p | (((0xCF00u >> h) & 1u) << 28) | (((0x300Fu >> h) & 1u) << 29) |
         (((0x8CCCu >> h) & 1u) << 30) | (((0xEAAAu >> h) & 1u) << 31);
}

__device__ __forceinline__ void load_perm(const PermTable& t, uint32_t* s) {
  for (uint32_t i = threadIdx.x; i < 512 * 16; i += blockDim.x) s[i] = perm_word(t.p[i >> 4]);
  __syncthreads();
}

// Permutation-table views: idx(j) = P[j] (a lattice index), grad(j) = the
// perm_word() of P[j] (its gradient case decoded).
struct Perm {
  const uint32_t* __restrict__ s;
  uint32_t lane;
  // j may carry a word's bits 28-31: the 32-bit shift drops them, and the
  // rest (an index below 512) stays inside the 8192-word table
  __device__ __forceinline__ uint32_t word(uint32_t j) const { return s[(j << 4) + lane]; }
  // the raw word: as the next lookup's index its bits 28-31 do not count
  __device__ __forceinline__ uint32_t idx(uint32_t j) const { return word(j); }
  __device__ __forceinline__ uint32_t grad(uint32_t j) const { return word(j); }
};

__device__ __forceinline__ Perm perm_view(const uint32_t* s) { return Perm{s, threadIdx.x & 15u}; }

// Single shared tables for several seeds side by side (the batched
// renderer; no per-lane copies, lookups may share banks): perm_word()
// entries, 2 KB per seed (measured 4 % faster on the batch), or plain bytes,
// 512 B per seed, for batches with many seeds.
struct PermWords {
  const uint32_t* __restrict__ s;
  __device__ __forceinline__ uint32_t idx(uint32_t j) const { return s[j] & 255u; }
  __device__ __forceinline__ uint32_t grad(uint32_t j) const { return s[j]; }
};

struct PermBytes {
  const uint8_t* __restrict__ s;
  __device__ __forceinline__ uint32_t idx(uint32_t j) const { return s[j]; }
  __device__ __forceinline__ uint32_t grad(uint32_t j) const { return perm_word(s[j]); }
};

// gradientDotV (sdf_functions.cuh:26-47) without branches: each case is a
// sum of two signed coordinates, picked here from the decoded case bits of
// perm_word().  The operands and their signs are exactly the reference's,
// so the single rounded addition is unchanged:
//   first operand is y for cases 8-11, 14, 15 (x otherwise), negated for
//   1, 3, 5, 7, 9, 11, 13, 14, 15; second operand is y for 0-3, 12 and 13
//   (z otherwise), negated for 2, 3, 6, 7, 10, 11, 15.
// Case 12 is the reference's y + x, taken here as x + y: IEEE addition is
// commutative, so the sum is the same, and the second operand needs one
// select instead of two.  Negating the first operand flips its sign bit
// with the word's bit 31.  (Measured on B200: the field evaluation is bound
// by the ALU pipe, where these selects run.)
// g: a grad() lookup.
__device__ __forceinline__ float grad_dot(uint32_t g, float x, float y, float z) {
  float u = (g & 0x10000000u) ? y : x;
  u = __uint_as_float(__float_as_uint(u) ^ (g & 0x80000000u));
  float v = (g & 0x20000000u) ? y : z;
  v = (g & 0x40000000u) ? -v : v;
  return u + v;
}

__device__ __forceinline__ float quintic(float t) {
  float in = __fmaf_rn(t, 6.0f, -15.0f);
  in = __fmaf_rn(t, in, 10.0f);
  return ((t * t) * t) * in;
}

// PT: a permutation-table view with idx() and grad() (Perm: interleaved
// shared copies; PermWords: one word table).  The table's second half repeats the
// first (P[256 + i] = P[i], RPerlinNoise), so the upper lattice corners
// index it with xi0 + 1 etc. unmasked, which reads the same entries as the
// reference's (xi0 + 1) & 255.
template <class PT>
__device__ __forceinline__ float perlin(const PT& P, float x, float y, float z) {
  float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  uint32_t xi0 = ((int)fx) & 255, yi0 = ((int)fy) & 255, zi0 = ((int)fz) & 255;
  uint32_t xi1 = xi0 + 1, yi1 = yi0 + 1, zi1 = zi0 + 1;
  float tx = x - fx, ty = y - fy, tz = z - fz;
  float u = quintic(tx), v = quintic(ty), w = quintic(tz);
  float x1 = tx - 1.0f, y1 = ty - 1.0f, z1 = tz - 1.0f;
  uint32_t px0 = P.idx(xi0), px1 = P.idx(xi1);
  uint32_t p00 = P.idx(px0 + yi0), p10 = P.idx(px1 + yi0);
  uint32_t p01 = P.idx(px0 + yi1), p11 = P.idx(px1 + yi1);
  float a = grad_dot(P.grad(p00 + zi0), tx, ty, tz);
  float b = grad_dot(P.grad(p10 + zi0), x1, ty, tz);
  float c = grad_dot(P.grad(p01 + zi0), tx, y1, tz);
  float d = grad_dot(P.grad(p11 + zi0), x1, y1, tz);
  float e = grad_dot(P.grad(p00 + zi1), tx, ty, z1);
  float f = grad_dot(P.grad(p10 + zi1), x1, ty, z1);
  float g = grad_dot(P.grad(p01 + zi1), tx, y1, z1);
  float h = grad_dot(P.grad(p11 + zi1), x1, y1, z1);
  float k1 = b - a;
  float k2 = c - a;
  float k3 = e - a;
  float k4 = ((a + d) - b) - c;
  float k5 = ((a + f) - b) - e;
  float k6 = ((a + g) - c) - e;
  float k7 = ((((((b + c) + e) + h) - a) - d) - f) - g;
  float r = __fmaf_rn(k1, u, a);
  r = __fmaf_rn(k2, v, r);
  r = __fmaf_rn(k3, w, r);
  r = __fmaf_rn(k4, u * v, r);
  r = __fmaf_rn(k5, u * w, r);
  r = __fmaf_rn(k6, v * w, r);
  r = __fmaf_rn(k7, (u * v) * w, r);
  return r;
}

template <class PT>
__device__ __forceinline__ float fbm(const PT& P, float x, float y, float z,
                                     uint32_t octaves, float lacunarity, float gain) {
  float sum = 0.0f, amp = 1.0f;
#pragma unroll 4
  for (uint32_t i = 0; i < octaves; ++i) {
    sum = __fmaf_rn(amp, perlin(P, x, y, z), sum);
    x *= lacunarity;
    y *= lacunarity;
    z *= lacunarity;
    amp *= gain;
  }
  return sum;
}

// d(p) = p.y - amp * fbm(scale * p), lacunarity 2, gain 0.5
template <class PT>
__device__ __forceinline__ float terrain_density(const PT& P, V3 p,
                                                 uint32_t octaves, float scale, float amp) {
  float f = fbm(P, scale * p.x, scale * p.y, scale * p.z, octaves, 2.0f, 0.5f);
  return __fmaf_rn(-amp, f, p.y);
}

// Gradient of perlin() at (x, y, z), from the same lattice, fade and blend
// differentiated in closed form.  With corner values a..h (corner gradient
// vector ga..gh dotted with the offset to the corner) the blend is
//   n = a + k1 u + k2 v + k3 w + k4 uv + k5 uw + k6 vw + k7 uvw,
// u = fade(tx) etc., so
//   dn/dx = [sum over corners of (its trilinear weight in u, v, w) g].x
//           + fade'(tx) (k1 + k4 v + k5 w + k7 vw),
// likewise for y and z, with fade'(t) = 30 t^2 (t - 1)^2.  A corner's
// gradient vector is s1 e_op1 + s2 e_op2 (grad_dot's operands and signs), so
// the weighted sum adds the signed weight to the operands' components
// instead of multiplying.
template <class PT>
__device__ __forceinline__ V3 perlin_grad(const PT& P, float x, float y, float z) {
  float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  uint32_t xi0 = ((int)fx) & 255, yi0 = ((int)fy) & 255, zi0 = ((int)fz) & 255;
  uint32_t xi1 = xi0 + 1, yi1 = yi0 + 1, zi1 = zi0 + 1;
  float tx = x - fx, ty = y - fy, tz = z - fz;
  float u = quintic(tx), v = quintic(ty), w = quintic(tz);
  float x1 = tx - 1.0f, y1 = ty - 1.0f, z1 = tz - 1.0f;
  float du = 30.0f * (tx * tx) * (x1 * x1);
  float dv = 30.0f * (ty * ty) * (y1 * y1);
  float dw = 30.0f * (tz * tz) * (z1 * z1);
  uint32_t px0 = P.idx(xi0), px1 = P.idx(xi1);
  uint32_t p00 = P.idx(px0 + yi0), p10 = P.idx(px1 + yi0);
  uint32_t p01 = P.idx(px0 + yi1), p11 = P.idx(px1 + yi1);
  const uint32_t G[8] = {P.grad(p00 + zi0), P.grad(p10 + zi0), P.grad(p01 + zi0),
                         P.grad(p11 + zi0), P.grad(p00 + zi1), P.grad(p10 + zi1),
                         P.grad(p01 + zi1), P.grad(p11 + zi1)};
  const float a = grad_dot(G[0], tx, ty, tz), b = grad_dot(G[1], x1, ty, tz);
  const float c = grad_dot(G[2], tx, y1, tz), d = grad_dot(G[3], x1, y1, tz);
  const float e = grad_dot(G[4], tx, ty, z1), f = grad_dot(G[5], x1, ty, z1);
  const float g = grad_dot(G[6], tx, y1, z1), h = grad_dot(G[7], x1, y1, z1);
  float k1 = b - a, k2 = c - a, k3 = e - a;
  float k4 = ((a + d) - b) - c;
  float k5 = ((a + f) - b) - e;
  float k6 = ((a + g) - c) - e;
  float k7 = ((((((b + c) + e) + h) - a) - d) - f) - g;
  float uv = u * v, uw = u * w, vw = v * w, uvw = uv * w;
  // trilinear weights of the corners (order a..h: x fastest, then y, z)
  const float cw[8] = {1.0f - u - v - w + uv + uw + vw - uvw, u - uv - uw + uvw,
                       v - uv - vw + uvw, uv - uvw, w - uw - vw + uvw, uw - uvw, vw - uvw, uvw};
  float sx = 0.f, sy = 0.f, sz = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t gk = G[k];
    const float c1 = __uint_as_float(__float_as_uint(cw[k]) ^ (gk & 0x80000000u));  // s1 w
    const float c2 = (gk & 0x40000000u) ? -cw[k] : cw[k];                          // s2 w
    // first operand x or y, second y or z
    sx += (gk & 0x10000000u) ? 0.0f : c1;
    sy += ((gk & 0x10000000u) ? c1 : 0.0f) + ((gk & 0x20000000u) ? c2 : 0.0f);
    sz += (gk & 0x20000000u) ? 0.0f : c2;
  }
  V3 r;
  r.x = sx + du * (k1 + k4 * v + k5 * w + k7 * vw);
  r.y = sy + dv * (k2 + k4 * u + k6 * w + k7 * uw);
  r.z = sz + dw * (k3 + k5 * u + k6 * v + k7 * uv);
  return r;
}

// Gradient of terrain_density: (0, 1, 0) - amp * scale * sum_i gain^i
// lacunarity^i grad perlin(lacunarity^i scale p), lacunarity 2, gain 0.5
// (each octave's amplitude x frequency is 1).
template <class PT>
__device__ __forceinline__ V3 terrain_gradient(const PT& P, V3 p, uint32_t octaves, float scale,
                                               float amp) {
  float x = scale * p.x, y = scale * p.y, z = scale * p.z;
  V3 s = v3(0.f, 0.f, 0.f);
  for (uint32_t i = 0; i < octaves; ++i) {
    V3 gi = perlin_grad(P, x, y, z);
    s = v3(s.x + gi.x, s.y + gi.y, s.z + gi.z);
    x *= 2.0f;
    y *= 2.0f;
    z *= 2.0f;
  }
  const float k = -amp * scale;
  return v3(k * s.x, __fmaf_rn(k, s.y, 1.0f), k * s.z);
}

}  // namespace re
