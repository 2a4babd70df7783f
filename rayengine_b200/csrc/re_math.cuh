// Device-side vector math with a fixed rounding policy.
//
// The library is compiled with -fmad=false, IEEE division and square root:
// every fused multiply-add is written out as __fmaf_rn, so results are
// reproducible and identical to the CPU checker built the same way.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace re {

struct V3 {
  float x, y, z;
};

__device__ __forceinline__ V3 v3(float x, float y, float z) { return {x, y, z}; }
__device__ __forceinline__ V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
__device__ __forceinline__ float dot(V3 a, V3 b) {
  return __fmaf_rn(a.z, b.z, __fmaf_rn(a.y, b.y, a.x * b.x));
}
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
  return {__fmaf_rn(a.y, b.z, -(a.z * b.y)), __fmaf_rn(a.z, b.x, -(a.x * b.z)),
          __fmaf_rn(a.x, b.y, -(a.y * b.x))};
}
__device__ __forceinline__ V3 normalize(V3 v) {
  float inv = 1.0f / sqrtf(dot(v, v));
  return {v.x * inv, v.y * inv, v.z * inv};
}
__device__ __forceinline__ float comp(V3 v, uint32_t k) {
  return k == 0 ? v.x : (k == 1 ? v.y : v.z);
}

// Camera constants computed on the host (see camera_basis()).
struct CamDev {
  V3 campos, middle, horizontal, vertical;
  float focal;
};

// generate_ray (RayEngine/src/cuda-src/ray_functions.cuh:14-55) for pixel
// (x, y), followed by the traversal's renormalisation (:267).
__device__ __forceinline__ void generate_ray(const CamDev& c, uint32_t w, uint32_t h,
                                             uint32_t x, uint32_t y, V3& o, V3& d) {
  float sx = (float)x / ((float)w - 1.0f);
  float sy = 1.0f - (float)y / ((float)h - 1.0f);
  float a = 2.0f * sx - 1.0f;
  float b = 2.0f * sy - 1.0f;
  V3 p1 = {__fmaf_rn(c.vertical.x, b, __fmaf_rn(c.horizontal.x, a, c.middle.x)),
           __fmaf_rn(c.vertical.y, b, __fmaf_rn(c.horizontal.y, a, c.middle.y)),
           __fmaf_rn(c.vertical.z, b, __fmaf_rn(c.horizontal.z, a, c.middle.z))};
  V3 pip = {__fmaf_rn(p1.x - c.campos.x, c.focal, c.campos.x),
            __fmaf_rn(p1.y - c.campos.y, c.focal, c.campos.y),
            __fmaf_rn(p1.z - c.campos.z, c.focal, c.campos.z)};
  d = normalize(normalize(normalize(sub(pip, c.campos))));
  o = c.campos;
}

// integer mixer shared with the CPU checker (counter-based sampling)
__device__ __forceinline__ uint32_t hash_u32(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u ^ (c + 0x165667B1u) * 0xC2B2AE3Du;
  h ^= h >> 16;
  h *= 0x7feb352du;
  h ^= h >> 15;
  h *= 0x846ca68bu;
  h ^= h >> 16;
  return h;
}

// sin/cos of 2*pi*u, u in [0,1): quadrant split + Taylor polynomials on
// [0, pi/2) (sin to x^11, cos to x^12), Horner form.
__device__ __forceinline__ void sincos_2pi(float u, float& s, float& c) {
  float x4 = u * 4.0f;
  float qf = floorf(x4);
  int q = ((int)qf) & 3;
  float a = (x4 - qf) * 1.57079637f;
  float a2 = a * a;
  float sp = __fmaf_rn(a2, -2.50521084e-08f, 2.75573192e-06f);
  sp = __fmaf_rn(a2, sp, -1.98412698e-04f);
  sp = __fmaf_rn(a2, sp, 8.33333333e-03f);
  sp = __fmaf_rn(a2, sp, -1.66666667e-01f);
  sp = __fmaf_rn(a2, sp, 1.0f);
  float sn = a * sp;
  float cp = __fmaf_rn(a2, 2.08767570e-09f, -2.75573192e-07f);
  cp = __fmaf_rn(a2, cp, 2.48015873e-05f);
  cp = __fmaf_rn(a2, cp, -1.38888889e-03f);
  cp = __fmaf_rn(a2, cp, 4.16666667e-02f);
  cp = __fmaf_rn(a2, cp, -0.5f);
  float cs = __fmaf_rn(a2, cp, 1.0f);
  switch (q) {
    case 0: s = sn; c = cs; break;
    case 1: s = cs; c = -sn; break;
    case 2: s = -sn; c = -cs; break;
    default: s = -cs; c = sn; break;
  }
}

}  // namespace re
