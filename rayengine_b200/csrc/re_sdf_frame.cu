// The shaded SDF terrain frame: the reference's live render path.
//
// The reference ships with `sphere_tracing` defined (RE/RayEngine/RayEngine.h:22),
// so its render call cuda_render_frame (RE/cuda-src/renderer.cu:702-738)
// launches render_sphere_trace (renderer.cu:143-285) every frame: march the
// terrain, shade the hit (paint_surface, sphere_tracing.cuh:408-440; the
// lighting of shade_terrain / sphere_trace_shadow, :276-360, with the soft
// shadow march of single_shadow_ray_sphere_trace, :246-273), paint misses
// with the atmosphere (compute_incident_light, material_functions.cuh:296-344,
// and the tone curve of renderer.cu:266-270), then fog, gamma and vignetting
// (renderer.cu:273-279), clamp and rgbaFloatToInt (cuda_helper_functions.h:61-68).
//
// Here the terrain is the exact SDF field d(p) = p.y - amp fBm(scale p)
// traced by re_sdf_trace (k_sdf), and a second kernel shades every pixel
// from that hit record.  Deviations (each stated where it is made):
//   * the reference's terrain shadow march never advances (its
//     `min_dist == get_terrain_distance(...)` compares instead of assigning,
//     sphere_tracing.cuh:230); the working volume variant is restated, and
//     it starts at shadow_tmin and steps by the field's step factor because
//     d(p) is not a distance bound;
//   * paint_surface's biome test has no return value for heights between
//     the ocean and snow bands (sdf_functions.cuh:139-144); those keep the
//     tile colour;
//   * the snow band's fBm reads the permutation table as a filtered texture
//     (sphere_tracing.cuh:389-400), unreproducible; it uses the library's
//     Perlin noise at y = 0;
//   * the fog distance of a hit is |hit - origin| (the march's t is not kept
//     in the hit record).
// Transcendentals use re_fmath.cuh's fixed-sequence functions.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "re_common.hpp"
#include "re_fmath.cuh"
#include "re_math.cuh"
#include "re_noise.cuh"

namespace re {
namespace sdfframe {

constexpr float kInf = 1e20f;     // K_INFINITY (RayEngine.h:24)
constexpr float kEps = 1e-4f;     // K_EPSILON (RayEngine.h:25)
constexpr double kPi = 3.14159265358979323846;

struct ShadeDev {
  // field
  uint32_t octaves;
  float scale, amp, step_factor;
  // light (illuminate, cuda_helper_functions.h:90-102, computed on the host)
  V3 lightpos, light_int;
  float light_dist;
  float soft_k, shadow_tmin, shadow_tmax;
  uint32_t shadow_max_steps;
  V3 sun;
  float max_y, fog_density, vignetting_k;
  uint32_t flags;
};

__device__ __forceinline__ float sat(float x) { return x > 0.0f ? (x < 1.0f ? x : 1.0f) : 0.0f; }

// smoothstep(a, b, x) of the reference's vector helpers
__device__ __forceinline__ float smooth(float a, float b, float x) {
  float y = (x - a) / (b - a);
  y = fminf(fmaxf(y, 0.0f), 1.0f);
  return (y * y) * (3.0f - (2.0f * y));
}

// 4-octave rotated fBm of the snow band (sphere_tracing.cuh:389-400) on the
// library's Perlin noise.
template <class PT>
__device__ __forceinline__ float snow_fbm(const PT& P, float x, float z) {
  const float w[4] = {0.5f, 0.25f, 0.125f, 0.0625f};
  const float lac[3] = {2.02f, 2.03f, 2.01f};
  float f = 0.0f;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    f = f + w[i] * perlin(P, x, 0.0f, z);  // w[i] * n is exact: one rounding, as in double
    if (i < 3) {
      float nx = 0.8f * x + (-0.6f) * z, nz = 0.6f * x + 0.8f * z;
      x = nx * lac[i];
      z = nz * lac[i];
    }
  }
  return (float)((double)f / 0.9375);
}

// paint_surface for the terrain (material -1): tile pattern, then biomes.
template <class PT>
__device__ __forceinline__ V3 paint(const PT& P, const ShadeDev& S, V3 p, V3 n) {
  int square = (int)floorf(p.x) + (int)floorf(p.z);
  float c = (square % 2 == 0) ? 0.0f : 1.0f;  // tile_pattern (material_functions.cuh:13-27)
  V3 col = {c, c, c};
  double y = p.y, e = S.max_y;
  if (y <= 0.2 * e) {  // ocean
    col = v3(0.1f, 0.1f, 0.8f);
  } else if (y >= 0.8 * e) {  // snow
    float sx = ((0.01f * p.x) / S.max_y) / 2.0f, sz = ((0.01f * p.z) / S.max_y) / 2.0f;
    float h = smooth(55.0f, 80.0f, (float)((double)(p.y / (S.max_y / 2.0f)) +
                                           25.0 * (double)snow_fbm(P, sx, sz)));
    float ee = smooth((float)(1.0 - 0.5 * (double)h), (float)(1.0 - 0.1 * (double)h), n.y);
    float o = (float)(0.3 + 0.7 * (double)smooth(0.0f, 0.1f, n.x + h * h));
    float s = (h * ee) * o;
    float m = smooth(0.1f, 0.9f, s);
    col = v3(sat(col.x + m * (0.29f * 0.62f)), sat(col.y + m * (0.29f * 0.65f)),
             sat(col.z + m * (0.29f * 0.7f)));
  }
  return col;
}

// The light of sphere_trace_shadow, in three parts so that the shading
// kernel can advance the soft-shadow march one field evaluation per trip:
// light_setup (illuminate: direction of the light from the hit), one march
// step of single_shadow_ray_sphere_trace per call of shadow_step, and
// light_terms (ambient, soft-shadowed diffuse and back light).
__device__ __forceinline__ void light_setup(const ShadeDev& S, V3 p, V3& L, float& ldx,
                                            float& ldz) {
  V3 ld = {(p.x - S.lightpos.x) / S.light_dist, (p.y - S.lightpos.y) / S.light_dist,
           (p.z - S.lightpos.z) / S.light_dist};
  L = normalize(v3(-ld.x, -ld.y, -ld.z));
  ldx = ld.x;
  ldz = ld.z;
}

// One step: returns false when the march is over (step bound, range, or the
// ray is occluded: prel = 0).  The march starts with t = shadow_tmin,
// prel = 1, i = 0.
template <class PT>
__device__ __forceinline__ bool shadow_step(const PT& P, const ShadeDev& S, V3 p, V3 L, float& t,
                                            float& prel, uint32_t& i, uint32_t& evals) {
  if (!(i < S.shadow_max_steps && t < S.shadow_tmax)) return false;
  V3 q = {__fmaf_rn(t, L.x, p.x), __fmaf_rn(t, L.y, p.y), __fmaf_rn(t, L.z, p.z)};
  float dd = terrain_density(P, q, S.octaves, S.scale, S.amp);
  ++evals;
  ++i;
  if (prel < kEps || dd <= 1e-5f) {
    prel = 0.0f;
    return false;
  }
  prel = fminf(prel, (S.soft_k * dd) / t);
  t = __fmaf_rn(S.step_factor, dd, t);
  return true;
}

__device__ __forceinline__ V3 light_terms(const ShadeDev& S, float prel, V3 n, V3 L, float ldx,
                                          float ldz) {
  float amb = sat((float)(0.5 + 0.5 * (double)n.y));
  float soft = sat(prel);
  float dif = fmaxf(0.0f, dot(n, L));
  V3 bv = normalize(v3(-ldx, 0.0f, ldz));
  float bac = sat((float)(0.2 + 0.8 * (double)dot(bv, n)));
  V3 pc = {(soft * S.light_int.x) * dif, (soft * S.light_int.y) * dif,
           (soft * S.light_int.z) * dif};
  pc = v3(pc.x + (amb * 0.40f) * 1.2f, pc.y + (amb * 0.60f) * 1.2f, pc.z + (amb * 1.00f) * 1.2f);
  pc = v3(pc.x + bac * 0.40f, pc.y + bac * 0.50f, pc.z + bac * 0.60f);
  return pc;
}

// gpu_ray_sphere_intersect + solve_quadratic (ray_functions.cuh:95-126)
__device__ __forceinline__ bool ray_sphere(V3 o, V3 d, float radius, float& t0, float& t1) {
  float a = dot(d, d);
  float b = 2.0f * dot(d, o);
  float c = dot(o, o) - radius * radius;
  float discr = b * b - (4.0f * a) * c;
  if (discr < 0.0f) return false;
  if (discr == 0.0f) {
    t0 = t1 = (-0.5f * b) / a;
  } else {
    float q = b > 0.0f ? -0.5f * (b + sqrtf(discr)) : -0.5f * (b - sqrtf(discr));
    t0 = q / a;
    t1 = c / q;
  }
  if (t0 > t1) {
    float x = t0;
    t0 = t1;
    t1 = x;
  }
  return true;
}

__device__ __forceinline__ float vlen(V3 v) { return sqrtf(dot(v, v)); }

// compute_incident_light (material_functions.cuh:296-344) with the
// Atmosphere defaults (Atmosphere.cuh:8-21), then the miss tone curve.
__device__ __noinline__ V3 sky(const ShadeDev& S, V3 dir) {
  const float R = 6360e3f, Ra = 6420e3f, Hr = 79945.0f, Hm = 1200.0f;
  const V3 betaR = {3.8e-6f, 13.5e-6f, 33.1e-6f};
  const float betaM = 21e-6f;
  const V3 orig = {0.0f, R + 10000.0f, 300000.0f};
  V3 col;
  float t0, t1;
  if (!ray_sphere(orig, dir, Ra, t0, t1) || t1 < 0.0f) {
    col = v3(1.0f, 1.0f, 1.0f);
  } else {
    float tmin = 0.0f, tmax = kInf;
    if (t0 > tmin && t0 > 0.0f) tmin = t0;
    if (t1 < tmax) tmax = t1;
    float seg = (tmax - tmin) / 32.0f;
    float tc = tmin;
    V3 sumR = {0.f, 0.f, 0.f}, sumM = {0.f, 0.f, 0.f};
    float odR = 0.0f, odM = 0.0f;
    float mu = dot(dir, S.sun);
    float phaseR = (float)((3.0 / (16.0 * kPi)) * (double)(1.0f + mu * mu));
    const float g = 0.76f;
    float pb = (1.0f - g * g) * (1.0f + mu * mu);
    float pc = (2.0f + g * g) * fm_pow(1.0f + g * g - (2.0f * g) * mu, 1.5f);
    float phaseM = (float)(((3.0 / (8.0 * kPi)) * (double)pb) / (double)pc);
    for (int i = 0; i < 32; ++i) {
      float s = tc + seg * 0.5f;
      V3 sp = {orig.x + s * dir.x, orig.y + s * dir.y, orig.z + s * dir.z};
      float height = vlen(sp) - R;
      float hr = fm_exp(-height / Hr) * seg;
      float hm = fm_exp(-height / Hm) * seg;
      odR += hr;
      odM += hm;
      float tl0 = 0.0f, tl1 = 0.0f;
      ray_sphere(sp, S.sun, Ra, tl0, tl1);
      float segl = tl1 / 8.0f, tcl = 0.0f;
      float odLR = 0.0f, odLM = 0.0f;
      int j;
      for (j = 0; j < 8; ++j) {
        float sl = tcl + segl * 0.5f;
        V3 spl = {sp.x + sl * S.sun.x, sp.y + sl * S.sun.y, sp.z + sl * S.sun.z};
        float hl = vlen(spl) - R;
        if (hl < 0.0f) break;
        odLR += fm_exp(-hl / Hr) * segl;
        odLM += fm_exp(-hl / Hm) * segl;
        tcl += segl;
      }
      if (j == 8) {
        float aR = odR + odLR, aM = (betaM * 1.1f) * (odM + odLM);
        V3 att = {fm_exp(-(betaR.x * aR + aM)), fm_exp(-(betaR.y * aR + aM)),
                  fm_exp(-(betaR.z * aR + aM))};
        sumR = v3(sumR.x + att.x * hr, sumR.y + att.y * hr, sumR.z + att.z * hr);
        sumM = v3(sumM.x + att.x * hm, sumM.y + att.y * hm, sumM.z + att.z * hm);
      }
      tc += seg;
    }
    float m100 = (100.0f * betaM) * phaseM;
    col = v3((((sumR.x * betaR.x) * phaseR + sumM.x) + m100) * 20.0f,
             (((sumR.y * betaR.y) * phaseR + sumM.y) + m100) * 20.0f,
             (((sumR.z * betaR.z) * phaseR + sumM.z) + m100) * 20.0f);
  }
  // tone curve of the sky (renderer.cu:268-270)
  float c[3] = {col.x, col.y, col.z};
#pragma unroll
  for (int k = 0; k < 3; ++k)
    c[k] = c[k] < 1.413f ? fm_pow(c[k] * 0.38317f, 1.0f / 2.2f) : 1.0f - fm_exp(-c[k]);
  return v3(c[0], c[1], c[2]);
}

__device__ __forceinline__ uint32_t rgba8(V3 c) {
  float r = sat(c.x), g = sat(c.y), b = sat(c.z);
  return (255u << 24) | ((uint32_t)(b * 255.0f) << 16) | ((uint32_t)(g * 255.0f) << 8) |
         (uint32_t)(r * 255.0f);
}

// Fog, gamma and vignetting of render_sphere_trace (renderer.cu:273-283)
// on a shaded colour, then the RGBA8 pack.  dist: the hit's distance
// (K_INFINITY for a miss).
__device__ __forceinline__ uint32_t finish_pixel(const ShadeDev& S, V3 col, V3 o, V3 d, float dist,
                                                 float u, float v) {
  if (S.flags & RE_SDF_FOG) {  // apply_fog (material_functions.cuh:53-63)
    float dens = S.fog_density;
    float e1 = fm_exp(-o.y * dens);
    float e2 = fm_exp(((-dist) * d.y) * dens);
    float f = sat((float)((((double)((0.0375f / dens) * e1)) * (1.0 - (double)e2)) / (double)d.y));
    col = v3(sat(col.x + f * (0.65f * 0.4f)), sat(col.y + f * (0.65f * 0.65f)),
             sat(col.z + f * (0.65f * 1.0f)));
  }
  if (S.flags & RE_SDF_GAMMA)
    col = v3(fm_pow(col.x, 1.0f / 2.2f), fm_pow(col.y, 1.0f / 2.2f), fm_pow(col.z, 1.0f / 2.2f));
  if (S.flags & RE_SDF_VIGNETTING) {
    float k = 0.5f + 0.5f * fm_pow((((16.0f * u) * v) * (1.0f - u)) * (1.0f - v), S.vignetting_k);
    col = v3(col.x * k, col.y * k, col.z * k);
  }
  return rgba8(col);
}

// Shading in two passes over the tracer's pixel order (lane i & 31 of 8x4
// tile i >> 5).
//
// k_sdf_shadow: the soft-shadow march of every lit hit, as a per-lane state
// machine: a lane takes a pixel, a lit hit then advances its shadow ray by
// one field evaluation per loop trip, so the lanes of a warp stay on the
// same code while their shadow rays take different numbers of steps; when
// at least kShadeRefill lanes are idle the warp claims that many new pixels
// with one atomic.  The pass writes each lit hit's shadow factor (prel, as
// float bits) into that pixel's word of the RGBA8 output, which the second
// pass reads and overwrites.
//
// k_sdf_finish: one thread per pixel paints it: the surface colour, the
// light with the shadow factor, or the atmosphere for a miss, then fog,
// gamma, vignetting and the pack.  Neighbouring pixels take the same branch
// (sky above the horizon, terrain below), so the warps stay converged; in
// one fused state machine the sky's 32 x 8 in-scattering samples and the
// surface shading of a refilled lane ran while the rest of its warp waited.
//
// Same operations, in the same order per pixel, as one loop per pixel.
constexpr uint32_t kShadeRefill = 4;

__global__ void __launch_bounds__(256) k_sdf_shadow(PermTable perm, ShadeDev S, uint32_t w,
                                                    uint32_t h, const float4* __restrict__ hits,
                                                    uint32_t* __restrict__ rgba,
                                                    uint32_t* __restrict__ cursor,
                                                    unsigned long long* __restrict__ evals_out) {
  extern __shared__ uint32_t perm_smem[];
  load_perm(perm, perm_smem);
  Perm P = perm_view(perm_smem);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t tiles_x = (w + 7) / 8;
  const uint32_t total = tiles_x * ((h + 3) / 4) * 32u;
  bool live = false, exhausted = false;
  uint32_t i = 0, evals = 0;
  size_t pix = 0;
  V3 p = {0.f, 0.f, 0.f}, L = p;
  float ldx = 0.f, ldz = 0.f, t = 0.f, prel = 0.f;
  for (;;) {
    uint32_t idle = __ballot_sync(0xFFFFFFFFu, !live);
    uint32_t nidle = __popc(idle);
    if (!exhausted && (nidle >= kShadeRefill || nidle == 32u)) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(cursor, nidle);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (base + nidle >= total) exhausted = true;
      if (!live) {
        uint32_t k = base + __popc(idle & ((1u << lane) - 1u));
        uint32_t tile = k >> 5, l = k & 31u;
        uint32_t x = (tile % tiles_x) * 8 + (l & 7u), y = (tile / tiles_x) * 4 + (l >> 3);
        if (k < total && x < w && y < h) {
          pix = (size_t)y * w + x;
          float4 r1 = __ldg(&hits[2 * pix + 1]);
          if (__float_as_uint(r1.w) == 1u) {
            float4 r0 = __ldg(&hits[2 * pix]);
            p = v3(r0.x, r0.y, r0.z);
            light_setup(S, p, L, ldx, ldz);
            t = S.shadow_tmin;
            prel = 1.0f;
            i = 0;
            live = true;
          }
        }
      }
    }
    if (__ballot_sync(0xFFFFFFFFu, live) == 0u) {
      if (exhausted) break;
      continue;
    }
    if (live && !shadow_step(P, S, p, L, t, prel, i, evals)) {
      rgba[pix] = __float_as_uint(prel);
      live = false;
    }
  }
  if (evals_out) {
    uint32_t s = __reduce_add_sync(0xFFFFFFFFu, evals);
    if (lane == 0) atomicAdd(evals_out, (unsigned long long)s);
  }
}

// The second pass; the permutation table (for the snow band's noise) as one
// word copy per entry: a pixel reads it at most once.
__global__ void __launch_bounds__(256) k_sdf_finish(PermTable perm, ShadeDev S, CamDev cam,
                                                    uint32_t w, uint32_t h,
                                                    const float4* __restrict__ hits,
                                                    uint32_t* __restrict__ rgba) {
  __shared__ uint32_t words[512];
  for (uint32_t j = threadIdx.x; j < 512u; j += blockDim.x) words[j] = perm_word(perm.p[j]);
  __syncthreads();
  PermWords P{words};
  const bool lit = (S.flags & RE_SDF_SHADE) != 0u;
  const uint32_t tiles_x = (w + 7) / 8;
  const uint32_t total = tiles_x * ((h + 3) / 4) * 32u;
  for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < total;
       k += gridDim.x * blockDim.x) {
    uint32_t tile = k >> 5, l = k & 31u;
    uint32_t x = (tile % tiles_x) * 8 + (l & 7u), y = (tile / tiles_x) * 4 + (l >> 3);
    if (x >= w || y >= h) continue;
    size_t pix = (size_t)y * w + x;
    float4 r1 = __ldg(&hits[2 * pix + 1]);
    V3 o, d;
    generate_ray(cam, w, h, x, y, o, d);
    float u = (float)x / (float)w, v = (float)y / (float)h;
    if (__float_as_uint(r1.w) == 1u) {
      float4 r0 = __ldg(&hits[2 * pix]);
      V3 p = v3(r0.x, r0.y, r0.z), n = v3(r0.w, r1.x, r1.y);
      V3 col = paint(P, S, p, n);
      if (lit) {
        V3 L;
        float ldx, ldz;
        light_setup(S, p, L, ldx, ldz);
        V3 pc = light_terms(S, __uint_as_float(rgba[pix]), n, L, ldx, ldz);
        col = v3(col.x * pc.x, col.y * pc.y, col.z * pc.z);
      }
      rgba[pix] = finish_pixel(S, col, o, d, vlen(sub(p, o)), u, v);
    } else {
      rgba[pix] = finish_pixel(S, sky(S, d), o, d, kInf, u, v);
    }
  }
}

// ------------------------------------------------------------------ host
PermTable perm_table(uint32_t seed) {
  uint32_t full[512];
  perlin_permutation(seed, full);
  PermTable t;
  for (int i = 0; i < 512; ++i) t.p[i] = (uint8_t)full[i];
  return t;
}

// Per-device scratch of the shading kernel: the tile cursor and the
// shadow-march evaluation count.
uint32_t* counters() {
  static uint32_t* ptrs[64] = {nullptr};
  static std::mutex mu;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(mu);
  if (!ptrs[dev] && cudaMalloc(&ptrs[dev], 64) != cudaSuccess) return nullptr;
  return ptrs[dev];
}

re_status check_shade(const re_sdf_shade_params* s, const char* fn) {
  if (!s) return fail(RE_ERR_INVALID_ARG, "%s: null shade parameters", fn);
  if (s->flags & ~(uint32_t)(RE_SDF_SHADE | RE_SDF_FOG | RE_SDF_GAMMA | RE_SDF_VIGNETTING))
    return fail(RE_ERR_INVALID_ARG, "%s: unknown flags", fn);
  if (s->shadow_max_steps > 4096) return fail(RE_ERR_LIMIT, "%s: shadow_max_steps > 4096", fn);
  if (!(s->shadow_tmin > 0.0f) || !(s->max_y > 0.0f))
    return fail(RE_ERR_INVALID_ARG, "%s: shadow_tmin and max_y must be positive", fn);
  if ((s->flags & RE_SDF_FOG) && !(s->fog_density > 0.0f))
    return fail(RE_ERR_INVALID_ARG, "%s: fog needs a positive density", fn);
  return RE_OK;
}

ShadeDev shade_dev(const re_sdf_params& f, const re_sdf_shade_params& s) {
  ShadeDev S;
  S.octaves = f.octaves;
  S.scale = f.scale;
  S.amp = f.amplitude;
  S.step_factor = f.step_factor;
  // illuminate (cuda_helper_functions.h:90-102): the distance is that of the
  // light from the origin, as in the reference
  float lx = s.light_pos[0], ly = s.light_pos[1];
  S.lightpos = {lx, ly, lx};
  float r2 = lx * lx + ly * ly + lx * lx;
  S.light_dist = std::sqrt(r2);
  float den = (float)(4.0 * kPi * (double)r2);
  S.light_int = {(0.86f * s.light_intensity) / den, (0.80f * s.light_intensity) / den,
                 (0.45f * s.light_intensity) / den};
  S.soft_k = s.soft_shadow_k;
  S.shadow_tmin = s.shadow_tmin;
  S.shadow_tmax = s.shadow_tmax;
  S.shadow_max_steps = s.shadow_max_steps;
  S.sun = {s.sun_dir[0], s.sun_dir[1], s.sun_dir[2]};
  S.max_y = s.max_y;
  S.fog_density = s.fog_density;
  S.vignetting_k = s.vignetting_k;
  S.flags = s.flags;
  return S;
}

re_status shade(const re_sdf_params& f, const re_sdf_shade_params& s, const re_camera& cam,
                uint32_t w, uint32_t h, const re_sdf_hit* d_hits, uint32_t* d_rgba,
                cudaStream_t st, uint64_t* d_evals) {
  uint32_t* ctr = counters();
  if (!ctr) return fail(RE_ERR_CUDA, "re_render_sdf_frame: counter allocation failed");
  CamBasis b;
  camera_basis(cam, b);
  CamDev cd;
  cd.campos = {b.campos[0], b.campos[1], b.campos[2]};
  cd.middle = {b.middle[0], b.middle[1], b.middle[2]};
  cd.horizontal = {b.horizontal[0], b.horizontal[1], b.horizontal[2]};
  cd.vertical = {b.vertical[0], b.vertical[1], b.vertical[2]};
  cd.focal = b.focal;
  if (s.flags & RE_SDF_SHADE) {
    RE_CUDA(cudaMemsetAsync(ctr, 0, 4, st));
    RE_CUDA(cudaFuncSetAttribute(k_sdf_shadow, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)kPermSmemBytes));
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sdf_shadow, 256,
                                                      kPermSmemBytes) != cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    k_sdf_shadow<<<per_sm * sm_count(), 256, kPermSmemBytes, st>>>(
        perm_table(f.seed), shade_dev(f, s), w, h, reinterpret_cast<const float4*>(d_hits),
        d_rgba, ctr, reinterpret_cast<unsigned long long*>(d_evals));
    RE_CHECK_LAUNCH("re_render_sdf_frame: shadow launch");
  }
  int fin_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fin_sm, k_sdf_finish, 256, 0) !=
          cudaSuccess ||
      fin_sm < 1)
    fin_sm = 1;
  k_sdf_finish<<<fin_sm * sm_count(), 256, 0, st>>>(
      perm_table(f.seed), shade_dev(f, s), cd, w, h, reinterpret_cast<const float4*>(d_hits),
      d_rgba);
  RE_CHECK_LAUNCH("re_render_sdf_frame: finish launch");
  return RE_OK;
}

// State for the reference-style cuda_render_frame() in SDF mode
// (initialize_volume_render keeps the reference's scene in globals).
struct BoundSdf {
  std::mutex mu;
  bool active = false;
  re_sdf_params field{};
  re_sdf_shade_params shade{};
  re_camera cam{};
  int animate = 0;
  float angle = 0.f;
  re_sdf_hit* d_hits = nullptr;
  size_t cap = 0;
};
BoundSdf& bound_sdf() {
  static BoundSdf b;
  return b;
}

}  // namespace sdfframe
}  // namespace re

extern "C" {

RE_API void re_sdf_shade_params_default(re_sdf_shade_params* s) {
  if (!s) return;
  std::memset(s, 0, sizeof(*s));
  s->light_pos[0] = 20.0f;
  s->light_pos[1] = 40.0f;
  s->light_intensity = 30000.0f;
  s->soft_shadow_k = 32.0f;  // SceneSettings::soft_shadow_k (RayEngine.h:113)
  s->shadow_tmin = 0.05f;
  s->shadow_tmax = 40.0f;
  s->shadow_max_steps = 128;
  // the sun of Craze's first frame after start (renderer.cu:287-298) is
  // straight up; a lower sun gives a visible sky gradient: (0, cos a, sin a)
  // at Craze's angle 0.3 (a = 0.18 pi), rounded to float
  s->sun_dir[0] = 0.0f;
  s->sun_dir[1] = 0.844327926f;
  s->sun_dir[2] = 0.535826795f;
  s->max_y = 2.0f;  // the terrain's lowest ~30 % of hits are ocean
  s->fog_density = 0.02f;
  s->vignetting_k = 0.25f;
  s->flags = RE_SDF_SHADE;
}

RE_API re_status re_sdf_shade(const re_sdf_params* field, const re_sdf_shade_params* shade,
                              const re_camera* cam, uint32_t w, uint32_t h,
                              const re_sdf_hit* d_hits, uint32_t* d_rgba, uint64_t* d_evals,
                              void* stream) {
  if (!field || !cam || !d_hits || !d_rgba || w < 2 || h < 2)
    return re::fail(RE_ERR_INVALID_ARG, "re_sdf_shade: bad arguments");
  if ((uint64_t)w * h > (1ull << 31)) return re::fail(RE_ERR_LIMIT, "re_sdf_shade: image too large");
  if (field->octaves > 32) return re::fail(RE_ERR_LIMIT, "re_sdf_shade: octaves > 32");
  re_status rs = re::sdfframe::check_shade(shade, "re_sdf_shade");
  if (rs != RE_OK) return rs;
  return re::sdfframe::shade(*field, *shade, *cam, w, h, d_hits, d_rgba, (cudaStream_t)stream,
                             d_evals);
}

RE_API re_status re_render_sdf_frame(const re_sdf_params* field,
                                     const re_sdf_shade_params* shade, const re_camera* cam,
                                     uint32_t w, uint32_t h, re_sdf_hit* d_hits,
                                     uint32_t* d_rgba, void* stream) {
  re_status rs = re::sdfframe::check_shade(shade, "re_render_sdf_frame");
  if (rs != RE_OK) return rs;
  if (!d_rgba) return re::fail(RE_ERR_INVALID_ARG, "re_render_sdf_frame: null output");
  rs = re_sdf_trace(field, cam, w, h, d_hits, stream);
  if (rs != RE_OK) return rs;
  return re::sdfframe::shade(*field, *shade, *cam, w, h, d_hits, d_rgba, (cudaStream_t)stream,
                             nullptr);
}

RE_API re_status re_sdf_frame_bind(const re_sdf_params* field, const re_sdf_shade_params* shade,
                                   const re_camera* cam, int animate_sun) {
  if (!field || !cam) return re::fail(RE_ERR_INVALID_ARG, "re_sdf_frame_bind: bad arguments");
  re_status rs = re::sdfframe::check_shade(shade, "re_sdf_frame_bind");
  if (rs != RE_OK) return rs;
  re::sdfframe::BoundSdf& b = re::sdfframe::bound_sdf();
  std::lock_guard<std::mutex> lk(b.mu);
  b.field = *field;
  b.shade = *shade;
  b.cam = *cam;
  b.animate = animate_sun;
  b.angle = 0.f;
  b.active = true;
  return RE_OK;
}

}  // extern "C"

namespace re {

// cuda_render_frame in SDF mode (called from re_frame.cu while an SDF
// terrain is bound): the frame on the default stream, then Craze's sun
// animation (renderer.cu:287-298: sun = (0, cos a, sin a), a = angle * pi *
// 0.6; angle += 0.001, wrapping past 1.1).  Returns false when no SDF
// terrain is bound.
bool sdf_render_bound(unsigned int* output, unsigned int width, unsigned int height) {
  sdfframe::BoundSdf& b = sdfframe::bound_sdf();
  std::lock_guard<std::mutex> lk(b.mu);
  if (!b.active) return false;
  size_t need = (size_t)width * height;
  if (b.cap < need) {
    cudaFree(b.d_hits);
    b.d_hits = nullptr;
    b.cap = 0;
    cudaError_t e = cudaMalloc(&b.d_hits, need * sizeof(re_sdf_hit));
    if (e != cudaSuccess) {
      cuda_fail(e, "cuda_render_frame: hit buffer");
      return true;
    }
    b.cap = need;
  }
  if (re_render_sdf_frame(&b.field, &b.shade, &b.cam, width, height, b.d_hits, output, nullptr) !=
      RE_OK)
    return true;
  cudaError_t e = cudaStreamSynchronize(nullptr);
  if (e != cudaSuccess) {
    cuda_fail(e, "cuda_render_frame");
    return true;
  }
  if (b.animate) {
    float ang = (float)((double)b.angle * sdfframe::kPi * 0.6);
    b.shade.sun_dir[0] = 0.0f;
    b.shade.sun_dir[1] = std::cos(ang);
    b.shade.sun_dir[2] = std::sin(ang);
    b.angle += 0.001f;
    if (b.angle > 1.1f) b.angle = 0.f;
  }
  return true;
}

void sdf_unbind() {
  sdfframe::BoundSdf& b = sdfframe::bound_sdf();
  std::lock_guard<std::mutex> lk(b.mu);
  b.active = false;
}

}  // namespace re

// ---------------------------------------------------------- checking
// The frame's elementary functions over device arrays, for checking them
// against CUDA's own (fn 0: e^x, 1: ln x, 2: x^y).
namespace re {
namespace {
__global__ void k_fmath(uint32_t fn, const float* __restrict__ x, const float* __restrict__ y,
                        uint32_t n, float* __restrict__ out) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    out[i] = fn == 0 ? fm_exp(x[i]) : (fn == 1 ? fm_log(x[i]) : fm_pow(x[i], y[i]));
}
}  // namespace
}  // namespace re

extern "C" RE_API re_status re_fmath(uint32_t fn, const float* d_x, const float* d_y, uint32_t n,
                                     float* d_out, void* stream) {
  if (fn > 2 || !d_x || !d_out || (fn == 2 && !d_y))
    return re::fail(RE_ERR_INVALID_ARG, "re_fmath: bad arguments");
  if (n == 0) return RE_OK;
  re::k_fmath<<<std::min<uint32_t>((n + 255) / 256, 4096), 256, 0, (cudaStream_t)stream>>>(
      fn, d_x, d_y, n, d_out);
  RE_CHECK_LAUNCH("re_fmath: launch");
  return RE_OK;
}
