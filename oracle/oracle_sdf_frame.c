/*
 * TEST INFRASTRUCTURE ONLY -- CPU restatement of the shaded SDF terrain
 * frame, the checker of the library's re_render_sdf_frame / re_sdf_shade.
 *
 * Follows the reference's live frame kernel render_sphere_trace
 * (RayEngine/src/cuda-src/renderer.cu:143-285):
 *   paint_surface            sphere_tracing.cuh:408-440 (tile_pattern,
 *                            material_functions.cuh:13-27; biomes,
 *                            sdf_functions.cuh:139-144)
 *   soft shadow + light      single_shadow_ray_sphere_trace and
 *                            sphere_trace_shadow, sphere_tracing.cuh:246-360;
 *                            illuminate, cuda_helper_functions.h:90-102
 *   sky                      compute_incident_light,
 *                            material_functions.cuh:296-344, Atmosphere.cuh:8-21;
 *                            gpu_ray_sphere_intersect, ray_functions.cuh:95-126;
 *                            tone curve renderer.cu:266-270
 *   fog, gamma, vignetting   material_functions.cuh:53-63, renderer.cu:273-279
 *   clip + rgbaFloatToInt    cuda_helper_functions.h:61-68,109-131
 * with the library's deviations (stated in re_sdf_frame.cu): the working
 * volume shadow march started at shadow_tmin with the field's step factor,
 * tile colour between the ocean and snow bands, Perlin noise in the snow
 * band's fBm, fog distance |hit - origin|.
 *
 * Elementary functions: e^x by Cody-Waite reduction (Cephes' split of ln 2,
 * 355/512 + -2.12194440e-4) and the Taylor polynomial of e^r to r^7; ln x by
 * 2 atanh((m-1)/(m+1)) to s^11; x^y = e^(y ln x).  Built with
 * -ffp-contract=off and explicit fmaf, like the kernels' __fmaf_rn.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

#define O_PI 3.14159265358979323846
#define K_INFINITY 1e20f /* RE/RayEngine/RayEngine.h:24 */

static inline float f_as(uint32_t u) {
  float f;
  memcpy(&f, &u, 4);
  return f;
}
static inline uint32_t u_as(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}

float o_fm_exp(float x) {
  x = fminf(fmaxf(x, -87.0f), 88.0f);
  float n = rintf(x * 1.44269504088896341f);
  float r = fmaf(-n, 0.693359375f, x);
  r = fmaf(-n, -2.12194440e-4f, r);
  float p = 1.0f / 5040.0f;
  p = fmaf(p, r, 1.0f / 720.0f);
  p = fmaf(p, r, 1.0f / 120.0f);
  p = fmaf(p, r, 1.0f / 24.0f);
  p = fmaf(p, r, 1.0f / 6.0f);
  p = fmaf(p, r, 0.5f);
  p = fmaf(p, r, 1.0f);
  p = fmaf(p, r, 1.0f);
  return p * f_as((uint32_t)(((int)n + 127) << 23));
}

float o_fm_log(float x) {
  uint32_t b = u_as(x);
  int e = (int)((b >> 23) & 255u) - 127;
  float m = f_as((b & 0x007FFFFFu) | 0x3F800000u);
  if (m > 2.0f * 0.707106781186547524f) {
    m *= 0.5f;
    e += 1;
  }
  float s = (m - 1.0f) / (m + 1.0f);
  float z = s * s;
  float q = 1.0f / 11.0f;
  q = fmaf(q, z, 1.0f / 9.0f);
  q = fmaf(q, z, 1.0f / 7.0f);
  q = fmaf(q, z, 1.0f / 5.0f);
  q = fmaf(q, z, 1.0f / 3.0f);
  q = fmaf(q, z, 1.0f);
  float lnm = 2.0f * (s * q);
  return fmaf((float)e, 0.693147180559945309f, lnm);
}

float o_fm_pow(float x, float y) {
  if (!(x >= 1.17549435e-38f)) return 0.0f;
  return o_fm_exp(y * o_fm_log(x));
}

static inline float sat(float x) { return x > 0.0f ? (x < 1.0f ? x : 1.0f) : 0.0f; }

static inline float smooth(float a, float b, float x) {
  float y = (x - a) / (b - a);
  y = fminf(fmaxf(y, 0.0f), 1.0f);
  return (y * y) * (3.0f - (2.0f * y));
}

static inline float dot3f(const float a[3], const float b[3]) {
  return fmaf(a[2], b[2], fmaf(a[1], b[1], a[0] * b[0]));
}
static inline void norm3f(float v[3]) {
  float inv = 1.0f / sqrtf(dot3f(v, v));
  v[0] *= inv;
  v[1] *= inv;
  v[2] *= inv;
}
static inline float len3f(const float v[3]) { return sqrtf(dot3f(v, v)); }

static float snow_fbm(const uint32_t P[512], float x, float z) {
  const float w[4] = {0.5f, 0.25f, 0.125f, 0.0625f};
  const float lac[3] = {2.02f, 2.03f, 2.01f};
  float f = 0.0f;
  for (int i = 0; i < 4; ++i) {
    f = f + w[i] * o_perlin(P, x, 0.0f, z);
    if (i < 3) {
      float nx = 0.8f * x + (-0.6f) * z, nz = 0.6f * x + 0.8f * z;
      x = nx * lac[i];
      z = nz * lac[i];
    }
  }
  return (float)((double)f / 0.9375);
}

static void paint(const uint32_t P[512], const o_sdf_shade* S, const float p[3],
                  const float n[3], float col[3]) {
  int square = (int)floorf(p[0]) + (int)floorf(p[2]);
  float c = (square % 2 == 0) ? 0.0f : 1.0f;
  col[0] = col[1] = col[2] = c;
  double y = p[1], e = S->max_y;
  if (y <= 0.2 * e) {
    col[0] = 0.1f;
    col[1] = 0.1f;
    col[2] = 0.8f;
  } else if (y >= 0.8 * e) {
    float sx = ((0.01f * p[0]) / S->max_y) / 2.0f, sz = ((0.01f * p[2]) / S->max_y) / 2.0f;
    float h = smooth(55.0f, 80.0f,
                     (float)((double)(p[1] / (S->max_y / 2.0f)) + 25.0 * (double)snow_fbm(P, sx, sz)));
    float ee = smooth((float)(1.0 - 0.5 * (double)h), (float)(1.0 - 0.1 * (double)h), n[1]);
    float o = (float)(0.3 + 0.7 * (double)smooth(0.0f, 0.1f, n[0] + h * h));
    float s = (h * ee) * o;
    float m = smooth(0.1f, 0.9f, s);
    col[0] = sat(col[0] + m * (0.29f * 0.62f));
    col[1] = sat(col[1] + m * (0.29f * 0.65f));
    col[2] = sat(col[2] + m * (0.29f * 0.7f));
  }
}

/* Light setup of illuminate(), as the library computes it on the host. */
typedef struct {
  float lightpos[3], light_int[3], light_dist;
} light_setup;

static light_setup setup_light(const o_sdf_shade* s) {
  light_setup L;
  float lx = s->light_pos[0], ly = s->light_pos[1];
  L.lightpos[0] = lx;
  L.lightpos[1] = ly;
  L.lightpos[2] = lx;
  float r2 = lx * lx + ly * ly + lx * lx;
  L.light_dist = sqrtf(r2);
  float den = (float)(4.0 * O_PI * (double)r2);
  L.light_int[0] = (0.86f * s->light_intensity) / den;
  L.light_int[1] = (0.80f * s->light_intensity) / den;
  L.light_int[2] = (0.45f * s->light_intensity) / den;
  return L;
}

static void lighting(const uint32_t P[512], const o_sdf_field* F, const o_sdf_shade* S,
                     const light_setup* LS, const float p[3], const float n[3], float pc[3],
                     uint32_t* evals) {
  float ld[3];
  for (int k = 0; k < 3; ++k) ld[k] = (p[k] - LS->lightpos[k]) / LS->light_dist;
  float L[3] = {-ld[0], -ld[1], -ld[2]};
  norm3f(L);
  float prel = 1.0f;
  float t = S->shadow_tmin;
  for (uint32_t i = 0; i < S->shadow_max_steps && t < S->shadow_tmax; ++i) {
    float q[3] = {fmaf(t, L[0], p[0]), fmaf(t, L[1], p[1]), fmaf(t, L[2], p[2])};
    float dd = o_terrain_density(P, q, (int)F->octaves, F->scale, F->amp);
    ++*evals;
    if (prel < 1e-4f || dd <= 1e-5f) {
      prel = 0.0f;
      break;
    }
    prel = fminf(prel, (S->soft_shadow_k * dd) / t);
    t = fmaf(F->step_factor, dd, t);
  }
  float amb = sat((float)(0.5 + 0.5 * (double)n[1]));
  float soft = sat(prel);
  float dif = fmaxf(0.0f, dot3f(n, L));
  float bv[3] = {-ld[0], 0.0f, ld[2]};
  norm3f(bv);
  float bac = sat((float)(0.2 + 0.8 * (double)dot3f(bv, n)));
  for (int k = 0; k < 3; ++k) pc[k] = (soft * LS->light_int[k]) * dif;
  pc[0] = pc[0] + (amb * 0.40f) * 1.2f;
  pc[1] = pc[1] + (amb * 0.60f) * 1.2f;
  pc[2] = pc[2] + (amb * 1.00f) * 1.2f;
  pc[0] = pc[0] + bac * 0.40f;
  pc[1] = pc[1] + bac * 0.50f;
  pc[2] = pc[2] + bac * 0.60f;
}

static int ray_sphere(const float o[3], const float d[3], float radius, float* t0, float* t1) {
  float a = dot3f(d, d);
  float b = 2.0f * dot3f(d, o);
  float c = dot3f(o, o) - radius * radius;
  float discr = b * b - (4.0f * a) * c;
  if (discr < 0.0f) return 0;
  if (discr == 0.0f) {
    *t0 = *t1 = (-0.5f * b) / a;
  } else {
    float q = b > 0.0f ? -0.5f * (b + sqrtf(discr)) : -0.5f * (b - sqrtf(discr));
    *t0 = q / a;
    *t1 = c / q;
  }
  if (*t0 > *t1) {
    float x = *t0;
    *t0 = *t1;
    *t1 = x;
  }
  return 1;
}

static void sky(const o_sdf_shade* S, const float dir[3], float col[3]) {
  const float R = 6360e3f, Ra = 6420e3f, Hr = 79945.0f, Hm = 1200.0f;
  const float betaR[3] = {3.8e-6f, 13.5e-6f, 33.1e-6f};
  const float betaM = 21e-6f;
  const float orig[3] = {0.0f, R + 10000.0f, 300000.0f};
  float t0 = 0.0f, t1 = 0.0f;
  if (!ray_sphere(orig, dir, Ra, &t0, &t1) || t1 < 0.0f) {
    col[0] = col[1] = col[2] = 1.0f;
  } else {
    float tmin = 0.0f, tmax = K_INFINITY;
    if (t0 > tmin && t0 > 0.0f) tmin = t0;
    if (t1 < tmax) tmax = t1;
    float seg = (tmax - tmin) / 32.0f;
    float tc = tmin;
    float sumR[3] = {0, 0, 0}, sumM[3] = {0, 0, 0};
    float odR = 0.0f, odM = 0.0f;
    float mu = dot3f(dir, S->sun_dir);
    float phaseR = (float)((3.0 / (16.0 * O_PI)) * (double)(1.0f + mu * mu));
    const float g = 0.76f;
    float pb = (1.0f - g * g) * (1.0f + mu * mu);
    float pcm = (2.0f + g * g) * o_fm_pow(1.0f + g * g - (2.0f * g) * mu, 1.5f);
    float phaseM = (float)(((3.0 / (8.0 * O_PI)) * (double)pb) / (double)pcm);
    for (int i = 0; i < 32; ++i) {
      float s = tc + seg * 0.5f;
      float sp[3] = {orig[0] + s * dir[0], orig[1] + s * dir[1], orig[2] + s * dir[2]};
      float height = len3f(sp) - R;
      float hr = o_fm_exp(-height / Hr) * seg;
      float hm = o_fm_exp(-height / Hm) * seg;
      odR += hr;
      odM += hm;
      float tl0 = 0.0f, tl1 = 0.0f;
      ray_sphere(sp, S->sun_dir, Ra, &tl0, &tl1);
      float segl = tl1 / 8.0f, tcl = 0.0f;
      float odLR = 0.0f, odLM = 0.0f;
      int j;
      for (j = 0; j < 8; ++j) {
        float sl = tcl + segl * 0.5f;
        float spl[3] = {sp[0] + sl * S->sun_dir[0], sp[1] + sl * S->sun_dir[1],
                        sp[2] + sl * S->sun_dir[2]};
        float hl = len3f(spl) - R;
        if (hl < 0.0f) break;
        odLR += o_fm_exp(-hl / Hr) * segl;
        odLM += o_fm_exp(-hl / Hm) * segl;
        tcl += segl;
      }
      if (j == 8) {
        float aR = odR + odLR, aM = (betaM * 1.1f) * (odM + odLM);
        for (int k = 0; k < 3; ++k) {
          float att = o_fm_exp(-(betaR[k] * aR + aM));
          sumR[k] = sumR[k] + att * hr;
          sumM[k] = sumM[k] + att * hm;
        }
      }
      tc += seg;
    }
    float m100 = (100.0f * betaM) * phaseM;
    for (int k = 0; k < 3; ++k) col[k] = (((sumR[k] * betaR[k]) * phaseR + sumM[k]) + m100) * 20.0f;
  }
  for (int k = 0; k < 3; ++k)
    col[k] = col[k] < 1.413f ? o_fm_pow(col[k] * 0.38317f, 1.0f / 2.2f) : 1.0f - o_fm_exp(-col[k]);
}

static uint32_t rgba8(const float c[3]) {
  float r = sat(c[0]), g = sat(c[1]), b = sat(c[2]);
  return (255u << 24) | ((uint32_t)(b * 255.0f) << 16) | ((uint32_t)(g * 255.0f) << 8) |
         (uint32_t)(r * 255.0f);
}

uint32_t o_sdf_shade_pixel(const uint32_t P[512], const o_sdf_field* F, const o_sdf_shade* S,
                           const float o[3], const float d[3], const o_sdf_hit* hit, float u,
                           float v, uint32_t* evals) {
  light_setup LS = setup_light(S);
  float col[3];
  float dist = K_INFINITY;
  if (hit->status == 1) {
    float po[3] = {hit->pos[0] - o[0], hit->pos[1] - o[1], hit->pos[2] - o[2]};
    dist = len3f(po);
    paint(P, S, hit->pos, hit->normal, col);
    if (S->flags & 1u) {
      float pc[3];
      lighting(P, F, S, &LS, hit->pos, hit->normal, pc, evals);
      for (int k = 0; k < 3; ++k) col[k] = col[k] * pc[k];
    }
  } else {
    sky(S, d, col);
  }
  if (S->flags & 2u) {
    float dens = S->fog_density;
    float e1 = o_fm_exp(-o[1] * dens);
    float e2 = o_fm_exp(((-dist) * d[1]) * dens);
    float f = sat((float)((((double)((0.0375f / dens) * e1)) * (1.0 - (double)e2)) / (double)d[1]));
    col[0] = sat(col[0] + f * (0.65f * 0.4f));
    col[1] = sat(col[1] + f * (0.65f * 0.65f));
    col[2] = sat(col[2] + f * (0.65f * 1.0f));
  }
  if (S->flags & 4u)
    for (int k = 0; k < 3; ++k) col[k] = o_fm_pow(col[k], 1.0f / 2.2f);
  if (S->flags & 8u) {
    float k = 0.5f + 0.5f * o_fm_pow((((16.0f * u) * v) * (1.0f - u)) * (1.0f - v), S->vignetting_k);
    for (int c = 0; c < 3; ++c) col[c] = col[c] * k;
  }
  return rgba8(col);
}

/* The whole frame on a pixel sample: the exact march (o_sdf_trace) and the
 * shading of each pixel.  out_evals (may be NULL): shadow-ray field
 * evaluations per pixel. */
void o_batch_sdf_frame(const uint32_t P[512], const o_camera* cam, uint32_t w, uint32_t h,
                       const o_sdf_field* F, const o_sdf_shade* S, const uint32_t* pixels,
                       int64_t npix, uint32_t* out_rgba, uint32_t* out_evals, int threads) {
  o_camera_basis b;
  o_camera_setup(cam, &b);
  if (!pixels) npix = (int64_t)w * h;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < npix; ++i) {
    uint32_t p = pixels ? pixels[i] : (uint32_t)i;
    uint32_t x = p % w, y = p / w;
    float o[3], d[3];
    o_generate_ray(&b, w, h, x, y, o, d);
    o_sdf_hit hit;
    o_sdf_trace(P, o, d, (int)F->octaves, F->scale, F->amp, F->step_factor, F->eps, F->tmax,
                F->max_steps, &hit);
    uint32_t ev = 0;
    out_rgba[i] = o_sdf_shade_pixel(P, F, S, o, d, &hit, (float)x / (float)w,
                                    (float)y / (float)h, &ev);
    if (out_evals) out_evals[i] = ev;
  }
}

/* The elementary functions over arrays (fn 0: e^x, 1: ln x, 2: x^y). */
void o_batch_fmath(uint32_t fn, const float* x, const float* y, int64_t n, float* out) {
  for (int64_t i = 0; i < n; ++i)
    out[i] = fn == 0 ? o_fm_exp(x[i]) : (fn == 1 ? o_fm_log(x[i]) : o_fm_pow(x[i], y[i]));
}
