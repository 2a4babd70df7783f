/*
 * TEST INFRASTRUCTURE ONLY -- CPU oracle for the RayEngine ray-query path.
 * Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline /
 * reference legs load this (as the checker).  Compiled with
 * -ffp-contract=off: every fused multiply-add below is an explicit fmaf().
 *
 * Citations are to the reference (hadalhw17/RayEngine), paths relative to
 * its repository root; "RE/" = RayEngine/src/.
 */
#include "oracle.h"

#include <math.h>
#include <string.h>

#define K_EPSILON 1e-4f   /* RE/RayEngine/RayEngine.h:25 */
#define K_INFINITY 1e20f  /* RE/RayEngine/RayEngine.h:24 */

/* ---------------------------------------------------------------- vectors */
static inline float dot3(const float a[3], const float b[3]) {
  return fmaf(a[2], b[2], fmaf(a[1], b[1], a[0] * b[0]));
}
static inline void cross3(const float a[3], const float b[3], float r[3]) {
  r[0] = fmaf(a[1], b[2], -(a[2] * b[1]));
  r[1] = fmaf(a[2], b[0], -(a[0] * b[2]));
  r[2] = fmaf(a[0], b[1], -(a[1] * b[0]));
}
static inline void normalize3(float v[3]) {
  float inv = 1.0f / sqrtf(dot3(v, v));
  v[0] *= inv;
  v[1] *= inv;
  v[2] *= inv;
}

/* ----------------------------------------------------------------- camera */
/* RE/cuda-src/ray_functions.cuh:26-37: the per-frame part of generate_ray.
 * fov is the full angle in degrees; the reference evaluates
 * fov * 0.5 * (M_PI / 180) in double and calls tanf on the result. */
void o_camera_setup(const o_camera* cam, o_camera_basis* out) {
  float view[3] = {cam->view[0], cam->view[1], cam->view[2]};
  float down[3] = {cam->camdown[0], cam->camdown[1], cam->camdown[2]};
  float h[3], v[3];
  normalize3(view);
  normalize3(down);
  cross3(view, down, h);
  normalize3(h);
  cross3(h, view, v);
  normalize3(v);
  float th = tanf((float)(cam->fov[0] * 0.5 * (3.14159265358979323846 / 180.0)));
  float tv = tanf((float)(cam->fov[1] * 0.5 * (3.14159265358979323846 / 180.0)));
  for (int k = 0; k < 3; ++k) {
    out->campos[k] = cam->campos[k];
    out->middle[k] = cam->campos[k] + view[k];
    out->horizontal[k] = h[k] * th;
    out->vertical[k] = v[k] * tv;
  }
  out->focal = cam->focal;
}

/* RE/cuda-src/ray_functions.cuh:23-51, plus the renormalisation the
 * traversal applies (ray_functions.cuh:267). */
void o_generate_ray(const o_camera_basis* b, uint32_t w, uint32_t h,
                    uint32_t x, uint32_t y, float o[3], float d[3]) {
  float sx = (float)x / ((float)w - 1.0f);
  float sy = 1.0f - (float)y / ((float)h - 1.0f);
  float a = 2.0f * sx - 1.0f;
  float c = 2.0f * sy - 1.0f;
  for (int k = 0; k < 3; ++k) {
    float p1 = fmaf(b->vertical[k], c, fmaf(b->horizontal[k], a, b->middle[k]));
    float pip = fmaf(p1 - b->campos[k], b->focal, b->campos[k]);
    d[k] = pip - b->campos[k];
    o[k] = b->campos[k];
  }
  normalize3(d); /* apertureToImagePlane = normalize(...)      :47 */
  normalize3(d); /* ray_dir = normalize(rayInWorldSpace)       :51 */
  normalize3(d); /* new_dir = normalize(new_dir) in traversal :267 */
}

/* ---------------------------------------------------------------- ray/box */
/* RE/cuda-src/ray_functions.cuh:62-92 */
int o_ray_box(const float bmin[3], const float bmax[3], const float o[3],
              const float d[3], float* t_near, float* t_far) {
  float inv0 = 1.0f / d[0], inv1 = 1.0f / d[1], inv2 = 1.0f / d[2];
  float t1 = (bmin[0] - o[0]) * inv0, t2 = (bmax[0] - o[0]) * inv0;
  float t3 = (bmin[1] - o[1]) * inv1, t4 = (bmax[1] - o[1]) * inv1;
  float t5 = (bmin[2] - o[2]) * inv2, t6 = (bmax[2] - o[2]) * inv2;
  float tmin = fmaxf(fmaxf(fminf(t1, t2), fminf(t3, t4)), fminf(t5, t6));
  float tmax = fminf(fminf(fmaxf(t1, t2), fmaxf(t3, t4)), fmaxf(t5, t6));
  if (tmax < 0.0f) return 0;
  if (tmin > tmax) return 0;
  *t_near = tmin >= 0.0f ? tmin : 0.0f; /* fsel(t_near, t_near, 0) */
  *t_far = tmax;
  return 1;
}

/* ----------------------------------------------------------- ray/triangle */
/* Moller-Trumbore.  mode 0 = RKDTreeCPU triIntersect (KDTree.cpp:909-949),
 * mode 1 = gpu_ray_tri_intersect (ray_functions.cuh:174-223). */
int o_ray_tri(const float o[3], const float d[3], const float v0[3],
              const float e1[3], const float e2[3], int mode, float* t,
              float* u, float* v) {
  float h[3], s[3], q[3];
  cross3(d, e2, h);
  float a = dot3(e1, h);
  if (mode == 0) {
    if (a > -0.00001f && a < 0.00001f) return 0;
  } else {
    if (a < K_EPSILON) return 0;
  }
  float f = 1.0f / a;
  s[0] = o[0] - v0[0];
  s[1] = o[1] - v0[1];
  s[2] = o[2] - v0[2];
  float uu = f * dot3(s, h);
  if (uu < 0.0f || uu > 1.0f) return 0;
  cross3(s, e1, q);
  float vv = f * dot3(d, q);
  if (vv < 0.0f || uu + vv > 1.0f) return 0;
  float tt = f * dot3(e2, q);
  if (!(tt > (mode == 0 ? 0.00001f : K_EPSILON))) return 0;
  *t = tt;
  *u = uu;
  *v = vv;
  return 1;
}

void o_trace_bruteforce(const float* tris, int32_t n, const float bmin[3],
                        const float bmax[3], const float o[3], const float d[3],
                        int mode, o_hit* out) {
  out->id = -1;
  out->t = K_INFINITY;
  out->u = 0.0f;
  out->v = 0.0f;
  float t_entry, t_exit;
  if (!o_ray_box(bmin, bmax, o, d, &t_entry, &t_exit)) return;
  /* while (t_entry < t_exit && limit < 50): one iteration for a single leaf */
  if (!(t_entry < t_exit)) return;
  for (int32_t i = 0; i < n; ++i) {
    const float* T = tris + 12 * (size_t)i;
    float t, u, v;
    if (o_ray_tri(o, d, T, T + 4, T + 8, mode, &t, &u, &v) && t < t_exit) {
      t_exit = t;
      out->id = i;
      out->t = t;
      out->u = u;
      out->v = v;
    }
  }
}

/* ------------------------------------------------------- kd-tree traversal */
static inline uint32_t fbits(float f) {
  uint32_t u;
  memcpy(&u, &f, 4);
  return u;
}

/* start: leaf node to begin in when the origin lies in its region (secondary
 * rays start in the leaf of their primary hit), else 0 = root.  out_leaf:
 * node index of the leaf the best hit was found in. */
void o_trace_kd_ex(const o_kdtree* kd, const float o[3], const float d[3], float tmax, int mode,
                   int anyhit, uint32_t max_leaf_visits, uint32_t start, o_hit* out,
                   o_counts* cnt, uint32_t* out_leaf) {
  o_counts c = {0, 0, 0, 0};
  if (out_leaf) *out_leaf = 0;
  out->id = -1;
  out->t = K_INFINITY;
  out->u = 0.0f;
  out->v = 0.0f;
  float t_entry, t_root_exit;
  if (!o_ray_box(kd->bmin, kd->bmax, o, d, &t_entry, &t_root_exit)) {
    if (cnt) *cnt = c;
    return;
  }
  float inv[3] = {1.0f / d[0], 1.0f / d[1], 1.0f / d[2]};
  float best_t = fminf(t_root_exit, tmax);
  int32_t best_id = -1;
  float best_u = 0.0f, best_v = 0.0f;
  uint32_t node = 0, best_leaf = 0;
  uint32_t visits = 0;
  int done = 0;
  if (start != 0) {
    uint32_t meta = fbits(kd->nodes[2 * start + 1]);
    if ((meta & 3u) == 3u) {
      const float* L = kd->leaves + 16 * (size_t)(meta >> 2);
      if (o[0] >= L[0] && o[0] <= L[3] && o[1] >= L[1] && o[1] <= L[4] && o[2] >= L[2] &&
          o[2] <= L[5])
        node = start;
    }
  }
  while (!done && t_entry < best_t) {
    uint32_t meta = fbits(kd->nodes[2 * node + 1]);
    while ((meta & 3u) != 3u) {
      uint32_t k = meta & 3u;
      float split = kd->nodes[2 * node];
      int left;
      if (d[k] > 0.0f)
        left = t_entry < (split - o[k]) * inv[k];
      else if (d[k] < 0.0f)
        left = t_entry >= (split - o[k]) * inv[k];
      else
        left = o[k] < split;
      node = (meta >> 2) + (left ? 0u : 1u);
      meta = fbits(kd->nodes[2 * node + 1]);
      c.inner_visits++;
    }
    const float* L = kd->leaves + 16 * (size_t)(meta >> 2);
    c.leaf_visits++;
    uint32_t first = fbits(L[6]), count = fbits(L[7]);
    for (uint32_t i = first; i < first + count; ++i) {
      const float* T = kd->tris + 12 * (size_t)i;
      int32_t id = (int32_t)fbits(T[3]);
      float t, u, v;
      c.tri_tests++;
      if (o_ray_tri(o, d, T, T + 4, T + 8, mode, &t, &u, &v)) {
        if (t < best_t || (t == best_t && id < best_id && best_id >= 0)) {
          best_t = t;
          best_id = id;
          best_u = u;
          best_v = v;
          best_leaf = node;
          if (anyhit) {
            done = 1;
            break;
          }
        }
      }
    }
    if (done) break;
    float lo[3] = {L[0], L[1], L[2]}, hi[3] = {L[3], L[4], L[5]};
    float texit = INFINITY;
    int face = -1;
    for (int k = 0; k < 3; ++k) {
      float tk;
      int f;
      if (d[k] > 0.0f) {
        tk = (hi[k] - o[k]) * inv[k];
        f = 2 * k + 1;
      } else if (d[k] < 0.0f) {
        tk = (lo[k] - o[k]) * inv[k];
        f = 2 * k;
      } else {
        continue;
      }
      if (tk < texit) {
        texit = tk;
        face = f;
      }
    }
    if (face < 0) break;
    t_entry = fmaxf(t_entry, texit);
    if (!(t_entry < best_t)) break;
    int32_t rope = (int32_t)fbits(L[8 + face]);
    if (rope < 0) break;
    node = (uint32_t)rope;
    if (++visits >= max_leaf_visits) {
      c.status = 1;
      break;
    }
  }
  if (best_id >= 0) {
    out->id = best_id;
    out->t = best_t;
    out->u = best_u;
    out->v = best_v;
    if (out_leaf) *out_leaf = best_leaf;
  }
  if (cnt) *cnt = c;
}

void o_trace_kd(const o_kdtree* kd, const float o[3], const float d[3], float tmax, int mode,
                int anyhit, uint32_t max_leaf_visits, o_hit* out, o_counts* cnt) {
  o_trace_kd_ex(kd, o, d, tmax, mode, anyhit, max_leaf_visits, 0, out, cnt, NULL);
}

/* ------------------------------------------------------------ Perlin/fBm */
/* std::mt19937 (32-bit) -- RPerlinNoise seeds one and takes raw 32-bit draws
 * through uniform_int_distribution<unsigned> over the full range
 * (PerlinNoise.h:43-47).  The float draws of dice() advance a copy made by
 * std::bind, so the swap sequence starts from the freshly seeded state. */
typedef struct {
  uint32_t mt[624];
  int idx;
} o_mt32;

static void mt32_seed(o_mt32* g, uint32_t seed) {
  g->mt[0] = seed;
  for (int i = 1; i < 624; ++i)
    g->mt[i] = 1812433253u * (g->mt[i - 1] ^ (g->mt[i - 1] >> 30)) + (uint32_t)i;
  g->idx = 624;
}

static uint32_t mt32_next(o_mt32* g) {
  if (g->idx >= 624) {
    for (int i = 0; i < 624; ++i) {
      uint32_t y = (g->mt[i] & 0x80000000u) | (g->mt[(i + 1) % 624] & 0x7fffffffu);
      g->mt[i] = g->mt[(i + 397) % 624] ^ (y >> 1) ^ ((y & 1u) ? 0x9908b0dfu : 0u);
    }
    g->idx = 0;
  }
  uint32_t y = g->mt[g->idx++];
  y ^= y >> 11;
  y ^= (y << 7) & 0x9d2c5680u;
  y ^= (y << 15) & 0xefc60000u;
  y ^= y >> 18;
  return y;
}

/* PerlinNoise.h:16-52 */
void o_perlin_permutation(uint32_t seed, uint32_t perm[512]) {
  o_mt32 g;
  mt32_seed(&g, seed);
  for (uint32_t i = 0; i < 256; ++i) perm[i] = i;
  for (uint32_t i = 0; i < 256; ++i) {
    uint32_t j = mt32_next(&g) & 255u;
    uint32_t t = perm[i];
    perm[i] = perm[j];
    perm[j] = t;
  }
  for (uint32_t i = 0; i < 256; ++i) perm[256 + i] = perm[i];
}

/* sdf_functions.cuh:26-47 */
static inline float grad_dot(uint32_t h, float x, float y, float z) {
  switch (h & 15u) {
    case 0: return x + y;
    case 1: return -x + y;
    case 2: return x - y;
    case 3: return -x - y;
    case 4: return x + z;
    case 5: return -x + z;
    case 6: return x - z;
    case 7: return -x - z;
    case 8: return y + z;
    case 9: return -y + z;
    case 10: return y - z;
    case 11: return -y - z;
    case 12: return y + x;
    case 13: return -x + y;
    case 14: return -y + z;
    default: return -y - z;
  }
}

/* sdf_functions.cuh:57-60 */
static inline float quintic(float t) {
  float in = fmaf(t, 6.0f, -15.0f);
  in = fmaf(t, in, 10.0f);
  return ((t * t) * t) * in;
}

/* sdf_functions.cuh:84-135, value only.  The reference's texture hash
 * (sdf_functions.cuh:77-81, a linearly-filtered normalised-float read of a
 * 256x256 uchar array) is not reproducible; the lattice hash here is
 * P[P[P[x] + y] + z] over the same RPerlinNoise table. */
float o_perlin(const uint32_t P[512], float x, float y, float z) {
  float fx = floorf(x), fy = floorf(y), fz = floorf(z);
  int xi0 = ((int)fx) & 255, yi0 = ((int)fy) & 255, zi0 = ((int)fz) & 255;
  int xi1 = (xi0 + 1) & 255, yi1 = (yi0 + 1) & 255, zi1 = (zi0 + 1) & 255;
  float tx = x - fx, ty = y - fy, tz = z - fz;
  float u = quintic(tx), v = quintic(ty), w = quintic(tz);
  float x0 = tx, x1 = tx - 1.0f;
  float y0 = ty, y1 = ty - 1.0f;
  float z0 = tz, z1 = tz - 1.0f;
  uint32_t px0 = P[xi0], px1 = P[xi1];
  uint32_t p00 = P[px0 + yi0], p10 = P[px1 + yi0];
  uint32_t p01 = P[px0 + yi1], p11 = P[px1 + yi1];
  float a = grad_dot(P[p00 + zi0], x0, y0, z0);
  float b = grad_dot(P[p10 + zi0], x1, y0, z0);
  float c = grad_dot(P[p01 + zi0], x0, y1, z0);
  float d = grad_dot(P[p11 + zi0], x1, y1, z0);
  float e = grad_dot(P[p00 + zi1], x0, y0, z1);
  float f = grad_dot(P[p10 + zi1], x1, y0, z1);
  float g = grad_dot(P[p01 + zi1], x0, y1, z1);
  float h = grad_dot(P[p11 + zi1], x1, y1, z1);
  float k0 = a;
  float k1 = b - a;
  float k2 = c - a;
  float k3 = e - a;
  float k4 = ((a + d) - b) - c;
  float k5 = ((a + f) - b) - e;
  float k6 = ((a + g) - c) - e;
  float k7 = ((((((b + c) + e) + h) - a) - d) - f) - g;
  float r = fmaf(k1, u, k0);
  r = fmaf(k2, v, r);
  r = fmaf(k3, w, r);
  r = fmaf(k4, u * v, r);
  r = fmaf(k5, u * w, r);
  r = fmaf(k6, v * w, r);
  r = fmaf(k7, (u * v) * w, r);
  return r;
}

/* plain fBm: sum_i gain^i * noise(lacunarity^i * p) (the configs' form of
 * terrainH/M, sdf_functions.cuh:147-186, without damping or rotation) */
float o_fbm(const uint32_t P[512], float x, float y, float z, int octaves,
            float lacunarity, float gain) {
  float sum = 0.0f, amp = 1.0f;
  for (int i = 0; i < octaves; ++i) {
    sum = fmaf(amp, o_perlin(P, x, y, z), sum);
    x *= lacunarity;
    y *= lacunarity;
    z *= lacunarity;
    amp *= gain;
  }
  return sum;
}

float o_height(const uint32_t P[512], float x, float z, int octaves, float amp) {
  return amp * o_fbm(P, x, 0.0f, z, octaves, 2.0f, 0.5f);
}

float o_terrain_density(const uint32_t P[512], const float p[3], int octaves,
                        float scale, float amp) {
  float f = o_fbm(P, scale * p[0], scale * p[1], scale * p[2], octaves, 2.0f, 0.5f);
  return fmaf(-amp, f, p[1]);
}

/* --------------------------------------------------------- scene makers */
/* std::mt19937_64 */
typedef struct {
  uint64_t mt[312];
  int idx;
} o_mt64;

static void mt64_seed(o_mt64* g, uint64_t seed) {
  g->mt[0] = seed;
  for (int i = 1; i < 312; ++i)
    g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
  g->idx = 312;
}

static uint64_t mt64_next(o_mt64* g) {
  if (g->idx >= 312) {
    for (int i = 0; i < 312; ++i) {
      uint64_t y = (g->mt[i] & 0xFFFFFFFF80000000ULL) | (g->mt[(i + 1) % 312] & 0x7FFFFFFFULL);
      g->mt[i] = g->mt[(i + 156) % 312] ^ (y >> 1) ^ ((y & 1ULL) ? 0xB5026F5AA96619E9ULL : 0ULL);
    }
    g->idx = 0;
  }
  uint64_t y = g->mt[g->idx++];
  y ^= (y >> 29) & 0x5555555555555555ULL;
  y ^= (y << 17) & 0x71D67FFFEDA60000ULL;
  y ^= (y << 37) & 0xFFF7EEE000000000ULL;
  y ^= y >> 43;
  return y;
}

uint64_t o_mt64_next(uint64_t* state) {
  /* state layout: 312 words + index in state[312] (for tests only) */
  o_mt64 g;
  memcpy(g.mt, state, sizeof(g.mt));
  g.idx = (int)state[312];
  uint64_t r = mt64_next(&g);
  memcpy(state, g.mt, sizeof(g.mt));
  state[312] = (uint64_t)g.idx;
  return r;
}

static double u01(o_mt64* g) { return (double)(mt64_next(g) >> 11) * 0x1.0p-53; }

/* Triangle soup: centroid ~ U[-1,1]^3, each vertex = centroid + N(0,0.02)
 * per axis (Box-Muller in double), mt19937_64(seed). */
void o_gen_soup(uint64_t seed, int32_t n, float* verts) {
  o_mt64 g;
  mt64_seed(&g, seed);
  for (int32_t i = 0; i < n; ++i) {
    double c[3], nz[10];
    for (int k = 0; k < 3; ++k) c[k] = -1.0 + 2.0 * u01(&g);
    for (int p = 0; p < 5; ++p) {
      double u1 = 1.0 - u01(&g);
      double u2 = u01(&g);
      double r = sqrt(-2.0 * log(u1));
      nz[2 * p] = r * cos(6.283185307179586 * u2);
      nz[2 * p + 1] = r * sin(6.283185307179586 * u2);
    }
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k)
        verts[9 * (size_t)i + 3 * j + k] = (float)(c[k] + 0.02 * nz[3 * j + k]);
  }
}

void o_gen_heightfield(const uint32_t P[512], int32_t cells, float lo, float hi,
                       int octaves, float amp, float* verts, uint32_t* faces) {
  float step = (hi - lo) / (float)cells;
  int32_t nv = cells + 1;
  for (int32_t j = 0; j < nv; ++j) {
    for (int32_t i = 0; i < nv; ++i) {
      float x = lo + (float)i * step;
      float z = lo + (float)j * step;
      float* V = verts + 3 * ((size_t)j * nv + i);
      V[0] = x;
      V[1] = o_height(P, x, z, octaves, amp);
      V[2] = z;
    }
  }
  for (int32_t j = 0; j < cells; ++j) {
    for (int32_t i = 0; i < cells; ++i) {
      uint32_t a = (uint32_t)(j * nv + i), b = a + 1, c = a + 1 + (uint32_t)nv,
               dd = a + (uint32_t)nv;
      uint32_t* F = faces + 6 * ((size_t)j * cells + i);
      F[0] = a; F[1] = b; F[2] = c;
      F[3] = a; F[4] = c; F[5] = dd;
    }
  }
}

/* --------------------------------------------------------- sphere tracer */
/* single_ray_sphere_trace (sphere_tracing.cuh:183-216) in the configs' form:
 * t += factor * d, hit when d < eps, bounded by max_steps and tmax.  The
 * normal uses central differences with delta = 0.002 t as
 * compute_terrain_normal does (sdf_functions.cuh:535-546). */
void o_sdf_trace(const uint32_t P[512], const float o[3], const float d[3],
                 int octaves, float scale, float amp, float step_factor,
                 float eps, float tmax, uint32_t max_steps, o_sdf_hit* out) {
  float t = 0.0f;
  float p[3] = {o[0], o[1], o[2]};
  uint32_t status = 2, steps = 0;
  for (uint32_t s = 0; s < max_steps; ++s) {
    p[0] = fmaf(t, d[0], o[0]);
    p[1] = fmaf(t, d[1], o[1]);
    p[2] = fmaf(t, d[2], o[2]);
    float dist = o_terrain_density(P, p, octaves, scale, amp);
    steps = s + 1;
    if (dist < eps) {
      status = 1;
      break;
    }
    t = fmaf(step_factor, dist, t);
    if (t > tmax) {
      status = 0;
      break;
    }
  }
  memset(out, 0, sizeof(*out));
  out->steps = steps;
  out->status = status;
  out->t = t;
  if (status == 1) {
    float delta = 0.002f * t;
    float n[3];
    for (int k = 0; k < 3; ++k) {
      float pp[3] = {p[0], p[1], p[2]}, pm[3] = {p[0], p[1], p[2]};
      pp[k] = p[k] + delta;
      pm[k] = p[k] - delta;
      n[k] = o_terrain_density(P, pp, octaves, scale, amp) -
             o_terrain_density(P, pm, octaves, scale, amp);
    }
    normalize3(n);
    for (int k = 0; k < 3; ++k) {
      out->pos[k] = p[k];
      out->normal[k] = n[k];
    }
  }
}

/* ------------------------------------------------ sampling (AO / shadow) */
/* integer mixer (lowbias32 finaliser) over a combination of three words */
uint32_t o_hash_u32(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t h = a * 0x9E3779B1u ^ (b + 0x7F4A7C15u) * 0x85EBCA77u ^ (c + 0x165667B1u) * 0xC2B2AE3Du;
  h ^= h >> 16;
  h *= 0x7feb352du;
  h ^= h >> 15;
  h *= 0x846ca68bu;
  h ^= h >> 16;
  return h;
}

/* sin and cos of 2*pi*u for u in [0,1): quadrant split, then Taylor series of
 * sin (to x^11) and cos (to x^12) on [0, pi/2) in Horner form. */
void o_sincos_2pi(float u, float* s, float* c) {
  float x4 = u * 4.0f;
  float qf = floorf(x4);
  int q = ((int)qf) & 3;
  float a = (x4 - qf) * 1.57079637f;
  float a2 = a * a;
  float sp = fmaf(a2, -2.50521084e-08f, 2.75573192e-06f);
  sp = fmaf(a2, sp, -1.98412698e-04f);
  sp = fmaf(a2, sp, 8.33333333e-03f);
  sp = fmaf(a2, sp, -1.66666667e-01f);
  sp = fmaf(a2, sp, 1.0f);
  float sn = a * sp;
  float cp = fmaf(a2, 2.08767570e-09f, -2.75573192e-07f);
  cp = fmaf(a2, cp, 2.48015873e-05f);
  cp = fmaf(a2, cp, -1.38888889e-03f);
  cp = fmaf(a2, cp, 4.16666667e-02f);
  cp = fmaf(a2, cp, -0.5f);
  float cs = fmaf(a2, cp, 1.0f);
  switch (q) {
    case 0: *s = sn; *c = cs; break;
    case 1: *s = cs; *c = -sn; break;
    case 2: *s = -sn; *c = -cs; break;
    default: *s = -cs; *c = sn; break;
  }
}

/* One shadow ray towards light_dir (any hit, unbounded) and four
 * cosine-weighted hemisphere rays of length 1 around n, all starting at
 * hitp + n * bias (the reference's shadow bias, material_functions.cuh:103).
 * The tangent frame is createCoordinateSystem (cuda_helper_functions.h:197-204)
 * and the local-to-world mix follows renderer.cu:574-577. */
void o_secondary_rays(const float hitp[3], const float n[3], uint32_t seed,
                      uint32_t pixel, const float light_dir[3], float bias,
                      float o_out[5][3], float d_out[5][3], float tmax_out[5]) {
  float org[3];
  for (int k = 0; k < 3; ++k) org[k] = fmaf(n[k], bias, hitp[k]);
  for (int k = 0; k < 3; ++k) {
    o_out[0][k] = org[k];
    d_out[0][k] = light_dir[k];
  }
  tmax_out[0] = K_INFINITY;
  float nt[3], nb[3];
  if (fabsf(n[0]) > fabsf(n[1])) {
    float inv = 1.0f / sqrtf(fmaf(n[2], n[2], n[0] * n[0]));
    nt[0] = n[2] * inv; nt[1] = 0.0f; nt[2] = -n[0] * inv;
  } else {
    float inv = 1.0f / sqrtf(fmaf(n[2], n[2], n[1] * n[1]));
    nt[0] = 0.0f; nt[1] = -n[2] * inv; nt[2] = n[1] * inv;
  }
  cross3(n, nt, nb);
  for (uint32_t j = 0; j < 4; ++j) {
    uint32_t h1 = o_hash_u32(seed, pixel, 2 * j);
    uint32_t h2 = o_hash_u32(seed, pixel, 2 * j + 1);
    float u1 = (float)(h1 >> 8) * 0x1.0p-24f;
    float u2 = (float)(h2 >> 8) * 0x1.0p-24f;
    float r = sqrtf(u1);
    float sn, cs;
    o_sincos_2pi(u2, &sn, &cs);
    float lx = r * cs, ly = sqrtf(1.0f - u1), lz = r * sn;
    for (int k = 0; k < 3; ++k) {
      o_out[1 + j][k] = org[k];
      d_out[1 + j][k] = fmaf(lz, nt[k], fmaf(ly, n[k], lx * nb[k]));
    }
    tmax_out[1 + j] = 1.0f;
  }
}

/* ------------------------------------------------------- FP64 arbiter */
/* The same lattice noise in double precision (exact quintic and trilinear
 * polynomial), for the error of float hit positions. */
static double quintic_d(double t) { return t * t * t * (t * (t * 6.0 - 15.0) + 10.0); }

static double grad_dot_d(uint32_t h, double x, double y, double z) {
  switch (h & 15u) {
    case 0: return x + y;
    case 1: return -x + y;
    case 2: return x - y;
    case 3: return -x - y;
    case 4: return x + z;
    case 5: return -x + z;
    case 6: return x - z;
    case 7: return -x - z;
    case 8: return y + z;
    case 9: return -y + z;
    case 10: return y - z;
    case 11: return -y - z;
    case 12: return y + x;
    case 13: return -x + y;
    case 14: return -y + z;
    default: return -y - z;
  }
}

double o_perlin_d(const uint32_t P[512], double x, double y, double z) {
  double fx = floor(x), fy = floor(y), fz = floor(z);
  int xi0 = ((int)fx) & 255, yi0 = ((int)fy) & 255, zi0 = ((int)fz) & 255;
  int xi1 = (xi0 + 1) & 255, yi1 = (yi0 + 1) & 255, zi1 = (zi0 + 1) & 255;
  double tx = x - fx, ty = y - fy, tz = z - fz;
  double u = quintic_d(tx), v = quintic_d(ty), w = quintic_d(tz);
  uint32_t px0 = P[xi0], px1 = P[xi1];
  uint32_t p00 = P[px0 + yi0], p10 = P[px1 + yi0], p01 = P[px0 + yi1], p11 = P[px1 + yi1];
  double a = grad_dot_d(P[p00 + zi0], tx, ty, tz), b = grad_dot_d(P[p10 + zi0], tx - 1, ty, tz);
  double c = grad_dot_d(P[p01 + zi0], tx, ty - 1, tz), d = grad_dot_d(P[p11 + zi0], tx - 1, ty - 1, tz);
  double e = grad_dot_d(P[p00 + zi1], tx, ty, tz - 1), f = grad_dot_d(P[p10 + zi1], tx - 1, ty, tz - 1);
  double g = grad_dot_d(P[p01 + zi1], tx, ty - 1, tz - 1), h = grad_dot_d(P[p11 + zi1], tx - 1, ty - 1, tz - 1);
  return a + (b - a) * u + (c - a) * v + (e - a) * w + (a + d - b - c) * u * v +
         (a + f - b - e) * u * w + (a + g - c - e) * v * w +
         (b + c + e + h - a - d - f - g) * u * v * w;
}

double o_terrain_density_d(const uint32_t P[512], const double p[3], int octaves, double scale,
                           double amp) {
  double x = scale * p[0], y = scale * p[1], z = scale * p[2], s = 0.0, a = 1.0;
  for (int i = 0; i < octaves; ++i) {
    s += a * o_perlin_d(P, x, y, z);
    x *= 2.0;
    y *= 2.0;
    z *= 2.0;
    a *= 0.5;
  }
  return p[1] - amp * s;
}

/* March the ray (o, d promoted to double) with t += factor * d until the
 * density falls below 1e-10 (the first sample at or inside the surface), or
 * t > tmax.  On a hit the root of the density between the last outside
 * sample and that one is refined by bisection (`refine` != 0), so a march
 * step that overshoots into the terrain shows up as position error.
 * Returns 1 and the position on a hit. */
int o_sdf_root_d(const uint32_t P[512], const float o[3], const float d[3], int octaves,
                 double scale, double amp, double factor, double tmax, int max_steps,
                 int refine, double pos[3], double* t_out) {
  double t = 0.0, t_prev = 0.0;
  for (int s = 0; s < max_steps; ++s) {
    double p[3] = {o[0] + t * (double)d[0], o[1] + t * (double)d[1], o[2] + t * (double)d[2]};
    double dist = o_terrain_density_d(P, p, octaves, scale, amp);
    if (dist < 1e-10) {
      if (refine && s > 0 && dist < 0.0) {
        double lo = t_prev, hi = t;
        for (int it = 0; it < 80; ++it) {
          double mid = 0.5 * (lo + hi);
          double q[3] = {o[0] + mid * (double)d[0], o[1] + mid * (double)d[1],
                         o[2] + mid * (double)d[2]};
          if (o_terrain_density_d(P, q, octaves, scale, amp) < 0.0) hi = mid;
          else lo = mid;
        }
        t = hi;
        p[0] = o[0] + t * (double)d[0];
        p[1] = o[1] + t * (double)d[1];
        p[2] = o[2] + t * (double)d[2];
      }
      pos[0] = p[0];
      pos[1] = p[1];
      pos[2] = p[2];
      *t_out = t;
      return 1;
    }
    t_prev = t;
    t += factor * dist;
    if (t > tmax) return 0;
  }
  return 0;
}

/* ------------------------------------------------- batched path tracing */
/* One pixel's path of the batched wavefront renderer: closest hits by
 * brute force (two-sided, equal to the rope traversal's hits), the exact
 * SDF march for terrains, cosine-weighted Lambertian bounces. */
static void cosine_dir(const float n[3], uint32_t seed, uint32_t pixel, uint32_t j, float d[3]) {
  float nt[3], nb[3];
  if (fabsf(n[0]) > fabsf(n[1])) {
    float inv = 1.0f / sqrtf(fmaf(n[2], n[2], n[0] * n[0]));
    nt[0] = n[2] * inv; nt[1] = 0.0f; nt[2] = -n[0] * inv;
  } else {
    float inv = 1.0f / sqrtf(fmaf(n[2], n[2], n[1] * n[1]));
    nt[0] = 0.0f; nt[1] = -n[2] * inv; nt[2] = n[1] * inv;
  }
  cross3(n, nt, nb);
  uint32_t h1 = o_hash_u32(seed, pixel, 2 * j), h2 = o_hash_u32(seed, pixel, 2 * j + 1);
  float u1 = (float)(h1 >> 8) * 0x1.0p-24f;
  float u2 = (float)(h2 >> 8) * 0x1.0p-24f;
  float r = sqrtf(u1);
  float sn, cs;
  o_sincos_2pi(u2, &sn, &cs);
  float lx = r * cs, ly = sqrtf(1.0f - u1), lz = r * sn;
  for (int k = 0; k < 3; ++k) d[k] = fmaf(lz, nt[k], fmaf(ly, n[k], lx * nb[k]));
}

uint32_t o_path_pixel(const o_path_scene* s, uint32_t gpix, uint32_t local_pix, uint32_t depth,
                      uint32_t seed, float mesh_bias, float* radiance, o_hit* primary) {
  o_camera_basis cb;
  o_camera_setup(&s->cam, &cb);
  float o[3], d[3];
  o_generate_ray(&cb, s->w, s->h, local_pix % s->w, local_pix / s->w, o, d);
  for (uint32_t b = 0; b < depth; ++b) {
    int hit = 0;
    float n[3] = {0, 0, 1}, hp[3] = {0, 0, 0};
    o_hit ph = {-1, K_INFINITY, 0.f, 0.f};
    if (s->kind == 0) {
      o_hit h;
      o_trace_bruteforce(s->tris, s->ntris, s->bmin, s->bmax, o, d, 0, &h);
      if (h.id >= 0) {
        hit = 1;
        ph = h;
        const float* T = s->tris + 12 * (size_t)h.id;
        cross3(T + 4, T + 8, n);
        normalize3(n);
        if (dot3(n, d) > 0.0f) {
          n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2];
        }
        for (int k = 0; k < 3; ++k) hp[k] = fmaf(n[k], mesh_bias, fmaf(h.t, d[k], o[k]));
      }
    } else {
      float t = 0.0f, v = 0.0f, p[3];
      uint32_t steps = 0;
      for (;;) {
        for (int k = 0; k < 3; ++k) p[k] = fmaf(t, d[k], o[k]);
        v = o_terrain_density(s->perm, p, s->octaves, s->scale, s->amp);
        ++steps;
        if (v < s->eps) {
          hit = 1;
          break;
        }
        t = fmaf(s->step_factor, v, t);
        if (t > s->tmax || steps >= s->max_steps) break;
      }
      if (hit) {
        float delta = fmaxf(0.002f * t, 1e-3f), g[3];
        for (int k = 0; k < 3; ++k) {
          float q[3] = {p[0], p[1], p[2]};
          q[k] = p[k] + delta;
          float plus = o_terrain_density(s->perm, q, s->octaves, s->scale, s->amp);
          q[k] = p[k] - delta;
          g[k] = plus - o_terrain_density(s->perm, q, s->octaves, s->scale, s->amp);
        }
        float gl = sqrtf(fmaf(g[2], g[2], fmaf(g[1], g[1], g[0] * g[0])));
        n[0] = g[0]; n[1] = g[1]; n[2] = g[2];
        normalize3(n);
        float off = fmaxf(-v, 0.0f) / (gl / (2.0f * delta)) + 2e-3f;
        for (int k = 0; k < 3; ++k) hp[k] = fmaf(n[k], off, p[k]);
        ph.id = 0;
        ph.t = t;
      }
    }
    if (b == 0 && primary) *primary = ph;
    if (!hit) {
      float pw = 1.0f;
      for (uint32_t i = 0; i < b; ++i) pw *= s->albedo;
      *radiance = pw * (0.5f * (1.0f + d[1]));
      return b + 1;
    }
    if (b + 1 == depth) {
      *radiance = 0.0f;
      return b + 1;
    }
    float nd[3];
    cosine_dir(n, seed, gpix, b, nd);
    for (int k = 0; k < 3; ++k) {
      o[k] = hp[k];
      d[k] = nd[k];
    }
  }
  return depth;
}

/* ------------------------------------------------------- shaded frame */
/* One pixel of the shaded frame (Phong with shadow rays, sky gradient,
 * rgbaFloatToInt pack): brute-force closest hits (mode for the primary
 * ray, two-sided shadow rays). */
static uint32_t pack_rgba(const float c[3]) {
  float v[3];
  for (int k = 0; k < 3; ++k) v[k] = c[k] < 0.0f ? 0.0f : (c[k] > 1.0f ? 1.0f : c[k]);
  return (255u << 24) | ((uint32_t)(v[2] * 255.0f) << 16) | ((uint32_t)(v[1] * 255.0f) << 8) |
         (uint32_t)(v[0] * 255.0f);
}

uint32_t o_frame_pixel(const float* tris, int32_t n, const float bmin[3], const float bmax[3],
                       const o_camera_basis* cb, uint32_t w, uint32_t h, uint32_t x, uint32_t y,
                       int mode, const float* light_pos, const float* light_int,
                       uint32_t num_lights, const float albedo[3], const float zenith[3],
                       const float horizon[3]) {
  float o[3], d[3], col[3];
  o_generate_ray(cb, w, h, x, y, o, d);
  o_hit hit;
  o_trace_bruteforce(tris, n, bmin, bmax, o, d, mode, &hit);
  if (hit.id < 0) {
    float s = d[1] > 0.0f ? d[1] : 0.0f;
    for (int k = 0; k < 3; ++k) col[k] = fmaf(s, zenith[k] - horizon[k], horizon[k]);
    return pack_rgba(col);
  }
  const float* T = tris + 12 * (size_t)hit.id;
  float nn[3], p[3], org[3];
  cross3(T + 4, T + 8, nn);
  normalize3(nn);
  if (dot3(nn, d) > 0.0f) {
    nn[0] = -nn[0]; nn[1] = -nn[1]; nn[2] = -nn[2];
  }
  for (int k = 0; k < 3; ++k) {
    p[k] = fmaf(hit.t, d[k], o[k]);
    org[k] = fmaf(nn[k], 1e-4f, p[k]);
    col[k] = albedo[k];
  }
  for (uint32_t i = 0; i < num_lights; ++i) {
    const float* L = light_pos + 3 * i;
    float pl[3] = {p[0] - L[0], p[1] - L[1], p[2] - L[2]};
    float r2 = dot3(pl, pl);
    float dist = sqrtf(r2);
    float l[3] = {pl[0] / dist, pl[1] / dist, pl[2] / dist};
    float kk = light_int[i] / (4.0f * 3.14159265358979f * r2);
    float li[3] = {0.86f * kk, 0.80f * kk, 0.45f * kk};
    float toward[3] = {-l[0], -l[1], -l[2]};
    o_hit sh;
    o_trace_bruteforce(tris, n, bmin, bmax, org, toward, 0, &sh);
    if (sh.id >= 0 && sh.t < dist) continue;
    float nl = dot3(nn, toward);
    nl = nl > 0.0f ? nl : 0.0f;
    float dn = dot3(nn, l);
    float R[3];
    for (int k = 0; k < 3; ++k) R[k] = fmaf(-2.0f * dn, nn[k], l[k]);
    float rv = -dot3(R, d);
    rv = rv > 0.0f ? rv : 0.0f;
    float r2v = rv * rv, r4 = r2v * r2v, r8 = r4 * r4;
    float spec = r8 * r2v;
    float dfac = 0.8f * (0.18f * nl), sfac = 0.2f * spec;
    for (int k = 0; k < 3; ++k) col[k] = fmaf(li[k], sfac, fmaf(li[k], dfac, col[k]));
  }
  return pack_rgba(col);
}

/* ------------------------------------------------------------ voxel SDF */
/* Grid lookups and the voxel sphere tracer (LOW nearest, MEDIUM trilinear,
 * HIGH tricubic B-spline), edge-clamped. */
static float vox_fetch(const o_voxel* g, int x, int y, int z) {
  x = x < 0 ? 0 : (x > g->dim[0] - 1 ? g->dim[0] - 1 : x);
  y = y < 0 ? 0 : (y > g->dim[1] - 1 ? g->dim[1] - 1 : y);
  z = z < 0 ? 0 : (z > g->dim[2] - 1 ? g->dim[2] - 1 : z);
  return g->v[2 * ((size_t)x + (size_t)g->dim[0] * ((size_t)y + (size_t)g->dim[1] * z))];
}

static float vox_bspline(float t) {
  t = fabsf(t);
  const float a = 2.0f - t;
  if (t < 1.0f) return 2.0f / 3.0f - 0.5f * t * t * a;
  if (t < 2.0f) return a * a * a / 6.0f;
  return 0.0f;
}

static float vox_bilerp(float tx, float ty, float c00, float c10, float c01, float c11) {
  return (1.0f - tx) * (1.0f - ty) * c00 + tx * (1.0f - ty) * c10 + (1.0f - tx) * ty * c01 +
         tx * ty * c11;
}

float o_voxel_sample(const o_voxel* g, uint32_t quality, const float p[3]) {
  float u[3];
  for (int k = 0; k < 3; ++k) u[k] = (p[k] - g->origin[k]) / g->spacing[k];
  if (quality == 0) return vox_fetch(g, (int)floorf(u[0]), (int)floorf(u[1]), (int)floorf(u[2]));
  if (quality == 1) {
    float fx = floorf(u[0]), fy = floorf(u[1]), fz = floorf(u[2]);
    int x = (int)fx, y = (int)fy, z = (int)fz;
    float tx = u[0] - fx, ty = u[1] - fy, tz = u[2] - fz;
    float e = vox_bilerp(tx, ty, vox_fetch(g, x, y, z), vox_fetch(g, x + 1, y, z),
                         vox_fetch(g, x, y + 1, z), vox_fetch(g, x + 1, y + 1, z));
    float f = vox_bilerp(tx, ty, vox_fetch(g, x, y, z + 1), vox_fetch(g, x + 1, y, z + 1),
                         vox_fetch(g, x, y + 1, z + 1), vox_fetch(g, x + 1, y + 1, z + 1));
    return e * (1.0f - tz) + f * tz;
  }
  float cg[3] = {u[0] - 0.5f, u[1] - 0.5f, u[2] - 0.5f};
  float idx[3] = {floorf(cg[0]), floorf(cg[1]), floorf(cg[2])};
  float fr[3] = {cg[0] - idx[0], cg[1] - idx[1], cg[2] - idx[2]};
  int ix = (int)idx[0], iy = (int)idx[1], iz = (int)idx[2];
  float result = 0.0f;
  for (int z = -1; z <= 2; ++z) {
    float bz = vox_bspline((float)z - fr[2]);
    for (int y = -1; y <= 2; ++y) {
      float byz = vox_bspline((float)y - fr[1]) * bz;
      for (int x = -1; x <= 2; ++x) {
        float bxyz = vox_bspline((float)x - fr[0]) * byz;
        result += bxyz * vox_fetch(g, ix + x, iy + y, iz + z);
      }
    }
  }
  return result;
}

void o_voxel_trace_pixel(const o_voxel* g, uint32_t quality, float step_factor, float eps,
                         float tmax, uint32_t max_steps, const o_camera_basis* cb, uint32_t w,
                         uint32_t h, uint32_t pix, o_sdf_hit* out) {
  float o[3], d[3];
  o_generate_ray(cb, w, h, pix % w, pix / w, o, d);
  float t0 = 0.0f, t1 = tmax;
  for (int k = 0; k < 3; ++k) {
    float lo = g->origin[k], hi = fmaf((float)(g->dim[k] - 1), g->spacing[k], g->origin[k]);
    float inv = 1.0f / d[k];
    float ta = (lo - o[k]) * inv, tb = (hi - o[k]) * inv;
    float mn = fminf(ta, tb), mx = fmaxf(ta, tb);
    t0 = fmaxf(t0, mn);
    t1 = fminf(t1, mx);
  }
  uint32_t steps = 0, status = 0;
  float p[3] = {0, 0, 0};
  if (t0 < t1) {
    float t = t0;
    for (;;) {
      for (int k = 0; k < 3; ++k) p[k] = fmaf(t, d[k], o[k]);
      float v = o_voxel_sample(g, quality, p);
      ++steps;
      if (v < eps) {
        status = 1;
        break;
      }
      t = fmaf(step_factor, v, t);
      if (t > t1) break;
      if (steps >= max_steps) {
        status = 2;
        break;
      }
    }
  }
  memset(out, 0, sizeof(*out));
  out->steps = steps;
  out->status = status;
  if (status == 1) {
    float s01 = g->spacing[1] < g->spacing[2] ? g->spacing[1] : g->spacing[2];
    float delta = 0.5f * (g->spacing[0] < s01 ? g->spacing[0] : s01);
    float n[3];
    for (int k = 0; k < 3; ++k) {
      float a[3] = {p[0], p[1], p[2]}, b[3] = {p[0], p[1], p[2]};
      a[k] = p[k] + delta;
      b[k] = p[k] - delta;
      n[k] = o_voxel_sample(g, quality, a) - o_voxel_sample(g, quality, b);
    }
    normalize3(n);
    for (int k = 0; k < 3; ++k) {
      out->pos[k] = p[k];
      out->normal[k] = n[k];
    }
  }
}

/* ------------------------------------------------------------ instances */
/* Closest hit over instances (object-space ray d' = normalize(Ry d),
 * o' = Ry o + location), brute force per instance; c, s = cos / sin of
 * each yaw as the library computes them. */
void o_trace_instances_pixel(const float* const* tris, const int32_t* ntris, const float* bmin,
                             const float* bmax, const float* cs, const float* loc, int32_t n,
                             const float o[3], const float d[3], int mode, o_hit* out,
                             int32_t* inst) {
  out->id = -1;
  out->t = K_INFINITY;
  out->u = out->v = 0.0f;
  *inst = -1;
  float best = INFINITY;
  for (int32_t k = 0; k < n; ++k) {
    float c = cs[2 * k], s = cs[2 * k + 1];
    float nd[3] = {d[0] * c + d[2] * s, d[1], -d[0] * s + d[2] * c};
    normalize3(nd);
    float no[3] = {o[0] * c + o[2] * s + loc[3 * k], o[1] + loc[3 * k + 1],
                   -o[0] * s + o[2] * c + loc[3 * k + 2]};
    o_hit h;
    o_trace_bruteforce(tris[k], ntris[k], bmin + 3 * k, bmax + 3 * k, no, nd, mode, &h);
    if (h.id >= 0 && h.t < best) {
      best = h.t;
      *out = h;
      *inst = k;
    }
  }
}

/* ---------------------------------------------------------- voxel brush */
static float len3f(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }

void o_voxel_brush(float* v, const int dim[3], const float spacing[3], const float origin[3],
                   uint32_t type, const float c[3], const float e[3], float mat, float k) {
  int64_t n = (int64_t)dim[0] * dim[1] * dim[2];
  for (int64_t i = 0; i < n; ++i) {
    int x = (int)(i % dim[0]), y = (int)((i / dim[0]) % dim[1]), z = (int)(i / ((int64_t)dim[0] * dim[1]));
    float qx = fmaf((float)x, spacing[0], origin[0]) - c[0];
    float qy = fmaf((float)y, spacing[1], origin[1]) - c[1];
    float qz = fmaf((float)z, spacing[2], origin[2]) - c[2];
    float ax = v[2 * i], ay = v[2 * i + 1], rx = ax, ry = ay;
    if (type <= 1) {
      float sd = len3f(qx, qy, qz) - e[0];
      if (type == 0) {
        float h = fmaxf(k - fabsf(ax - sd), 0.0f) / k;
        float mx = ax < sd ? ax : sd, my = ax < sd ? ay : mat;
        float cc = h * h * k * 0.25f;
        rx = mx - cc;
        ry = my;
      } else if (!(ax > -sd)) {
        rx = -sd;
        ry = mat;
      }
    } else {
      float dx = fabsf(qx) - e[0], dy = fabsf(qy) - e[1], dz = fabsf(qz) - e[2];
      float bd = len3f(fmaxf(dx, 0.0f), fmaxf(dy, 0.0f), fmaxf(dz, 0.0f)) +
                 fminf(fmaxf(dx, fmaxf(dy, dz)), 0.0f);
      if (type == 2) {
        rx = fminf(ax, bd);
        ry = fminf(ay, mat);
      } else if (!(ax > -bd)) {
        rx = -bd;
        ry = mat;
      }
    }
    v[2 * i] = rx;
    v[2 * i + 1] = ry;
  }
}
