/*
 * TEST INFRASTRUCTURE ONLY -- OpenMP batch drivers over the CPU oracle
 * (oracle.c), so tests and the CPU baseline can check or time whole images.
 * The parallel loops follow RRayTracer::trace's
 * `#pragma omp parallel for schedule(dynamic)` over pixels
 * (RayEngine/src/Engine/RayTracer.cpp:154).
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <string.h>

#include "oracle.h"

int o_max_threads(void) { return omp_get_max_threads(); }

/* pixels: list of pixel indices (y*w+x), or NULL for all w*h pixels. */
void o_batch_primary_bruteforce(const float* tris, int32_t n, const float bmin[3],
                                const float bmax[3], const o_camera* cam, uint32_t w,
                                uint32_t h, int mode, const uint32_t* pixels, int64_t npix,
                                o_hit* out, int threads) {
  o_camera_basis b;
  o_camera_setup(cam, &b);
  if (!pixels) npix = (int64_t)w * h;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < npix; ++i) {
    uint32_t p = pixels ? pixels[i] : (uint32_t)i;
    float o[3], d[3];
    o_generate_ray(&b, w, h, p % w, p / w, o, d);
    o_trace_bruteforce(tris, n, bmin, bmax, o, d, mode, &out[i]);
  }
}

void o_batch_primary_kd(const o_kdtree* kd, const o_camera* cam, uint32_t w, uint32_t h,
                        int mode, uint32_t max_visits, const uint32_t* pixels, int64_t npix,
                        o_hit* out, o_counts* counts, int threads) {
  o_camera_basis b;
  o_camera_setup(cam, &b);
  if (!pixels) npix = (int64_t)w * h;
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < npix; ++i) {
    uint32_t p = pixels ? pixels[i] : (uint32_t)i;
    float o[3], d[3];
    o_generate_ray(&b, w, h, p % w, p / w, o, d);
    o_trace_kd(kd, o, d, INFINITY, mode, 0, max_visits, &out[i], counts ? &counts[i] : NULL);
  }
}

/* rays: n x 8 floats {o.xyz, tmax, d.xyz, tag} */
void o_batch_rays_kd(const o_kdtree* kd, const float* rays, int64_t n, int mode, int anyhit,
                     uint32_t max_visits, o_hit* out, int threads) {
#pragma omp parallel for schedule(dynamic, 64) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < n; ++i) {
    const float* R = rays + 8 * i;
    o_trace_kd(kd, R, R + 4, R[3], mode, anyhit, max_visits, &out[i], NULL);
  }
}

/* Primary + shadow + 4 AO rays per pixel; mask bits as re_render_ao (bit 6:
 * a ray of the pixel stopped at the leaf-visit cap).  packed: the scene's
 * triangles in input order (12 floats each), used for the hit triangle's
 * geometric normal.  totals[0..7]: inner/leaf/tests/rays of the primary and
 * of the secondary pass; totals[8], totals[9]: primary and secondary rays
 * stopped at the cap. */
static inline void cross3c(const float a[3], const float b[3], float r[3]) {
  r[0] = fmaf(a[1], b[2], -(a[2] * b[1]));
  r[1] = fmaf(a[2], b[0], -(a[0] * b[2]));
  r[2] = fmaf(a[0], b[1], -(a[1] * b[0]));
}
static inline float dot3c(const float a[3], const float b[3]) {
  return fmaf(a[2], b[2], fmaf(a[1], b[1], a[0] * b[0]));
}

void o_batch_frame_ao(const o_kdtree* kd, const float* packed, const o_camera* cam, uint32_t w,
                      uint32_t h, const float light_dir[3], float ao_length, float bias,
                      uint32_t seed, uint32_t max_visits, const uint32_t* pixels, int64_t npix,
                      o_hit* out, uint32_t* mask, uint32_t* nsec, uint64_t* totals,
                      int threads) {
  o_camera_basis b;
  o_camera_setup(cam, &b);
  if (!pixels) npix = (int64_t)w * h;
  uint64_t total = 0;
  uint64_t pi = 0, pl = 0, pt = 0, si = 0, sl = 0, stt = 0, ptr = 0, str_ = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : total, pi, pl, pt, si, sl, stt, ptr, str_) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < npix; ++i) {
    uint32_t p = pixels ? pixels[i] : (uint32_t)i;
    float o[3], d[3];
    o_generate_ray(&b, w, h, p % w, p / w, o, d);
    o_hit hit;
    o_counts c;
    uint32_t leaf = 0;
    o_trace_kd_ex(kd, o, d, INFINITY, 0, 0, max_visits, 0, &hit, &c, &leaf);
    pi += c.inner_visits;
    pl += c.leaf_visits;
    pt += c.tri_tests;
    out[i] = hit;
    uint32_t m = 0;
    if (c.status == 1) {
      m |= 1u << 6;
      ptr++;
    }
    if (hit.id >= 0) {
      m |= 1u;
      const float* T = packed + 12 * (size_t)hit.id;
      float n[3];
      cross3c(T + 4, T + 8, n);
      float inv = 1.0f / sqrtf(dot3c(n, n));
      n[0] *= inv;
      n[1] *= inv;
      n[2] *= inv;
      if (dot3c(n, d) > 0.0f) {
        n[0] = -n[0];
        n[1] = -n[1];
        n[2] = -n[2];
      }
      float hp[3];
      for (int k = 0; k < 3; ++k) hp[k] = fmaf(hit.t, d[k], o[k]);
      float so[5][3], sd[5][3], st[5];
      o_secondary_rays(hp, n, seed, p, light_dir, bias, so, sd, st);
      st[1] = st[2] = st[3] = st[4] = ao_length;
      for (int j = 0; j < 5; ++j) {
        o_hit sh;
        o_counts sc;
        o_trace_kd_ex(kd, so[j], sd[j], st[j], 0, 1, max_visits, leaf, &sh, &sc, NULL);
        si += sc.inner_visits;
        sl += sc.leaf_visits;
        stt += sc.tri_tests;
        if (sh.id < 0) m |= 1u << (1 + j);
        if (sc.status == 1) {
          m |= 1u << 6;
          str_++;
        }
      }
      total += 5;
    }
    mask[i] = m;
  }
  if (nsec) *nsec = (uint32_t)total;
  if (totals) {
    totals[0] = pi; totals[1] = pl; totals[2] = pt; totals[3] = (uint64_t)npix;
    totals[4] = si; totals[5] = sl; totals[6] = stt; totals[7] = total;
    totals[8] = ptr; totals[9] = str_;
  }
}

/* n points (3 floats each) -> amplitude * fbm(scale * p) */
void o_batch_fbm(const uint32_t perm[512], const float* pts, int64_t n, int octaves,
                 float lacunarity, float gain, float scale, float amplitude, float* out,
                 int threads) {
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < n; ++i) {
    const float* p = pts + 3 * i;
    out[i] = amplitude * o_fbm(perm, scale * p[0], scale * p[1], scale * p[2], octaves,
                               lacunarity, gain);
  }
}

void o_batch_sdf(const uint32_t perm[512], const o_camera* cam, uint32_t w, uint32_t h,
                 int octaves, float scale, float amp, float step_factor, float eps, float tmax,
                 uint32_t max_steps, const uint32_t* pixels, int64_t npix, o_sdf_hit* out,
                 int threads) {
  o_camera_basis b;
  o_camera_setup(cam, &b);
  if (!pixels) npix = (int64_t)w * h;
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < npix; ++i) {
    uint32_t p = pixels ? pixels[i] : (uint32_t)i;
    float o[3], d[3];
    o_generate_ray(&b, w, h, p % w, p / w, o, d);
    o_sdf_trace(perm, o, d, octaves, scale, amp, step_factor, eps, tmax, max_steps, &out[i]);
  }
}

/* The reference as shipped over the AO frame: one leaf, so every ray (primary,
 * shadow, AO) is a brute-force MT loop over all triangles.  Occlusion of a
 * secondary ray = closest hit closer than its length.  Same mask bits. */
void o_batch_frame_ao_bruteforce(const float* packed, int32_t n, const float bmin[3],
                                 const float bmax[3], const o_camera* cam, uint32_t w, uint32_t h,
                                 const float light_dir[3], float ao_length, float bias,
                                 uint32_t seed, const uint32_t* pixels, int64_t npix, o_hit* out,
                                 uint32_t* mask, uint32_t* nsec, int threads) {
  o_camera_basis b;
  o_camera_setup(cam, &b);
  uint64_t total = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < npix; ++i) {
    uint32_t p = pixels[i];
    float o[3], d[3];
    o_generate_ray(&b, w, h, p % w, p / w, o, d);
    o_hit hit;
    o_trace_bruteforce(packed, n, bmin, bmax, o, d, 0, &hit);
    out[i] = hit;
    uint32_t m = 0;
    if (hit.id >= 0) {
      m = 1;
      const float* T = packed + 12 * (size_t)hit.id;
      float nn[3];
      cross3c(T + 4, T + 8, nn);
      float inv = 1.0f / sqrtf(dot3c(nn, nn));
      nn[0] *= inv; nn[1] *= inv; nn[2] *= inv;
      if (dot3c(nn, d) > 0.0f) { nn[0] = -nn[0]; nn[1] = -nn[1]; nn[2] = -nn[2]; }
      float hp[3];
      for (int k = 0; k < 3; ++k) hp[k] = fmaf(hit.t, d[k], o[k]);
      float so[5][3], sd[5][3], st[5];
      o_secondary_rays(hp, nn, seed, p, light_dir, bias, so, sd, st);
      st[1] = st[2] = st[3] = st[4] = ao_length;
      for (int j = 0; j < 5; ++j) {
        o_hit sh;
        o_trace_bruteforce(packed, n, bmin, bmax, so[j], sd[j], 0, &sh);
        if (!(sh.id >= 0 && sh.t < st[j])) m |= 1u << (1 + j);
      }
      total += 5;
    }
    mask[i] = m;
  }
  if (nsec) *nsec = (uint32_t)total;
}

double o_terrain_density_d(const uint32_t P[512], const double p[3], int octaves, double scale,
                           double amp);
int o_sdf_root_d(const uint32_t P[512], const float o[3], const float d[3], int octaves,
                 double scale, double amp, double factor, double tmax, int max_steps,
                 int refine, double pos[3], double* t_out);

/* FP64 arbiter over pixels: out[i] = {x, y, z, hit} of the surface point
 * (refine != 0: bisected root of the first crossing the march reaches). */
void o_batch_sdf_arbiter(const uint32_t perm[512], const o_camera* cam, uint32_t w, uint32_t h,
                       int octaves, double scale, double amp, double factor, double tmax,
                       int max_steps, int refine, const uint32_t* pixels, int64_t npix,
                       double* out, int threads) {
  o_camera_basis b;
  o_camera_setup(cam, &b);
#pragma omp parallel for schedule(dynamic, 8) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < npix; ++i) {
    uint32_t p = pixels[i];
    float o[3], d[3];
    o_generate_ray(&b, w, h, p % w, p / w, o, d);
    double pos[3] = {0, 0, 0}, t = 0;
    int hit = o_sdf_root_d(perm, o, d, octaves, scale, amp, factor, tmax, max_steps, refine, pos, &t);
    out[4 * i] = pos[0];
    out[4 * i + 1] = pos[1];
    out[4 * i + 2] = pos[2];
    out[4 * i + 3] = hit;
  }
}

/* FP64 terrain density at n points (3 doubles each). */
void o_batch_density_d(const uint32_t perm[512], const double* pts, int64_t n, int octaves,
                       double scale, double amp, double* out, int threads) {
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < n; ++i) out[i] = o_terrain_density_d(perm, pts + 3 * i, octaves, scale, amp);
}

/* Batched path tracing over `npix` global pixels of `nscenes` scenes
 * (offsets[s] = first global pixel of scene s). */
void o_batch_path(const o_path_scene* scenes, int nscenes, const uint64_t* offsets,
                  const uint32_t* gpix, int64_t npix, uint32_t depth, uint32_t seed,
                  float mesh_bias, float* radiance, o_hit* primary, uint32_t* nrays,
                  int threads) {
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < npix; ++i) {
    uint32_t g = gpix[i];
    int s = 0;
    while (s + 1 < nscenes && offsets[s + 1] <= g) ++s;
    uint32_t r = o_path_pixel(&scenes[s], g, (uint32_t)(g - offsets[s]), depth, seed, mesh_bias,
                              &radiance[i], primary ? &primary[i] : NULL);
    if (nrays) nrays[i] = r;
  }
}

/* Shaded frame over the given pixels (or all when pixels == NULL). */
void o_batch_frame(const float* tris, int32_t n, const float bmin[3], const float bmax[3],
                   const o_camera* cam, uint32_t w, uint32_t h, int mode, const float* light_pos,
                   const float* light_int, uint32_t num_lights, const float albedo[3],
                   const float zenith[3], const float horizon[3], const uint32_t* pixels,
                   int64_t npix, uint32_t* out, int threads) {
  o_camera_basis b;
  o_camera_setup(cam, &b);
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < npix; ++i) {
    uint32_t p = pixels ? pixels[i] : (uint32_t)i;
    out[i] = o_frame_pixel(tris, n, bmin, bmax, &b, w, h, p % w, p / w, mode, light_pos, light_int,
                           num_lights, albedo, zenith, horizon);
  }
}

void o_batch_voxel_sample(const o_voxel* g, uint32_t quality, const float* pts, int64_t n,
                          float* out, int threads) {
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < n; ++i) out[i] = o_voxel_sample(g, quality, pts + 3 * i);
}

void o_batch_voxel_trace(const o_voxel* g, uint32_t quality, float step_factor, float eps,
                         float tmax, uint32_t max_steps, const o_camera* cam, uint32_t w,
                         uint32_t h, const uint32_t* pixels, int64_t npix, o_sdf_hit* out,
                         int threads) {
  o_camera_basis b;
  o_camera_setup(cam, &b);
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < npix; ++i)
    o_voxel_trace_pixel(g, quality, step_factor, eps, tmax, max_steps, &b, w, h,
                        pixels ? pixels[i] : (uint32_t)i, &out[i]);
}

/* FP32 density at grid points origin + (i, j, k) * spacing (the bake). */
void o_batch_voxel_bake(const uint32_t perm[512], int octaves, float scale, float amp,
                        const int dim[3], const float spacing[3], const float origin[3],
                        float* out, int threads) {
  int64_t n = (int64_t)dim[0] * dim[1] * dim[2];
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < n; ++i) {
    int x = (int)(i % dim[0]), y = (int)((i / dim[0]) % dim[1]), z = (int)(i / ((int64_t)dim[0] * dim[1]));
    float p[3] = {fmaf((float)x, spacing[0], origin[0]), fmaf((float)y, spacing[1], origin[1]),
                  fmaf((float)z, spacing[2], origin[2])};
    out[2 * i] = o_terrain_density(perm, p, octaves, scale, amp);
    out[2 * i + 1] = 0.0f;
  }
}

void o_batch_instances(const float* const* tris, const int32_t* ntris, const float* bmin,
                       const float* bmax, const float* cs, const float* loc, int32_t n,
                       const o_camera* cam, uint32_t w, uint32_t h, int mode, o_hit* out,
                       int32_t* inst, int threads) {
  o_camera_basis b;
  o_camera_setup(cam, &b);
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < (int64_t)w * h; ++i) {
    float o[3], d[3];
    o_generate_ray(&b, w, h, (uint32_t)(i % w), (uint32_t)(i / w), o, d);
    o_trace_instances_pixel(tris, ntris, bmin, bmax, cs, loc, n, o, d, mode, &out[i], &inst[i]);
  }
}
