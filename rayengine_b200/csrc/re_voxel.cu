// Voxel-SDF path: bake a field into a grid, the .rsdf file format, and
// sphere tracing of the sampled grid at three quality levels.
//
// Replaces, in the reference (hadalhw17/RayEngine, "RE/" = RayEngine/src/):
//   generate_noise (bake)   RE/cuda-src/renderer.cu:106-126,813-836
//   .rsdf read / write      RE/World/Grid.cpp:23-64, renderer.cu:839-870
//                           (int dim[3], float spacing[3], then float2
//                           {distance, material} per voxel, x fastest)
//   get_distance            RE/cuda-src/sdf_functions.cuh:394-419 with
//     LOW    nearest voxel                       (tex3D point lookup)
//     MEDIUM trilinear between voxels            (interpolate, :231-262)
//     HIGH   tricubic B-spline, 64 voxels        (cubicTex3DSimple, :296-329)
//
// Grid coordinates: u = (p - origin) / spacing per axis; voxel (i, j, k)
// holds the field at origin + (i, j, k) * spacing.  Lookups outside the grid
// clamp to the edge voxels (the reference's texture uses a zero border,
// which reads as a surface along the grid boundary).  The reference's
// texture fetches filter in hardware (linear mode with 8-bit weights); here
// every lookup reads exact voxel values and blends in FP32 with the
// reference's formulas, so results are reproducible on the CPU.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "re_common.hpp"
#include "re_math.cuh"
#include "re_noise.cuh"

namespace re {
namespace voxel {

struct GridDev {
  const float2* __restrict__ v;
  int dim[3];
  float spacing[3], origin[3];
};

__device__ __forceinline__ float fetch(const GridDev& g, int x, int y, int z) {
  x = min(max(x, 0), g.dim[0] - 1);
  y = min(max(y, 0), g.dim[1] - 1);
  z = min(max(z, 0), g.dim[2] - 1);
  return __ldg(&g.v[(size_t)x + (size_t)g.dim[0] * ((size_t)y + (size_t)g.dim[1] * z)]).x;
}

__device__ __forceinline__ float bspline(float t) {
  t = fabsf(t);
  const float a = 2.0f - t;
  if (t < 1.0f) return 2.0f / 3.0f - 0.5f * t * t * a;
  if (t < 2.0f) return a * a * a / 6.0f;
  return 0.0f;
}

__device__ __forceinline__ float bilerp(float tx, float ty, float c00, float c10, float c01,
                                        float c11) {
  return (1.0f - tx) * (1.0f - ty) * c00 + tx * (1.0f - ty) * c10 + (1.0f - tx) * ty * c01 +
         tx * ty * c11;
}

__device__ __forceinline__ float sample(const GridDev& g, uint32_t quality, V3 p) {
  float u[3] = {(p.x - g.origin[0]) / g.spacing[0], (p.y - g.origin[1]) / g.spacing[1],
                (p.z - g.origin[2]) / g.spacing[2]};
  if (quality == RE_VOXEL_LOW)
    return fetch(g, (int)floorf(u[0]), (int)floorf(u[1]), (int)floorf(u[2]));
  if (quality == RE_VOXEL_MEDIUM) {
    float fx = floorf(u[0]), fy = floorf(u[1]), fz = floorf(u[2]);
    int x = (int)fx, y = (int)fy, z = (int)fz;
    float tx = u[0] - fx, ty = u[1] - fy, tz = u[2] - fz;
    float e = bilerp(tx, ty, fetch(g, x, y, z), fetch(g, x + 1, y, z), fetch(g, x, y + 1, z),
                     fetch(g, x + 1, y + 1, z));
    float f = bilerp(tx, ty, fetch(g, x, y, z + 1), fetch(g, x + 1, y, z + 1),
                     fetch(g, x, y + 1, z + 1), fetch(g, x + 1, y + 1, z + 1));
    return e * (1.0f - tz) + f * tz;
  }
  // HIGH: B-spline weights about the voxel below u - 0.5
  float cg[3] = {u[0] - 0.5f, u[1] - 0.5f, u[2] - 0.5f};
  float idx[3] = {floorf(cg[0]), floorf(cg[1]), floorf(cg[2])};
  float fr[3] = {cg[0] - idx[0], cg[1] - idx[1], cg[2] - idx[2]};
  int ix = (int)idx[0], iy = (int)idx[1], iz = (int)idx[2];
  float result = 0.0f;
  for (int z = -1; z <= 2; ++z) {
    float bz = bspline((float)z - fr[2]);
    for (int y = -1; y <= 2; ++y) {
      float byz = bspline((float)y - fr[1]) * bz;
      for (int x = -1; x <= 2; ++x) {
        float bxyz = bspline((float)x - fr[0]) * byz;
        result += bxyz * fetch(g, ix + x, iy + y, iz + z);
      }
    }
  }
  return result;
}

__global__ void k_bake(PermTable perm, uint32_t octaves, float scale, float amp, GridDev g,
                       float2* __restrict__ out) {
  extern __shared__ uint32_t perm_smem[];
  load_perm(perm, perm_smem);
  Perm P = perm_view(perm_smem);
  size_t n = (size_t)g.dim[0] * g.dim[1] * g.dim[2];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    uint32_t x = (uint32_t)(i % g.dim[0]), y = (uint32_t)((i / g.dim[0]) % g.dim[1]),
             z = (uint32_t)(i / ((size_t)g.dim[0] * g.dim[1]));
    V3 p = v3(__fmaf_rn((float)x, g.spacing[0], g.origin[0]), __fmaf_rn((float)y, g.spacing[1], g.origin[1]),
              __fmaf_rn((float)z, g.spacing[2], g.origin[2]));
    out[i] = make_float2(terrain_density(P, p, octaves, scale, amp), 0.0f);
  }
}

__global__ void k_sample(GridDev g, uint32_t quality, const float* __restrict__ pts, uint32_t n,
                         float* __restrict__ out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = sample(g, quality, v3(pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2]));
}

struct MarchDev {
  float step_factor, eps, tmax;
  uint32_t max_steps;
};

// Sphere tracing of the sampled grid inside its box (the box holds the
// voxel centres, origin .. origin + (dim - 1) spacing): the exact tracer's
// rule t += step_factor * d, hit when d < eps; normal by central
// differences with delta = half the smallest spacing.  Output as re_sdf_hit.
__global__ void __launch_bounds__(256) k_trace(GridDev g, uint32_t quality, MarchDev m, CamDev cam,
                                               uint32_t w, uint32_t h, float4* __restrict__ out) {
  uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= w * h) return;
  V3 o, d;
  generate_ray(cam, w, h, pix % w, pix / w, o, d);
  float o3[3] = {o.x, o.y, o.z}, d3[3] = {d.x, d.y, d.z};
  float t0 = 0.0f, t1 = m.tmax;
  for (int k = 0; k < 3; ++k) {
    float lo = g.origin[k], hi = __fmaf_rn((float)(g.dim[k] - 1), g.spacing[k], g.origin[k]);
    float inv = 1.0f / d3[k];
    float ta = (lo - o3[k]) * inv, tb = (hi - o3[k]) * inv;
    t0 = fmaxf(t0, fminf(ta, tb));
    t1 = fminf(t1, fmaxf(ta, tb));
  }
  uint32_t steps = 0, status = 0;
  V3 p = {0.f, 0.f, 0.f};
  if (t0 < t1) {
    float t = t0;
    for (;;) {
      p = v3(__fmaf_rn(t, d.x, o.x), __fmaf_rn(t, d.y, o.y), __fmaf_rn(t, d.z, o.z));
      float v = sample(g, quality, p);
      ++steps;
      if (v < m.eps) {
        status = 1;
        break;
      }
      t = __fmaf_rn(m.step_factor, v, t);
      if (t > t1) break;
      if (steps >= m.max_steps) {
        status = 2;
        break;
      }
    }
  }
  float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1;
  if (status == 1) {
    float delta = 0.5f * fminf(g.spacing[0], fminf(g.spacing[1], g.spacing[2]));
    float n3[3];
    for (int k = 0; k < 3; ++k) {
      V3 a = p, b = p;
      if (k == 0) { a.x = p.x + delta; b.x = p.x - delta; }
      else if (k == 1) { a.y = p.y + delta; b.y = p.y - delta; }
      else { a.z = p.z + delta; b.z = p.z - delta; }
      n3[k] = sample(g, quality, a) - sample(g, quality, b);
    }
    V3 n = normalize(v3(n3[0], n3[1], n3[2]));
    r0 = make_float4(p.x, p.y, p.z, n.x);
    r1 = make_float4(n.y, n.z, __uint_as_float(steps), __uint_as_float(status));
  } else {
    r1 = make_float4(0.f, 0.f, __uint_as_float(steps), __uint_as_float(status));
  }
  out[2 * (size_t)pix] = r0;
  out[2 * (size_t)pix + 1] = r1;
}

// Brush edit of every voxel (insert_sphere_to_texture, renderer.cu:31-92):
// q = voxel position - centre; SPHERE_ADD smooth union (sdf_smin, k),
// SPHERE_SUBTRACT max(v, -sphere), CUBE_ADD component-wise min of the
// {distance, material} pairs (as the reference's fminf on float2),
// CUBE_SUBTRACT max(v, -box); sphere = |q| - r, box as aabb_distance
// (sdf_functions.cuh:424-436).
__device__ __forceinline__ float len3(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }

__global__ void k_brush(GridDev g, uint32_t type, float cx, float cy, float cz, float ex, float ey,
                        float ez, float mat, float k, float2* __restrict__ v) {
  size_t n = (size_t)g.dim[0] * g.dim[1] * g.dim[2];
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
       i += (size_t)gridDim.x * blockDim.x) {
    uint32_t x = (uint32_t)(i % g.dim[0]), y = (uint32_t)((i / g.dim[0]) % g.dim[1]),
             z = (uint32_t)(i / ((size_t)g.dim[0] * g.dim[1]));
    float qx = __fmaf_rn((float)x, g.spacing[0], g.origin[0]) - cx;
    float qy = __fmaf_rn((float)y, g.spacing[1], g.origin[1]) - cy;
    float qz = __fmaf_rn((float)z, g.spacing[2], g.origin[2]) - cz;
    float2 a = v[i], r = a;
    if (type == RE_BRUSH_SPHERE_ADD || type == RE_BRUSH_SPHERE_SUBTRACT) {
      float sd = len3(qx, qy, qz) - ex;
      if (type == RE_BRUSH_SPHERE_ADD) {
        float h = fmaxf(k - fabsf(a.x - sd), 0.0f) / k;
        float2 m = a.x < sd ? a : make_float2(sd, mat);
        float c = h * h * k * 0.25f;
        r = make_float2(m.x - c, m.y);
      } else {
        r = a.x > -sd ? a : make_float2(-sd, mat);
      }
    } else {
      float dx = fabsf(qx) - ex, dy = fabsf(qy) - ey, dz = fabsf(qz) - ez;
      float bd = len3(fmaxf(dx, 0.0f), fmaxf(dy, 0.0f), fmaxf(dz, 0.0f)) +
                 fminf(fmaxf(dx, fmaxf(dy, dz)), 0.0f);
      if (type == RE_BRUSH_CUBE_ADD) r = make_float2(fminf(a.x, bd), fminf(a.y, mat));
      else r = a.x > -bd ? a : make_float2(-bd, mat);
    }
    v[i] = r;
  }
}

}  // namespace voxel
}  // namespace re

namespace re {
namespace {

re_status check_grid(const re_voxel_grid* g, const char* fn) {
  if (!g) return fail(RE_ERR_INVALID_ARG, "%s: null grid", fn);
  for (int k = 0; k < 3; ++k) {
    if (g->dim[k] < 2 || g->dim[k] > 4096) return fail(RE_ERR_INVALID_ARG, "%s: dim out of [2, 4096]", fn);
    if (!(g->spacing[k] > 0.f)) return fail(RE_ERR_INVALID_ARG, "%s: spacing must be > 0", fn);
  }
  if ((uint64_t)g->dim[0] * g->dim[1] * g->dim[2] > (1ull << 31))
    return fail(RE_ERR_LIMIT, "%s: more than 2^31 voxels", fn);
  return RE_OK;
}

voxel::GridDev grid_dev(const re_voxel_grid* g, const float* d_grid) {
  voxel::GridDev d;
  d.v = reinterpret_cast<const float2*>(d_grid);
  for (int k = 0; k < 3; ++k) {
    d.dim[k] = (int)g->dim[k];
    d.spacing[k] = g->spacing[k];
    d.origin[k] = g->origin[k];
  }
  return d;
}

CamDev cam_of_voxel(const re_camera& c) {
  CamBasis b;
  camera_basis(c, b);
  CamDev d;
  d.campos = {b.campos[0], b.campos[1], b.campos[2]};
  d.middle = {b.middle[0], b.middle[1], b.middle[2]};
  d.horizontal = {b.horizontal[0], b.horizontal[1], b.horizontal[2]};
  d.vertical = {b.vertical[0], b.vertical[1], b.vertical[2]};
  d.focal = b.focal;
  return d;
}

}  // namespace
}  // namespace re

extern "C" {

RE_API re_status re_voxel_bake(const re_sdf_params* field, const re_voxel_grid* g, float* d_grid,
                               void* stream) {
  re_status st = re::check_grid(g, "re_voxel_bake");
  if (st != RE_OK) return st;
  if (!field || !d_grid || field->octaves < 1 || field->octaves > 16)
    return re::fail(RE_ERR_INVALID_ARG, "re_voxel_bake: bad arguments");
  uint32_t full[512];
  re::perlin_permutation(field->seed, full);
  re::PermTable t;
  for (int i = 0; i < 512; ++i) t.p[i] = (uint8_t)full[i];
  RE_CUDA(cudaFuncSetAttribute(re::voxel::k_bake, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)re::kPermSmemBytes));
  re::voxel::k_bake<<<2 * re::sm_count(), 256, re::kPermSmemBytes, (cudaStream_t)stream>>>(
      t, field->octaves, field->scale, field->amplitude, re::grid_dev(g, d_grid),
      reinterpret_cast<float2*>(d_grid));
  RE_CHECK_LAUNCH("re_voxel_bake: launch");
  return RE_OK;
}

RE_API re_status re_voxel_sample(const float* d_grid, const re_voxel_grid* g, uint32_t quality,
                                 const float* d_pts, uint32_t n, float* d_out, void* stream) {
  re_status st = re::check_grid(g, "re_voxel_sample");
  if (st != RE_OK) return st;
  if (!d_grid || !d_pts || !d_out || quality > RE_VOXEL_HIGH)
    return re::fail(RE_ERR_INVALID_ARG, "re_voxel_sample: bad arguments");
  if (n == 0) return RE_OK;
  re::voxel::k_sample<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(re::grid_dev(g, d_grid),
                                                                          quality, d_pts, n, d_out);
  RE_CHECK_LAUNCH("re_voxel_sample: launch");
  return RE_OK;
}

RE_API re_status re_voxel_trace(const float* d_grid, const re_voxel_grid* g, uint32_t quality,
                                const re_sdf_params* march, const re_camera* cam, uint32_t w,
                                uint32_t h, re_sdf_hit* d_out, void* stream) {
  re_status st = re::check_grid(g, "re_voxel_trace");
  if (st != RE_OK) return st;
  if (!d_grid || !march || !cam || !d_out || quality > RE_VOXEL_HIGH || w < 2 || h < 2 ||
      !(march->step_factor > 0.f) || march->max_steps == 0)
    return re::fail(RE_ERR_INVALID_ARG, "re_voxel_trace: bad arguments");
  if ((uint64_t)w * h > (1ull << 30)) return re::fail(RE_ERR_LIMIT, "re_voxel_trace: image too large");
  re::voxel::MarchDev m{march->step_factor, march->eps, march->tmax, march->max_steps};
  uint32_t n = w * h;
  re::voxel::k_trace<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(
      re::grid_dev(g, d_grid), quality, m, re::cam_of_voxel(*cam), w, h,
      reinterpret_cast<float4*>(d_out));
  RE_CHECK_LAUNCH("re_voxel_trace: launch");
  return RE_OK;
}

RE_API re_status re_voxel_brush(float* d_grid, const re_voxel_grid* g, const re_voxel_brush_params* b,
                                void* stream) {
  re_status st = re::check_grid(g, "re_voxel_brush");
  if (st != RE_OK) return st;
  if (!d_grid || !b || b->type > RE_BRUSH_CUBE_SUBTRACT ||
      (b->type == RE_BRUSH_SPHERE_ADD && !(b->smooth > 0.f)))
    return re::fail(RE_ERR_INVALID_ARG, "re_voxel_brush: bad arguments");
  re::voxel::k_brush<<<4 * re::sm_count(), 256, 0, (cudaStream_t)stream>>>(
      re::grid_dev(g, d_grid), b->type, b->center[0], b->center[1], b->center[2], b->extent[0],
      b->extent[1], b->extent[2], b->material, b->smooth, reinterpret_cast<float2*>(d_grid));
  RE_CHECK_LAUNCH("re_voxel_brush: launch");
  return RE_OK;
}

// .rsdf: int32 dim[3], float spacing[3], then {distance, material} float
// pairs with x fastest (Grid.cpp:23-64; the reference's save_map writes
// the same order).  The origin is not stored (0 on load).
RE_API re_status re_voxel_save(const char* path, const re_voxel_grid* g, const float* host_grid) {
  re_status st = re::check_grid(g, "re_voxel_save");
  if (st != RE_OK) return st;
  if (!path || !host_grid) return re::fail(RE_ERR_INVALID_ARG, "re_voxel_save: bad arguments");
  FILE* f = std::fopen(path, "wb");
  if (!f) return re::fail(RE_ERR_INVALID_ARG, "re_voxel_save: cannot open %s", path);
  int32_t dim[3] = {(int32_t)g->dim[0], (int32_t)g->dim[1], (int32_t)g->dim[2]};
  size_t n = (size_t)dim[0] * dim[1] * dim[2];
  bool ok = std::fwrite(dim, 4, 3, f) == 3 && std::fwrite(g->spacing, 4, 3, f) == 3 &&
            std::fwrite(host_grid, 8, n, f) == n;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return re::fail(RE_ERR_INTERNAL, "re_voxel_save: write failed for %s", path);
  return RE_OK;
}

RE_API re_status re_voxel_load(const char* path, re_voxel_grid* g, float* host_grid,
                               uint64_t capacity_voxels) {
  if (!path || !g) return re::fail(RE_ERR_INVALID_ARG, "re_voxel_load: bad arguments");
  FILE* f = std::fopen(path, "rb");
  if (!f) return re::fail(RE_ERR_INVALID_ARG, "re_voxel_load: cannot open %s", path);
  int32_t dim[3];
  float sp[3];
  bool ok = std::fread(dim, 4, 3, f) == 3 && std::fread(sp, 4, 3, f) == 3;
  re_voxel_grid tmp;
  std::memset(&tmp, 0, sizeof(tmp));
  if (ok)
    for (int k = 0; k < 3; ++k) {
      tmp.dim[k] = dim[k] > 0 ? (uint32_t)dim[k] : 0u;
      tmp.spacing[k] = sp[k];
    }
  re_status st = ok ? re::check_grid(&tmp, "re_voxel_load")
                    : re::fail(RE_ERR_INVALID_ARG, "re_voxel_load: %s: short header", path);
  if (st != RE_OK) {
    std::fclose(f);
    return st;
  }
  *g = tmp;
  size_t n = (size_t)tmp.dim[0] * tmp.dim[1] * tmp.dim[2];
  if (host_grid) {
    if (capacity_voxels < n) {
      std::fclose(f);
      return re::fail(RE_ERR_LIMIT, "re_voxel_load: buffer holds %llu of %zu voxels",
                      (unsigned long long)capacity_voxels, n);
    }
    ok = std::fread(host_grid, 8, n, f) == n;
  }
  std::fclose(f);
  if (!ok) return re::fail(RE_ERR_INVALID_ARG, "re_voxel_load: %s: truncated", path);
  return RE_OK;
}

}  // extern "C"
