// Noise kernels (fBm batch evaluation, heightfield bake) and the exact-SDF
// sphere tracer.
//
// Replaces, in the reference ("RE/" = RayEngine/src/):
//   generate_noise kernel + host wrapper   RE/cuda-src/renderer.cu:106-126, :813-836
//     (block (2,2,2) bake of get_terrain_distance into a voxel grid)
//   terrainH/M fBm + get_terrain_distance  RE/cuda-src/sdf_functions.cuh:147-206, :477-503
//   single_ray_sphere_trace / terrain march RE/cuda-src/sphere_tracing.cuh:183-216,
//                                          RE/cuda-src/renderer.cu:215-235
//   compute_terrain_normal                 RE/cuda-src/sdf_functions.cuh:535-546
//
// The permutation table travels as a 512-byte kernel parameter and is
// expanded into shared memory by every block (one copy per lane, so
// lattice lookups with divergent indices never conflict on a bank).  The
// march is FP32-ALU bound; it runs as a per-lane state machine with lane
// refills so sky rays (few steps) and grazing rays (hundreds) keep the warps
// full.
#include <cuda_runtime.h>

#include <cstring>

#include "re_common.hpp"
#include "re_noise.cuh"

namespace re {

__global__ void __launch_bounds__(256) k_fbm(PermTable perm, const float* __restrict__ pts,
                                             uint32_t n, float* __restrict__ out,
                                             uint32_t octaves, float lac, float gain,
                                             float scale, float amplitude) {
  extern __shared__ uint32_t perm_smem[];
  load_perm(perm, perm_smem);
  Perm P = perm_view(perm_smem);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float x = __ldg(&pts[3 * (size_t)i]), y = __ldg(&pts[3 * (size_t)i + 1]),
          z = __ldg(&pts[3 * (size_t)i + 2]);
    out[i] = amplitude * fbm(P, scale * x, scale * y, scale * z, octaves, lac, gain);
  }
}

__global__ void __launch_bounds__(256) k_heightfield(PermTable perm, uint32_t cells, float lo,
                                                     float step, float* __restrict__ verts,
                                                     uint32_t octaves, float lac, float gain,
                                                     float scale, float amplitude) {
  extern __shared__ uint32_t perm_smem[];
  load_perm(perm, perm_smem);
  Perm P = perm_view(perm_smem);
  uint32_t nv = cells + 1;
  uint32_t total = nv * nv;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    uint32_t ix = i % nv, iz = i / nv;
    float x = lo + (float)ix * step;
    float z = lo + (float)iz * step;
    float y = amplitude * fbm(P, scale * x, 0.0f, scale * z, octaves, lac, gain);
    verts[3 * (size_t)i] = x;
    verts[3 * (size_t)i + 1] = y;
    verts[3 * (size_t)i + 2] = z;
  }
}

struct SdfDev {
  uint32_t octaves, max_steps;
  float scale, amp, step_factor, eps, tmax;
};

// Sphere tracing as a per-lane state machine with one field evaluation per
// loop trip: phase 0 marches (t += step_factor * d), phases 1..6 evaluate
// the central-difference taps of the normal at the hit.  Every trip runs the
// same density code on all live lanes (a single call site keeps the loop in
// the instruction cache), and when at least kSdfRefill lanes of a warp are
// idle the warp claims new pixels with one atomic.  Pixel i of the claim
// order is lane (i & 31) of 8x4 tile (i >> 5), so claims stay coherent.
constexpr uint32_t kSdfRefill = 4;

__global__ void __launch_bounds__(256) k_sdf(PermTable perm, SdfDev sp, CamDev cam, uint32_t w,
                                             uint32_t h, float4* __restrict__ out,
                                             uint32_t* __restrict__ cursor) {
  extern __shared__ uint32_t perm_smem[];
  load_perm(perm, perm_smem);
  Perm P = perm_view(perm_smem);
  uint32_t lane = threadIdx.x & 31u;
  uint32_t tiles_x = (w + 7) / 8;
  uint32_t total = tiles_x * ((h + 3) / 4) * 32u;
  bool live = false, exhausted = false;
  uint32_t pix = 0, steps = 0, phase = 0;
  V3 o = {0, 0, 0}, d = {0, 0, 1}, p = {0, 0, 0};
  float t = 0.f, delta = 0.f, nx = 0.f, ny = 0.f, nz = 0.f, plus = 0.f;
  for (;;) {
    uint32_t idle = __ballot_sync(0xFFFFFFFFu, !live);
    uint32_t nidle = __popc(idle);
    if (!exhausted && (nidle >= kSdfRefill || nidle == 32u)) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(cursor, nidle);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (base + nidle >= total) exhausted = true;
      if (!live) {
        uint32_t i = base + __popc(idle & ((1u << lane) - 1u));
        uint32_t tile = i >> 5, l = i & 31u;
        uint32_t x = (tile % tiles_x) * 8 + (l & 7u), y = (tile / tiles_x) * 4 + (l >> 3);
        if (i < total && x < w && y < h) {
          generate_ray(cam, w, h, x, y, o, d);
          pix = y * w + x;
          t = 0.f;
          steps = 0;
          phase = 0;
          live = true;
        }
      }
    }
    if (__ballot_sync(0xFFFFFFFFu, live) == 0u) {
      if (exhausted) break;
      continue;
    }
    if (!live) continue;
    V3 q;
    if (phase == 0) {
      q = v3(__fmaf_rn(t, d.x, o.x), __fmaf_rn(t, d.y, o.y), __fmaf_rn(t, d.z, o.z));
    } else {
      float sgn_delta = (phase & 1u) ? delta : -delta;
      q = p;
      if (phase <= 2) q.x = p.x + sgn_delta;
      else if (phase <= 4) q.y = p.y + sgn_delta;
      else q.z = p.z + sgn_delta;
    }
    float v = terrain_density(P, q, sp.octaves, sp.scale, sp.amp);
    uint32_t status = 3;  // 3 = keep going
    if (phase == 0) {
      ++steps;
      if (v < sp.eps) {
        p = q;
        delta = 0.002f * t;
        phase = 1;
      } else {
        t = __fmaf_rn(sp.step_factor, v, t);
        if (t > sp.tmax) status = 0;
        else if (steps >= sp.max_steps) status = 2;
      }
    } else {
      if (phase & 1u) {
        plus = v;
      } else {
        float diff = plus - v;
        if (phase == 2) nx = diff;
        else if (phase == 4) ny = diff;
        else nz = diff;
      }
      if (phase == 6) status = 1;
      else ++phase;
    }
    if (status != 3) {
      float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1;
      if (status == 1) {
        V3 n = normalize(v3(nx, ny, nz));
        r0 = make_float4(p.x, p.y, p.z, n.x);
        r1 = make_float4(n.y, n.z, __uint_as_float(steps), __uint_as_float(status));
      } else {
        r1 = make_float4(0.f, 0.f, __uint_as_float(steps), __uint_as_float(status));
      }
      out[2 * (size_t)pix] = r0;
      out[2 * (size_t)pix + 1] = r1;
      live = false;
    }
  }
}

namespace {
PermTable make_perm(uint32_t seed) {
  uint32_t full[512];
  perlin_permutation(seed, full);
  PermTable t;
  for (int i = 0; i < 512; ++i) t.p[i] = (uint8_t)full[i];
  return t;
}

int blocks_for(uint64_t n) {
  uint64_t b = (n + 255) / 256;
  uint64_t cap = (uint64_t)sm_count() * 8;
  return (int)(b < cap ? (b ? b : 1) : cap);
}

// Claim cursor of the SDF kernel, one per device.
uint32_t* sdf_counter() {
  static uint32_t* ptrs[64] = {nullptr};
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
  if (!ptrs[dev] && cudaMalloc(&ptrs[dev], 16) != cudaSuccess) return nullptr;
  return ptrs[dev];
}
}  // namespace

}  // namespace re

extern "C" {

RE_API re_status re_noise_fbm(const re_fbm_params* p, const float* d_pts, uint32_t n,
                              float* d_out, void* stream) {
  if (!p || !d_pts || !d_out) return re::fail(RE_ERR_INVALID_ARG, "re_noise_fbm: null argument");
  if (p->octaves > 32) return re::fail(RE_ERR_LIMIT, "re_noise_fbm: octaves > 32");
  if (n == 0) return RE_OK;
  re::PermTable t = re::make_perm(p->seed);
  RE_CUDA(cudaFuncSetAttribute(re::k_fbm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)re::kPermSmemBytes));
  re::k_fbm<<<re::blocks_for(n), 256, re::kPermSmemBytes, (cudaStream_t)stream>>>(
      t, d_pts, n, d_out, p->octaves, p->lacunarity, p->gain, p->scale, p->amplitude);
  RE_CHECK_LAUNCH("re_noise_fbm: launch");
  return RE_OK;
}

RE_API re_status re_heightfield(const re_fbm_params* p, uint32_t cells, float lo, float hi,
                                float* d_verts, void* stream) {
  if (!p || !d_verts || cells == 0 || !(hi > lo))
    return re::fail(RE_ERR_INVALID_ARG, "re_heightfield: bad arguments");
  if (cells > 16384) return re::fail(RE_ERR_LIMIT, "re_heightfield: cells > 16384");
  if (p->octaves > 32) return re::fail(RE_ERR_LIMIT, "re_heightfield: octaves > 32");
  re::PermTable t = re::make_perm(p->seed);
  float step = (hi - lo) / (float)cells;
  uint64_t total = (uint64_t)(cells + 1) * (cells + 1);
  RE_CUDA(cudaFuncSetAttribute(re::k_heightfield, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)re::kPermSmemBytes));
  re::k_heightfield<<<re::blocks_for(total), 256, re::kPermSmemBytes, (cudaStream_t)stream>>>(
      t, cells, lo, step, d_verts, p->octaves, p->lacunarity, p->gain, p->scale, p->amplitude);
  RE_CHECK_LAUNCH("re_heightfield: launch");
  return RE_OK;
}

RE_API re_status re_sdf_trace(const re_sdf_params* p, const re_camera* cam, uint32_t w,
                              uint32_t h, re_sdf_hit* d_out, void* stream) {
  if (!p || !cam || !d_out || w < 2 || h < 2)
    return re::fail(RE_ERR_INVALID_ARG, "re_sdf_trace: bad arguments");
  if ((uint64_t)w * h > (1ull << 31)) return re::fail(RE_ERR_LIMIT, "re_sdf_trace: image too large");
  if (p->octaves > 32) return re::fail(RE_ERR_LIMIT, "re_sdf_trace: octaves > 32");
  if (p->max_steps == 0 || p->max_steps > (1u << 20))
    return re::fail(RE_ERR_LIMIT, "re_sdf_trace: max_steps must be in [1, 2^20]");
  uint32_t* counter = re::sdf_counter();
  if (!counter) return re::fail(RE_ERR_CUDA, "re_sdf_trace: counter allocation failed");
  re::PermTable t = re::make_perm(p->seed);
  re::SdfDev sp;
  sp.octaves = p->octaves;
  sp.max_steps = p->max_steps;
  sp.scale = p->scale;
  sp.amp = p->amplitude;
  sp.step_factor = p->step_factor;
  sp.eps = p->eps;
  sp.tmax = p->tmax;
  re::CamBasis b;
  re::camera_basis(*cam, b);
  re::CamDev cd;
  cd.campos = {b.campos[0], b.campos[1], b.campos[2]};
  cd.middle = {b.middle[0], b.middle[1], b.middle[2]};
  cd.horizontal = {b.horizontal[0], b.horizontal[1], b.horizontal[2]};
  cd.vertical = {b.vertical[0], b.vertical[1], b.vertical[2]};
  cd.focal = b.focal;
  cudaStream_t st = (cudaStream_t)stream;
  RE_CUDA(cudaMemsetAsync(counter, 0, 4, st));
  RE_CUDA(cudaFuncSetAttribute(re::k_sdf, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)re::kPermSmemBytes));
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, re::k_sdf, 256, re::kPermSmemBytes) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  re::k_sdf<<<per_sm * re::sm_count(), 256, re::kPermSmemBytes, st>>>(
      t, sp, cd, w, h, reinterpret_cast<float4*>(d_out), counter);
  RE_CHECK_LAUNCH("re_sdf_trace: launch");
  return RE_OK;
}

}  // extern "C"
