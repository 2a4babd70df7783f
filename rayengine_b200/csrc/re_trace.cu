// Rope kd-tree scenes on the device and the traversal kernels.
//
// Replaces, in the reference (hadalhw17/RayEngine, "RE/" = RayEngine/src/):
//   copy_memory            RE/cuda-src/cuda_memory_functions.cuh:58-211
//   stackless_kdtree_traversal, gpu_ray_box_intersect, gpu_ray_tri_intersect,
//   is_point_to_the_left_of_split, get_neighboring_node_index
//                          RE/cuda-src/ray_functions.cuh:62-92,174-360,
//                          RE/cuda-src/kd_tree_functions.cuh:10-62
//   trace_primary_rays     RE/cuda-src/renderer.cu:390-410
//   trace_shadow / shade   RE/cuda-src/ray_functions.cuh:366-374,
//                          RE/cuda-src/material_functions.cuh:99-119
//   hemisphere sampling    RE/cuda-src/renderer.cu:537-613,
//                          RE/cuda-src/cuda_helper_functions.h:197-216
//
// Kernel design (sm_100a):
//   * persistent warps: each warp takes 8x4 pixel tiles (or 32 queued rays)
//     from a global counter until the frame is done, so long and short rays
//     are balanced across the 148 SMs;
//   * the breadth-first top of the node array is staged in shared memory
//     once per resident block;
//   * nodes are 8 bytes, leaves 64 bytes, triangle references 48 bytes, all
//     read with 8/16-byte vector loads through the read-only path;
//   * secondary rays are appended to a queue with one warp-aggregated atomic
//     per warp (ballot + popc).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>

#include "kd_build.hpp"
#include "re_common.hpp"
#include "re_kd.cuh"
#include "re_scene.hpp"
#include "re_math.cuh"

namespace re {

// --------------------------------------------------------------- kernels
// Lane-refill driver shared by the ray kernels: each lane runs its ray one
// leaf at a time (trav_step) and, as soon as at least refill_min lanes of the
// warp are idle, the warp claims that many consecutive work indices with one
// atomic, so lanes need not wait for the slowest ray of the warp and the
// frame has no warp-sized tail.  gen(i, o, d, tmax) -> false for an index
// without a ray; done(i, s, c) gets the finished walk (c: the ray's own
// counters when COUNT).
template <int MODE, bool ANYHIT, bool COUNT, class Gen, class Done>
__device__ __forceinline__ void refill_walk(const KdDev& kd, const uint2* snodes, uint32_t n,
                                            uint32_t refill_min, uint32_t* counter, Gen gen,
                                            Done done) {
  uint32_t lane = threadIdx.x & 31u;
  Trav s;
  s.live = false;
  Counters c = {0, 0, 0, 0};
  uint32_t cur = 0;
  bool exhausted = false;
  for (;;) {
    uint32_t idle = __ballot_sync(0xFFFFFFFFu, !s.live);
    uint32_t nidle = __popc(idle);
    if (!exhausted && (nidle >= refill_min || nidle == 32u)) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(counter, nidle);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (base + nidle >= n) exhausted = true;
      if (!s.live) {
        uint32_t i = base + __popc(idle & ((1u << lane) - 1u));
        V3 o, d;
        float tmax;
        if (i < n && gen(i, o, d, tmax)) {
          cur = i;
          if (COUNT) c = {0, 0, 0, 0};
          trav_init(s, kd, o, d, tmax, 0u);
          if (!s.live) done(cur, s, c);
        }
      }
    }
    if (__ballot_sync(0xFFFFFFFFu, s.live) == 0u) {
      if (exhausted) break;
      continue;
    }
    if (s.live) {
      trav_step<MODE, ANYHIT, COUNT>(s, kd, snodes, c);
      if (!s.live) done(cur, s, c);
    }
  }
}

// Launch bounds measured on B200: the primary and caller-ray kernels run 6
// blocks of 256 threads per SM (40 registers, a few dozen bytes of spills):
// the 2^20-triangle soup's primary pass is 3 % faster than at 5 blocks (48
// registers) and 9 % faster than at 4; the AO frame's kernels keep 5 blocks
// (at 6 its secondary pass is 2.6 % slower).
//
// Primary rays, persistent warps over 8x4 pixel tiles, each lane running its
// ray to the end (ray_refill_min 32: no per-leaf bookkeeping; fastest when
// rays of a tile take similar work).
template <int MODE, bool COUNT>
__global__ void __launch_bounds__(256, 6) k_primary_tiles(KdDev kd, CamDev cam, uint32_t w,
                                                       uint32_t h, re_hit* __restrict__ out,
                                                       uint4* __restrict__ counts,
                                                       uint32_t* __restrict__ tile_counter,
                                                       uint32_t) {
  extern __shared__ uint2 snodes[];
  stage_nodes(kd, snodes);
  uint32_t lane = threadIdx.x & 31u;
  uint32_t tiles_x = (w + 7) / 8, tiles = tiles_x * ((h + 3) / 4);
  for (;;) {
    uint32_t tile = warp_fetch(tile_counter);
    if (tile >= tiles) break;
    uint32_t x = (tile % tiles_x) * 8 + (lane & 7u);
    uint32_t y = (tile / tiles_x) * 4 + (lane >> 3);
    if (x >= w || y >= h) continue;
    V3 o, d;
    generate_ray(cam, w, h, x, y, o, d);
    HitState hs;
    Counters c = {0, 0, 0, 0};
    traverse<MODE, false, COUNT>(kd, snodes, o, d, __int_as_float(0x7f800000), 0u, hs, c);
    size_t pix = (size_t)y * w + x;
    if (COUNT)
      counts[pix] = make_uint4(c.inner, c.leaf, c.tests, c.status);
    else
      store_hit(out, pix, hs);
  }
}

// Primary rays with G lanes per ray (ray_lanes 2, 4 or 8): persistent warps
// over tiles of 32 / G pixels, 4 wide; the lanes of a ray split each leaf's
// triangle tests (trav_step with G).  For frames whose pass time is set by
// the longest walks rather than by throughput (a 512x512 frame of a 2^20-
// triangle soup takes as long as a 64x64 one), the G-fold shorter test
// chain per leaf shortens the critical path.
template <int MODE, uint32_t G>
__global__ void __launch_bounds__(256, 6) k_primary_lanes(KdDev kd, CamDev cam, uint32_t w,
                                                       uint32_t h, re_hit* __restrict__ out,
                                                       uint4* __restrict__,
                                                       uint32_t* __restrict__ tile_counter,
                                                       uint32_t) {
  constexpr uint32_t kRows = 32u / G / 4u;  // tile height; 4 pixels wide
  extern __shared__ uint2 snodes[];
  stage_nodes(kd, snodes);
  const uint32_t lane = threadIdx.x & 31u, r = lane / G;
  const uint32_t tiles_x = (w + 3) / 4, tiles = tiles_x * ((h + kRows - 1) / kRows);
  for (;;) {
    uint32_t tile = warp_fetch(tile_counter);
    if (tile >= tiles) break;
    uint32_t x = (tile % tiles_x) * 4 + (r & 3u);
    uint32_t y = (tile / tiles_x) * kRows + (r >> 2);
    if (x >= w || y >= h) continue;  // the whole group skips
    V3 o, d;
    generate_ray(cam, w, h, x, y, o, d);
    Trav s;
    Counters c = {0, 0, 0, 0};
    trav_init(s, kd, o, d, __int_as_float(0x7f800000), 0u);
    while (s.live) trav_step<MODE, false, false, G>(s, kd, snodes, c);
    HitState hs;
    trav_result(s, hs);
    if ((lane & (G - 1u)) == 0u) store_hit(out, (size_t)y * w + x, hs);
  }
}

// Primary rays, persistent warps over 8x4 pixel tiles, the warp testing the
// triangles of all its lanes' leaves together (ray_lanes 32,
// trav_step_warp): lanes whose rays have finished help the others, so the
// longest walks of frames too small to fill the GPU get a shorter chain of
// triangle tests.
template <int MODE>
__global__ void __launch_bounds__(256, 4) k_primary_warp(KdDev kd, CamDev cam, uint32_t w,
                                                      uint32_t h, re_hit* __restrict__ out,
                                                      uint4* __restrict__,
                                                      uint32_t* __restrict__ tile_counter,
                                                      uint32_t) {
  extern __shared__ uint2 snodes[];
  __shared__ unsigned long long wkey[8][32];
  __shared__ float4 wrec[8][32];
  stage_nodes(kd, snodes);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  const uint32_t tiles_x = (w + 7) / 8, tiles = tiles_x * ((h + 3) / 4);
  for (;;) {
    uint32_t tile = warp_fetch(tile_counter);
    if (tile >= tiles) break;
    uint32_t x = (tile % tiles_x) * 8 + (lane & 7u);
    uint32_t y = (tile / tiles_x) * 4 + (lane >> 3);
    const bool valid = x < w && y < h;
    Trav s;
    s.live = false;
    if (valid) {
      V3 o, d;
      generate_ray(cam, w, h, x, y, o, d);
      trav_init(s, kd, o, d, __int_as_float(0x7f800000), 0u);
    }
    while (__any_sync(0xFFFFFFFFu, s.live)) trav_step_warp<MODE>(s, kd, snodes, wkey[warp], wrec[warp]);
    if (valid) {
      HitState hs;
      trav_result(s, hs);
      store_hit(out, (size_t)y * w + x, hs);
    }
  }
}

// Primary rays with lane refill (ray_refill_min < 32).  Work index i is lane
// i % 32 of 8x4 pixel tile i / 32, so a warp's claims stay in one screen
// region.
template <int MODE, bool COUNT>
__global__ void __launch_bounds__(256, 6) k_primary(KdDev kd, CamDev cam, uint32_t w, uint32_t h,
                                                 re_hit* __restrict__ out,
                                                 uint4* __restrict__ counts,
                                                 uint32_t* __restrict__ tile_counter,
                                                 uint32_t refill_min) {
  extern __shared__ uint2 snodes[];
  stage_nodes(kd, snodes);
  uint32_t tiles_x = (w + 7) / 8, tiles = tiles_x * ((h + 3) / 4);
  auto gen = [&](uint32_t i, V3& o, V3& d, float& tmax) {
    uint32_t tile = i >> 5, l = i & 31u;
    uint32_t x = (tile % tiles_x) * 8 + (l & 7u);
    uint32_t y = (tile / tiles_x) * 4 + (l >> 3);
    if (x >= w || y >= h) return false;
    generate_ray(cam, w, h, x, y, o, d);
    tmax = __int_as_float(0x7f800000);
    return true;
  };
  auto done = [&](uint32_t i, const Trav& s, const Counters& c) {
    uint32_t tile = i >> 5, l = i & 31u;
    uint32_t x = (tile % tiles_x) * 8 + (l & 7u);
    uint32_t y = (tile / tiles_x) * 4 + (l >> 3);
    size_t pix = (size_t)y * w + x;
    if (COUNT) {
      counts[pix] = make_uint4(c.inner, c.leaf, c.tests, c.status);
    } else {
      HitState hs;
      trav_result(s, hs);
      store_hit(out, pix, hs);
    }
  };
  refill_walk<MODE, false, COUNT>(kd, snodes, tiles * 32u, refill_min, tile_counter, gen, done);
}

// Caller rays (re_ray), persistent warps over 32-ray chunks, each lane
// running its ray to the end (ray_refill_min 32).
template <int MODE, bool ANYHIT>
__global__ void __launch_bounds__(256, 6) k_rays_chunks(KdDev kd, const float4* __restrict__ rays,
                                                     uint32_t n, re_hit* __restrict__ out,
                                                     uint32_t* __restrict__ counter, uint32_t) {
  extern __shared__ uint2 snodes[];
  stage_nodes(kd, snodes);
  uint32_t lane = threadIdx.x & 31u;
  for (;;) {
    uint32_t chunk = warp_fetch(counter);
    uint32_t i = chunk * 32 + lane;
    if (chunk * 32 >= n) break;
    if (i >= n) continue;
    float4 R0 = __ldg(&rays[2 * (size_t)i]), R1 = __ldg(&rays[2 * (size_t)i + 1]);
    V3 o = {R0.x, R0.y, R0.z}, d = {R1.x, R1.y, R1.z};
    HitState hs;
    Counters c = {0, 0, 0, 0};
    traverse<MODE, ANYHIT, false>(kd, snodes, o, d, R0.w, 0u, hs, c);
    store_hit(out, i, hs);
  }
}

// Caller rays (re_ray), lane refill over ray indices (ray_refill_min < 32).
template <int MODE, bool ANYHIT>
__global__ void __launch_bounds__(256, 6) k_rays(KdDev kd, const float4* __restrict__ rays,
                                              uint32_t n, re_hit* __restrict__ out,
                                              uint32_t* __restrict__ counter,
                                              uint32_t refill_min) {
  extern __shared__ uint2 snodes[];
  stage_nodes(kd, snodes);
  auto gen = [&](uint32_t i, V3& o, V3& d, float& tmax) {
    float4 R0 = __ldg(&rays[2 * (size_t)i]), R1 = __ldg(&rays[2 * (size_t)i + 1]);
    o = {R0.x, R0.y, R0.z};
    d = {R1.x, R1.y, R1.z};
    tmax = R0.w;
    return true;
  };
  auto done = [&](uint32_t i, const Trav& s, const Counters&) {
    HitState hs;
    trav_result(s, hs);
    store_hit(out, i, hs);
  };
  refill_walk<MODE, ANYHIT, false>(kd, snodes, n, refill_min, counter, gen, done);
}

// Pixel mask bit of the AO frame: one of the pixel's rays (primary, shadow
// or AO) stopped at the leaf-visit cap.  Bits 0..5: hit, light visible, AO
// rays 1..4 unoccluded.
constexpr uint32_t kMaskTruncated = 1u << 6;

// Primary + secondary-ray generation for the AO frame.
struct AoDev {
  V3 light;
  float ao_length, bias;
  uint32_t seed;
};

// Secondary-ray queue and its tuning.  The r-th hit's shadow ray (kind 0)
// and AO rays j = 0..3 (kinds 1..4) are stored, by `mode`:
//   0 pixel-major   5r, 5r + 1 + j          a pixel's five rays together
//                                          (one start leaf, cache reuse)
//   1 kind-major    r, (1 + j) cap + r      a warp gets rays of one kind
//                                          from neighbouring pixels
//   2 shadow-first  r, cap + 4r + j         the shadow rays (one direction)
//                                          side by side, then each pixel's
//                                          four AO rays together
// and traced in record order.  refill_min: idle lanes a warp waits for
// before claiming new rays (32 = whole warps only).
struct AoQueue {
  float4* q;
  uint32_t mode, cap, refill_min;
};

__device__ __forceinline__ size_t shadow_record(const AoQueue& aq, uint32_t r) {
  return aq.mode == 0u ? 5 * (size_t)r : (size_t)r;
}
__device__ __forceinline__ size_t ao_record(const AoQueue& aq, uint32_t r, uint32_t j) {
  return aq.mode == 0u   ? 5 * (size_t)r + 1 + j
         : aq.mode == 1u ? (size_t)(1 + j) * aq.cap + r
                         : (size_t)aq.cap + 4 * (size_t)r + j;
}

// Warp-sum of per-thread work counters, one 64-bit atomic per warp and field.
__device__ __forceinline__ void flush_counts(const Counters& c, uint32_t rays,
                                             unsigned long long* totals) {
  uint32_t v[4] = {c.inner, c.leaf, c.tests, rays};
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    uint32_t x = v[f];
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xFFFFFFFFu, x, off);
    if ((threadIdx.x & 31u) == 0) atomicAdd(&totals[f], (unsigned long long)x);
  }
}

// Primary rays of the AO frame: closest hit, pixel mask bit 0, and the five
// secondary rays of every hit appended to the queue.
//
// Records go to the AoQueue layout; one warp-aggregated atomic per warp
// (ballot + popc) assigns hit ranks.  counters: [0] tile cursor, [1] hits,
// [2] secondary cursor, [3] secondary rays.  COUNT: also sum the traversal
// work into totals[0..3].
template <bool COUNT>
__global__ void __launch_bounds__(256, 5) k_ao_primary(KdDev kd, CamDev cam, AoDev ao, uint32_t w,
                                                    uint32_t h, re_hit* __restrict__ out,
                                                    uint32_t* __restrict__ mask,
                                                    AoQueue aq, uint32_t* __restrict__ counters,
                                                    unsigned long long* __restrict__ totals) {
  extern __shared__ uint2 snodes[];
  stage_nodes(kd, snodes);
  uint32_t lane = threadIdx.x & 31u;
  uint32_t tiles_x = (w + 7) / 8, tiles = tiles_x * ((h + 3) / 4);
  Counters c = {0, 0, 0, 0};
  uint32_t rays = 0;
  for (;;) {
    uint32_t tile = warp_fetch(&counters[0]);
    if (tile >= tiles) break;
    uint32_t x = (tile % tiles_x) * 8 + (lane & 7u);
    uint32_t y = (tile / tiles_x) * 4 + (lane >> 3);
    bool valid = x < w && y < h;
    HitState hs;
    hs.id = -1;
    V3 o = {0, 0, 0}, d = {0, 0, 1};
    if (valid) {
      generate_ray(cam, w, h, x, y, o, d);
      bool cut = traverse<0, false, COUNT>(kd, snodes, o, d, __int_as_float(0x7f800000), 0u,
                                           hs, c);
      ++rays;
      size_t pix = (size_t)y * w + x;
      if (!COUNT) {
        store_hit(out, pix, hs);
        mask[pix] = (hs.id >= 0 ? 1u : 0u) | (cut ? kMaskTruncated : 0u);
      }
    }
    bool hit = valid && hs.id >= 0;
    uint32_t ballot = __ballot_sync(0xFFFFFFFFu, hit);
    if (!ballot) continue;
    uint32_t base = 0;
    if (lane == 0) {
      base = atomicAdd(&counters[1], (uint32_t)__popc(ballot));
      atomicAdd(&counters[3], 5u * __popc(ballot));
    }
    base = __shfl_sync(0xFFFFFFFFu, base, 0);
    if (!hit) continue;
    uint32_t rank = base + __popc(ballot & ((1u << lane) - 1u));
    // geometric normal of the hit triangle, facing the incoming ray
    const float4* T = kd.tris + 3 * (size_t)hs.ref;
    float4 T1 = __ldg(T + 1), T2 = __ldg(T + 2);
    V3 n = normalize(cross(v3(T1.x, T1.y, T1.z), v3(T2.x, T2.y, T2.z)));
    if (dot(n, d) > 0.0f) n = v3(-n.x, -n.y, -n.z);
    V3 p = {__fmaf_rn(hs.t, d.x, o.x), __fmaf_rn(hs.t, d.y, o.y), __fmaf_rn(hs.t, d.z, o.z)};
    V3 org = {__fmaf_rn(n.x, ao.bias, p.x), __fmaf_rn(n.y, ao.bias, p.y),
              __fmaf_rn(n.z, ao.bias, p.z)};
    uint32_t pix = y * w + x;
    // record: {origin, start leaf node} {direction, pixel*8 + mask bit}; the
    // shadow ray (bit 1) is unbounded, AO rays (bits 2..5) have ao_length.
    // The start leaf is checked here, once for the hit's five rays (0: the
    // origin left the leaf, start at the root); the secondary pass trusts it.
    float start = __uint_as_float(origin_in_leaf(kd, org, hs.leaf_node) ? hs.leaf_node : 0u);
    float4* queue = aq.q;
    size_t q0 = shadow_record(aq, rank);
    queue[2 * q0] = make_float4(org.x, org.y, org.z, start);
    queue[2 * q0 + 1] = make_float4(ao.light.x, ao.light.y, ao.light.z,
                                    __uint_as_float(pix * 8u + 1u));
    // createCoordinateSystem (cuda_helper_functions.h:197-204)
    V3 nt;
    if (fabsf(n.x) > fabsf(n.y)) {
      float iv = 1.0f / sqrtf(__fmaf_rn(n.z, n.z, n.x * n.x));
      nt = v3(n.z * iv, 0.0f, -n.x * iv);
    } else {
      float iv = 1.0f / sqrtf(__fmaf_rn(n.z, n.z, n.y * n.y));
      nt = v3(0.0f, -n.z * iv, n.y * iv);
    }
    V3 nb = cross(n, nt);
#pragma unroll
    for (uint32_t j = 0; j < 4; ++j) {
      uint32_t h1 = hash_u32(ao.seed, pix, 2 * j), h2 = hash_u32(ao.seed, pix, 2 * j + 1);
      float u1 = (float)(h1 >> 8) * 5.9604644775390625e-08f;
      float u2 = (float)(h2 >> 8) * 5.9604644775390625e-08f;
      float r = sqrtf(u1);
      float sn, cs;
      sincos_2pi(u2, sn, cs);
      float lx = r * cs, ly = sqrtf(1.0f - u1), lz = r * sn;
      V3 dir = {__fmaf_rn(lz, nt.x, __fmaf_rn(ly, n.x, lx * nb.x)),
                __fmaf_rn(lz, nt.y, __fmaf_rn(ly, n.y, lx * nb.y)),
                __fmaf_rn(lz, nt.z, __fmaf_rn(ly, n.z, lx * nb.z))};
      size_t q = ao_record(aq, rank, j);
      queue[2 * q] = make_float4(org.x, org.y, org.z, start);
      queue[2 * q + 1] = make_float4(dir.x, dir.y, dir.z, __uint_as_float(pix * 8u + 2u + j));
    }
  }
  if (COUNT) flush_counts(c, rays, totals);
}

// Any-hit pass over the queued secondary rays; unoccluded rays set their bit
// in the pixel mask.  Each lane runs its ray one leaf at a time; when at
// least aq.refill_min lanes of a warp are idle the warp claims that many new
// rays with one atomic, so lanes need not wait for the slowest ray of the
// warp.  The number of hits is read on the device.
template <bool COUNT>
__global__ void __launch_bounds__(256, 5) k_ao_secondary(KdDev kd, AoDev ao, AoQueue aq,
                                                      uint32_t* __restrict__ mask,
                                                      uint32_t* __restrict__ counters,
                                                      unsigned long long* __restrict__ totals) {
  extern __shared__ uint2 snodes[];
  stage_nodes(kd, snodes);
  uint32_t lane = threadIdx.x & 31u;
  uint32_t nh = counters[1];
  uint32_t n = 5u * nh;
  Counters c = {0, 0, 0, 0};
  uint32_t rays = 0;
  Trav s;
  s.live = false;
  uint32_t tag = 0;
  bool exhausted = false;
  for (;;) {
    uint32_t idle = __ballot_sync(0xFFFFFFFFu, !s.live);
    uint32_t nidle = __popc(idle);
    if (!exhausted && (nidle >= aq.refill_min || nidle == 32u)) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(&counters[2], nidle);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (base + nidle >= n) exhausted = true;
      if (!s.live) {
        uint32_t i = base + __popc(idle & ((1u << lane) - 1u));
        if (i < n) {
          // claim index i -> record e in the layout's order; kind 0 = shadow
          uint32_t kind;
          size_t e;
          if (aq.mode == 0u) {
            e = i;
            kind = i % 5u;
          } else if (aq.mode == 1u) {
            kind = i / nh;
            e = (size_t)kind * aq.cap + (i - kind * nh);
          } else {
            kind = i < nh ? 0u : 1u;
            e = i < nh ? (size_t)i : (size_t)aq.cap + (i - nh);
          }
          float4 R0 = __ldg(&aq.q[2 * (size_t)e]), R1 = __ldg(&aq.q[2 * (size_t)e + 1]);
          tag = __float_as_uint(R1.w);
          float tmax = kind == 0 ? K_INF : ao.ao_length;
          trav_init<false>(s, kd, v3(R0.x, R0.y, R0.z), v3(R1.x, R1.y, R1.z), tmax,
                           __float_as_uint(R0.w));
          ++rays;
          if (!s.live && !COUNT) atomicOr(&mask[tag >> 3], 1u << (tag & 7u));
        }
      }
    }
    if (__ballot_sync(0xFFFFFFFFu, s.live) == 0u) {
      if (exhausted) break;
      continue;
    }
    if (s.live) {
      trav_step<0, true, COUNT>(s, kd, snodes, c);
      if (!s.live && !COUNT) {
        uint32_t bits = (s.best_id < 0 ? 1u << (tag & 7u) : 0u) |
                        (trav_truncated(s) ? kMaskTruncated : 0u);
        if (bits) atomicOr(&mask[tag >> 3], bits);
      }
    }
  }
  if (COUNT) flush_counts(c, rays, totals + 4);
}

}  // namespace re

// ------------------------------------------------------------------ host
namespace re {
namespace {

constexpr uint32_t kMaxStage = 8192;  // 64 KB of shared memory
// Default staging depth: the top 1024 nodes (8 KB).  Measured on the
// primary pass of the 2^20- and 65,536-triangle soups: 0-4096 staged nodes
// are within 3 % of each other, 8192 (64 KB, fewer resident blocks) is
// 13-20 % slower.  re_autotune_ao / re_scene_set_tuning override it.
constexpr uint32_t kDefaultStage = 1024;

KdDev kd_view(const re_scene* s) {
  KdDev kd;
  kd.nodes = s->d_nodes;
  kd.leaves = s->d_leaves;
  kd.tris = s->d_tris;
  kd.bmin = {s->host.bmin[0], s->host.bmin[1], s->host.bmin[2]};
  kd.bmax = {s->host.bmax[0], s->host.bmax[1], s->host.bmax[2]};
  kd.max_visits = s->max_visits;
  kd.stage = s->stage;
  kd.trunc = s->d_counters + RE_SCENE_TRUNC_SLOT;
  kd.num_refs = s->host.num_refs;
  if (s->d_entry) {
    kd.entry = s->d_entry;
    kd.entry_res = kEntryRes;
    float sc[3];
    for (int k = 0; k < 3; ++k) {
      const float ext = s->host.bmax[k] - s->host.bmin[k];
      sc[k] = ext > 0.f ? (float)kEntryRes / ext : 0.f;
    }
    kd.entry_scale = {sc[0], sc[1], sc[2]};
  }
  return kd;
}

CamDev cam_view(const re_camera& c) {
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

re_status check_scene(const re_scene* s, const char* fn) {
  if (!s) return fail(RE_ERR_INVALID_ARG, "%s: null scene", fn);
  if (s->device < 0) return fail(RE_ERR_NO_DEVICE, "%s: scene was built host-only", fn);
  int dev = -1;
  RE_CUDA(cudaGetDevice(&dev));
  if (dev != s->device)
    return fail(RE_ERR_INVALID_ARG, "%s: scene lives on device %d, current device is %d", fn,
                s->device, dev);
  return RE_OK;
}

template <typename K>
int grid_for(K kernel, size_t smem) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  return per_sm * sm_count();
}

re_status upload(re_scene* s) {
  const FlatTree& h = s->host;
  RE_CUDA(cudaMalloc(&s->d_nodes, h.nodes.size() * 4));
  RE_CUDA(cudaMalloc(&s->d_leaves, h.leaves.size() * 4));
  RE_CUDA(cudaMalloc(&s->d_tris, h.tris.size() * 4));
  RE_CUDA(cudaMalloc(&s->d_counters, 64));
  if (!h.entry.empty()) {
    RE_CUDA(cudaMalloc(&s->d_entry, h.entry.size() * 4));
    RE_CUDA(cudaMemcpy(s->d_entry, h.entry.data(), h.entry.size() * 4, cudaMemcpyHostToDevice));
  }
  RE_CUDA(cudaMemcpy(s->d_nodes, h.nodes.data(), h.nodes.size() * 4, cudaMemcpyHostToDevice));
  RE_CUDA(cudaMemcpy(s->d_leaves, h.leaves.data(), h.leaves.size() * 4, cudaMemcpyHostToDevice));
  RE_CUDA(cudaMemcpy(s->d_tris, h.tris.data(), h.tris.size() * 4, cudaMemcpyHostToDevice));
  RE_CUDA(cudaMemset(s->d_counters, 0, 64));
  s->stage = std::min<uint32_t>(h.bfs_nodes, kDefaultStage);
  s->tune.stage_nodes = s->stage;
  return RE_OK;
}

AoQueue ao_queue(const re_scene* s, float4* q, uint32_t capacity) {
  AoQueue aq;
  aq.q = q;
  aq.mode = s->tune.queue_kind_major;
  aq.cap = capacity;
  aq.refill_min = s->tune.refill_min;
  return aq;
}

void release(re_scene* s) {
  if (!s) return;
  cudaFree(s->d_nodes);
  cudaFree(s->d_leaves);
  cudaFree(s->d_tris);
  cudaFree(s->d_entry);
  cudaFree(s->d_counters);
  cudaFree(s->d_queue);
  delete s;
}

re_status create_from_packed(const float* tris, uint32_t n, const re_kd_params* params,
                             re_scene** out, bool host_only = false) {
  re_kd_params p;
  re_kd_params_default(&p);
  if (params) p = *params;
  if (p.leaf_size == 0 || p.max_depth == 0 || p.max_depth > 64)
    return fail(RE_ERR_INVALID_ARG, "re_scene_create: bad kd params");
  int dev = -1;
  if (!host_only) RE_CUDA(cudaGetDevice(&dev));
  re_scene* s = new (std::nothrow) re_scene();
  if (!s) return fail(RE_ERR_OUT_OF_MEMORY, "re_scene_create: host allocation");
  s->device = dev;
  s->max_visits = p.max_leaf_visits ? p.max_leaf_visits : 16384;
  const char* err = nullptr;
  try {
    if (!build_kdtree(tris, n, p, s->host, &err)) {
      delete s;
      return fail(RE_ERR_INVALID_ARG, "%s", err ? err : "kd build failed");
    }
  } catch (const std::bad_alloc&) {
    delete s;
    return fail(RE_ERR_OUT_OF_MEMORY, "re_scene_create: host allocation during build");
  }
  if (host_only) {
    *out = s;
    return RE_OK;
  }
  re_status st = upload(s);
  if (st != RE_OK) {
    release(s);
    return st;
  }
  *out = s;
  return RE_OK;
}

}  // namespace
}  // namespace re

namespace re {
namespace {

// One primary pass: G lanes per ray when ray_lanes > 1 (hits only), else
// whole-warp tiles when ray_refill_min is 32, else lane refill.  All
// kernels take the same arguments.
template <int MODE, bool COUNT>
re_status launch_primary(re_scene* s, const re_camera& cam, uint32_t w, uint32_t h, re_hit* out,
                         uint4* counts, cudaStream_t st) {
  KdDev kd = kd_view(s);
  // the counting walk descends from the root, as the oracle's does
  if (COUNT) kd.entry = nullptr;
  CamDev cd = cam_view(cam);
  size_t smem = kd.stage * sizeof(uint2);
  uint32_t refill = s->tune.ray_refill_min, lanes = COUNT ? 1u : s->tune.ray_lanes;
  auto k = lanes == 2u    ? k_primary_lanes<MODE, 2>
           : lanes == 4u  ? k_primary_lanes<MODE, 4>
           : lanes == 8u  ? k_primary_lanes<MODE, 8>
           : lanes == 32u ? k_primary_warp<MODE>
           : refill >= 32u ? k_primary_tiles<MODE, COUNT>
                           : k_primary<MODE, COUNT>;
  RE_CUDA(cudaMemsetAsync(s->d_counters, 0, RE_SCENE_RESET_BYTES, st));
  RE_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k<<<grid_for(k, smem), 256, smem, st>>>(kd, cd, w, h, out, counts, s->d_counters, refill);
  RE_CHECK_LAUNCH(COUNT ? "re_count_primary: launch" : "re_trace_primary: launch");
  return RE_OK;
}

template <int MODE, bool ANYHIT>
re_status launch_rays(re_scene* s, const float4* rays, uint32_t n, re_hit* out, cudaStream_t st) {
  KdDev kd = kd_view(s);
  size_t smem = kd.stage * sizeof(uint2);
  uint32_t refill = s->tune.ray_refill_min;
  auto k = refill >= 32u ? k_rays_chunks<MODE, ANYHIT> : k_rays<MODE, ANYHIT>;
  RE_CUDA(cudaMemsetAsync(s->d_counters, 0, RE_SCENE_RESET_BYTES, st));
  RE_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k<<<grid_for(k, smem), 256, smem, st>>>(kd, rays, n, out, s->d_counters, refill);
  RE_CHECK_LAUNCH("re_trace_rays: launch");
  return RE_OK;
}

}  // namespace
}  // namespace re

extern "C" {

RE_API void re_kd_params_default(re_kd_params* p) {
  if (!p) return;
  // Measured on B200 (AO frame of the 2.1M-triangle heightfield, primary
  // pass of 2^16- and 2^20-triangle soups): depth 24 cut the heightfield
  // tree short (+18 % frame time against depth >= 28); splitting down to
  // leaves of <= 2 references (splits stop early only when a side does not
  // shrink or the reference budget is spent) with an empty-side bonus of
  // 0.1 gave the fastest heightfield frame (3.14 ms; leaves of 4: 3.24 ms;
  // depth 24, leaf 8, bonus 0.2: 3.91 ms).  Random soups of large
  // overlapping triangles prefer leaves of 8 (finer splits duplicate
  // references): SoupConfig asks for that.
  p->max_depth = 40;
  p->leaf_size = 2;
  p->cost_traversal = 1.0f;
  p->cost_intersect = 2.0f;
  p->empty_bonus = 0.1f;
  p->bfs_levels = 12;
  p->threads = 0;
  p->max_leaf_visits = 16384;
}

RE_API re_status re_scene_create(const float* verts, uint32_t num_verts, const uint32_t* faces,
                                 uint32_t num_faces, const re_kd_params* params,
                                 re_scene** out) {
  if (!verts || !faces || !out || num_faces == 0 || num_verts == 0)
    return re::fail(RE_ERR_INVALID_ARG, "re_scene_create: null or empty mesh");
  if (num_faces > (1u << 30)) return re::fail(RE_ERR_LIMIT, "re_scene_create: > 2^30 faces");
  std::vector<float> packed;
  try {
    packed.resize(12 * (size_t)num_faces);
  } catch (const std::bad_alloc&) {
    return re::fail(RE_ERR_OUT_OF_MEMORY, "re_scene_create: host allocation");
  }
  // RTScene::init_triangles packing (RTScene.cpp:228-242)
  for (uint32_t i = 0; i < num_faces; ++i) {
    uint32_t a = faces[3 * (size_t)i], b = faces[3 * (size_t)i + 1], c = faces[3 * (size_t)i + 2];
    if (a >= num_verts || b >= num_verts || c >= num_verts)
      return re::fail(RE_ERR_INVALID_ARG, "re_scene_create: face %u indexes past the vertices", i);
    float* P = &packed[12 * (size_t)i];
    for (int k = 0; k < 3; ++k) {
      float v0 = verts[3 * (size_t)a + k];
      P[k] = v0;
      P[4 + k] = verts[3 * (size_t)b + k] - v0;
      P[8 + k] = verts[3 * (size_t)c + k] - v0;
    }
    P[3] = P[7] = P[11] = 0.f;
  }
  return re::create_from_packed(packed.data(), num_faces, params, out);
}

RE_API re_status re_scene_create_packed(const float* tris, uint32_t num_tris,
                                        const re_kd_params* params, re_scene** out) {
  if (!tris || !out || num_tris == 0)
    return re::fail(RE_ERR_INVALID_ARG, "re_scene_create_packed: null or empty input");
  if (num_tris > (1u << 30)) return re::fail(RE_ERR_LIMIT, "re_scene_create_packed: > 2^30 tris");
  return re::create_from_packed(tris, num_tris, params, out);
}

RE_API re_status re_scene_build_host(const float* tris, uint32_t num_tris,
                                     const re_kd_params* params, re_scene** out) {
  if (!tris || !out || num_tris == 0)
    return re::fail(RE_ERR_INVALID_ARG, "re_scene_build_host: null or empty input");
  if (num_tris > (1u << 30)) return re::fail(RE_ERR_LIMIT, "re_scene_build_host: > 2^30 tris");
  return re::create_from_packed(tris, num_tris, params, out, true);
}

RE_API re_status re_scene_stats_get(const re_scene* s, re_scene_stats* o) {
  if (!s || !o) return re::fail(RE_ERR_INVALID_ARG, "re_scene_stats_get: null argument");
  const re::FlatTree& h = s->host;
  std::memset(o, 0, sizeof(*o));
  o->num_tris = h.num_tris;
  o->num_nodes = h.num_nodes;
  o->num_leaves = h.num_leaves;
  o->num_refs = h.num_refs;
  o->max_depth = h.max_depth;
  o->max_leaf_size = h.max_leaf_size;
  o->bfs_nodes = h.bfs_nodes;
  for (int k = 0; k < 3; ++k) {
    o->bmin[k] = h.bmin[k];
    o->bmax[k] = h.bmax[k];
  }
  o->build_seconds = h.build_seconds;
  o->device_bytes = (h.nodes.size() + h.leaves.size() + h.tris.size()) * 4ull;
  return RE_OK;
}

RE_API re_status re_scene_export(const re_scene* s, uint32_t* nodes, uint32_t* leaves,
                                 float* tris) {
  if (!s) return re::fail(RE_ERR_INVALID_ARG, "re_scene_export: null scene");
  const re::FlatTree& h = s->host;
  if (nodes) std::memcpy(nodes, h.nodes.data(), h.nodes.size() * 4);
  if (leaves) std::memcpy(leaves, h.leaves.data(), h.leaves.size() * 4);
  if (tris) std::memcpy(tris, h.tris.data(), h.tris.size() * 4);
  return RE_OK;
}

RE_API re_status re_scene_export_entry(const re_scene* s, uint32_t* out, uint32_t* res) {
  if (!s || !res) return re::fail(RE_ERR_INVALID_ARG, "re_scene_export_entry: bad arguments");
  *res = re::kEntryRes;
  if (out) std::memcpy(out, s->host.entry.data(), s->host.entry.size() * 4);
  return RE_OK;
}

RE_API re_status re_scene_destroy(re_scene* s) {
  re::release(s);
  return RE_OK;
}

RE_API re_status re_trace_primary(re_scene* s, const re_camera* cam, uint32_t w, uint32_t h,
                                  uint32_t flags, re_hit* d_out, void* stream) {
  re_status st = re::check_scene(s, "re_trace_primary");
  if (st != RE_OK) return st;
  if (!cam || !d_out || w < 2 || h < 2)
    return re::fail(RE_ERR_INVALID_ARG, "re_trace_primary: bad arguments");
  if ((uint64_t)w * h > (1ull << 31)) return re::fail(RE_ERR_LIMIT, "re_trace_primary: image too large");
  if (flags & ~1u) return re::fail(RE_ERR_INVALID_ARG, "re_trace_primary: unknown flags");
  if (flags & RE_TRACE_ONE_SIDED)
    return re::launch_primary<1, false>(s, *cam, w, h, d_out, nullptr, (cudaStream_t)stream);
  return re::launch_primary<0, false>(s, *cam, w, h, d_out, nullptr, (cudaStream_t)stream);
}

RE_API re_status re_count_primary(re_scene* s, const re_camera* cam, uint32_t w, uint32_t h,
                                  uint32_t flags, uint32_t* d_counts, void* stream) {
  re_status st = re::check_scene(s, "re_count_primary");
  if (st != RE_OK) return st;
  if (!cam || !d_counts || w < 2 || h < 2)
    return re::fail(RE_ERR_INVALID_ARG, "re_count_primary: bad arguments");
  if ((uint64_t)w * h > (1ull << 31)) return re::fail(RE_ERR_LIMIT, "re_count_primary: image too large");
  if (flags & ~1u) return re::fail(RE_ERR_INVALID_ARG, "re_count_primary: unknown flags");
  uint4* c4 = reinterpret_cast<uint4*>(d_counts);
  if (flags & RE_TRACE_ONE_SIDED)
    return re::launch_primary<1, true>(s, *cam, w, h, nullptr, c4, (cudaStream_t)stream);
  return re::launch_primary<0, true>(s, *cam, w, h, nullptr, c4, (cudaStream_t)stream);
}

RE_API re_status re_scene_truncated(const re_scene* s, uint32_t* d_count, void* stream) {
  re_status st = re::check_scene(s, "re_scene_truncated");
  if (st != RE_OK) return st;
  if (!d_count) return re::fail(RE_ERR_INVALID_ARG, "re_scene_truncated: null output");
  RE_CUDA(cudaMemcpyAsync(d_count, s->d_counters + RE_SCENE_TRUNC_SLOT, 4,
                          cudaMemcpyDeviceToDevice, (cudaStream_t)stream));
  return RE_OK;
}

RE_API re_status re_trace_rays(re_scene* s, const re_ray* d_rays, uint32_t n, uint32_t flags,
                               re_hit* d_out, void* stream) {
  re_status st = re::check_scene(s, "re_trace_rays");
  if (st != RE_OK) return st;
  if (!d_rays || !d_out) return re::fail(RE_ERR_INVALID_ARG, "re_trace_rays: null buffer");
  if (n == 0) return RE_OK;
  if (n > (1u << 31)) return re::fail(RE_ERR_LIMIT, "re_trace_rays: n > 2^31");
  if (flags & ~3u) return re::fail(RE_ERR_INVALID_ARG, "re_trace_rays: unknown flags");
  const float4* r4 = reinterpret_cast<const float4*>(d_rays);
  cudaStream_t st_ = (cudaStream_t)stream;
  switch (flags & 3u) {
    case 0: return re::launch_rays<0, false>(s, r4, n, d_out, st_);
    case 1: return re::launch_rays<1, false>(s, r4, n, d_out, st_);
    case 2: return re::launch_rays<0, true>(s, r4, n, d_out, st_);
    default: return re::launch_rays<1, true>(s, r4, n, d_out, st_);
  }
}

}  // extern "C"

namespace re {
namespace {

re_status ao_prepare(re_scene* s, const re_camera* cam, uint32_t w, uint32_t h,
                     const re_ao_params* p, const char* fn, cudaStream_t st, CamDev& cd,
                     AoDev& ao) {
  re_status rs = check_scene(s, fn);
  if (rs != RE_OK) return rs;
  if (!cam || !p || w < 2 || h < 2) return fail(RE_ERR_INVALID_ARG, "%s: bad arguments", fn);
  if ((uint64_t)w * h > (1ull << 28)) return fail(RE_ERR_LIMIT, "%s: image > 2^28 pixels", fn);
  size_t need = 5ull * w * h;
  s->queue_stride = w * h;
  if (s->queue_cap < need) {
    // The queue grows outside stream order: wait until no earlier frame on
    // this stream still reads the old one.
    RE_CUDA(cudaStreamSynchronize(st));
    cudaFree(s->d_queue);
    s->d_queue = nullptr;
    s->queue_cap = 0;
    RE_CUDA(cudaMalloc(&s->d_queue, need * 32));
    s->queue_cap = need;
  }
  cd = cam_view(*cam);
  ao.light = {p->light_dir[0], p->light_dir[1], p->light_dir[2]};
  ao.ao_length = p->ao_length;
  ao.bias = p->bias;
  ao.seed = p->seed;
  s->ao_length = p->ao_length;
  return RE_OK;
}

template <bool COUNT>
re_status ao_primary(re_scene* s, const CamDev& cd, const AoDev& ao, uint32_t w, uint32_t h,
                     re_hit* d_primary, uint32_t* d_mask, unsigned long long* totals,
                     cudaStream_t st) {
  KdDev kd = kd_view(s);
  // the counting walk descends from the root, as the oracle's does
  if (COUNT) kd.entry = nullptr;
  size_t smem = kd.stage * sizeof(uint2);
  RE_CUDA(cudaMemsetAsync(s->d_counters, 0, RE_SCENE_RESET_BYTES, st));
  auto k = k_ao_primary<COUNT>;
  RE_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k<<<grid_for(k, smem), 256, smem, st>>>(kd, cd, ao, w, h, d_primary, d_mask,
                                          ao_queue(s, s->d_queue, s->queue_stride), s->d_counters,
                                          totals);
  RE_CHECK_LAUNCH("ao primary launch");
  return RE_OK;
}

template <bool COUNT>
re_status ao_secondary(re_scene* s, uint32_t* d_mask, unsigned long long* totals,
                       cudaStream_t st) {
  KdDev kd = kd_view(s);
  AoDev ao{};
  ao.ao_length = s->ao_length;
  size_t smem = kd.stage * sizeof(uint2);
  auto k = k_ao_secondary<COUNT>;
  RE_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k<<<grid_for(k, smem), 256, smem, st>>>(kd, ao, ao_queue(s, s->d_queue, s->queue_stride),
                                          d_mask, s->d_counters, totals);
  RE_CHECK_LAUNCH("ao secondary launch");
  return RE_OK;
}

}  // namespace
}  // namespace re

extern "C" {

RE_API re_status re_render_ao_primary(re_scene* s, const re_camera* cam, uint32_t w, uint32_t h,
                                      const re_ao_params* p, re_hit* d_primary,
                                      uint32_t* d_mask, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  re::CamDev cd;
  re::AoDev ao;
  re_status rs = re::ao_prepare(s, cam, w, h, p, "re_render_ao_primary", st, cd, ao);
  if (rs != RE_OK) return rs;
  if (!d_primary || !d_mask) return re::fail(RE_ERR_INVALID_ARG, "re_render_ao_primary: null output");
  return re::ao_primary<false>(s, cd, ao, w, h, d_primary, d_mask, nullptr, st);
}

RE_API re_status re_render_ao_secondary(re_scene* s, uint32_t* d_mask, uint32_t* d_num_secondary,
                                        void* stream) {
  re_status rs = re::check_scene(s, "re_render_ao_secondary");
  if (rs != RE_OK) return rs;
  if (!d_mask) return re::fail(RE_ERR_INVALID_ARG, "re_render_ao_secondary: null mask");
  if (!s->d_queue) return re::fail(RE_ERR_INVALID_ARG, "re_render_ao_secondary: no primary pass ran");
  cudaStream_t st = (cudaStream_t)stream;
  rs = re::ao_secondary<false>(s, d_mask, nullptr, st);
  if (rs != RE_OK) return rs;
  if (d_num_secondary)
    RE_CUDA(cudaMemcpyAsync(d_num_secondary, s->d_counters + 3, 4, cudaMemcpyDeviceToDevice, st));
  return RE_OK;
}

RE_API re_status re_render_ao(re_scene* s, const re_camera* cam, uint32_t w, uint32_t h,
                              const re_ao_params* p, re_hit* d_primary, uint32_t* d_mask,
                              uint32_t* d_num_secondary, void* stream) {
  re_status rs = re_render_ao_primary(s, cam, w, h, p, d_primary, d_mask, stream);
  if (rs != RE_OK) return rs;
  return re_render_ao_secondary(s, d_mask, d_num_secondary, stream);
}

RE_API re_status re_render_ao_counts(re_scene* s, const re_camera* cam, uint32_t w, uint32_t h,
                                     const re_ao_params* p, uint64_t* d_totals, void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  re::CamDev cd;
  re::AoDev ao;
  re_status rs = re::ao_prepare(s, cam, w, h, p, "re_render_ao_counts", st, cd, ao);
  if (rs != RE_OK) return rs;
  if (!d_totals) return re::fail(RE_ERR_INVALID_ARG, "re_render_ao_counts: null totals");
  unsigned long long* t = reinterpret_cast<unsigned long long*>(d_totals);
  RE_CUDA(cudaMemsetAsync(t, 0, 8 * sizeof(uint64_t), st));
  rs = re::ao_primary<true>(s, cd, ao, w, h, nullptr, nullptr, t, st);
  if (rs != RE_OK) return rs;
  return re::ao_secondary<true>(s, nullptr, t, st);
}

}  // extern "C"

// ------------------------------------------------ allocation-free AO frame
// Some callers cannot allocate device memory while they render: an engine
// that reserves all device memory up front through its own pool, or a frame
// loop that cannot afford cudaMalloc's implicit synchronisation or an
// out-of-memory failure in the middle of a frame.  re_render_ao grows its
// secondary-ray queue with cudaMalloc on first use; re_render_ao_noalloc
// instead uses the fixed array below (held by every GPU that loads the
// library, until the process exits).
namespace re {
namespace {

constexpr size_t kNoAllocCounterBytes = 256;
constexpr size_t kNoAllocQueueBytes = (size_t)5 * 32 * RE_NOALLOC_MAX_PIXELS;
constexpr size_t kNoAllocScratchBytes = kNoAllocCounterBytes + kNoAllocQueueBytes;

// counters (tile cursor, queue size, queue cursor) followed by the queue
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch on the current device.  In host code
// the symbol's name is only a host-side handle; the address comes from
// cudaGetSymbolAddress with the device current.  It is looked up on every
// call (a lookup allocates nothing), so no address outlives the context it
// belongs to: after a device reset the next call finds the new one.
re_status noalloc_scratch(unsigned char** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
  *out = static_cast<unsigned char*>(p);
  return RE_OK;
}

}  // namespace
}  // namespace re

extern "C" {

RE_API re_status re_render_ao_noalloc(re_scene* s, const re_camera* cam, uint32_t w, uint32_t h,
                                      const re_ao_params* p, re_hit* d_primary, uint32_t* d_mask,
                                      uint32_t* d_num_secondary, void* stream) {
  re_status rs = re::check_scene(s, "re_render_ao_noalloc");
  if (rs != RE_OK) return rs;
  if (!cam || !p || !d_primary || !d_mask || w < 2 || h < 2)
    return re::fail(RE_ERR_INVALID_ARG, "re_render_ao_noalloc: bad arguments");
  if ((uint64_t)w * h > RE_NOALLOC_MAX_PIXELS)
    return re::fail(RE_ERR_LIMIT,
                    "re_render_ao_noalloc: %ux%u = %llu pixels exceeds the fixed scratch of %u "
                    "pixels (5 secondary rays of 32 bytes each per pixel); use re_render_ao",
                    w, h, (unsigned long long)w * h, (unsigned)RE_NOALLOC_MAX_PIXELS);
  unsigned char* scratch = nullptr;
  rs = re::noalloc_scratch(&scratch);
  if (rs != RE_OK) return rs;
  uint32_t* counters = reinterpret_cast<uint32_t*>(scratch);
  float4* queue = reinterpret_cast<float4*>(scratch + re::kNoAllocCounterBytes);
  cudaStream_t st = (cudaStream_t)stream;
  re::KdDev kd = re::kd_view(s);
  kd.trunc = counters + RE_SCENE_TRUNC_SLOT;
  re::CamDev cd = re::cam_view(*cam);
  re::AoDev ao;
  ao.light = {p->light_dir[0], p->light_dir[1], p->light_dir[2]};
  ao.ao_length = p->ao_length;
  ao.bias = p->bias;
  ao.seed = p->seed;
  size_t smem = kd.stage * sizeof(uint2);
  // the array keeps the previous call's contents: the cursors must restart at zero
  RE_CUDA(cudaMemsetAsync(counters, 0, RE_SCENE_RESET_BYTES, st));
  {
    auto k = re::k_ao_primary<false>;
    RE_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<re::grid_for(k, smem), 256, smem, st>>>(kd, cd, ao, w, h, d_primary, d_mask,
                                                re::ao_queue(s, queue, w * h), counters, nullptr);
    RE_CHECK_LAUNCH("re_render_ao_noalloc: primary launch");
  }
  {
    auto k = re::k_ao_secondary<false>;
    RE_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k<<<re::grid_for(k, smem), 256, smem, st>>>(kd, ao, re::ao_queue(s, queue, w * h), d_mask,
                                                counters, nullptr);
    RE_CHECK_LAUNCH("re_render_ao_noalloc: secondary launch");
  }
  if (d_num_secondary)
    RE_CUDA(cudaMemcpyAsync(d_num_secondary, counters + 3, 4, cudaMemcpyDeviceToDevice, st));
  return RE_OK;
}

}  // extern "C"

// ------------------------------------------------------------- autotuner
extern "C" {

RE_API re_status re_scene_get_tuning(const re_scene* s, re_tuning* out) {
  if (!s || !out) return re::fail(RE_ERR_INVALID_ARG, "re_scene_get_tuning: null argument");
  *out = s->tune;
  return RE_OK;
}

RE_API re_status re_scene_set_tuning(re_scene* s, const re_tuning* t) {
  if (!s || !t) return re::fail(RE_ERR_INVALID_ARG, "re_scene_set_tuning: null argument");
  if (t->refill_min < 1 || t->refill_min > 32 || t->ray_refill_min < 1 || t->ray_refill_min > 32)
    return re::fail(RE_ERR_INVALID_ARG,
                    "re_scene_set_tuning: refill_min and ray_refill_min must be in [1, 32]");
  if (t->queue_kind_major > 2)
    return re::fail(RE_ERR_INVALID_ARG, "re_scene_set_tuning: queue_kind_major must be 0, 1 or 2");
  if ((t->ray_lanes > 8 && t->ray_lanes != 32) || (t->ray_lanes & (t->ray_lanes - 1u)))
    return re::fail(RE_ERR_INVALID_ARG,
                    "re_scene_set_tuning: ray_lanes must be 0, 1, 2, 4, 8 or 32");
  s->tune = *t;
  if (s->tune.ray_lanes == 0) s->tune.ray_lanes = 1;
  s->tune.stage_nodes = std::min(std::min(t->stage_nodes, s->host.bfs_nodes), re::kMaxStage);
  s->stage = s->tune.stage_nodes;
  return RE_OK;
}

// Times the AO frame for every combination of staging depth, queue layout
// and refill threshold (one warm-up and three timed frames each, CUDA events
// on the caller's stream) and keeps the fastest on the scene.  Set-up time
// only: it allocates its own output buffers.
RE_API re_status re_autotune_ao(re_scene* s, const re_camera* cam, uint32_t w, uint32_t h,
                                const re_ao_params* p, re_tuning* best_out, float* best_ms_out,
                                void* stream) {
  re_status rs = re::check_scene(s, "re_autotune_ao");
  if (rs != RE_OK) return rs;
  if (!cam || !p || w < 2 || h < 2) return re::fail(RE_ERR_INVALID_ARG, "re_autotune_ao: bad arguments");
  if ((uint64_t)w * h > (1ull << 28)) return re::fail(RE_ERR_LIMIT, "re_autotune_ao: image > 2^28 pixels");
  cudaStream_t st = (cudaStream_t)stream;
  re_hit* hits = nullptr;
  uint32_t* mask = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  RE_CUDA(cudaMalloc(&hits, (size_t)w * h * sizeof(re_hit)));
  cudaError_t ce = cudaMalloc(&mask, (size_t)w * h * 4);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  re_tuning keep = s->tune, best = s->tune;
  float best_ms = 1e30f;
  uint32_t bfs = std::min(s->host.bfs_nodes, re::kMaxStage);
  const uint32_t stages[4] = {0u, std::min(1024u, bfs), std::min(4096u, bfs), bfs};
  const uint32_t refills[4] = {4u, 8u, 16u, 32u};
  for (int si = 0; si < 4 && ce == cudaSuccess && rs == RE_OK; ++si) {
    if (si > 0 && stages[si] == stages[si - 1]) continue;
    for (uint32_t km = 0; km < 3 && rs == RE_OK; ++km) {
      for (int ri = 0; ri < 4 && rs == RE_OK; ++ri) {
        re_tuning t = keep;
        t.stage_nodes = stages[si];
        t.queue_kind_major = km;
        t.refill_min = refills[ri];
        rs = re_scene_set_tuning(s, &t);
        if (rs != RE_OK) break;
        rs = re_render_ao(s, cam, w, h, p, hits, mask, nullptr, stream);
        if (rs != RE_OK) break;
        ce = cudaEventRecord(e0, st);
        for (int r = 0; r < 3 && rs == RE_OK; ++r) rs = re_render_ao(s, cam, w, h, p, hits, mask, nullptr, stream);
        if (ce == cudaSuccess) ce = cudaEventRecord(e1, st);
        if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
        float ms = 0.f;
        if (ce == cudaSuccess) ce = cudaEventElapsedTime(&ms, e0, e1);
        if (ce != cudaSuccess) break;
        if (ms < best_ms) {
          best_ms = ms;
          best = s->tune;
        }
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(hits);
  cudaFree(mask);
  if (ce != cudaSuccess) {
    s->tune = keep;
    s->stage = keep.stage_nodes;
    return re::cuda_fail(ce, "re_autotune_ao");
  }
  if (rs != RE_OK) {
    s->tune = keep;
    s->stage = keep.stage_nodes;
    return rs;
  }
  re_scene_set_tuning(s, &best);
  if (best_out) *best_out = best;
  if (best_ms_out) *best_ms_out = best_ms / 3.0f;
  return RE_OK;
}

// Times the primary pass (re_trace_primary with `flags`) for every
// combination of staging depth and walk form (one lane per ray with each
// refill threshold, or 2, 4 or 8 lanes per ray; one warm-up and three timed
// passes each, CUDA events on the caller's stream) and keeps the fastest on
// the scene.  Each timed pass follows a write of twice the L2 size, so the
// forms are compared on a frame whose tree is not cached (as after other
// work; back-to-back passes with a warm L2 favoured forms that lose on a
// cold one).  Set-up time only: it allocates its own output and the
// scratch it writes.
RE_API re_status re_autotune_primary(re_scene* s, const re_camera* cam, uint32_t w, uint32_t h,
                                     uint32_t flags, re_tuning* best_out, float* best_ms_out,
                                     void* stream) {
  re_status rs = re::check_scene(s, "re_autotune_primary");
  if (rs != RE_OK) return rs;
  if (!cam || w < 2 || h < 2 || (flags & ~1u))
    return re::fail(RE_ERR_INVALID_ARG, "re_autotune_primary: bad arguments");
  if ((uint64_t)w * h > (1ull << 28))
    return re::fail(RE_ERR_LIMIT, "re_autotune_primary: image > 2^28 pixels");
  cudaStream_t st = (cudaStream_t)stream;
  re_hit* hits = nullptr;
  void* scratch = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int l2 = 0;
  RE_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, s->device));
  const size_t scratch_bytes = 2 * (size_t)std::max(l2, 1 << 20);
  RE_CUDA(cudaMalloc(&hits, (size_t)w * h * sizeof(re_hit)));
  cudaError_t ce = cudaMalloc(&scratch, scratch_bytes);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e0);
  if (ce == cudaSuccess) ce = cudaEventCreate(&e1);
  re_tuning keep = s->tune, best = s->tune;
  float best_ms = 1e30f;
  uint32_t bfs = std::min(s->host.bfs_nodes, re::kMaxStage);
  const uint32_t stages[3] = {0u, std::min(1024u, bfs), std::min(4096u, bfs)};
  // {ray_lanes, ray_refill_min}
  const uint32_t forms[8][2] = {{1u, 32u}, {1u, 16u}, {1u, 8u}, {1u, 4u},
                                {2u, 32u}, {4u, 32u}, {8u, 32u}, {32u, 32u}};
  for (int si = 0; si < 3 && ce == cudaSuccess && rs == RE_OK; ++si) {
    if (si > 0 && stages[si] == stages[si - 1]) continue;
    for (int fi = 0; fi < 8 && rs == RE_OK; ++fi) {
      re_tuning t = keep;
      t.stage_nodes = stages[si];
      t.ray_lanes = forms[fi][0];
      t.ray_refill_min = forms[fi][1];
      rs = re_scene_set_tuning(s, &t);
      if (rs != RE_OK) break;
      rs = re_trace_primary(s, cam, w, h, flags, hits, stream);
      if (rs != RE_OK) break;
      float ms = 0.f;
      for (int r = 0; r < 3 && rs == RE_OK && ce == cudaSuccess; ++r) {
        ce = cudaMemsetAsync(scratch, r, scratch_bytes, st);
        if (ce == cudaSuccess) ce = cudaEventRecord(e0, st);
        if (ce == cudaSuccess) rs = re_trace_primary(s, cam, w, h, flags, hits, stream);
        if (ce == cudaSuccess) ce = cudaEventRecord(e1, st);
        if (ce == cudaSuccess) ce = cudaEventSynchronize(e1);
        float one = 0.f;
        if (ce == cudaSuccess) ce = cudaEventElapsedTime(&one, e0, e1);
        ms += one;
      }
      if (ce != cudaSuccess || rs != RE_OK) break;
      if (ms < best_ms) {
        best_ms = ms;
        best = s->tune;
      }
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(hits);
  cudaFree(scratch);
  if (ce != cudaSuccess || rs != RE_OK) {
    s->tune = keep;
    s->stage = keep.stage_nodes;
    return ce != cudaSuccess ? re::cuda_fail(ce, "re_autotune_primary") : rs;
  }
  re_scene_set_tuning(s, &best);
  if (best_out) *best_out = best;
  if (best_ms_out) *best_ms_out = best_ms / 3.0f;
  return RE_OK;
}

}  // extern "C"
