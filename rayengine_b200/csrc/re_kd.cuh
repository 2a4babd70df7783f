// Rope kd-tree traversal on the device, shared by the frame kernels
// (re_trace.cu) and the batched wavefront renderer (re_batch.cu).
//
// Restates, in the reference (hadalhw17/RayEngine, "RE/" = RayEngine/src/):
//   gpu_ray_box_intersect, gpu_ray_tri_intersect, stackless_kdtree_traversal
//                          RE/cuda-src/ray_functions.cuh:62-92,174-360
//   is_point_to_the_left_of_split, get_neighboring_node_index
//                          RE/cuda-src/kd_tree_functions.cuh:10-62
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "re_common.hpp"
#include "re_math.cuh"

namespace re {

constexpr float K_INF = 1e20f;  // RE/RayEngine/RayEngine.h:24

struct KdDev {
  const uint2* __restrict__ nodes;
  const float4* __restrict__ leaves;
  const float4* __restrict__ tris;
  V3 bmin, bmax;
  uint32_t max_visits;
  uint32_t stage;  // nodes [0, stage) are read from shared memory
  // rays stopped by the leaf-visit cap are counted here (may be null); the
  // reference stops at its cap silently (ray_functions.cuh:284)
  uint32_t* trunc;
  // triangle slots in `tris`; lanes that share a ray fetch their first
  // triangle of a leaf before its record only below this bound (0: never)
  uint32_t num_refs = 0;
  // start nodes of rays entering the root box through a face (the host's
  // entry table: 6 faces x entry_res^2 cells; null: every walk starts at the
  // root).  entry_scale = entry_res / extent per axis.
  const uint32_t* __restrict__ entry = nullptr;
  uint32_t entry_res = 0;
  V3 entry_scale = {0.f, 0.f, 0.f};
};

// Trav::visits of a walk that stopped at the leaf-visit cap.
constexpr uint32_t kTruncated = 0xFFFFFFFFu;

struct Counters {
  uint32_t inner, leaf, tests, status;
};

// gpu_ray_box_intersect (ray_functions.cuh:62-92)
__device__ __forceinline__ bool ray_box(V3 lo, V3 hi, V3 o, V3 inv, float& tn, float& tf) {
  float t1 = (lo.x - o.x) * inv.x, t2 = (hi.x - o.x) * inv.x;
  float t3 = (lo.y - o.y) * inv.y, t4 = (hi.y - o.y) * inv.y;
  float t5 = (lo.z - o.z) * inv.z, t6 = (hi.z - o.z) * inv.z;
  float tmin = fmaxf(fmaxf(fminf(t1, t2), fminf(t3, t4)), fminf(t5, t6));
  float tmax = fminf(fminf(fmaxf(t1, t2), fmaxf(t3, t4)), fmaxf(t5, t6));
  if (tmax < 0.0f) return false;
  if (tmin > tmax) return false;
  tn = tmin >= 0.0f ? tmin : 0.0f;
  tf = tmax;
  return true;
}

// Moller-Trumbore.  MODE 0: two-sided (KDTree.cpp:909-949), MODE 1:
// back faces culled (ray_functions.cuh:174-223).
template <int MODE>
__device__ __forceinline__ bool ray_tri(V3 o, V3 d, float4 T0, float4 T1, float4 T2,
                                        float& t, float& u, float& v) {
  // The reference's early-out tests, evaluated as one predicate so that the
  // lanes of a warp do not diverge on them; every value is computed exactly
  // as in the early-out form (a division by a rejected determinant is
  // computed and discarded).
  V3 v0 = {T0.x, T0.y, T0.z}, e1 = {T1.x, T1.y, T1.z}, e2 = {T2.x, T2.y, T2.z};
  V3 h = cross(d, e2);
  float a = dot(e1, h);
  bool ok = MODE == 0 ? !(a > -0.00001f && a < 0.00001f) : !(a < 1e-4f);
  float f = 1.0f / a;
  V3 s = sub(o, v0);
  float uu = f * dot(s, h);
  ok = ok & !(uu < 0.0f || uu > 1.0f);
  V3 q = cross(s, e1);
  float vv = f * dot(d, q);
  ok = ok & !(vv < 0.0f || uu + vv > 1.0f);
  float tt = f * dot(e2, q);
  ok = ok & (tt > (MODE == 0 ? 0.00001f : 1e-4f));
  t = tt;
  u = uu;
  v = vv;
  return ok;
}

struct HitState {
  float t, u, v;
  int32_t id;
  uint32_t ref;        // leaf-order triangle slot of the best hit
  uint32_t leaf_node;  // node index of the leaf the best hit was found in
};

__device__ __forceinline__ uint2 load_node(const KdDev& kd, const uint2* snodes, uint32_t i) {
  return i < kd.stage ? snodes[i] : __ldg(&kd.nodes[i]);
}

// Stackless rope traversal (stackless_kdtree_traversal,
// ray_functions.cuh:231-360) with the exit face taken from the slab test and
// split decisions made on the ray parameter so that a point on a split plane
// goes to the side the ray moves into.
//
// The walk is a per-lane state machine: trav_init() clips the ray to the
// root box, each trav_step() descends to one leaf, tests its triangles and
// follows one rope.  Kernels either run a ray to completion (traverse()) or
// interleave steps of many rays and refill finished lanes (k_ao_secondary).
//
// start: a leaf node to begin in instead of descending from the root (a
// secondary ray starts where its primary ray hit); used only when the ray
// origin lies in that leaf's region, otherwise the walk starts at the root.
// Either way every leaf the ray crosses is visited, so hits are unchanged.
struct Trav {
  V3 o, d, inv;
  float t_entry, best_t, best_u, best_v;
  int32_t best_id;
  uint32_t best_ref, best_leaf, node, visits;
  bool live;
};

// Whether origin o lies in the region of leaf node `start` (the condition
// under which a walk may begin there instead of at the root).
__device__ __forceinline__ bool origin_in_leaf(const KdDev& kd, V3 o, uint32_t start) {
  uint2 sn = __ldg(&kd.nodes[start]);
  if ((sn.y & 3u) != 3u) return false;
  const float4* SL = kd.leaves + 4 * (size_t)(sn.y >> 2);
  float4 A = __ldg(SL), B = __ldg(SL + 1);
  return o.x >= A.x && o.x <= A.w && o.y >= A.y && o.y <= B.x && o.z >= A.z && o.z <= B.y;
}

// The node a ray entering the root box at t_entry > 0 starts its first
// descent from: the entry table's cell of the face it entered through (the
// axis whose slab it entered last; the -k face when it moves in +k).  The
// table was built so that every entry point in a cell takes the root
// descent's path down to the cell's node, so the walk (and every hit) is
// that of a descent from the root.  0 (the root) without a table or for an
// origin inside the box.
__device__ __forceinline__ uint32_t entry_node(const KdDev& kd, V3 o, V3 d, V3 inv,
                                               float t_entry) {
  if (kd.entry == nullptr || !(t_entry > 0.0f)) return 0u;
  const float nx = fminf((kd.bmin.x - o.x) * inv.x, (kd.bmax.x - o.x) * inv.x);
  const float ny = fminf((kd.bmin.y - o.y) * inv.y, (kd.bmax.y - o.y) * inv.y);
  const float nz = fminf((kd.bmin.z - o.z) * inv.z, (kd.bmax.z - o.z) * inv.z);
  const uint32_t k = (nx >= ny && nx >= nz) ? 0u : (ny >= nz ? 1u : 2u);
  const uint32_t side = comp(d, k) > 0.0f ? 0u : 1u;
  // the face's axes a < b
  const uint32_t a = k == 0u ? 1u : 0u, b = k == 2u ? 1u : 2u;
  const float lim = (float)(kd.entry_res - 1u);
  const float pa = __fmaf_rn(t_entry, comp(d, a), comp(o, a));
  const float pb = __fmaf_rn(t_entry, comp(d, b), comp(o, b));
  const float fa = fminf(fmaxf((pa - comp(kd.bmin, a)) * comp(kd.entry_scale, a), 0.0f), lim);
  const float fb = fminf(fmaxf((pb - comp(kd.bmin, b)) * comp(kd.entry_scale, b), 0.0f), lim);
  const uint32_t i = (uint32_t)fa, j = (uint32_t)fb;
  return __ldg(&kd.entry[((k * 2u + side) * kd.entry_res + i) * kd.entry_res + j]);
}

// CHECKED false: the caller has already established origin_in_leaf(start)
// (or passes start 0), so the walk begins at `start` without loading it.
// CHECKED true: a start leaf the origin is not in, or start 0, begins at the
// entry table's node (entry_node).
template <bool CHECKED = true>
__device__ __forceinline__ void trav_init(Trav& s, const KdDev& kd, V3 o, V3 d, float tmax,
                                          uint32_t start) {
  s.o = o;
  s.d = d;
  s.inv = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
  s.best_id = -1;
  s.best_u = 0.f;
  s.best_v = 0.f;
  s.best_ref = 0xFFFFFFFFu;
  s.best_leaf = 0;
  s.node = 0;
  s.visits = 0;
  float t_root_exit;
  s.live = ray_box(kd.bmin, kd.bmax, o, s.inv, s.t_entry, t_root_exit);
  if (!s.live) return;
  s.best_t = fminf(t_root_exit, tmax);
  s.live = s.t_entry < s.best_t;
  if (CHECKED) {
    if (s.live && start != 0 && origin_in_leaf(kd, o, start)) s.node = start;
    else if (s.live) s.node = entry_node(kd, o, d, s.inv, s.t_entry);
  } else {
    s.node = start;
  }
}

// G > 1: G consecutive lanes walk the same ray in lockstep (same state,
// same loads) and split each leaf's triangle tests, lane j taking slots
// first + j, first + j + G, ...; the group then keeps the smallest (t, id)
// of its lanes' bests.  The sequential acceptance rule (smaller t, or equal
// t and smaller id, with id -1 for "no hit yet") is that same lexicographic
// minimum, and a leaf holds each triangle once, so the merged best, its
// slot and its leaf equal the one-lane walk's.  Closest hit only.
template <int MODE, bool ANYHIT, bool COUNT, uint32_t G = 1>
__device__ __forceinline__ void trav_step(Trav& s, const KdDev& kd, const uint2* snodes,
                                          Counters& c) {
  static_assert(G == 1 || G == 2 || G == 4 || G == 8, "lanes per ray: 1, 2, 4 or 8");
  static_assert(G == 1 || (!ANYHIT && !COUNT), "shared rays: closest hit, no counters");
  const uint32_t sub = G > 1 ? (threadIdx.x & (G - 1u)) : 0u;
  const V3 o = s.o, d = s.d, inv = s.inv;
  const float t_entry = s.t_entry;
  uint32_t node = s.node;
  uint2 nd = load_node(kd, snodes, node);
  while ((nd.y & 3u) != 3u) {
    uint32_t k = nd.y & 3u;
    float split = __uint_as_float(nd.x);
    float ok = comp(o, k), dk = comp(d, k), ik = comp(inv, k);
    // branch-free form of: dk > 0: t_entry < ts; dk < 0: t_entry >= ts;
    // dk == 0: ok < split (ts is computed but unused when dk == 0)
    float ts = (split - ok) * ik;
    bool left = dk > 0.0f ? (t_entry < ts) : (dk < 0.0f ? (t_entry >= ts) : (ok < split));
    node = (nd.y >> 2) + (left ? 0u : 1u);
    nd = load_node(kd, snodes, node);
    if (COUNT) c.inner++;
  }
  // a leaf node carries its first triangle reference (bit 31: empty leaf):
  // closest-hit walks fetch that triangle together with the leaf record
  // (measured: any-hit walks, which often stop at the first hit of a leaf,
  // run faster without the extra live registers)
  constexpr bool kEarlyFirst = !ANYHIT;
  uint32_t first = nd.x & 0x7FFFFFFFu;
  // this lane's first slot; with G > 1 it may lie past the leaf (fetched
  // only inside the triangle array, and used only if the leaf reaches it)
  const uint32_t mine = first + sub;
  const float4* T = kd.tris + 3 * (size_t)mine;
  float4 T0 = make_float4(0.f, 0.f, 0.f, 0.f), T1 = T0, T2 = T0;
  if (kEarlyFirst && !(nd.x >> 31) && (G == 1 || mine < kd.num_refs)) {
    T0 = __ldg(T);
    T1 = __ldg(T + 1);
    T2 = __ldg(T + 2);
  }
  const float4* L = kd.leaves + 4 * (size_t)(nd.y >> 2);
  float4 A = __ldg(L), B = __ldg(L + 1);
  if (COUNT) c.leaf++;
  uint32_t count = __float_as_uint(B.w);
  // The exit face of the leaf box and the rope behind it are taken before
  // the triangle tests, so that the rope load overlaps them.  Per axis the
  // ray leaves through +k when d.k > 0 and -k when d.k < 0; an axis with
  // d.k == 0 gets the distance +inf, which the strict comparisons below
  // never accept.  Written with selects so that lanes of different
  // direction signs do not diverge.
  const float kInf = __int_as_float(0x7f800000);
  float texit = kInf;
  int face = -1;
  {
    float tx = d.x != 0.0f ? ((d.x > 0.0f ? A.w : A.x) - o.x) * inv.x : kInf;
    float ty = d.y != 0.0f ? ((d.y > 0.0f ? B.x : A.y) - o.y) * inv.y : kInf;
    float tz = d.z != 0.0f ? ((d.z > 0.0f ? B.y : A.z) - o.z) * inv.z : kInf;
    if (tx < texit) { texit = tx; face = d.x > 0.0f ? 1 : 0; }
    if (ty < texit) { texit = ty; face = d.y > 0.0f ? 3 : 2; }
    if (tz < texit) { texit = tz; face = d.z > 0.0f ? 5 : 4; }
  }
  int32_t rope = face >= 0 ? __ldg(reinterpret_cast<const int32_t*>(L + 2) + face) : -1;
  for (uint32_t i = mine, end = first + count; i < end; i += G) {
    if (!kEarlyFirst || i != mine || (G > 1 && mine >= kd.num_refs)) {
      T = kd.tris + 3 * (size_t)i;
      T0 = __ldg(T);
      T1 = __ldg(T + 1);
      T2 = __ldg(T + 2);
    }
    int32_t id = __float_as_int(T0.w);
    float t, u, v;
    if (COUNT) c.tests++;
    if (ray_tri<MODE>(o, d, T0, T1, T2, t, u, v)) {
      if (t < s.best_t || (t == s.best_t && id < s.best_id && s.best_id >= 0)) {
        s.best_t = t;
        s.best_id = id;
        s.best_u = u;
        s.best_v = v;
        s.best_ref = i;
        s.best_leaf = node;
        if (ANYHIT) {
          s.live = false;
          return;
        }
      }
    }
  }
  if (G > 1) {
    const uint32_t gmask = ((1u << G) - 1u) << ((threadIdx.x & 31u) & ~(G - 1u));
#pragma unroll
    for (uint32_t off = 1; off < G; off <<= 1) {
      float ot = __shfl_xor_sync(gmask, s.best_t, off);
      int32_t oid = __shfl_xor_sync(gmask, s.best_id, off);
      float ou = __shfl_xor_sync(gmask, s.best_u, off);
      float ov = __shfl_xor_sync(gmask, s.best_v, off);
      uint32_t oref = __shfl_xor_sync(gmask, s.best_ref, off);
      // the other lane differs only if it accepted a triangle of this leaf
      if (ot < s.best_t || (ot == s.best_t && oid < s.best_id)) {
        s.best_t = ot;
        s.best_id = oid;
        s.best_u = ou;
        s.best_v = ov;
        s.best_ref = oref;
        s.best_leaf = node;
      }
    }
  }
  if (face < 0) {
    s.live = false;
    return;
  }
  s.t_entry = fmaxf(t_entry, texit);
  if (!(s.t_entry < s.best_t)) {
    s.live = false;
    return;
  }
  if (rope < 0) {
    s.live = false;
    return;
  }
  s.node = (uint32_t)rope;
  if (++s.visits >= kd.max_visits) {
    c.status = 1;
    s.live = false;
    s.visits = kTruncated;
    if (kd.trunc && sub == 0u) atomicAdd(kd.trunc, 1u);
  }
}

// Warp-cooperative closest-hit step: every lane of the warp calls it, live
// or not.  Each live lane descends to its next leaf as in trav_step; then the
// warp tests the (ray, triangle) pairs of all its live lanes' leaves
// together, 32 at a time, so a lane whose ray has finished helps the others
// and a leaf's tests no longer run one after another on its own lane.  Pair
// p belongs to the lane whose exclusive prefix of test counts is the last
// one <= p.  Each owner's best is reduced in shared memory as the 64-bit key
// (t bits << 32 | id): t > 0, so the key order is the (t, id) lexicographic
// order, and seeding the owner's slot with (best t, best id) — or (best t,
// 0) before any hit, so that an equal t is never accepted then — makes the
// minimum exactly the sequential acceptance rule's result (strictly
// smaller t, or equal t and smaller id once a hit exists; a leaf holds each
// triangle once).  The tester whose key is the minimum writes u, v and the
// triangle slot for its owner.  key and rec: this warp's 32 slots.
template <int MODE>
__device__ __forceinline__ void trav_step_warp(Trav& s, const KdDev& kd, const uint2* snodes,
                                               unsigned long long* key, float4* rec) {
  const uint32_t lane = threadIdx.x & 31u;
  const bool live = s.live;
  const V3 o = s.o, d = s.d, inv = s.inv;
  uint32_t node = s.node, first = 0, count = 0;
  const float kInf = __int_as_float(0x7f800000);
  float texit = kInf;
  int face = -1;
  int32_t rope = -1;
  if (live) {
    const float t_entry = s.t_entry;
    uint2 nd = load_node(kd, snodes, node);
    while ((nd.y & 3u) != 3u) {
      uint32_t k = nd.y & 3u;
      float split = __uint_as_float(nd.x);
      float ok = comp(o, k), dk = comp(d, k), ik = comp(inv, k);
      float ts = (split - ok) * ik;
      bool left = dk > 0.0f ? (t_entry < ts) : (dk < 0.0f ? (t_entry >= ts) : (ok < split));
      node = (nd.y >> 2) + (left ? 0u : 1u);
      nd = load_node(kd, snodes, node);
    }
    first = nd.x & 0x7FFFFFFFu;
    const float4* L = kd.leaves + 4 * (size_t)(nd.y >> 2);
    float4 A = __ldg(L), B = __ldg(L + 1);
    count = __float_as_uint(B.w);
    float tx = d.x != 0.0f ? ((d.x > 0.0f ? A.w : A.x) - o.x) * inv.x : kInf;
    float ty = d.y != 0.0f ? ((d.y > 0.0f ? B.x : A.y) - o.y) * inv.y : kInf;
    float tz = d.z != 0.0f ? ((d.z > 0.0f ? B.y : A.z) - o.z) * inv.z : kInf;
    if (tx < texit) { texit = tx; face = d.x > 0.0f ? 1 : 0; }
    if (ty < texit) { texit = ty; face = d.y > 0.0f ? 3 : 2; }
    if (tz < texit) { texit = tz; face = d.z > 0.0f ? 5 : 4; }
    rope = face >= 0 ? __ldg(reinterpret_cast<const int32_t*>(L + 2) + face) : -1;
  }
  uint32_t incl = count;
#pragma unroll
  for (uint32_t off = 1; off < 32; off <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, off);
    if (lane >= off) incl += y;
  }
  const uint32_t excl = incl - count, total = __shfl_sync(0xFFFFFFFFu, incl, 31);
  if (total > 0u) {
    unsigned long long seed = 0ull;
    if (live) {
      seed = ((unsigned long long)__float_as_uint(s.best_t) << 32) |
             (uint32_t)(s.best_id >= 0 ? s.best_id : 0);
      key[lane] = seed;
    }
    __syncwarp();
    for (uint32_t base = 0; base < total; base += 32u) {
      const uint32_t p = base + lane;
      uint32_t own = 0;
#pragma unroll
      for (uint32_t step = 16; step > 0; step >>= 1) {
        const uint32_t cand = own + step;
        if (__shfl_sync(0xFFFFFFFFu, excl, cand) <= p) own = cand;
      }
      const uint32_t oex = __shfl_sync(0xFFFFFFFFu, excl, own);
      const uint32_t ofirst = __shfl_sync(0xFFFFFFFFu, first, own);
      const V3 ro = {__shfl_sync(0xFFFFFFFFu, o.x, own), __shfl_sync(0xFFFFFFFFu, o.y, own),
                     __shfl_sync(0xFFFFFFFFu, o.z, own)};
      const V3 rd = {__shfl_sync(0xFFFFFFFFu, d.x, own), __shfl_sync(0xFFFFFFFFu, d.y, own),
                     __shfl_sync(0xFFFFFFFFu, d.z, own)};
      bool hit = false;
      unsigned long long k = 0ull;
      float u = 0.f, v = 0.f;
      uint32_t ref = 0;
      if (p < total) {
        ref = ofirst + (p - oex);
        const float4* T = kd.tris + 3 * (size_t)ref;
        float4 T0 = __ldg(T), T1 = __ldg(T + 1), T2 = __ldg(T + 2);
        float t;
        if (ray_tri<MODE>(ro, rd, T0, T1, T2, t, u, v)) {
          k = ((unsigned long long)__float_as_uint(t) << 32) | (uint32_t)__float_as_int(T0.w);
          hit = true;
          atomicMin(&key[own], k);
        }
      }
      __syncwarp();
      if (hit && key[own] == k) rec[own] = make_float4(u, v, __uint_as_float(ref), 0.f);
      __syncwarp();
    }
    if (live) {
      const unsigned long long k = key[lane];
      if (k != seed) {
        const float4 r = rec[lane];
        s.best_t = __uint_as_float((uint32_t)(k >> 32));
        s.best_id = (int32_t)(uint32_t)k;
        s.best_u = r.x;
        s.best_v = r.y;
        s.best_ref = __float_as_uint(r.z);
        s.best_leaf = node;
      }
    }
    __syncwarp();
  }
  if (!live) return;
  if (face < 0) {
    s.live = false;
    return;
  }
  s.t_entry = fmaxf(s.t_entry, texit);
  if (!(s.t_entry < s.best_t) || rope < 0) {
    s.live = false;
    return;
  }
  s.node = (uint32_t)rope;
  if (++s.visits >= kd.max_visits) {
    s.live = false;
    s.visits = kTruncated;
    if (kd.trunc) atomicAdd(kd.trunc, 1u);
  }
}

// The walk ended at the leaf-visit cap (its hit, if any, is the closest one
// found among the leaves it reached).
__device__ __forceinline__ bool trav_truncated(const Trav& s) { return s.visits == kTruncated; }

__device__ __forceinline__ void trav_result(const Trav& s, HitState& hs) {
  if (s.best_id >= 0) {
    hs.t = s.best_t;
    hs.u = s.best_u;
    hs.v = s.best_v;
    hs.id = s.best_id;
    hs.ref = s.best_ref;
    hs.leaf_node = s.best_leaf;
  } else {
    hs.t = K_INF;
    hs.u = 0.f;
    hs.v = 0.f;
    hs.id = -1;
    hs.ref = 0xFFFFFFFFu;
    hs.leaf_node = 0;
  }
}

// Runs one ray to the end; returns true when it stopped at the leaf-visit cap.
template <int MODE, bool ANYHIT, bool COUNT>
__device__ __forceinline__ bool traverse(const KdDev& kd, const uint2* snodes, V3 o, V3 d,
                                         float tmax, uint32_t start, HitState& hs, Counters& c) {
  Trav s;
  trav_init(s, kd, o, d, tmax, start);
  while (s.live) trav_step<MODE, ANYHIT, COUNT>(s, kd, snodes, c);
  trav_result(s, hs);
  return trav_truncated(s);
}

__device__ __forceinline__ void stage_nodes(const KdDev& kd, uint2* snodes) {
  for (uint32_t i = threadIdx.x; i < kd.stage; i += blockDim.x) snodes[i] = __ldg(&kd.nodes[i]);
  __syncthreads();
}

__device__ __forceinline__ uint32_t warp_fetch(uint32_t* counter) {
  uint32_t lane = threadIdx.x & 31u;
  uint32_t t = 0;
  if (lane == 0) t = atomicAdd(counter, 1u);
  return __shfl_sync(0xFFFFFFFFu, t, 0);
}

__device__ __forceinline__ void store_hit(re_hit* out, size_t i, const HitState& hs) {
  reinterpret_cast<int4*>(out)[i] =
      make_int4(hs.id, __float_as_int(hs.t), __float_as_int(hs.u), __float_as_int(hs.v));
}

}  // namespace re
