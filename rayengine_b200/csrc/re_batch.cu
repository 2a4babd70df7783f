// Batched wavefront path tracer: many scenes of uneven size (rope kd-tree
// meshes and exact-SDF terrains, each with its own camera and resolution)
// rendered by ONE persistent launch that pulls rays from per-bounce queues.
//
// The reference renders one scene per frame (cuda_render_frame,
// RE/cuda-src/renderer.cu:702-738, with trace_secondary_rays :435-492 for
// the bounce rays); batching is new.  Ray queries restate the reference's
// traversal (re_kd.cuh) and the exact SDF march (sphere_tracing.cuh:183-216,
// re_noise.cuh).
//
// Path (per pixel, 1 sample): ray 0 from the scene's camera; at a hit with
// bounce b < depth - 1 the path continues with a cosine-weighted Lambertian
// direction about the normal (createCoordinateSystem /
// uniformSampleHemisphere, RE/cuda-src/cuda_helper_functions.h:197-216, with
// cosine weighting), so the throughput after b bounces is albedo^b.  A miss
// at bounce b writes albedo^b * sky(d), sky(d) = 0.5 (1 + d.y); a hit at the
// last bounce writes 0.  Each pixel is written exactly once.
//
// Work distribution (no grid-wide barrier):
//   * primary rays come from a global pixel cursor over all scenes' pixels;
//   * a ray that continues is appended to the queue of (next bounce, scene
//     kind): a warp reserves slots with one atomic per distinct queue, writes
//     the 32-byte records and publishes each slot with a release store of the
//     frame's epoch into the slot's flag;
//   * idle lanes refill from the deepest non-empty queue (preferring the kind
//     the warp is already running, so meshes and terrains rarely share a
//     warp), claiming only published-or-reserved slots (compare-and-swap up to
//     the reserved count) and waiting, without blocking the warp, for a
//     claimed slot's flag;
//   * a warp leaves when the cursor is exhausted and every created ray has
//     finished (children are counted as created before their parent counts
//     as finished, so finished == created means nothing is in flight);
//   * the last block to leave resets the counters and advances the epoch, so
//     the same launch can be replayed from a CUDA graph.
// Every wait has an iteration bound after which the kernel sets the error
// flag and drops the ray.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "re_common.hpp"
#include "re_kd.cuh"
#include "re_math.cuh"
#include "re_noise.cuh"
#include "re_scene.hpp"

namespace re {
namespace batch {

constexpr uint32_t kMaxScenes = 64;
constexpr uint32_t kMaxDepth = 8;
constexpr uint32_t kMaxQueues = 2 * (kMaxDepth - 1);
constexpr uint32_t kMesh = RE_BATCH_MESH, kTerrain = RE_BATCH_TERRAIN;

// Counters (uint32), each contended one on its own 128-byte line so that
// atomics on different counters do not queue behind each other in one L2
// slice: the pixel cursor, finished rays per bounce, the frame epoch,
// blocks done and the error flag, reserved[q] / claimed[q] per queue; then
// (cold) the last frame's statistics.  Rays created of bounce 0 = pixels,
// of bounce b = the reserved counts of bounce b's two queues.
constexpr uint32_t kLine = 32;
enum : uint32_t {
  kCursor = 0 * kLine,
  kFin = 1 * kLine,  // + bounce * kLine: finished rays of that bounce
  kEpoch = (1 + kMaxDepth) * kLine,
  kDone = (2 + kMaxDepth) * kLine,
  kError = (2 + kMaxDepth) * kLine + 1,
  kReserved = (3 + kMaxDepth) * kLine,  // + q * kLine
  kClaimed = kReserved + kMaxQueues * kLine,
  kStats = kClaimed + kMaxQueues * kLine,  // + q
  kStatsPrimary = kStats + kMaxQueues,
  kStatsError = kStatsPrimary + 1,
  kNumCounters = kStats + kLine
};
static_assert(kStatsError < kNumCounters, "counter layout");
__host__ __device__ constexpr uint32_t fin_at(uint32_t b) { return kFin + b * kLine; }
__host__ __device__ constexpr uint32_t reserved_at(uint32_t q) { return kReserved + q * kLine; }
__host__ __device__ constexpr uint32_t claimed_at(uint32_t q) { return kClaimed + q * kLine; }

struct __align__(16) SceneDev {
  const uint2* nodes;
  const float4* leaves;
  const float4* tris;
  float bmin[3], bmax[3];
  uint32_t max_visits, stage, stage_off;
  uint32_t perm_slot, octaves, max_steps;
  float scale, amp, step_factor, eps, tmax;
  float ceiling;  // terrain: no surface above this height (|fBm| bound)
  CamDev cam;
  uint32_t w, h, kind, pix_off;
  float albedo;
  // the mesh's entry table (re_kd.cuh entry_node) for its camera rays
  const uint32_t* entry;
  float entry_scale[3];
  uint32_t entry_res;
};
// Shared memory holds SceneDev[num_scenes], then the noise tables (multiples
// of 512 bytes), then the staged nodes (uint2): the nodes stay 8-byte
// aligned only while the scene records are a multiple of 16 bytes.
static_assert(sizeof(SceneDev) % 16 == 0, "SceneDev must keep the staged nodes aligned");

struct BatchDev {
  const SceneDev* scenes;
  const uint8_t* perms;  // perm_count tables of 512 bytes (words in shared memory)
  uint32_t num_scenes, perm_count, stage_total, total_pixels;
  uint32_t depth, seed, refill_min, steps_per_trip;
  uint32_t pending_bound, loop_bound;  // polls of one slot flag, trips of the loop
  float mesh_bias;
  float4* queue;        // records: 2 float4 per slot
  uint32_t* flags;      // one per slot
  uint64_t qoff[kMaxQueues];  // first slot of queue q
  uint32_t qcap[kMaxQueues];  // slots of queue q (pixels of its kind)
  uint32_t* ctr;
  float* radiance;
  int4* primary;        // optional re_hit per pixel
  unsigned long long* totals;  // COUNT: inner nodes, leaves, triangle tests, field evaluations
};

__device__ __forceinline__ uint32_t ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ uint32_t scene_of(const SceneDev* sc, uint32_t n, uint32_t gpix) {
  uint32_t lo = 0, hi = n - 1;
  while (lo < hi) {
    uint32_t mid = (lo + hi + 1) >> 1;
    if (sc[mid].pix_off <= gpix) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ KdDev kd_of(const SceneDev& s) {
  KdDev kd;
  kd.nodes = s.nodes;
  kd.leaves = s.leaves;
  kd.tris = s.tris;
  kd.bmin = v3(s.bmin[0], s.bmin[1], s.bmin[2]);
  kd.bmax = v3(s.bmax[0], s.bmax[1], s.bmax[2]);
  kd.max_visits = s.max_visits;
  kd.stage = s.stage;
  kd.trunc = nullptr;
  return kd;
}

// kd_of with the mesh's entry table, for camera rays (which enter the scene
// box from outside); the counting kernel descends from the root, as the
// oracle does.
__device__ __forceinline__ KdDev kd_entry_of(const SceneDev& s) {
  KdDev kd = kd_of(s);
  kd.entry = s.entry;
  kd.entry_res = s.entry_res;
  kd.entry_scale = v3(s.entry_scale[0], s.entry_scale[1], s.entry_scale[2]);
  return kd;
}

// cosine-weighted direction about n (the AO frame's construction)
__device__ __forceinline__ V3 cosine_dir(V3 n, uint32_t seed, uint32_t gpix, uint32_t bounce) {
  V3 nt;
  if (fabsf(n.x) > fabsf(n.y)) {
    float iv = 1.0f / sqrtf(__fmaf_rn(n.z, n.z, n.x * n.x));
    nt = v3(n.z * iv, 0.0f, -n.x * iv);
  } else {
    float iv = 1.0f / sqrtf(__fmaf_rn(n.z, n.z, n.y * n.y));
    nt = v3(0.0f, -n.z * iv, n.y * iv);
  }
  V3 nb = cross(n, nt);
  uint32_t h1 = hash_u32(seed, gpix, 2u * bounce), h2 = hash_u32(seed, gpix, 2u * bounce + 1u);
  float u1 = (float)(h1 >> 8) * 5.9604644775390625e-08f;
  float u2 = (float)(h2 >> 8) * 5.9604644775390625e-08f;
  float r = sqrtf(u1);
  float sn, cs;
  sincos_2pi(u2, sn, cs);
  float lx = r * cs, ly = sqrtf(1.0f - u1), lz = r * sn;
  return v3(__fmaf_rn(lz, nt.x, __fmaf_rn(ly, n.x, lx * nb.x)),
            __fmaf_rn(lz, nt.y, __fmaf_rn(ly, n.y, lx * nb.y)),
            __fmaf_rn(lz, nt.z, __fmaf_rn(ly, n.z, lx * nb.z)));
}

__device__ __forceinline__ float miss_radiance(float albedo, uint32_t bounce, V3 d) {
  float pw = 1.0f;
  for (uint32_t i = 0; i < bounce; ++i) pw *= albedo;
  return pw * (0.5f * (1.0f + d.y));
}

enum : uint32_t { kIdle = 0, kPending = 1, kLive = 2 };
enum : uint32_t { kMarch = 0, kNormal = 1 };
// Default wait bounds (re_batch_set_wait_bounds lowers them for tests).
constexpr uint32_t kPendingBound = 1u << 22;  // polls of one slot flag
constexpr uint32_t kLoopBound = 1u << 22;     // trips of the persistent loop

// Bounce b's queues are closed (no ray of bounce b can still be created)
// once the pixel cursor is exhausted and every ray of bounce b - 1 has
// finished.  Bit b of the result, b = 1 .. depth; bit depth = the frame is
// done.  Each bounce's created count is read only after its predecessor's
// finished count compared equal (a control dependency orders the loads), so
// it is final when read: its producers all finished first.
__device__ __forceinline__ uint32_t closed_mask(const uint32_t* ctr, const BatchDev& B) {
  uint32_t mask = 0, created = B.total_pixels;
  for (uint32_t b = 1; b <= B.depth; ++b) {
    if (ld_relaxed(&ctr[fin_at(b - 1)]) != created) break;
    mask |= 1u << b;
    if (b == B.depth) break;
    created = ld_relaxed(&ctr[reserved_at(2 * (b - 1))]) + ld_relaxed(&ctr[reserved_at(2 * (b - 1) + 1)]);
  }
  return mask;
}

// Launch bounds: blocks of up to 256 threads, 4 resident per SM (64
// registers, 32 warps per SM).  Measured on the 8-scene batch: 22.0 ms
// against 30.4 ms with 122 registers and 16 warps, despite the spills.
#ifndef RE_BATCH_MIN_BLOCKS
#define RE_BATCH_MIN_BLOCKS 4
#endif
#ifndef RE_BATCH_MAX_THREADS
#define RE_BATCH_MAX_THREADS 256
#endif

// WORDS: the terrain permutation tables in shared memory as perm_word()
// entries (2 KB per seed), else as bytes (512 B per seed; batches with
// more than kWordTablesMax seeds, where word tables would cost blocks per SM).
template <bool COUNT, bool WORDS>
__global__ void __launch_bounds__(RE_BATCH_MAX_THREADS, RE_BATCH_MIN_BLOCKS) k_batch(BatchDev B) {
  extern __shared__ uint4 smem_u4[];
  SceneDev* sc = reinterpret_cast<SceneDev*>(smem_u4);
  uint8_t* sperm = reinterpret_cast<uint8_t*>(sc + B.num_scenes);
  uint32_t* sperm_w = reinterpret_cast<uint32_t*>(sperm);
  uint2* snodes = reinterpret_cast<uint2*>(sperm + (WORDS ? 4u : 1u) * 512u * B.perm_count);
  uint32_t* sfin = reinterpret_cast<uint32_t*>(snodes + B.stage_total);  // [warp][bounce]
  {
    const uint32_t* src = reinterpret_cast<const uint32_t*>(B.scenes);
    uint32_t* dst = reinterpret_cast<uint32_t*>(sc);
    for (uint32_t i = threadIdx.x; i < B.num_scenes * (uint32_t)(sizeof(SceneDev) / 4); i += blockDim.x)
      dst[i] = src[i];
    for (uint32_t i = threadIdx.x; i < 512u * B.perm_count; i += blockDim.x) {
      if (WORDS)
        sperm_w[i] = perm_word(B.perms[i]);
      else
        sperm[i] = B.perms[i];
    }
    for (uint32_t i = threadIdx.x; i < (blockDim.x / 32u) * kMaxDepth; i += blockDim.x) sfin[i] = 0u;
    __syncthreads();
    for (uint32_t s = 0; s < B.num_scenes; ++s)
      for (uint32_t i = threadIdx.x; i < sc[s].stage; i += blockDim.x)
        snodes[sc[s].stage_off + i] = __ldg(&sc[s].nodes[i]);
    __syncthreads();
  }
  uint32_t* ctr = B.ctr;
  const uint32_t epoch = ld_relaxed(&ctr[kEpoch]);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lt_mask = (1u << lane) - 1u;
  const uint32_t nq = 2u * (B.depth - 1u);
  uint32_t* wfin = sfin + (threadIdx.x >> 5) * kMaxDepth;  // this warp's unpublished counts

  uint32_t state = kIdle;
  uint32_t gpix = 0, scene = 0, bounce = 0, kind = kMesh;
  Trav tr;
  tr.live = false;
  // Terrain march state, kept in the Trav fields that a terrain ray leaves
  // unused (its ray is tr.o / tr.d) so that it takes no registers of its
  // own in this register-bound kernel: nx, ny, nz as float bits, the mode
  // (bit 3) and the normal tap (bits 0-2) in one word.  Every field is set
  // by a ray's start (trav_init or the terrain start below) before use.
  float& t = tr.t_entry;
  float& v_hit = tr.best_t;
  float& delta = tr.best_u;
  float& plus = tr.best_v;
  V3& p = tr.inv;
  uint32_t& steps = tr.visits;
  uint32_t& mode_tap = tr.node;
  uint32_t& nx_bits = tr.best_ref;
  uint32_t& ny_bits = tr.best_leaf;
  int32_t& nz_bits = tr.best_id;
  // A pending claim (queue, slot, polls so far) likewise: a lane waiting
  // for its record has no ray yet, and the ray's start overwrites these
  // fields only after the record has been read.
  uint32_t& pq = tr.best_ref;
  uint32_t& pslot = tr.best_leaf;
  uint32_t& polls = tr.visits;
  Counters cnt = {0, 0, 0, 0};
  uint32_t errors = 0;
  uint32_t fin_pending = 0;   // lane 0: finished rays in wfin
  uint32_t backoff = 32;      // lane 0: idle sleep, ns
  bool primary_done = false;  // lane 0: the pixel cursor has passed the end

  // publishes this warp's finished counts (after its reservations, which
  // completed when their atomics returned)
  auto flush = [&]() {
    __syncwarp();
    if (lane == 0 && fin_pending) {
      __threadfence();
      for (uint32_t b = 0; b < B.depth; ++b) {
        uint32_t v = wfin[b];
        if (v) {
          atomicAdd(&ctr[fin_at(b)], v);
          wfin[b] = 0u;
        }
      }
      fin_pending = 0;
    }
    __syncwarp();
  };

  uint32_t trip = 0;
  for (; trip < B.loop_bound; ++trip) {
    // ---- pending claims: the slot's record is published once its flag holds this epoch
    if (state == kPending) {
      // The flag is polled with a relaxed load (an acquire load would
      // invalidate this SM's L1, which every other warp's traversal uses).
      // The record is read only after the flag compared equal (a control
      // dependency: GPUs do not issue loads past an unresolved branch) and
      // from L2 (ld.global.cg), where the producer's release store made it
      // visible before the flag.
      if (ld_relaxed(&B.flags[B.qoff[pq] + pslot]) == epoch) {
        const float4* rec = B.queue + 2 * (B.qoff[pq] + pslot);
        float4 A = __ldcg(rec), Bv = __ldcg(rec + 1);
        uint32_t tag = __float_as_uint(Bv.w);
        gpix = tag & 0x0FFFFFFFu;
        bounce = tag >> 28;
        scene = scene_of(sc, B.num_scenes, gpix);
        kind = sc[scene].kind;
        V3 o = v3(A.x, A.y, A.z), d = v3(Bv.x, Bv.y, Bv.z);
        if (kind == kMesh) {
          trav_init(tr, kd_of(sc[scene]), o, d, K_INF, __float_as_uint(A.w));
        } else {
          tr.o = o;
          tr.d = d;
          t = 0.f;
          steps = 0;
          mode_tap = kMarch << 3;
        }
        state = kLive;
      } else {
        ++polls;
      }
    }
    // a warp with no live ray publishes its finished counts: its pending
    // claims may wait on exactly those counts to see their queue close
    if (__ballot_sync(0xFFFFFFFFu, state == kLive) == 0u && __shfl_sync(0xFFFFFFFFu, fin_pending, 0) != 0u)
      flush();
    // claims ahead of the producers: retire those whose queue closed short
    // of their slot (checked every 64 unsuccessful polls)
    if (__ballot_sync(0xFFFFFFFFu, state == kPending && polls != 0u && (polls & 63u) == 0u)) {
      uint32_t mask = 0;
      if (lane == 0) mask = closed_mask(ctr, B);
      mask = __shfl_sync(0xFFFFFFFFu, mask, 0);
      if (state == kPending && ((mask >> (pq / 2u + 1u)) & 1u)) {
        if (pslot >= ld_relaxed(&ctr[reserved_at(pq)])) state = kIdle;  // never filled
      }
      if (state == kPending && polls >= B.pending_bound) {
        errors = 1;
        state = kIdle;
      }
    }
    // ---- refill idle lanes
    uint32_t idle = __ballot_sync(0xFFFFFFFFu, state == kIdle);
    uint32_t nidle = __popc(idle);
    if (nidle != 0u && (nidle >= B.refill_min || nidle == 32u)) {
      uint32_t live_mesh = __ballot_sync(0xFFFFFFFFu, state != kIdle && kind == kMesh);
      uint32_t live_terr = __ballot_sync(0xFFFFFFFFu, state != kIdle && kind == kTerrain);
      // lane q reads queue q's counters: one round trip for all queues
      uint32_t avail = 0;
      if (lane < nq) {
        uint32_t r = ld_relaxed(&ctr[reserved_at(lane)]), c = ld_relaxed(&ctr[claimed_at(lane)]);
        avail = r > c ? r - c : 0u;
      }
      uint32_t src = 0xFFFFFFFFu, base = 0, k = 0;
      const uint32_t first = live_terr > live_mesh ? kTerrain : kMesh;
      for (int b = (int)B.depth - 1; b >= 1 && k == 0; --b) {
        for (uint32_t j = 0; j < 2 && k == 0; ++j) {
          uint32_t q = 2u * (uint32_t)(b - 1) + (j == 0 ? first : 1u - first);
          uint32_t av = __shfl_sync(0xFFFFFFFFu, avail, q);
          if (av == 0u) continue;
          // atomicAdd claims pipeline in L2 (a compare-and-swap loop
          // serialises thousands of warps); a claim that races past the
          // reserved count waits for its slot or retires when the queue closes
          k = min(nidle, av);
          if (lane == 0) base = atomicAdd(&ctr[claimed_at(q)], k);
          src = q;
        }
      }
      if (k == 0 && lane == 0 && !primary_done) {
        base = atomicAdd(&ctr[kCursor], nidle);
        k = base < B.total_pixels ? min(nidle, B.total_pixels - base) : 0u;
        if (k) src = 0xFFFFFFFEu;
        if (base + nidle >= B.total_pixels) primary_done = true;
      }
      src = __shfl_sync(0xFFFFFFFFu, src, 0);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      k = __shfl_sync(0xFFFFFFFFu, k, 0);
      uint32_t rank = __popc(idle & lt_mask);
      if (state == kIdle && rank < k) {
        if (src == 0xFFFFFFFEu) {
          gpix = base + rank;
          bounce = 0;
          scene = scene_of(sc, B.num_scenes, gpix);
          kind = sc[scene].kind;
          const SceneDev& S = sc[scene];
          uint32_t lp = gpix - S.pix_off;
          V3 o, d;
          generate_ray(S.cam, S.w, S.h, lp % S.w, lp / S.w, o, d);
          if (kind == kMesh) {
            trav_init(tr, COUNT ? kd_of(S) : kd_entry_of(S), o, d, K_INF, 0u);
          } else {
            tr.o = o;
            tr.d = d;
            t = 0.f;
            steps = 0;
            mode_tap = kMarch << 3;
          }
          state = kLive;
        } else if (base + rank < B.qcap[src]) {
          // a claim at or past the queue's capacity can never be filled
          // (each pixel adds at most one ray per bounce): it is dropped
          // here and its flag is never read
          pq = src;
          pslot = base + rank;
          polls = 0;
          state = kPending;
          kind = src & 1u;
        }
      }
    }
    if (__ballot_sync(0xFFFFFFFFu, state != kIdle) == 0u) {
      // nothing in this warp: publish its finished counts, then leave once
      // every bounce is closed (all created rays have finished)
      flush();
      uint32_t leave = 0;
      if (lane == 0) {
        if (!primary_done) primary_done = ld_relaxed(&ctr[kCursor]) >= B.total_pixels;
        if (primary_done) leave = (closed_mask(ctr, B) >> B.depth) & 1u;
        if (!leave) {
          __nanosleep(backoff);
          backoff = min(2u * backoff, 4096u);
        }
      }
      if (__shfl_sync(0xFFFFFFFFu, leave, 0)) break;
      continue;
    }
    backoff = 32;
    // ---- one step of every live ray
    bool done = false, hit = false;
    V3 n = {0.f, 0.f, 1.f}, hp = {0.f, 0.f, 0.f};
    uint32_t start_leaf = 0;
    float hit_t = 0.f, hit_u = 0.f, hit_v = 0.f;
    int32_t hit_id = -1;
    if (state == kLive) {
      const SceneDev& S = sc[scene];
      if (kind == kMesh) {
        KdDev kd = kd_of(S);
        // up to steps_per_trip leaves before the warp's bookkeeping runs again
        for (uint32_t it = 0; it < B.steps_per_trip && tr.live; ++it)
          trav_step<0, false, COUNT>(tr, kd, snodes + S.stage_off, cnt);
        if (!tr.live) {
          done = true;
          hit = tr.best_id >= 0;
          if (hit) {
            hit_t = tr.best_t;
            hit_u = tr.best_u;
            hit_v = tr.best_v;
            hit_id = tr.best_id;
            start_leaf = tr.best_leaf;
            const float4* T = S.tris + 3 * (size_t)tr.best_ref;
            float4 T1 = __ldg(T + 1), T2 = __ldg(T + 2);
            n = normalize(cross(v3(T1.x, T1.y, T1.z), v3(T2.x, T2.y, T2.z)));
            if (dot(n, tr.d) > 0.0f) n = v3(-n.x, -n.y, -n.z);
            V3 q = v3(__fmaf_rn(hit_t, tr.d.x, tr.o.x), __fmaf_rn(hit_t, tr.d.y, tr.o.y),
                      __fmaf_rn(hit_t, tr.d.z, tr.o.z));
            hp = v3(__fmaf_rn(n.x, B.mesh_bias, q.x), __fmaf_rn(n.y, B.mesh_bias, q.y),
                    __fmaf_rn(n.z, B.mesh_bias, q.z));
          }
        }
      } else {
        const auto P = [&] {
          if constexpr (WORDS)
            return PermWords{sperm_w + 512u * S.perm_slot};
          else
            return PermBytes{sperm + 512u * S.perm_slot};
        }();
        for (uint32_t it = 0; it < B.steps_per_trip && !done; ++it) {
        V3 qp;
        if ((mode_tap >> 3) == kMarch) {
          qp = v3(__fmaf_rn(t, tr.d.x, tr.o.x), __fmaf_rn(t, tr.d.y, tr.o.y),
                  __fmaf_rn(t, tr.d.z, tr.o.z));
        } else {
          uint32_t tap = mode_tap & 7u;
          float sd = (tap & 1u) ? -delta : delta;
          qp = p;
          if (tap < 2) qp.x = p.x + sd;
          else if (tap < 4) qp.y = p.y + sd;
          else qp.z = p.z + sd;
        }
        float v = terrain_density(P, qp, S.octaves, S.scale, S.amp);
        if (COUNT) ++cnt.status;  // field evaluations
        if ((mode_tap >> 3) == kMarch) {
          ++steps;
          if (v < S.eps) {
            p = qp;
            v_hit = v;
            delta = fmaxf(0.002f * t, 1e-3f);
            mode_tap = kNormal << 3;  // tap 0
          } else {
            t = __fmaf_rn(S.step_factor, v, t);
            // going up above the ceiling it can only miss: stop early (the
            // result, a miss with this direction, is what the march reaches)
            if (t > S.tmax || steps >= S.max_steps || (tr.d.y >= 0.0f && qp.y > S.ceiling))
              done = true;
          }
        } else {
          uint32_t tap = mode_tap & 7u;
          if ((tap & 1u) == 0u) {
            plus = v;
          } else {
            float diff = plus - v;
            if (tap == 1) nx_bits = __float_as_uint(diff);
            else if (tap == 3) ny_bits = __float_as_uint(diff);
            else nz_bits = __float_as_int(diff);
          }
          if (tap == 5) {
            float nx = __uint_as_float(nx_bits), ny = __uint_as_float(ny_bits),
                  nz = __int_as_float(nz_bits);
            done = true;
            hit = true;
            hit_t = t;
            hit_id = 0;
            float gl = sqrtf(__fmaf_rn(nz, nz, __fmaf_rn(ny, ny, nx * nx)));
            n = normalize(v3(nx, ny, nz));
            // leave the surface: the march may stop inside (v_hit < 0)
            float off = fmaxf(-v_hit, 0.0f) / (gl / (2.0f * delta)) + 2e-3f;
            hp = v3(__fmaf_rn(n.x, off, p.x), __fmaf_rn(n.y, off, p.y), __fmaf_rn(n.z, off, p.z));
          } else {
            ++mode_tap;
          }
        }
        }
      }
    }
    // ---- finished rays: write or continue the path
    bool push = false;
    float4 R0 = make_float4(0.f, 0.f, 0.f, 0.f), R1 = R0;
    uint32_t qn = 0;
    if (done) {
      const SceneDev& S = sc[scene];
      if (bounce == 0 && B.primary)
        B.primary[gpix] = make_int4(hit_id, __float_as_int(hit ? hit_t : K_INF),
                                    __float_as_int(hit_u), __float_as_int(hit_v));
      if (hit && bounce + 1u < B.depth) {
        V3 nd = cosine_dir(n, B.seed, gpix, bounce);
        push = true;
        qn = 2u * bounce + kind;
        R0 = make_float4(hp.x, hp.y, hp.z, __uint_as_float(start_leaf));
        R1 = make_float4(nd.x, nd.y, nd.z, __uint_as_float(gpix | ((bounce + 1u) << 28)));
      } else {
        B.radiance[gpix] = hit ? 0.0f : miss_radiance(S.albedo, bounce, tr.d);
      }
      state = kIdle;
    }
    // ---- append continuations, one atomic per distinct queue
    uint32_t pushers = __ballot_sync(0xFFFFFFFFu, push);
    if (pushers) {
      uint32_t slot = 0;
      if (push) {
        uint32_t peers = __match_any_sync(pushers, qn);
        uint32_t leader = __ffs(peers) - 1u;
        uint32_t b0 = 0;
        if (lane == leader) b0 = atomicAdd(&ctr[reserved_at(qn)], (uint32_t)__popc(peers));
        b0 = __shfl_sync(peers, b0, leader);
        slot = b0 + __popc(peers & lt_mask);
        float4* rec = B.queue + 2 * (B.qoff[qn] + slot);
        __stcg(rec, R0);
        __stcg(rec + 1, R1);
        // the release store orders this lane's record before its flag
        st_release(&B.flags[B.qoff[qn] + slot], epoch);
      }
    }
    // finished rays are counted per warp and bounce in shared memory and
    // published when the warp runs dry (or every 1024): their children were
    // reserved first, so a published count never runs ahead of the created
    // count
    uint32_t fin = __ballot_sync(0xFFFFFFFFu, done);
    if (done) atomicAdd(&wfin[bounce], 1u);
    if (lane == 0) fin_pending += (uint32_t)__popc(fin);
    if (__shfl_sync(0xFFFFFFFFu, fin_pending, 0) >= 1024u) flush();
  }
  flush();
  if (trip >= B.loop_bound) errors = 1;
  if (COUNT) {
    uint32_t v4[4] = {cnt.inner, cnt.leaf, cnt.tests, cnt.status};
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      uint32_t x = __reduce_add_sync(0xFFFFFFFFu, v4[f]);
      if (lane == 0) atomicAdd(&B.totals[f], (unsigned long long)x);
    }
  }
  if (errors) atomicExch(&ctr[kError], 1u);
  // ---- the last block resets the counters for the next frame
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    uint32_t dn = atomicAdd(&ctr[kDone], 1u);
    if (dn == gridDim.x - 1u) {
      __threadfence();
      for (uint32_t q = 0; q < nq; ++q) {
        ctr[kStats + q] = ctr[reserved_at(q)];
        ctr[reserved_at(q)] = 0u;
        ctr[claimed_at(q)] = 0u;
      }
      for (uint32_t b = 0; b < kMaxDepth; ++b) ctr[fin_at(b)] = 0u;
      ctr[kStatsPrimary] = min(ctr[kCursor], B.total_pixels);
      ctr[kStatsError] = ctr[kError];
      ctr[kCursor] = 0u;
      ctr[kError] = 0u;
      ctr[kDone] = 0u;
      __threadfence();
      ctr[kEpoch] = epoch + 1u;
    }
  }
}

}  // namespace batch
}  // namespace re

// ------------------------------------------------------------------ host
struct re_batch {
  int device = 0;
  uint32_t num_scenes = 0, depth = 4, seed = 0;
  float mesh_bias = 1e-4f;
  std::vector<re::batch::SceneDev> host_scenes;
  std::vector<const re_scene*> meshes;
  std::vector<uint8_t> perms;
  uint64_t total_pixels = 0;
  std::vector<uint64_t> offsets;
  uint64_t cap[2] = {0, 0};  // pixels of mesh / terrain scenes (queue capacity)
  re::batch::SceneDev* d_scenes = nullptr;
  uint8_t* d_perms = nullptr;
  float4* d_queue = nullptr;
  uint32_t* d_flags = nullptr;
  uint32_t* d_ctr = nullptr;
  uint64_t qoff[re::batch::kMaxQueues] = {};
  re_batch_tuning tune = {256, 8, 0, 8};
  uint32_t pending_bound = 0, loop_bound = 0;  // 0: the kernel's defaults
  // captured frame
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  float* g_radiance = nullptr;
  re_hit* g_primary = nullptr;
  re_batch_tuning g_tune = {0, 0, 0, 0};
  cudaStream_t g_stream = nullptr;
};

namespace re {
namespace {

using namespace batch;

CamDev cam_of(const re_camera& c) {
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

void free_graph(re_batch* b) {
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  b->exec = nullptr;
  b->graph = nullptr;
}

// Staging: the first `stage_nodes` nodes (breadth-first top of the tree) of
// every mesh scene are copied to shared memory.
uint32_t layout_stage(re_batch* b, uint32_t stage_nodes) {
  uint32_t off = 0;
  for (uint32_t i = 0; i < b->num_scenes; ++i) {
    SceneDev& s = b->host_scenes[i];
    if (s.kind != kMesh) {
      s.stage = 0;
      s.stage_off = 0;
      continue;
    }
    uint32_t n = (uint32_t)std::min<size_t>(stage_nodes, b->meshes[i]->host.nodes.size());
    s.stage = n;
    s.stage_off = off;
    off += n;
  }
  return off;
}

// Word tables while the batch has at most this many terrain seeds (32 KB).
constexpr uint32_t kWordTablesMax = 16;

bool word_tables(const re_batch* b) { return b->perms.size() / 512 <= kWordTablesMax; }

size_t smem_bytes(const re_batch* b, uint32_t stage_total, uint32_t block_threads) {
  return b->num_scenes * sizeof(SceneDev) + (word_tables(b) ? 4u : 1u) * b->perms.size() +
         (size_t)stage_total * sizeof(uint2) + (size_t)(block_threads / 32) * kMaxDepth * 4;
}

// Scene table (with this tuning's staging offsets) to the device and the
// kernel's shared-memory limit; outside any stream capture.
re_status prepare(re_batch* b, const re_batch_tuning& tn, cudaStream_t st) {
  uint32_t stage_total = layout_stage(b, tn.stage_nodes);
  RE_CUDA(cudaMemcpyAsync(b->d_scenes, b->host_scenes.data(), b->num_scenes * sizeof(SceneDev),
                          cudaMemcpyHostToDevice, st));
  RE_CUDA(cudaStreamSynchronize(st));
  int bytes = (int)smem_bytes(b, stage_total, 512);
  RE_CUDA(cudaFuncSetAttribute(k_batch<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  RE_CUDA(cudaFuncSetAttribute(k_batch<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  RE_CUDA(cudaFuncSetAttribute(k_batch<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  RE_CUDA(cudaFuncSetAttribute(k_batch<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
  return RE_OK;
}

// One frame: a single launch of the persistent kernel (prepare() first).
re_status launch(re_batch* b, float* d_radiance, re_hit* d_primary, cudaStream_t st,
                 const re_batch_tuning& tn, unsigned long long* totals = nullptr) {
  uint32_t stage_total = layout_stage(b, tn.stage_nodes);
  size_t smem = smem_bytes(b, stage_total, tn.block_threads);
  int per_sm = 0;
  auto kern = word_tables(b) ? (totals ? k_batch<true, true> : k_batch<false, true>)
                             : (totals ? k_batch<true, false> : k_batch<false, false>);
  RE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, (int)tn.block_threads,
                                                        smem));
  if (per_sm < 1) return fail(RE_ERR_LIMIT, "re_batch: tuning does not fit on an SM");
  BatchDev B;
  B.scenes = b->d_scenes;
  B.perms = b->d_perms;
  B.num_scenes = b->num_scenes;
  B.perm_count = (uint32_t)(b->perms.size() / 512);
  B.stage_total = stage_total;
  B.total_pixels = (uint32_t)b->total_pixels;
  B.depth = b->depth;
  B.seed = b->seed;
  B.refill_min = tn.refill_min;
  B.steps_per_trip = tn.steps_per_trip ? tn.steps_per_trip : 1u;
  B.pending_bound = b->pending_bound ? b->pending_bound : kPendingBound;
  B.loop_bound = b->loop_bound ? b->loop_bound : kLoopBound;
  B.mesh_bias = b->mesh_bias;
  B.queue = b->d_queue;
  B.flags = b->d_flags;
  for (uint32_t q = 0; q < kMaxQueues; ++q) {
    B.qoff[q] = b->qoff[q];
    B.qcap[q] = q < 2 * (b->depth - 1) ? (uint32_t)b->cap[q & 1u] : 0u;
  }
  B.ctr = b->d_ctr;
  B.radiance = d_radiance;
  B.primary = reinterpret_cast<int4*>(d_primary);
  B.totals = totals;
  kern<<<per_sm * sm_count(), tn.block_threads, smem, st>>>(B);
  RE_CHECK_LAUNCH("re_batch: launch");
  return RE_OK;
}

re_status check_tuning(const re_batch_tuning& t) {
  if (t.block_threads == 0 || t.block_threads % 32 != 0 || t.block_threads > RE_BATCH_MAX_THREADS)
    return fail(RE_ERR_INVALID_ARG, "re_batch: block_threads must be a multiple of 32 in [32, %d]",
                RE_BATCH_MAX_THREADS);
  if (t.refill_min == 0 || t.refill_min > 32)
    return fail(RE_ERR_INVALID_ARG, "re_batch: refill_min must be in [1, 32]");
  if (t.stage_nodes > 4096) return fail(RE_ERR_INVALID_ARG, "re_batch: stage_nodes > 4096");
  if (t.steps_per_trip > 256) return fail(RE_ERR_INVALID_ARG, "re_batch: steps_per_trip > 256");
  return RE_OK;
}

}  // namespace
}  // namespace re

extern "C" {

RE_API re_status re_batch_create(const re_batch_scene* scenes, uint32_t n, const re_path_params* pp,
                                 re_batch** out) {
  using namespace re::batch;
  if (!scenes || !pp || !out || n == 0) return re::fail(RE_ERR_INVALID_ARG, "re_batch_create: bad arguments");
  *out = nullptr;
  if (n > kMaxScenes) return re::fail(RE_ERR_LIMIT, "re_batch_create: more than %u scenes", kMaxScenes);
  if (pp->max_depth < 1 || pp->max_depth > kMaxDepth)
    return re::fail(RE_ERR_INVALID_ARG, "re_batch_create: max_depth must be in [1, %u]", kMaxDepth);
  re_batch* b = new (std::nothrow) re_batch();
  if (!b) return re::fail(RE_ERR_OUT_OF_MEMORY, "re_batch_create: host allocation");
  RE_CUDA(cudaGetDevice(&b->device));
  b->num_scenes = n;
  b->depth = pp->max_depth;
  b->seed = pp->seed;
  b->mesh_bias = pp->mesh_bias;
  b->host_scenes.resize(n);
  b->meshes.assign(n, nullptr);
  b->offsets.resize(n);
  std::vector<uint32_t> perm_seeds;
  uint64_t off = 0;
  for (uint32_t i = 0; i < n; ++i) {
    const re_batch_scene& s = scenes[i];
    SceneDev d;
    std::memset(&d, 0, sizeof(d));
    if (s.width < 2 || s.height < 2 || !(s.albedo >= 0.f && s.albedo <= 1.f)) {
      delete b;
      return re::fail(RE_ERR_INVALID_ARG, "re_batch_create: scene %u: bad size or albedo", i);
    }
    d.cam = re::cam_of(s.camera);
    d.w = s.width;
    d.h = s.height;
    d.kind = s.kind;
    d.albedo = s.albedo;
    d.pix_off = (uint32_t)off;
    if (s.kind == RE_BATCH_MESH) {
      const re_scene* m = s.mesh;
      int dev = -1;
      if (!m || !m->d_nodes || (cudaGetDevice(&dev), dev != m->device)) {
        delete b;
        return re::fail(RE_ERR_INVALID_ARG, "re_batch_create: scene %u: no mesh on this device", i);
      }
      b->meshes[i] = m;
      d.nodes = m->d_nodes;
      d.leaves = m->d_leaves;
      d.tris = m->d_tris;
      for (int k = 0; k < 3; ++k) {
        d.bmin[k] = m->host.bmin[k];
        d.bmax[k] = m->host.bmax[k];
      }
      d.max_visits = m->max_visits;
      d.entry = m->d_entry;
      d.entry_res = m->d_entry ? re::kEntryRes : 0u;
      for (int k = 0; k < 3; ++k) {
        const float ext = m->host.bmax[k] - m->host.bmin[k];
        d.entry_scale[k] = ext > 0.f ? (float)re::kEntryRes / ext : 0.f;
      }
      b->cap[0] += (uint64_t)s.width * s.height;
    } else if (s.kind == RE_BATCH_TERRAIN) {
      const re_sdf_params& f = s.field;
      if (f.octaves < 1 || f.octaves > 16 || !(f.step_factor > 0.f) || !(f.tmax > 0.f) ||
          f.max_steps == 0) {
        delete b;
        return re::fail(RE_ERR_INVALID_ARG, "re_batch_create: scene %u: bad field", i);
      }
      auto it = std::find(perm_seeds.begin(), perm_seeds.end(), f.seed);
      d.perm_slot = (uint32_t)(it - perm_seeds.begin());
      if (it == perm_seeds.end()) {
        perm_seeds.push_back(f.seed);
        uint32_t full[512];
        re::perlin_permutation(f.seed, full);
        for (int k = 0; k < 512; ++k) b->perms.push_back((uint8_t)full[k]);
      }
      d.octaves = f.octaves;
      d.max_steps = f.max_steps;
      d.scale = f.scale;
      d.amp = f.amplitude;
      d.step_factor = f.step_factor;
      d.eps = f.eps;
      d.tmax = f.tmax;
      // |Perlin| <= 2 (corner terms |g . r| <= 2, convex blend), so
      // |fBm| <= 2 (2 - 2^(1 - octaves)) and the density is positive above
      d.ceiling = 2.0f * std::fabs(f.amplitude) * (2.0f - std::ldexp(1.0f, 1 - (int)f.octaves)) + 1e-3f;
      b->cap[1] += (uint64_t)s.width * s.height;
    } else {
      delete b;
      return re::fail(RE_ERR_INVALID_ARG, "re_batch_create: scene %u: unknown kind", i);
    }
    b->offsets[i] = off;
    off += (uint64_t)s.width * s.height;
    b->host_scenes[i] = d;
  }
  if (off >= (1ull << 28)) {
    delete b;
    return re::fail(RE_ERR_LIMIT, "re_batch_create: more than 2^28 pixels in the batch");
  }
  b->total_pixels = off;
  // queue q = 2 * (bounce - 1) + kind holds at most one ray per pixel of that kind
  uint64_t slots = 0;
  uint32_t nq = 2 * (b->depth - 1);
  for (uint32_t q = 0; q < nq; ++q) {
    b->qoff[q] = slots;
    slots += b->cap[q & 1u];
  }
  cudaError_t e = cudaMalloc(&b->d_scenes, n * sizeof(SceneDev));
  if (e == cudaSuccess && !b->perms.empty()) e = cudaMalloc(&b->d_perms, b->perms.size());
  if (e == cudaSuccess && slots) e = cudaMalloc(&b->d_queue, slots * 2 * sizeof(float4));
  if (e == cudaSuccess && slots) e = cudaMalloc(&b->d_flags, slots * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_ctr, kNumCounters * sizeof(uint32_t));
  if (e == cudaSuccess && !b->perms.empty())
    e = cudaMemcpy(b->d_perms, b->perms.data(), b->perms.size(), cudaMemcpyHostToDevice);
  if (e == cudaSuccess && slots) e = cudaMemset(b->d_flags, 0, slots * sizeof(uint32_t));
  if (e == cudaSuccess) e = cudaMemset(b->d_ctr, 0, kNumCounters * sizeof(uint32_t));
  if (e == cudaSuccess) {
    uint32_t one = 1;  // epoch of the first frame (flags start at 0)
    e = cudaMemcpy(b->d_ctr + kEpoch, &one, 4, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    re_batch_destroy(b);
    return re::cuda_fail(e, "re_batch_create");
  }
  *out = b;
  return RE_OK;
}

RE_API re_status re_batch_destroy(re_batch* b) {
  if (!b) return RE_OK;
  re::free_graph(b);
  cudaFree(b->d_scenes);
  cudaFree(b->d_perms);
  cudaFree(b->d_queue);
  cudaFree(b->d_flags);
  cudaFree(b->d_ctr);
  delete b;
  return RE_OK;
}

RE_API re_status re_batch_pixels(const re_batch* b, uint64_t* total, uint64_t* offsets) {
  if (!b || !total) return re::fail(RE_ERR_INVALID_ARG, "re_batch_pixels: bad arguments");
  *total = b->total_pixels;
  if (offsets) std::memcpy(offsets, b->offsets.data(), b->num_scenes * sizeof(uint64_t));
  return RE_OK;
}

RE_API re_status re_batch_set_wait_bounds(re_batch* b, uint32_t pending_polls,
                                          uint32_t loop_trips) {
  if (!b) return re::fail(RE_ERR_INVALID_ARG, "re_batch_set_wait_bounds: null batch");
  b->pending_bound = pending_polls;
  b->loop_bound = loop_trips;
  re::free_graph(b);  // a captured frame holds the old bounds
  return RE_OK;
}

RE_API re_status re_batch_render(re_batch* b, float* d_radiance, re_hit* d_primary, void* stream) {
  if (!b || !d_radiance) return re::fail(RE_ERR_INVALID_ARG, "re_batch_render: bad arguments");
  re_status s = re::prepare(b, b->tune, (cudaStream_t)stream);
  if (s != RE_OK) return s;
  return re::launch(b, d_radiance, d_primary, (cudaStream_t)stream, b->tune);
}

RE_API re_status re_batch_render_graph(re_batch* b, float* d_radiance, re_hit* d_primary,
                                       void* stream) {
  if (!b || !d_radiance) return re::fail(RE_ERR_INVALID_ARG, "re_batch_render_graph: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  bool same = b->exec && b->g_radiance == d_radiance && b->g_primary == d_primary &&
              b->g_stream == st && std::memcmp(&b->g_tune, &b->tune, sizeof(b->tune)) == 0;
  if (!same) {
    re::free_graph(b);
    // the scene table and shared-memory limit are set outside the capture
    re_status ps = re::prepare(b, b->tune, st);
    if (ps != RE_OK) return ps;
    cudaStream_t cap = nullptr;
    RE_CUDA(cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal);
    re_status s = RE_OK;
    if (e == cudaSuccess) {
      s = re::launch(b, d_radiance, d_primary, cap, b->tune);
      cudaError_t e2 = cudaStreamEndCapture(cap, &b->graph);
      if (e == cudaSuccess) e = e2;
    }
    if (e == cudaSuccess && s == RE_OK) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
    cudaStreamDestroy(cap);
    if (s != RE_OK) return s;
    if (e != cudaSuccess) {
      re::free_graph(b);
      return re::cuda_fail(e, "re_batch_render_graph: capture");
    }
    b->g_radiance = d_radiance;
    b->g_primary = d_primary;
    b->g_stream = st;
    b->g_tune = b->tune;
  }
  RE_CUDA(cudaGraphLaunch(b->exec, st));
  return RE_OK;
}

// A frame with the work counters on: totals[0..3] = inner-node visits, leaf
// visits, triangle tests, terrain field evaluations.
RE_API re_status re_batch_counts(re_batch* b, float* d_radiance, void* stream, uint64_t* totals) {
  if (!b || !d_radiance || !totals) return re::fail(RE_ERR_INVALID_ARG, "re_batch_counts: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  unsigned long long* d = nullptr;
  RE_CUDA(cudaMalloc(&d, 4 * sizeof(unsigned long long)));
  cudaError_t e = cudaMemsetAsync(d, 0, 4 * sizeof(unsigned long long), st);
  re_status s = e == cudaSuccess ? re::prepare(b, b->tune, st) : re::cuda_fail(e, "re_batch_counts");
  if (s == RE_OK) s = re::launch(b, d_radiance, nullptr, st, b->tune, d);
  if (s == RE_OK) {
    e = cudaMemcpyAsync(totals, d, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) s = re::cuda_fail(e, "re_batch_counts");
  }
  cudaFree(d);
  return s;
}

RE_API re_status re_batch_stats_get(re_batch* b, uint64_t* rays, int* error) {
  using namespace re::batch;
  if (!b || !rays) return re::fail(RE_ERR_INVALID_ARG, "re_batch_stats_get: bad arguments");
  uint32_t c[kNumCounters];
  RE_CUDA(cudaMemcpy(c, b->d_ctr, sizeof(c), cudaMemcpyDeviceToHost));
  // rays[2 * bounce + kind]: bounce 0 counts every primary ray under kind 0
  for (uint32_t i = 0; i < 2 * b->depth; ++i) rays[i] = 0;
  rays[0] = c[kStatsPrimary];
  for (uint32_t q = 0; q < 2 * (b->depth - 1); ++q) rays[2 + q] = c[kStats + q];
  if (error) *error = (int)c[kStatsError];
  return RE_OK;
}

RE_API re_status re_batch_get_tuning(const re_batch* b, re_batch_tuning* out) {
  if (!b || !out) return re::fail(RE_ERR_INVALID_ARG, "re_batch_get_tuning: bad arguments");
  *out = b->tune;
  return RE_OK;
}

RE_API re_status re_batch_set_tuning(re_batch* b, const re_batch_tuning* t) {
  if (!b || !t) return re::fail(RE_ERR_INVALID_ARG, "re_batch_set_tuning: bad arguments");
  re_status s = re::check_tuning(*t);
  if (s != RE_OK) return s;
  b->tune = *t;
  return RE_OK;
}

// Times one frame per candidate (after a warm-up frame) and keeps the
// fastest: block size x refill threshold x staged nodes per mesh scene x
// leaves / field evaluations per trip.
RE_API re_status re_batch_autotune(re_batch* b, float* d_radiance, void* stream,
                                   re_batch_tuning* out, float* best_ms) {
  if (!b || !d_radiance) return re::fail(RE_ERR_INVALID_ARG, "re_batch_autotune: bad arguments");
  cudaStream_t st = (cudaStream_t)stream;
  const uint32_t blocks[] = {128, 256};
  const uint32_t refills[] = {8, 32};
  const uint32_t stages[] = {0, 512};
  const uint32_t trips[] = {1, 8, 64};
  cudaEvent_t e0, e1;
  RE_CUDA(cudaEventCreate(&e0));
  RE_CUDA(cudaEventCreate(&e1));
  re_batch_tuning best = b->tune;
  float best_t = 1e30f;
  re_status s = RE_OK;
  for (uint32_t bt : blocks)
    for (uint32_t rf : refills)
      for (uint32_t sg : stages)
        for (uint32_t tp : trips) {
        re_batch_tuning t = {bt, rf, sg, tp};
        size_t smem = re::smem_bytes(b, re::layout_stage(b, sg), bt);
        if (smem > 200 * 1024) continue;
        s = re::prepare(b, t, st);
        if (s != RE_OK) break;
        s = re::launch(b, d_radiance, nullptr, st, t);  // warm-up
        if (s != RE_OK) break;
        cudaEventRecord(e0, st);
        s = re::launch(b, d_radiance, nullptr, st, t);
        if (s != RE_OK) break;
        cudaEventRecord(e1, st);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) {
          s = re::cuda_fail(e, "re_batch_autotune");
          break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_t) {
          best_t = ms;
          best = t;
        }
      }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (s != RE_OK) return s;
  b->tune = best;
  s = re::prepare(b, best, st);
  if (s != RE_OK) return s;
  if (out) *out = best;
  if (best_ms) *best_ms = best_t;
  return RE_OK;
}

}  // extern "C"
