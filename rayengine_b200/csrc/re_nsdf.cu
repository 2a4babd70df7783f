// Neural SDF surrogate of the volumetric terrain (config 3 of the path).
//
// The reference has no learned component.  The network stands in for the
// fBm terrain density (sdf_functions.cuh:147-206, d(p) = p.y - 3 fBm(p/4) in
// the configs) during sphere tracing; the exact field stays the arbiter and
// finishes every hit (sphere_tracing.cuh:183-216 restated in re_noise.cu).
//
//   data      k_nsdf_data: 50% points uniform in the view box, 50% near the
//             surface (exact-traced camera hits + N(0, 0.02) offsets),
//             labelled by the exact field's first-order distance d / |grad d|
//   training  tcgen05 as well: k_tc_train_fwd (features, 4 MMA layers with
//             FP32 bias + softplus epilogues, head, L1 loss) and
//             k_tc_train_bwd per layer (dA_prev = dZ W and dW^T = A^T dZ, the
//             weight gradient accumulated in tensor memory over the CTA's
//             tiles), BF16 operands and FP32 accumulation; then k_reduce and
//             hand-written Adam; one step is captured once in a CUDA graph
//             and replayed
//   inference tcgen05 (sm_100a): 128-point tiles, BF16 operands in shared
//             memory (K-major canonical layout, no swizzle), FP32
//             accumulators in tensor memory, one elected thread issues the
//             MMAs and commits to an mbarrier; softplus epilogue from TMEM
//   tracing   k_nsdf_march (persistent, lane refill) steps by the network's
//             distance scaled by its measured Lipschitz bound until it is
//             within `switch_dist` of the surface, then k_sdf_refine finishes
//             the ray with exact-field steps and the exact normal.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <random>
#include <vector>

#include "re_common.hpp"
#include "re_noise.cuh"
#include "re_nsdf.cuh"

namespace re {
namespace nsdf {

// ------------------------------------------------------------ shared
struct FieldDev {
  uint32_t octaves, max_steps;
  float scale, amp, step_factor, eps, tmax;
};

__device__ __forceinline__ uint32_t mix32(uint32_t a, uint32_t b, uint32_t c) {
  return hash_u32(a, b, c);
}
__device__ __forceinline__ float u01(uint32_t h) { return (float)(h >> 8) * 5.9604644775390625e-08f; }

// ------------------------------------------------------ data generation
__global__ void __launch_bounds__(256) k_nsdf_data(PermTable perm, FieldDev f, CamDev cam,
                                                   uint32_t w, uint32_t h, float3 bmin, float3 bmax,
                                                   uint32_t n, uint32_t seed,
                                                   float4* __restrict__ out) {
  extern __shared__ uint32_t perm_smem[];
  load_perm(perm, perm_smem);
  Perm P = perm_view(perm_smem);
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float px = 0.f, py = 0.f, pz = 0.f;
    bool placed = false;
    if (i & 1u) {
      // near-surface sample: an exact-traced camera hit plus N(0, 0.02) per axis
      uint32_t pix = mix32(seed, i, 11u) % (w * h);
      V3 o, d;
      generate_ray(cam, w, h, pix % w, pix / w, o, d);
      float t = 0.f;
      for (uint32_t s = 0; s < f.max_steps; ++s) {
        V3 p = v3(__fmaf_rn(t, d.x, o.x), __fmaf_rn(t, d.y, o.y), __fmaf_rn(t, d.z, o.z));
        float dist = terrain_density(P, p, f.octaves, f.scale, f.amp);
        if (dist < f.eps) {
          float u1 = fmaxf(u01(mix32(seed, i, 12u)), 1e-7f), u2 = u01(mix32(seed, i, 13u));
          float u3 = fmaxf(u01(mix32(seed, i, 14u)), 1e-7f), u4 = u01(mix32(seed, i, 15u));
          float r1 = sqrtf(-2.f * __logf(u1)), r2 = sqrtf(-2.f * __logf(u3));
          float s1, c1, s2, c2;
          __sincosf(6.28318531f * u2, &s1, &c1);
          __sincosf(6.28318531f * u4, &s2, &c2);
          px = p.x + 0.02f * r1 * c1;
          py = p.y + 0.02f * r1 * s1;
          pz = p.z + 0.02f * r2 * c2;
          placed = px >= bmin.x && px <= bmax.x && py >= bmin.y && py <= bmax.y &&
                   pz >= bmin.z && pz <= bmax.z;
          break;
        }
        t = __fmaf_rn(f.step_factor, dist, t);
        if (t > f.tmax) break;
      }
    }
    if (!placed) {
      px = bmin.x + (bmax.x - bmin.x) * u01(mix32(seed, i, 1u));
      py = bmin.y + (bmax.y - bmin.y) * u01(mix32(seed, i, 2u));
      pz = bmin.z + (bmax.z - bmin.z) * u01(mix32(seed, i, 3u));
    }
    // label: first-order distance d / |grad d| of the exact field, clipped
    const float e = 1e-3f;
    float d0 = terrain_density(P, v3(px, py, pz), f.octaves, f.scale, f.amp);
    float gx = terrain_density(P, v3(px + e, py, pz), f.octaves, f.scale, f.amp) -
               terrain_density(P, v3(px - e, py, pz), f.octaves, f.scale, f.amp);
    float gy = terrain_density(P, v3(px, py + e, pz), f.octaves, f.scale, f.amp) -
               terrain_density(P, v3(px, py - e, pz), f.octaves, f.scale, f.amp);
    float gz = terrain_density(P, v3(px, py, pz + e), f.octaves, f.scale, f.amp) -
               terrain_density(P, v3(px, py, pz - e), f.octaves, f.scale, f.amp);
    float g = sqrtf(gx * gx + gy * gy + gz * gz) / (2.f * e);
    float label = d0 / fmaxf(g, 0.25f);
    label = fminf(fmaxf(label, -4.f), 4.f);
    out[i] = make_float4(px, py, pz, label);
  }
}

// ------------------------------------------------------------- training
// One step on a batch of B rows (a multiple of 512): k_pack_train packs the
// BF16 weights, k_tc_train_fwd runs the four hidden layers and the head on
// the tensor cores (128-row tiles) and stores what the backward pass needs,
// then k_tc_train_bwd runs once per hidden layer (4 -> 1): dZ = dA softplus'(Z),
// dA_prev = dZ W and the weight gradient dW^T = A_prev^T dZ, accumulated in
// tensor memory over the CTA's tiles; k_reduce sums the CTAs' partial
// gradients and k_adam updates the parameters.
constexpr int kRowsBwd = 512;   // batch granularity of the training API
constexpr int kTrRows = 128;    // rows per tensor-core tile (one thread each)

struct TrainBufs {
  __nv_bfloat16* x0;  // [B][128] BF16 features (the first layer's input)
  float* z[4];        // [B][64] pre-activations
  __nv_bfloat16* a[3];  // [B][64] BF16 activations of layers 1-3 (inputs of 2-4)
  float* da;          // [B][64] gradient w.r.t. the current layer's output
  float* da2;         // [B][64]
  float* part;        // [grid][kNumParams] partial gradients of W1..W4, b1..b4
  float* part_head;   // [B / 128][kHidden + 2] partial gradients of w5, b5 and the loss
};

// grad[p] = sum of the partial gradients; the loss of the step is appended
// to loss_hist.
__global__ void k_reduce(TrainBufs tb, uint32_t nbwd, uint32_t nfwd, float* __restrict__ grad,
                         float* __restrict__ loss_hist, const uint32_t* __restrict__ step_ctr,
                         uint32_t batch) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < (uint32_t)OFF_W5) {
    float s = 0.f;
    for (uint32_t b = 0; b < nbwd; ++b) s += tb.part[(size_t)b * kNumParams + p];
    grad[p] = s;
  } else if (p < (uint32_t)kNumParams + 1) {
    uint32_t c = p - OFF_W5;  // 0..63 w5, 64 b5, 65 loss
    float s = 0.f;
    for (uint32_t b = 0; b < nfwd; ++b) s += tb.part_head[(size_t)b * (kHidden + 2) + c];
    if (p < (uint32_t)kNumParams)
      grad[p] = s;
    else if (loss_hist)
      loss_hist[*step_ctr] = s / (float)batch;
  }
}

__global__ void k_adam(float* __restrict__ params, const float* __restrict__ grad,
                       float* __restrict__ m, float* __restrict__ v, uint32_t* __restrict__ step_ctr,
                       float lr) {
  uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t step = *step_ctr + 1;
  if (p < (uint32_t)kNumParams) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    float g = grad[p];
    float mm = b1 * m[p] + (1.f - b1) * g;
    float vv = b2 * v[p] + (1.f - b2) * g * g;
    m[p] = mm;
    v[p] = vv;
    float mh = mm / (1.f - powf(b1, (float)step));
    float vh = vv / (1.f - powf(b2, (float)step));
    params[p] -= lr * mh / (sqrtf(vh) + eps);
  }
}

__global__ void k_step_inc(uint32_t* step_ctr) { *step_ctr += 1; }

// ------------------------------------------------ tensor-core inference
// Canonical K-major BF16 layout without swizzle: 8 rows x 8 k-elements
// (16 B per row) form a 128-byte core matrix; core matrices follow each
// other along K every 128 B (LBO) and along rows every K*16 B (SBO).
__host__ __device__ __forceinline__ uint32_t canon_off(uint32_t row, uint32_t k, uint32_t K) {
  return (row >> 3) * (K * 16u) + (k >> 3) * 128u + (row & 7u) * 16u + (k & 7u) * 2u;
}

// Packed inference weights: W1 (64x128), W2..W4 (64x64) in the canonical
// layout, then FP32 b1..b4, w5 (BF16-rounded) and b5.
constexpr uint32_t kPackW1 = kHidden * kIn * 2;            // 16384
constexpr uint32_t kPackWh = kHidden * kHidden * 2;        // 8192
constexpr uint32_t kPackWBytes = kPackW1 + 3 * kPackWh;    // 40960
constexpr uint32_t kPackFloats = 4 * kHidden + kHidden + 1;
constexpr uint32_t kPackBytes = kPackWBytes + kPackFloats * 4;
constexpr uint32_t kBiasCol = 99;    // feature = 1.0; W1 column = BF16(b1)
constexpr uint32_t kBiasColLo = 100; // feature = 1.0; W1 column = b1 - BF16(b1)

// The inference kernels feed 1.0 at W1 columns 99 and 100 (unused by the
// features), so those columns carry b1 as a BF16 high part and a BF16
// remainder and the first layer's bias comes out of the MMA.
__global__ void k_pack(const float* __restrict__ params, unsigned char* __restrict__ pack) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < (uint32_t)(kHidden * kIn)) {
    uint32_t n = i / kIn, k = i % kIn;
    float v = params[OFF_W1 + i];
    if (k == kBiasCol) v = bf16_round(params[OFF_B1 + n]);
    if (k == kBiasColLo) v = params[OFF_B1 + n] - bf16_round(params[OFF_B1 + n]);
    *reinterpret_cast<__nv_bfloat16*>(pack + canon_off(n, k, kIn)) = __float2bfloat16_rn(v);
  }
  if (i < (uint32_t)(3 * kHidden * kHidden)) {
    uint32_t l = i / (kHidden * kHidden), e = i % (kHidden * kHidden);
    uint32_t n = e / kHidden, k = e % kHidden;
    *reinterpret_cast<__nv_bfloat16*>(pack + kPackW1 + l * kPackWh + canon_off(n, k, kHidden)) =
        __float2bfloat16_rn(params[w_off(1 + l) + e]);
  }
  if (i < kPackFloats) {
    float* f = reinterpret_cast<float*>(pack + kPackWBytes);
    float v;
    if (i < 4u * kHidden)
      v = params[b_off(i / kHidden) + i % kHidden];
    else if (i < 5u * kHidden)
      v = bf16_round(params[OFF_W5 + i - 4 * kHidden]);
    else
      v = params[OFF_B5];
    f[i] = v;
  }
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t sbo_bytes) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) |
         ((uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// kind::f16 instruction descriptor: D FP32, A/B BF16, both K-major, N = 64, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((64u >> 3) << 17) |
                            ((128u >> 4) << 24);

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile(
      "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
          smem_addr(bar))
      : "memory");
}

// Bounded wait on an mbarrier phase; false if the bound was reached.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  uint32_t a = smem_addr(bar);
  for (uint32_t i = 0; i < (1u << 24); ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,"
      "%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t*>(&v);
}

// ---- packed BF16x2 arithmetic (two activations per instruction)
__device__ __forceinline__ uint32_t bf2_fma(uint32_t a, uint32_t b, uint32_t c) {
  uint32_t d;
  asm("fma.rn.bf16x2 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(c));
  return d;
}
__device__ __forceinline__ uint32_t bf2_mul(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("mul.rn.bf16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
__device__ __forceinline__ uint32_t bf2_max(uint32_t a, uint32_t b) {
  uint32_t d;
  asm("max.bf16x2 %0, %1, %2;" : "=r"(d) : "r"(a), "r"(b));
  return d;
}
__device__ __forceinline__ uint32_t bf2_ex2(uint32_t a) {
  uint32_t d;
  asm("ex2.approx.ftz.bf16x2 %0, %1;" : "=r"(d) : "r"(a));
  return d;
}

// BF16 pairs {lo, hi} of constants
constexpr uint32_t bf2_const(uint32_t bits) { return bits | (bits << 16); }
constexpr uint32_t kBf2Log2e = bf2_const(0x3FB9u);   // 1.4453125 ~ log2(e)
constexpr uint32_t kBf2C1 = bf2_const(0x3F7Cu);      // 0.984375
constexpr uint32_t kBf2C2 = bf2_const(0xBECFu);      // -0.404296875
constexpr uint32_t kBf2C3 = bf2_const(0x3DE6u);      // 0.1123046875

// softplus of two BF16 pre-activations in BF16 arithmetic:
// max(z, 0) + u (c1 + u (c2 + u c3)) with u = 2^(-|z| log2 e), the cubic a
// least-squares fit of log1p(u) / u on [0, 1] (coefficients rounded to
// BF16).  Against softplus in FP32 rounded once to BF16 (the training
// arithmetic) the pre-activation is rounded twice; the difference is at
// most one BF16 unit in the last place of the activation.
__device__ __forceinline__ uint32_t softplus_bf16x2(uint32_t z) {
  uint32_t u = bf2_ex2(bf2_mul(z | 0x80008000u, kBf2Log2e));
  uint32_t q = bf2_fma(kBf2C3, u, kBf2C2);
  q = bf2_fma(q, u, kBf2C1);
  return bf2_fma(q, u, bf2_max(z, 0u));
}

// Tensor-core inference: each CTA runs kGroups independent pipelines of 128
// rows (one thread per row, 4 warps per group, one warp of every group on
// each SM sub-partition).  A group computes its rows' features, then for
// each layer: one elected thread issues the MMAs into the group's 64 TMEM
// columns and commits to the group's mbarrier; the group reads its
// accumulators back, applies bias and softplus, and writes the next
// layer's BF16 input.  While one group waits on its MMAs the others run
// their epilogues, which hides the tensor-core latency.
constexpr int kGroups = 4;
constexpr int kGroupRows = 128;
constexpr int kTcThreads = kGroups * kGroupRows;  // 512
constexpr uint32_t kTmemCols = 64 * kGroups;      // 256

struct __align__(1024) TcSmem {
  unsigned char w[kPackWBytes];               // W1..W4, canonical
  unsigned char x[kGroups][kGroupRows * kIn * 2];  // per-group layer input (K = 128 or 64)
  float bias[3][kHidden];                     // b2..b4 (b1 rides in W1)
  float w5[kHidden];
  float b5;
  uint64_t bar[kGroups];
  uint32_t tmem;
};

__device__ __forceinline__ void group_sync(int g) {
  asm volatile("bar.sync %0, 128;" ::"r"(g + 1) : "memory");
}
__device__ __forceinline__ bool group_and(int g, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\t"
      "bar.red.and.pred q, %2, 128, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(g + 1)
      : "memory");
  return r != 0u;
}
__device__ __forceinline__ bool group_or(int g, bool v) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\tsetp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, %2, 128, p;\n\tselp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)v), "r"(g + 1)
      : "memory");
  return r != 0u;
}

__device__ __forceinline__ void store_chunk(unsigned char* x, int row, int k, uint32_t K, uint32_t a,
                                            uint32_t b, uint32_t c, uint32_t d) {
  *reinterpret_cast<uint4*>(x + canon_off(row, k, K)) = make_uint4(a, b, c, d);
}

// Network value of this thread's row (q = normalised point).  Called by the
// 128 threads of group g together; `ok` turns false if an MMA did not
// complete within the wait bound (the caller makes it group-uniform).
__device__ __forceinline__ float mlp_row(TcSmem& s, const InputMap& m, int g, int row,
                                         const float q[3], uint32_t& phase, bool& ok) {
  unsigned char* x = s.x[g];
  {
    float v[48];
#pragma unroll
    for (int chain = 0; chain < 2; ++chain) {
      chain_features(m, q, chain, v);
#pragma unroll
      for (int c = 0; c < 6; ++c)
        store_chunk(x, row, (chain * 6 + c) * 8, kIn, pack_bf16x2(v[c * 8 + 0], v[c * 8 + 1]),
                    pack_bf16x2(v[c * 8 + 2], v[c * 8 + 3]), pack_bf16x2(v[c * 8 + 4], v[c * 8 + 5]),
                    pack_bf16x2(v[c * 8 + 6], v[c * 8 + 7]));
    }
    // k = 96..103: q.xyz, the two bias inputs (1.0), zeros; 104..127 zero
    store_chunk(x, row, 96, kIn, pack_bf16x2(q[0], q[1]), pack_bf16x2(q[2], 1.0f),
                pack_bf16x2(1.0f, 0.f), 0u);
#pragma unroll
    for (int c = 13; c < 16; ++c) store_chunk(x, row, c * 8, kIn, 0u, 0u, 0u, 0u);
  }
  const uint32_t wq = (uint32_t)(row >> 5);  // warp within the group = TMEM lane quarter
  const uint32_t tcol = s.tmem + ((32u * wq) << 16) + 64u * (uint32_t)g;
  float d = 0.f;
#pragma unroll 1
  for (int layer = 0; layer < 4; ++layer) {
    const uint32_t K = layer == 0 ? kIn : kHidden;
    fence_async_smem();
    fence_before();
    group_sync(g);
    fence_after();
    if (row == 0) {
      uint32_t xa = smem_addr(x);
      uint32_t wa = smem_addr(s.w + (layer == 0 ? 0u : kPackW1 + (layer - 1) * kPackWh));
#pragma unroll 1
      for (uint32_t kk = 0; kk < K / 16; ++kk)
        mma_bf16(s.tmem + 64u * (uint32_t)g, umma_desc(xa + kk * 256u, K * 16u),
                 umma_desc(wa + kk * 256u, K * 16u), kk > 0 ? 1u : 0u);
      mma_commit(&s.bar[g]);
    }
    ok = mbar_wait(&s.bar[g], phase) && ok;
    phase ^= 1u;
    __syncwarp();
    fence_after();
#pragma unroll
    for (int half = 0; half < 2; ++half) {
      float acc[32];
      tmem_ld32(tcol + 32u * (uint32_t)half, acc);
      if (layer > 0) {
        const float4* b4 = reinterpret_cast<const float4*>(s.bias[layer - 1]) + 8 * half;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          float4 bb = b4[j];
          acc[4 * j] += bb.x;
          acc[4 * j + 1] += bb.y;
          acc[4 * j + 2] += bb.z;
          acc[4 * j + 3] += bb.w;
        }
      }
      uint32_t a[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) a[j] = softplus_bf16x2(pack_bf16x2(acc[2 * j], acc[2 * j + 1]));
      if (layer < 3) {
#pragma unroll
        for (int c = 0; c < 4; ++c)
          store_chunk(x, row, 32 * half + 8 * c, kHidden, a[4 * c], a[4 * c + 1], a[4 * c + 2],
                      a[4 * c + 3]);
      } else {
        const float4* w4 = reinterpret_cast<const float4*>(s.w5) + 8 * half;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          float4 ww = w4[j];
          d = __fmaf_rn(__uint_as_float(a[2 * j] << 16), ww.x, d);
          d = __fmaf_rn(__uint_as_float(a[2 * j] & 0xFFFF0000u), ww.y, d);
          d = __fmaf_rn(__uint_as_float(a[2 * j + 1] << 16), ww.z, d);
          d = __fmaf_rn(__uint_as_float(a[2 * j + 1] & 0xFFFF0000u), ww.w, d);
        }
      }
    }
    // every thread has read its accumulators before the next MMA overwrites them
    fence_before();
  }
  return d + s.b5;
}

__device__ __forceinline__ void tc_setup(TcSmem& s, const unsigned char* __restrict__ pack) {
  int tid = threadIdx.x;
  for (uint32_t i = tid; i < kPackWBytes / 16; i += blockDim.x)
    reinterpret_cast<uint4*>(s.w)[i] = __ldg(reinterpret_cast<const uint4*>(pack) + i);
  const float* f = reinterpret_cast<const float*>(pack + kPackWBytes);
  for (uint32_t i = tid; i < 3 * kHidden; i += blockDim.x)
    s.bias[i / kHidden][i % kHidden] = f[kHidden + i];
  for (uint32_t i = tid; i < kHidden; i += blockDim.x) s.w5[i] = f[4 * kHidden + i];
  if (tid == 0) {
    s.b5 = f[5 * kHidden];
    for (int g = 0; g < kGroups; ++g)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&s.bar[g])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if ((tid >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&s.tmem)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
}

__device__ __forceinline__ void tc_teardown(TcSmem& s) {
  fence_before();
  __syncthreads();
  fence_after();
  if ((threadIdx.x >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem),
                 "r"(kTmemCols));
}

__device__ __forceinline__ TcSmem& tc_smem(unsigned char* raw) {
  return *reinterpret_cast<TcSmem*>((reinterpret_cast<uintptr_t>(raw) + 1023) & ~uintptr_t(1023));
}

// Batch evaluation: out[i] = network(pts[i]).  Group tiles are claimed
// round-robin: tile = (block * kGroups + g) + k * (grid * kGroups).
__global__ void __launch_bounds__(kTcThreads, 1) k_tc_eval(InputMap m,
                                                           const unsigned char* __restrict__ pack,
                                                           const float* __restrict__ pts, uint32_t n,
                                                           float* __restrict__ out,
                                                           int* __restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  TcSmem& s = tc_smem(smem_raw);
  tc_setup(s, pack);
  const int tid = threadIdx.x, g = tid >> 7, row = tid & 127;
  uint32_t phase = 0;
  const uint32_t tiles = (n + kGroupRows - 1) / kGroupRows;
  const uint32_t stride = gridDim.x * kGroups;
  bool ok = true;
  for (uint32_t tile = blockIdx.x * kGroups + g; tile < tiles; tile += stride) {
    uint32_t i = tile * kGroupRows + row;
    bool live = i < n;
    float p0 = live ? pts[3 * (size_t)i] : 0.f, p1 = live ? pts[3 * (size_t)i + 1] : 0.f,
          p2 = live ? pts[3 * (size_t)i + 2] : 0.f;
    float q[3];
    normalise(m, p0, p1, p2, q);
    float dv = mlp_row(s, m, g, row, q, phase, ok);
    if (live) out[i] = dv;
    if (!group_and(g, ok)) break;
  }
  if (!ok && row == 0) atomicExch(err, 1);
  tc_teardown(s);
}

// Reference evaluation with the training arithmetic (SIMT FP32, BF16-rounded
// weights and activations), one thread per point.
__global__ void __launch_bounds__(128) k_ref_eval(InputMap m, const float* __restrict__ params,
                                                  const float* __restrict__ pts, uint32_t n,
                                                  float* __restrict__ out) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float x[kIn];
  float q[3];
  normalise(m, pts[3 * (size_t)i], pts[3 * (size_t)i + 1], pts[3 * (size_t)i + 2], q);
  float v[48];
  chain_features(m, q, 0, v);
  for (int k = 0; k < 48; ++k) x[k] = bf16_round(v[k]);
  chain_features(m, q, 1, v);
  for (int k = 0; k < 48; ++k) x[48 + k] = bf16_round(v[k]);
  x[96] = bf16_round(q[0]);
  x[97] = bf16_round(q[1]);
  x[98] = bf16_round(q[2]);
  for (int k = 99; k < kIn; ++k) x[k] = 0.f;
  float h[kHidden], h2[kHidden];
  for (int c = 0; c < kHidden; ++c) {
    float z = 0.f;
    for (int k = 0; k < kIn; ++k) z = __fmaf_rn(x[k], bf16_round(params[OFF_W1 + c * kIn + k]), z);
    h[c] = bf16_round(softplus_approx(z + params[OFF_B1 + c]));
  }
  for (int l = 1; l < 4; ++l) {
    for (int c = 0; c < kHidden; ++c) {
      float z = 0.f;
      for (int k = 0; k < kHidden; ++k)
        z = __fmaf_rn(h[k], bf16_round(params[w_off(l) + c * kHidden + k]), z);
      h2[c] = bf16_round(softplus_approx(z + params[b_off(l) + c]));
    }
    for (int c = 0; c < kHidden; ++c) h[c] = h2[c];
  }
  float d = 0.f;
  for (int c = 0; c < kHidden; ++c) d = __fmaf_rn(h[c], bf16_round(params[OFF_W5 + c]), d);
  out[i] = d + params[OFF_B5];
}

// ------------------------------------------------ tensor-core training
// Training weight pack: the forward's W1..W4 as in the inference pack but
// without the first-layer bias columns (the training adds b1 in FP32), then
// W2^T..W4^T (canonical rows = layer inputs), the B operands of dA_prev = dZ W.
constexpr uint32_t kTrPackBytes = kPackWBytes + 3 * kPackWh;  // 65536

__global__ void k_pack_train(const float* __restrict__ params, unsigned char* __restrict__ pack) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < (uint32_t)(kHidden * kIn)) {
    uint32_t n = i / kIn, k = i % kIn;
    *reinterpret_cast<__nv_bfloat16*>(pack + canon_off(n, k, kIn)) =
        __float2bfloat16_rn(params[OFF_W1 + i]);
  }
  if (i < (uint32_t)(3 * kHidden * kHidden)) {
    uint32_t l = i / (kHidden * kHidden), e = i % (kHidden * kHidden);
    uint32_t n = e / kHidden, k = e % kHidden;
    __nv_bfloat16 w = __float2bfloat16_rn(params[w_off(1 + l) + e]);
    *reinterpret_cast<__nv_bfloat16*>(pack + kPackW1 + l * kPackWh + canon_off(n, k, kHidden)) = w;
    *reinterpret_cast<__nv_bfloat16*>(pack + kPackWBytes + l * kPackWh +
                                      canon_off(k, n, kHidden)) = w;
  }
}

// Issues `steps` MMAs of K = 16 (M 128, N 64): D (+)= A B^T, A and B K-major
// canonical with rows of `ka` / `kb` elements.
__device__ __forceinline__ void mma_chain(uint32_t d_tmem, uint32_t a, uint32_t ka, uint32_t b,
                                          uint32_t kb, uint32_t steps, bool accumulate) {
#pragma unroll 1
  for (uint32_t kk = 0; kk < steps; ++kk)
    mma_bf16(d_tmem, umma_desc(a + kk * 256u, ka * 16u), umma_desc(b + kk * 256u, kb * 16u),
             (accumulate || kk > 0) ? 1u : 0u);
}

struct __align__(1024) TrFwdSmem {
  unsigned char w[kPackWBytes];          // W1..W4, canonical
  unsigned char x[kTrRows * kIn * 2];    // layer input (K 128 or 64); FP32 scratch for the head
  float bias[4][kHidden];
  float w5[kHidden];
  float gs[kTrRows], ls[kTrRows];
  float b5;
  uint64_t bar;
  uint32_t tmem;
};
constexpr size_t kTrFwdSmemBytes = sizeof(TrFwdSmem) + 1024;

// Forward of one training step: features, four hidden layers (MMA + FP32
// bias + softplus, Z kept in FP32 and the activations in BF16 for the
// backward pass), head, L1 loss and its gradient dA4 = sign(out - label) / B
// * w5; partial gradients of w5, b5 and the loss per tile.
__global__ void __launch_bounds__(kTrRows) k_tc_train_fwd(InputMap m,
                                                          const float4* __restrict__ data,
                                                          uint32_t npts,
                                                          const uint32_t* __restrict__ step_ctr,
                                                          uint32_t seed, int direct,
                                                          const unsigned char* __restrict__ pack,
                                                          const float* __restrict__ params,
                                                          TrainBufs tb, uint32_t batch,
                                                          float* __restrict__ pred_out,
                                                          int* __restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  TrFwdSmem& s = *reinterpret_cast<TrFwdSmem*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int row = threadIdx.x;
  for (uint32_t i = row; i < kPackWBytes / 16; i += kTrRows)
    reinterpret_cast<uint4*>(s.w)[i] = __ldg(reinterpret_cast<const uint4*>(pack) + i);
  for (uint32_t i = row; i < 4 * kHidden; i += kTrRows)
    s.bias[i / kHidden][i % kHidden] = params[b_off(i / kHidden) + i % kHidden];
  if (row < kHidden) s.w5[row] = bf16_round(params[OFF_W5 + row]);
  if (row == 0) {
    s.b5 = params[OFF_B5];
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&s.bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if ((row >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&s.tmem)),
                 "r"(64));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t tcol = s.tmem + ((32u * (uint32_t)(row >> 5)) << 16);
  const uint32_t step = *step_ctr;
  uint32_t phase = 0;
  bool ok = true;
  const uint32_t tiles = batch / kTrRows;
  for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    uint32_t b = tile * kTrRows + row;
    uint32_t idx = direct ? b : mix32(seed, step, b) % npts;
    float4 pt = __ldg(&data[idx]);
    float q[3];
    normalise(m, pt.x, pt.y, pt.z, q);
    {
      uint4* xg = reinterpret_cast<uint4*>(tb.x0 + (size_t)b * kIn);
      float v[48];
#pragma unroll
      for (int chain = 0; chain < 2; ++chain) {
        chain_features(m, q, chain, v);
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          uint4 u = make_uint4(pack_bf16x2(v[c * 8 + 0], v[c * 8 + 1]),
                               pack_bf16x2(v[c * 8 + 2], v[c * 8 + 3]),
                               pack_bf16x2(v[c * 8 + 4], v[c * 8 + 5]),
                               pack_bf16x2(v[c * 8 + 6], v[c * 8 + 7]));
          store_chunk(s.x, row, (chain * 6 + c) * 8, kIn, u.x, u.y, u.z, u.w);
          xg[chain * 6 + c] = u;
        }
      }
      uint4 u = make_uint4(pack_bf16x2(q[0], q[1]), pack_bf16x2(q[2], 0.f), 0u, 0u);
      store_chunk(s.x, row, 96, kIn, u.x, u.y, u.z, u.w);
      xg[12] = u;
#pragma unroll
      for (int c = 13; c < 16; ++c) {
        store_chunk(s.x, row, c * 8, kIn, 0u, 0u, 0u, 0u);
        xg[c] = make_uint4(0u, 0u, 0u, 0u);
      }
    }
    float d = 0.f;
    uint32_t a4[32];
#pragma unroll 1
    for (int layer = 0; layer < 4; ++layer) {
      const uint32_t K = layer == 0 ? kIn : kHidden;
      fence_async_smem();
      fence_before();
      __syncthreads();
      fence_after();
      if (row == 0) {
        mma_chain(s.tmem, smem_addr(s.x), K,
                  smem_addr(s.w + (layer == 0 ? 0u : kPackW1 + (layer - 1) * kPackWh)), K, K / 16,
                  false);
        mma_commit(&s.bar);
      }
      ok = __syncthreads_and(mbar_wait(&s.bar, phase) && ok);  // CTA-uniform
      phase ^= 1u;
      fence_after();
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        float acc[32];
        tmem_ld32(tcol + 32u * (uint32_t)half, acc);
        float4* zg = reinterpret_cast<float4*>(tb.z[layer] + (size_t)b * kHidden + 32 * half);
#pragma unroll
        for (int j = 0; j < 32; ++j) acc[j] += s.bias[layer][32 * half + j];
#pragma unroll
        for (int j = 0; j < 8; ++j)
          zg[j] = make_float4(acc[4 * j], acc[4 * j + 1], acc[4 * j + 2], acc[4 * j + 3]);
        uint32_t a[16];
#pragma unroll
        for (int j = 0; j < 16; ++j)
          a[j] = pack_bf16x2(softplus_approx(acc[2 * j]), softplus_approx(acc[2 * j + 1]));
        if (layer < 3) {
          uint4* ag = reinterpret_cast<uint4*>(tb.a[layer] + (size_t)b * kHidden + 32 * half);
#pragma unroll
          for (int c = 0; c < 4; ++c) {
            store_chunk(s.x, row, 32 * half + 8 * c, kHidden, a[4 * c], a[4 * c + 1],
                        a[4 * c + 2], a[4 * c + 3]);
            ag[c] = make_uint4(a[4 * c], a[4 * c + 1], a[4 * c + 2], a[4 * c + 3]);
          }
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            a4[16 * half + j] = a[j];
            int c = 32 * half + 2 * j;
            d = __fmaf_rn(__uint_as_float(a[j] << 16), s.w5[c], d);
            d = __fmaf_rn(__uint_as_float(a[j] & 0xFFFF0000u), s.w5[c + 1], d);
          }
        }
      }
      fence_before();
    }
    // head and L1 loss
    float pred = d + s.b5;
    float diff = pred - pt.w;
    float g = (diff > 0.f ? 1.f : (diff < 0.f ? -1.f : 0.f)) / (float)batch;
    if (pred_out) pred_out[b] = pred;
    float4* dag = reinterpret_cast<float4*>(tb.da + (size_t)b * kHidden);
#pragma unroll
    for (int j = 0; j < 16; ++j)
      dag[j] = make_float4(g * s.w5[4 * j], g * s.w5[4 * j + 1], g * s.w5[4 * j + 2],
                           g * s.w5[4 * j + 3]);
    // every MMA of the tile has completed: the input buffer is free for the
    // head's reduction (row-major FP32 [128][64])
    __syncthreads();
    float* red = reinterpret_cast<float*>(s.x);
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      red[row * kHidden + 2 * j] = g * __uint_as_float(a4[j] << 16);
      red[row * kHidden + 2 * j + 1] = g * __uint_as_float(a4[j] & 0xFFFF0000u);
    }
    s.gs[row] = g;
    s.ls[row] = fabsf(diff);
    __syncthreads();
    float* ph = tb.part_head + (size_t)tile * (kHidden + 2);
    if (row < kHidden) {
      float acc = 0.f;
      for (int r = 0; r < kTrRows; ++r) acc += red[r * kHidden + row];
      ph[row] = acc;
    } else if (row == kHidden) {
      float acc = 0.f;
      for (int r = 0; r < kTrRows; ++r) acc += s.gs[r];
      ph[kHidden] = acc;
    } else if (row == kHidden + 1) {
      float acc = 0.f;
      for (int r = 0; r < kTrRows; ++r) acc += s.ls[r];
      ph[kHidden + 1] = acc;
    }
    __syncthreads();  // the reduction has read the scratch before the next tile's features
  }
  if (!ok && row == 0) atomicExch(err, 1);
  fence_before();
  __syncthreads();
  fence_after();
  if ((row >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem), "r"(64));
}

struct __align__(1024) TrBwdSmem {
  unsigned char wt[kPackWh];                // W^T of this layer (rows = inputs), canonical
  unsigned char dz[kTrRows * kHidden * 2];  // dZ, rows = batch rows, K = 64
  unsigned char dzt[kHidden * kTrRows * 2]; // dZ^T, rows = outputs, K = 128 batch rows
  unsigned char at[kIn * kTrRows * 2];      // A_prev^T, rows = inputs (128), K = 128 batch rows
  uint64_t bar;
  uint32_t tmem;
};
constexpr size_t kTrBwdSmemBytes = sizeof(TrBwdSmem) + 1024;

__device__ __forceinline__ void st_bf16(unsigned char* base, uint32_t off, uint32_t bits16) {
  *reinterpret_cast<uint16_t*>(base + off) = (uint16_t)bits16;
}

// Backward through hidden layer `layer` (0-based) over 128-row tiles:
//   dZ      = dA * softplus'(Z)                      (FP32, then BF16)
//   dA_prev = dZ W          (layers > 0)            TMEM columns [0, 64)
//   dW^T   += A_prev^T dZ   over the CTA's tiles     TMEM columns [64, 128)
// The bias gradient rides in dW^T: the A_prev^T row just past the inputs
// (row 64; row 99, an always-zero feature, for the first layer) is all ones,
// so that accumulator row is sum_b dZ.  The CTA's dW, db go to its slot of
// the partial-gradient buffer.
__global__ void __launch_bounds__(kTrRows) k_tc_train_bwd(int layer,
                                                          const unsigned char* __restrict__ pack,
                                                          TrainBufs tb,
                                                          const float* __restrict__ da_in,
                                                          float* __restrict__ da_out,
                                                          uint32_t batch, int* __restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  TrBwdSmem& s = *reinterpret_cast<TrBwdSmem*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const int row = threadIdx.x;
  const uint32_t Kin = layer == 0 ? kIn : kHidden;
  const uint32_t ones_row = layer == 0 ? 99u : (uint32_t)kHidden;
  const uint32_t one = 0x3F80u;  // BF16 1.0
  if (layer > 0)
    for (uint32_t i = row; i < kPackWh / 16; i += kTrRows)
      reinterpret_cast<uint4*>(s.wt)[i] = __ldg(
          reinterpret_cast<const uint4*>(pack + kPackWBytes + (layer - 1) * kPackWh) + i);
  // rows of A_prev^T past the inputs: the ones row, then zeros (hidden layers)
  if (layer > 0)
    for (uint32_t k = kHidden; k < (uint32_t)kIn; ++k)
      st_bf16(s.at, canon_off(k, row, kTrRows), k == ones_row ? one : 0u);
  if (row == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&s.bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if ((row >> 5) == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_addr(&s.tmem)),
                 "r"(128));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  fence_before();
  __syncthreads();
  fence_after();
  const uint32_t lane_off = (32u * (uint32_t)(row >> 5)) << 16;
  uint32_t phase = 0;
  bool ok = true, first = true;
  const uint32_t tiles = batch / kTrRows;
  for (uint32_t tile = blockIdx.x; tile < tiles && ok; tile += gridDim.x) {
    size_t b = (size_t)tile * kTrRows + row;
    const float4* dg = reinterpret_cast<const float4*>(da_in + b * kHidden);
    const float4* zg = reinterpret_cast<const float4*>(tb.z[layer] + b * kHidden);
#pragma unroll
    for (int c = 0; c < 8; ++c) {  // 8 dZ values per 16-byte chunk
      float dz[8];
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float4 dd = dg[2 * c + h], zz = zg[2 * c + h];
        dz[4 * h] = dd.x * softplus_approx_deriv(zz.x);
        dz[4 * h + 1] = dd.y * softplus_approx_deriv(zz.y);
        dz[4 * h + 2] = dd.z * softplus_approx_deriv(zz.z);
        dz[4 * h + 3] = dd.w * softplus_approx_deriv(zz.w);
      }
      uint32_t p0 = pack_bf16x2(dz[0], dz[1]), p1 = pack_bf16x2(dz[2], dz[3]);
      uint32_t p2 = pack_bf16x2(dz[4], dz[5]), p3 = pack_bf16x2(dz[6], dz[7]);
      store_chunk(s.dz, row, 8 * c, kHidden, p0, p1, p2, p3);
      uint32_t pk[4] = {p0, p1, p2, p3};
#pragma unroll
      for (int e = 0; e < 8; ++e)
        st_bf16(s.dzt, canon_off(8 * c + e, row, kTrRows), (pk[e >> 1] >> (16 * (e & 1))) & 0xFFFFu);
    }
    const uint4* ag = layer == 0 ? reinterpret_cast<const uint4*>(tb.x0 + b * kIn)
                                 : reinterpret_cast<const uint4*>(tb.a[layer - 1] + b * kHidden);
    for (uint32_t c = 0; c < Kin / 8; ++c) {
      uint4 u = ag[c];
      uint32_t w4[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
      for (int e = 0; e < 8; ++e) {
        uint32_t k = 8 * c + e;
        uint32_t v = (w4[e >> 1] >> (16 * (e & 1))) & 0xFFFFu;
        st_bf16(s.at, canon_off(k, row, kTrRows), k == ones_row ? one : v);
      }
    }
    fence_async_smem();
    fence_before();
    __syncthreads();
    fence_after();
    if (row == 0) {
      if (layer > 0)
        mma_chain(s.tmem, smem_addr(s.dz), kHidden, smem_addr(s.wt), kHidden, kHidden / 16, false);
      mma_chain(s.tmem + 64u, smem_addr(s.at), kTrRows, smem_addr(s.dzt), kTrRows, kTrRows / 16,
                !first);
      mma_commit(&s.bar);
    }
    ok = __syncthreads_and(mbar_wait(&s.bar, phase) && ok);  // CTA-uniform
    phase ^= 1u;
    fence_after();
    if (layer > 0) {
      float4* og = reinterpret_cast<float4*>(da_out + b * kHidden);
#pragma unroll
      for (int half = 0; half < 2; ++half) {
        float acc[32];
        tmem_ld32(s.tmem + lane_off + 32u * (uint32_t)half, acc);
#pragma unroll
        for (int j = 0; j < 8; ++j)
          og[8 * half + j] = make_float4(acc[4 * j], acc[4 * j + 1], acc[4 * j + 2], acc[4 * j + 3]);
      }
    }
    fence_before();
    __syncthreads();  // the next tile overwrites the operands and dA_prev
    fence_after();
    first = false;
  }
  // this CTA's weight and bias gradients: TMEM lane = input index k', column = output n
  float* pp = tb.part + (size_t)blockIdx.x * kNumParams;
  const uint32_t k = (uint32_t)row;
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    float acc[32];
    if (!first) {
      tmem_ld32(s.tmem + lane_off + 64u + 32u * (uint32_t)half, acc);
    } else {
#pragma unroll
      for (int j = 0; j < 32; ++j) acc[j] = 0.f;
    }
#pragma unroll
    for (int j = 0; j < 32; ++j) {
      uint32_t n = 32u * (uint32_t)half + (uint32_t)j;
      if (k == ones_row)
        pp[b_off(layer) + n] = acc[j];
      if (k < Kin) pp[w_off(layer) + n * Kin + k] = k == ones_row ? 0.f : acc[j];
    }
  }
  if (!ok && row == 0) atomicExch(err, 1);
  fence_before();
  __syncthreads();
  fence_after();
  if ((row >> 5) == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem), "r"(128));
}

// ------------------------------------------------------------- tracing
struct MarchDev {
  float alpha;        // network step = alpha * network distance (safety / Lipschitz bound)
  float switch_dist;  // hand over to the exact field below this network distance
  float min_step;     // floor of a network step
  float tmax;
  uint32_t max_steps;  // network steps before handing over regardless
  float bmin[3], bmax[3];  // the network's box; the march stays inside it
};

// Exact phase parameters.
struct RefineDev {
  uint32_t max_steps;   // exact evaluations per ray (march + bracket + root)
  uint32_t root_steps;  // regula-falsi steps on a bracketed crossing
  float relax;          // an exact step may grow to relax x (step_factor * d) along a secant
  float root_tol;       // the root search ends when the secant point moves less than this
  float ceiling;        // no surface above this height (bound of the field)
  uint32_t normal_taps;  // 6: central differences; 4: tetrahedral; 1: none here (k_sdf_grad_normal)
  // cone starts (direct mode): pixel (x, y) starts at tile_t[(y / cone_tile)
  // * cone_tiles_x + x / cone_tile]; null: every pixel starts at t = 0
  const float* tile_t;
  uint32_t cone_tile, cone_tiles_x;
};

// Tap k of the tetrahedral normal (compute_sdf_normal_tet,
// sdf_functions.cuh:518-532): 0.5773 (2 b - 1) with b = (((k + 3) >> 1) & 1,
// (k >> 1) & 1, k & 1), i.e. the corners (+,-,-), (-,-,+), (-,+,-), (+,+,+)
// of a cube scaled to length ~1.
__device__ __forceinline__ V3 tet_dir(uint32_t k) {
  const float c = 0.5773f;
  return v3((((k + 3u) >> 1) & 1u) ? c : -c, ((k >> 1) & 1u) ? c : -c, (k & 1u) ? c : -c);
}

// Slab test of the ray against the box: [t0, t1] with t0 >= 0 (empty if t0 >= t1).
__device__ __forceinline__ void box_span(const MarchDev& md, const V3& o, const V3& d, float& t0,
                                         float& t1) {
  float o3[3] = {o.x, o.y, o.z}, d3[3] = {d.x, d.y, d.z};
  t0 = 0.f;
  t1 = md.tmax;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float inv = 1.0f / d3[k];
    float ta = (md.bmin[k] - o3[k]) * inv, tb = (md.bmax[k] - o3[k]) * inv;
    t0 = fmaxf(t0, fminf(ta, tb));
    t1 = fminf(t1, fmaxf(ta, tb));
  }
}

// Appends this lane's entry to the exact-phase queue (warp-aggregated).
__device__ __forceinline__ void queue_push(bool push, uint4 e, uint32_t* counters,
                                           uint4* __restrict__ queue) {
  uint32_t lane = threadIdx.x & 31u;
  uint32_t pm = __ballot_sync(0xFFFFFFFFu, push);
  if (pm == 0u) return;
  uint32_t leader = __ffs(pm) - 1u, base = 0;
  if (lane == leader) base = atomicAdd(&counters[1], (uint32_t)__popc(pm));
  base = __shfl_sync(0xFFFFFFFFu, base, leader);
  if (push) queue[base + __popc(pm & ((1u << lane) - 1u))] = e;
}

// Neural phase.  Each group of 128 threads marches 128 rays (one per
// thread) through the network; a warp refills its idle rows from the pixel
// cursor (claim order = 8x4 pixel tiles) once 8 of them are idle.  A ray
// starts where it enters the network's box and steps by
// max(alpha * d_net, min_step).  It is queued for the exact phase as
// {pixel, t, t_lo, steps} when d_net < switch_dist (t_lo = the previous
// network point, a bracket candidate), when it leaves the box before tmax
// (t = t_lo = exit), or after max_steps network steps; rays that reach tmax
// inside the box are written as misses.
__global__ void __launch_bounds__(kTcThreads, 1) k_nsdf_march(InputMap m,
                                                              const unsigned char* __restrict__ pack,
                                                              MarchDev md, CamDev cam, uint32_t w,
                                                              uint32_t h, uint32_t* __restrict__ counters,
                                                              unsigned long long* __restrict__ totals,
                                                              uint4* __restrict__ queue,
                                                              float4* __restrict__ out,
                                                              int* __restrict__ err) {
  extern __shared__ unsigned char smem_raw[];
  TcSmem& s = tc_smem(smem_raw);
  tc_setup(s, pack);
  const int tid = threadIdx.x, g = tid >> 7, row = tid & 127;
  const uint32_t lane = tid & 31u;
  uint32_t phase = 0;
  const uint32_t tiles_x = (w + 7) / 8;
  const uint32_t total = tiles_x * ((h + 3) / 4) * 32u;
  bool live = false, exhausted = false, ok = true;
  uint32_t pix = 0, steps = 0;
  V3 o = {0.f, 0.f, 0.f}, d = {0.f, 0.f, 1.f};
  float t = 0.f, t_lo = 0.f, t_end = 0.f;
  uint32_t n_live = 0, n_rows = 0;  // network evaluations of rays / rows computed
  for (uint32_t guard = 0; guard < (1u << 24); ++guard) {
    bool outside = false;  // a new ray that misses the box goes straight to the exact phase
    uint32_t idle = __ballot_sync(0xFFFFFFFFu, !live);
    uint32_t nidle = __popc(idle);
    if (!exhausted && nidle >= 8u) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(&counters[0], nidle);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (base + nidle >= total) exhausted = true;
      if (!live) {
        uint32_t i = base + __popc(idle & ((1u << lane) - 1u));
        uint32_t tile = i >> 5, l = i & 31u;
        uint32_t x = (tile % tiles_x) * 8 + (l & 7u), y = (tile / tiles_x) * 4 + (l >> 3);
        if (i < total && x < w && y < h) {
          generate_ray(cam, w, h, x, y, o, d);
          pix = y * w + x;
          steps = 0;
          float t0, t1;
          box_span(md, o, d, t0, t1);
          if (t0 < t1) {
            t = t0;
            t_lo = t0;
            t_end = t1;
            live = true;
          } else {
            outside = true;
          }
        }
      }
    }
    queue_push(outside, make_uint4(pix, 0u, 0u, 0u), counters, queue);
    if (!group_or(g, live || !exhausted)) break;
    float q[3];
    normalise(m, __fmaf_rn(t, d.x, o.x), __fmaf_rn(t, d.y, o.y), __fmaf_rn(t, d.z, o.z), q);
    float dn = mlp_row(s, m, g, row, q, phase, ok);
    if (!group_and(g, ok)) break;
    ++n_rows;
    n_live += live ? 1u : 0u;
    bool push = false;
    uint4 e = make_uint4(0u, 0u, 0u, 0u);
    if (live) {
      ++steps;
      if (dn < md.switch_dist) {
        push = true;
        e = make_uint4(pix, __float_as_uint(t), __float_as_uint(t_lo), steps);
      } else {
        t_lo = t;
        t += fmaxf(md.alpha * dn, md.min_step);
        if (t >= t_end) {
          if (t_end >= md.tmax) {
            out[2 * (size_t)pix] = make_float4(0.f, 0.f, 0.f, 0.f);
            out[2 * (size_t)pix + 1] =
                make_float4(0.f, 0.f, __uint_as_float(steps), __uint_as_float(0u));
            live = false;
          } else {
            push = true;
            e = make_uint4(pix, __float_as_uint(t_end), __float_as_uint(t_end), steps);
          }
        } else if (steps >= md.max_steps) {
          push = true;
          e = make_uint4(pix, __float_as_uint(t), __float_as_uint(t), steps);
        }
      }
      if (push) live = false;
    }
    queue_push(push, e, counters, queue);
  }
  n_live = __reduce_add_sync(0xFFFFFFFFu, n_live);
  n_rows = __reduce_add_sync(0xFFFFFFFFu, n_rows);
  if (lane == 0) {
    atomicAdd(&totals[0], (unsigned long long)n_live);
    atomicAdd(&totals[3], (unsigned long long)n_rows);
  }
  if (!ok && row == 0) atomicExch(err, 1);
  tc_teardown(s);
}

// Cone tiles of the network phase: tile x tile pixels, tiles_x x tiles_y of
// them; parent (may be null): start parameters of coarser tiles of
// parent_tile pixels (a multiple of tile), parent_tiles_x per row.
struct ConeDev {
  uint32_t tile, tiles_x, tiles_y;
  const float* parent;
  uint32_t parent_tile, parent_tiles_x;
};

// Cone phase.  Each tile's cone is marched by K consecutive lanes of a
// warp.  The axis is the normalised sum of the tile's four corner rays, and
// `s` the largest chord from the axis direction to a corner ray's.  The
// angle to the axis is quasi-convex over the image plane, so the corners
// bound it: every ray of the tile lies within t s of the axis point at the
// same parameter t, and a point of a tile ray within a further dt lies
// within dt + t s of the axis point.  The clearance c = d_net - t s (the
// network distance shrunk by the cone's radius) therefore bounds a step of
// alpha c for every ray of the tile, the per-ray rule's step.
//
// Speculation: in one pass lane j of a tile evaluates the axis at t + dt
// (r + r^2 + ... + r^j), dt the last accepted step and r = 0.9 x the ratio
// of the last two (the steps of a cone closing in on a surface shrink
// geometrically, in open space they grow).  The lanes' spheres are chained
// in order: a point that lies inside the part already cleared extends it to
// t_j + alpha c_j, a point beyond it ends the chain, and the first chained
// point whose clearance is below switch_dist stops the tile there.  Lane 0
// is at t, so a pass advances at least one sequential step, and up to K
// when the guesses land; K = 1 is plain cone marching.
//
// The axis starts at its entry into the network's box (or the parent tile's
// start, if later); a tile whose axis leaves the box stops at the exit, and
// one that makes max_steps passes stops where it is.  Every pixel of the
// tile then starts its exact phase at the tile's parameter (k_sdf_refine).
template <uint32_t K>
__global__ void __launch_bounds__(kTcThreads, 1) k_nsdf_cone(InputMap m,
                                                             const unsigned char* __restrict__ pack,
                                                             MarchDev md, ConeDev cd, CamDev cam,
                                                             uint32_t w, uint32_t h,
                                                             uint32_t* __restrict__ cursor,
                                                             unsigned long long* __restrict__ totals,
                                                             float* __restrict__ tile_t,
                                                             int* __restrict__ err) {
  static_assert(K == 1 || K == 2 || K == 4 || K == 8 || K == 16,
                "lanes per cone: 1, 2, 4, 8 or 16");
  extern __shared__ unsigned char smem_raw[];
  TcSmem& s = tc_smem(smem_raw);
  tc_setup(s, pack);
  const int tid = threadIdx.x, g = tid >> 7, row = tid & 127;
  const uint32_t lane = tid & 31u;
  const uint32_t j = lane & (K - 1u), lead = lane & ~(K - 1u);
  const uint32_t kmask = (K == 1 ? 1u : ((1u << K) - 1u)) << lead;
  uint32_t phase = 0;
  const uint32_t total = cd.tiles_x * cd.tiles_y;
  bool live = false, exhausted = false, ok = true;
  uint32_t tile = 0, passes = 0;
  V3 o = {0.f, 0.f, 0.f}, ax = {0.f, 0.f, 1.f};
  float t = 0.f, dt = 0.f, ratio = 1.f, t_end = 0.f, chord = 0.f;
  uint32_t n_live = 0, n_rows = 0;
  for (uint32_t guard = 0; guard < (1u << 24); ++guard) {
    // the K lanes of a tile share `live`, so a tile's first lane speaks for it
    const uint32_t idle = __ballot_sync(0xFFFFFFFFu, !live && j == 0u);
    const uint32_t nidle = __popc(idle);
    if (!exhausted && nidle * K >= 8u) {
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(cursor, nidle);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (base + nidle >= total) exhausted = true;
      const uint32_t i =
          __shfl_sync(0xFFFFFFFFu, base + __popc(idle & ((1u << lane) - 1u)), lead);
      if (!live && i < total) {
        // every lane of the tile computes the same set-up
        tile = i;
        const uint32_t x0 = (i % cd.tiles_x) * cd.tile, y0 = (i / cd.tiles_x) * cd.tile;
        const uint32_t x1 = min(x0 + cd.tile - 1u, w - 1u), y1 = min(y0 + cd.tile - 1u, h - 1u);
        V3 c[4];
        generate_ray(cam, w, h, x0, y0, o, c[0]);
        generate_ray(cam, w, h, x1, y0, o, c[1]);
        generate_ray(cam, w, h, x0, y1, o, c[2]);
        generate_ray(cam, w, h, x1, y1, o, c[3]);
        ax = normalize(v3(c[0].x + c[1].x + c[2].x + c[3].x, c[0].y + c[1].y + c[2].y + c[3].y,
                          c[0].z + c[1].z + c[2].z + c[3].z));
        chord = 0.f;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          V3 e = sub(c[k], ax);
          chord = fmaxf(chord, sqrtf(dot(e, e)));
        }
        // rounding of the corner rays and of the axis
        chord = chord * 1.001f + 1e-6f;
        float t0, t1;
        box_span(md, o, ax, t0, t1);
        float start =
            cd.parent ? cd.parent[(y0 / cd.parent_tile) * cd.parent_tiles_x + x0 / cd.parent_tile]
                      : 0.f;
        t = fmaxf(t0, start);
        t_end = t1;
        dt = 0.f;
        ratio = 1.f;
        passes = 0;
        if (t < t_end) live = true;
        else if (j == 0u) tile_t[tile] = start;
      }
    }
    if (!group_or(g, live || !exhausted)) break;
    float off = 0.f;
    {
      const float r = 0.9f * ratio;
      float rp = 1.f;
      for (uint32_t i = 0; i < j; ++i) {
        rp *= r;
        off += rp;
      }
    }
    const float tj = __fmaf_rn(off, dt, t);
    float q[3];
    normalise(m, __fmaf_rn(tj, ax.x, o.x), __fmaf_rn(tj, ax.y, o.y), __fmaf_rn(tj, ax.z, o.z), q);
    float dn = mlp_row(s, m, g, row, q, phase, ok);
    if (!group_and(g, ok)) break;
    ++n_rows;
    n_live += live ? 1u : 0u;
    if (live) {
      // all K lanes of the tile are here together and reach the same verdict
      const float cj = dn - tj * chord;
      float cov = t, t_stop = 0.f, s_last = dt, s_prev = dt;
      bool chained = true, stop = false;
#pragma unroll
      for (uint32_t k = 0; k < K; ++k) {
        const float tk = K == 1 ? tj : __shfl_sync(kmask, tj, lead + k);
        const float ck = K == 1 ? cj : __shfl_sync(kmask, cj, lead + k);
        if (chained && !stop) {
          if (tk > cov) {
            chained = false;
          } else if (ck < md.switch_dist) {
            stop = true;
            t_stop = tk;
          } else {
            cov = fmaxf(cov, tk + md.alpha * ck);
            s_prev = s_last;
            s_last = md.alpha * ck;
          }
        }
      }
      ++passes;
      if (stop) {
        if (j == 0u) tile_t[tile] = t_stop;
        live = false;
      } else {
        t = cov;
        ratio = s_prev > 0.f ? fminf(fmaxf(s_last / s_prev, 0.25f), 4.f) : 1.f;
        dt = s_last;
        if (t >= t_end) {
          if (j == 0u) tile_t[tile] = t_end;
          live = false;
        } else if (passes >= md.max_steps) {
          if (j == 0u) tile_t[tile] = t;
          live = false;
        }
      }
    }
  }
  n_live = __reduce_add_sync(0xFFFFFFFFu, n_live);
  n_rows = __reduce_add_sync(0xFFFFFFFFu, n_rows);
  if (lane == 0) {
    atomicAdd(&totals[0], (unsigned long long)n_live);
    atomicAdd(&totals[3], (unsigned long long)n_rows);
  }
  if (!ok && row == 0) atomicExch(err, 1);
  tc_teardown(s);
}

// Exact phase, one lane per ray with lane refill (from the queue, or from
// the pixel cursor when `direct`: every pixel from t = 0, the same method
// without the network).  One field evaluation per trip of a state machine:
//   march  t += step_factor * d (the exact tracer's rule); the step may
//          grow along the secant through the last two samples up to relax x
//          that (relax <= 1: plain rule).  d < eps: hit at t.  d < 0 (the
//          sample is inside): the crossing is bracketed by the last outside
//          sample and refined.  Going up above `ceiling`: miss.
//   probe  the ray arrived inside from the network: check the bracket
//          candidate t_lo; if it is outside the crossing lies in
//          [t_lo, t], else march again from t = 0 (the network skipped
//          over the surface).
//   root   Illinois regula falsi on the bracket, root_steps evaluations or
//          until |d| < 1e-6, or until the next secant point moves less than
//          root_tol (that point is the hit, unevaluated; a bracket already
//          narrower than root_tol gives its secant root at once).
//   normal the exact tracer's central differences (delta = 0.002 t), or,
//          with normal_taps 4, the reference's tetrahedral normal
//          (compute_sdf_normal_tet) at the same radius: sum of e_k d(p +
//          delta e_k) over the four tetrahedron directions e_k.  With
//          normal_taps 1 the hit is written without a normal and
//          k_sdf_grad_normal adds the field's analytic gradient afterwards.
// With cone starts a ray begins its march where its tile's cone stopped; a
// start that is already inside the terrain (the network overestimated the
// distance) marches again from the camera.
// The step count written is network steps + exact march/probe/root
// evaluations (normals excluded, as in the exact tracer).
enum : uint32_t { kMarch = 0, kProbe = 1, kRoot = 2, kNormal = 3 };

// NT: the normal (RefineDev::normal_taps), fixed at compile time so that
// the analytic-gradient form (1) carries no stencil state.
template <uint32_t NT>
__global__ void __launch_bounds__(256) k_sdf_refine(PermTable perm, FieldDev f, RefineDev rd,
                                                    CamDev cam, uint32_t w, uint32_t h, int direct,
                                                    const uint4* __restrict__ queue,
                                                    uint32_t* __restrict__ counters,
                                                    unsigned long long* __restrict__ totals,
                                                    float4* __restrict__ out) {
  extern __shared__ uint32_t perm_smem[];
  // Per-warp ring of set-up rays (64 entries): the warp claims 32 work
  // indices at a time and all its lanes set those rays up together (pixel,
  // two divisions and three normalisations for the direction, the cone
  // tile's start), so the set-up runs with every lane active instead of on
  // the few lanes that happen to be idle; idle lanes then take entries.
  // Entry: {d.xyz, t} and {pixel (0xFFFFFFFF: no ray), t_lo bits, base
  // steps, 0}.
  __shared__ float4 ring_a[8][64];
  __shared__ uint4 ring_b[8][64];
  load_perm(perm, perm_smem);
  Perm P = perm_view(perm_smem);
  const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
  // direct mode claims pixels in 8x4 tiles (claim i = lane i & 31 of tile
  // i >> 5), so a warp's rays start close together
  const uint32_t dtiles_x = (w + 7) / 8;
  const uint32_t total = direct ? dtiles_x * ((h + 3) / 4) * 32u : counters[1];
  bool live = false, claimed_all = false, have_lo = false, restarted = false;
  uint32_t head = 0, tail = 0;  // ring positions (warp-uniform)
  uint32_t pix = 0, steps = 0, base_steps = 0, mode = kMarch, tap = 0, iters = 0;
  int side = 0;
  V3 o = cam.campos, d = {0, 0, 1}, p = {0, 0, 0};
  float t = 0.f, t_lo = 0.f, a = 0.f, va = 0.f, b = 0.f, vb = 0.f, delta = 0.f;
  float nx = 0.f, ny = 0.f, nz = 0.f, plus = 0.f;
  uint32_t n_exact = 0, n_normal = 0;  // evaluations: march/probe/root, normal taps
  for (;;) {
    uint32_t idle = __ballot_sync(0xFFFFFFFFu, !live);
    uint32_t nidle = __popc(idle);
    if (nidle >= 4u && (!claimed_all || head != tail)) {
      if (tail - head < nidle && !claimed_all) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&counters[2], 32u);
        base = __shfl_sync(0xFFFFFFFFu, base, 0);
        if (base + 32u >= total) claimed_all = true;
        const uint32_t i = base + lane;
        uint32_t dx = 0, dy = 0;
        if (direct) {
          dx = ((i >> 5) % dtiles_x) * 8 + (i & 7u);
          dy = ((i >> 5) / dtiles_x) * 4 + ((i >> 3) & 3u);
        }
        float4 ea = make_float4(0.f, 0.f, 1.f, 0.f);
        uint4 eb = make_uint4(0xFFFFFFFFu, 0u, 0u, 0u);
        if (i < total && (!direct || (dx < w && dy < h))) {
          uint4 e = direct ? make_uint4(dy * w + dx, 0u, 0u, 0u) : queue[i];
          V3 ro, rd3;
          generate_ray(cam, w, h, e.x % w, e.x / w, ro, rd3);
          float t0 = __uint_as_float(e.y), tl = __uint_as_float(e.z);
          if (direct && rd.tile_t) {
            t0 = rd.tile_t[((e.x / w) / rd.cone_tile) * rd.cone_tiles_x + (e.x % w) / rd.cone_tile];
            tl = t0;
          }
          ea = make_float4(rd3.x, rd3.y, rd3.z, t0);
          eb = make_uint4(e.x, __float_as_uint(tl), e.w, 0u);
        }
        ring_a[warp][(tail + lane) & 63u] = ea;
        ring_b[warp][(tail + lane) & 63u] = eb;
        __syncwarp();
        tail += 32u;
      }
      const uint32_t avail = tail - head;
      if (!live) {
        const uint32_t r = __popc(idle & ((1u << lane) - 1u));
        if (r < avail) {
          const float4 ea = ring_a[warp][(head + r) & 63u];
          const uint4 eb = ring_b[warp][(head + r) & 63u];
          if (eb.x != 0xFFFFFFFFu) {
            pix = eb.x;
            d = v3(ea.x, ea.y, ea.z);
            t = ea.w;
            t_lo = __uint_as_float(eb.y);
            base_steps = eb.z;
            steps = 0;
            mode = kMarch;
            have_lo = false;
            restarted = false;
            live = true;
          }
        }
      }
      head += min(nidle, avail);
      __syncwarp();
    }
    if (__ballot_sync(0xFFFFFFFFu, live) == 0u) {
      if (claimed_all && head == tail) break;
      continue;
    }
    if (!live) continue;
    V3 qp;
    if (mode == kMarch) {
      qp = v3(__fmaf_rn(t, d.x, o.x), __fmaf_rn(t, d.y, o.y), __fmaf_rn(t, d.z, o.z));
    } else if (mode == kProbe) {
      qp = v3(__fmaf_rn(a, d.x, o.x), __fmaf_rn(a, d.y, o.y), __fmaf_rn(a, d.z, o.z));
    } else if (NT == 1u || mode == kRoot) {
      qp = v3(__fmaf_rn(t, d.x, o.x), __fmaf_rn(t, d.y, o.y), __fmaf_rn(t, d.z, o.z));
    } else if (NT == 4u) {
      V3 e = tet_dir(tap);
      qp = v3(__fmaf_rn(e.x, delta, p.x), __fmaf_rn(e.y, delta, p.y), __fmaf_rn(e.z, delta, p.z));
    } else {
      float sd = (tap & 1u) ? -delta : delta;
      qp = p;
      if (tap < 2) qp.x = p.x + sd;
      else if (tap < 4) qp.y = p.y + sd;
      else qp.z = p.z + sd;
    }
    float v = terrain_density(P, qp, f.octaves, f.scale, f.amp);
    if (NT != 1u && mode == kNormal) ++n_normal;
    else ++n_exact;
    uint32_t status = 3;  // 3 = still running
    bool begin_root = false, hit_here = false;
    if (mode == kMarch) {
      ++steps;
      if (v < 0.f) {
        if (have_lo) {
          b = t;
          vb = v;
          begin_root = true;
        } else if (t_lo < t && !restarted) {
          b = t;
          vb = v;
          a = t_lo;
          mode = kProbe;
        } else if (rd.tile_t && !restarted) {
          // the cone start lies inside: march again from the camera
          t = 0.f;
          t_lo = 0.f;
          restarted = true;
          if (steps >= rd.max_steps) status = 2;
        } else {
          hit_here = true;
        }
      } else if (v < f.eps) {
        hit_here = true;
      } else if (d.y >= 0.f && qp.y > rd.ceiling) {
        status = 0;
      } else {
        float step = f.step_factor * v;
        if (have_lo && va > v && rd.relax > 1.f) {
          float sec = v * (t - a) / (va - v);  // distance to the secant's root
          step = fminf(fmaxf(step, sec), rd.relax * step);
        }
        a = t;
        va = v;
        have_lo = true;
        t += step;
        if (t > f.tmax) status = 0;
        else if (steps >= rd.max_steps) status = 2;
      }
    } else if (mode == kProbe) {
      ++steps;
      if (v > 0.f) {
        va = v;
        begin_root = true;
      } else {
        // the network passed the crossing: march again from the camera
        t = 0.f;
        t_lo = 0.f;
        have_lo = false;
        restarted = true;
        mode = kMarch;
        if (steps >= rd.max_steps) status = 2;
      }
    } else if (NT == 1u || mode == kRoot) {
      ++steps;
      if (fabsf(v) < 1e-6f || ++iters >= rd.root_steps) {
        hit_here = true;
      } else {
        if (v < 0.f) {
          b = t;
          vb = v;
          if (side < 0) va *= 0.5f;
          side = -1;
        } else {
          a = t;
          va = v;
          if (side > 0) vb *= 0.5f;
          side = 1;
        }
        const float tn = b - vb * (b - a) / (vb - va);
        // the next secant point moves less than root_tol: take it unevaluated
        if (fabsf(tn - t) < rd.root_tol) hit_here = true;
        t = tn;
      }
    } else if (NT == 4u) {
      V3 e = tet_dir(tap);
      nx = __fmaf_rn(e.x, v, nx);
      ny = __fmaf_rn(e.y, v, ny);
      nz = __fmaf_rn(e.z, v, nz);
      if (tap == 3) status = 1;
      else ++tap;
    } else {
      if ((tap & 1u) == 0u) {
        plus = v;
      } else {
        float diff = plus - v;
        if (tap == 1) nx = diff;
        else if (tap == 3) ny = diff;
        else nz = diff;
      }
      if (tap == 5) status = 1;
      else ++tap;
    }
    if (begin_root) {
      mode = kRoot;
      side = 0;
      iters = 0;
      t = b - vb * (b - a) / (vb - va);
      // a bracket narrower than root_tol: its secant root is the hit
      if (b - a < rd.root_tol) hit_here = true;
    }
    if (hit_here) {
      p = v3(__fmaf_rn(t, d.x, o.x), __fmaf_rn(t, d.y, o.y), __fmaf_rn(t, d.z, o.z));
      if (NT == 1u) {
        // the hit is final here; k_sdf_grad_normal adds the normal
        status = 1;
      } else {
        delta = 0.002f * t;
        mode = kNormal;
        tap = 0;
        nx = ny = nz = 0.f;
      }
    }
    if (status != 3) {
      float4 r0 = make_float4(0.f, 0.f, 0.f, 0.f), r1;
      uint32_t total_steps = base_steps + steps;
      if (status == 1) {
        V3 n = NT == 1u ? v3(0.f, 0.f, 0.f) : normalize(v3(nx, ny, nz));
        r0 = make_float4(p.x, p.y, p.z, n.x);
        r1 = make_float4(n.y, n.z, __uint_as_float(total_steps), __uint_as_float(status));
      } else {
        r1 = make_float4(0.f, 0.f, __uint_as_float(total_steps), __uint_as_float(status));
      }
      out[2 * (size_t)pix] = r0;
      out[2 * (size_t)pix + 1] = r1;
      live = false;
    }
  }
  n_exact = __reduce_add_sync(0xFFFFFFFFu, n_exact);
  n_normal = __reduce_add_sync(0xFFFFFFFFu, n_normal);
  if (lane == 0) {
    atomicAdd(&totals[1], (unsigned long long)n_exact);
    atomicAdd(&totals[2], (unsigned long long)n_normal);
  }
}

// normal_taps 1: the normal of every hit in `out` (status 1) is the exact
// field's analytic gradient at the hit position, normalised
// (terrain_gradient: one lattice walk per octave, about 1.5 field
// evaluations of work, against 4 or 6 for the finite-difference stencils,
// which at radius 0.002 t are coarse estimates of this gradient).  A
// separate pass, so that the exact phase's state machine keeps a single
// field call site and the gradient's lanes do not diverge from the march.
__global__ void __launch_bounds__(256) k_sdf_grad_normal(PermTable perm, FieldDev f, uint32_t n,
                                                         float4* __restrict__ out,
                                                         unsigned long long* __restrict__ totals) {
  extern __shared__ uint32_t perm_smem[];
  load_perm(perm, perm_smem);
  Perm P = perm_view(perm_smem);
  uint32_t count = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 r1 = out[2 * (size_t)i + 1];
    if (__float_as_uint(r1.w) != 1u) continue;
    float4 r0 = out[2 * (size_t)i];
    V3 nn = normalize(terrain_gradient(P, v3(r0.x, r0.y, r0.z), f.octaves, f.scale, f.amp));
    r0.w = nn.x;
    r1.x = nn.y;
    r1.y = nn.z;
    out[2 * (size_t)i] = r0;
    out[2 * (size_t)i + 1] = r1;
    ++count;
  }
  count = __reduce_add_sync(0xFFFFFFFFu, count);
  if ((threadIdx.x & 31u) == 0u && count) atomicAdd(&totals[2], (unsigned long long)count);
}

// Finite-difference gradient norm of the network at n sample points (vals
// holds 4 evaluations per point: p, p+hx, p+hy, p+hz).
__global__ void k_grad_norm(const float* __restrict__ vals, uint32_t n, float h,
                            float* __restrict__ norms) {
  uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float v0 = vals[4 * (size_t)i];
  float gx = (vals[4 * (size_t)i + 1] - v0) / h, gy = (vals[4 * (size_t)i + 2] - v0) / h,
        gz = (vals[4 * (size_t)i + 3] - v0) / h;
  norms[i] = sqrtf(gx * gx + gy * gy + gz * gz);
}

}  // namespace nsdf
}  // namespace re

// ----------------------------------------------------------------- host
struct re_nsdf {
  int device = 0;
  re::nsdf::InputMap map;
  uint32_t seed = 1;
  float* params = nullptr;  // [kNumParams]
  float* grad = nullptr;
  float* adam_m = nullptr;
  float* adam_v = nullptr;
  unsigned char* pack = nullptr;
  bool pack_valid = false;
  uint32_t* step_ctr = nullptr;
  float4* data = nullptr;
  uint32_t npts = 0;
  // training buffers for `batch` rows
  uint32_t batch = 0;
  re::nsdf::TrainBufs tb{};
  float* loss_hist = nullptr;
  uint32_t loss_cap = 0;
  unsigned char* train_pack = nullptr;  // BF16 weights of the training kernels
  int fwd_grid = 0, bwd_grid = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  float graph_lr = -1.f;
  // tracing scratch
  // [0] pixel cursor [1] queue size [2] refine cursor; from byte 16, u64
  // totals of the last trace: network evaluations of rays, exact
  // evaluations (march/probe/root), exact normal taps, network rows computed
  uint32_t* counters = nullptr;
  uint4* queue = nullptr;
  size_t queue_cap = 0;
  int* err = nullptr;
  // cone phase: start parameters of the fine tiles, then of the coarse ones;
  // the image and fine tile size of the last network phase that wrote them
  float* cone_t = nullptr;
  size_t cone_cap = 0;
  uint32_t cone_w = 0, cone_h = 0, cone_tile = 0, cone_tiles_x = 0;
  float lipschitz = 0.f;
  uint32_t total_steps_done = 0;
};

namespace re {
namespace {

using namespace nsdf;

void free_train(re_nsdf* s) {
  if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
  if (s->graph) cudaGraphDestroy(s->graph);
  s->graph_exec = nullptr;
  s->graph = nullptr;
  cudaFree(s->tb.x0);
  for (int l = 0; l < 4; ++l) cudaFree(s->tb.z[l]);
  for (int l = 0; l < 3; ++l) cudaFree(s->tb.a[l]);
  cudaFree(s->tb.da);
  cudaFree(s->tb.da2);
  cudaFree(s->tb.part);
  cudaFree(s->tb.part_head);
  cudaFree(s->train_pack);
  s->train_pack = nullptr;
  s->tb = TrainBufs{};
  s->batch = 0;
}

// Persistent grids of the training kernels: as many CTAs per SM as shared
// memory holds (the occupancy API answers 1 for these tensor-memory kernels,
// measured, where the SM fits 2 forward or 3 backward CTAs), and never more
// than tensor memory holds (512 columns: 64 per forward CTA, 128 per
// backward CTA), so that no tcgen05.alloc has to wait.
template <typename K>
int train_grid(K kernel, size_t smem, int tmem_cols, uint32_t tiles) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTrRows, smem) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  int dev = 0, smem_sm = 0, reserved = 0;
  if (cudaGetDevice(&dev) == cudaSuccess &&
      cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) ==
          cudaSuccess &&
      cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) ==
          cudaSuccess)
    per_sm = std::max(per_sm, smem_sm / (int)(smem + (size_t)reserved));
  per_sm = std::min(per_sm, 512 / tmem_cols);
  return (int)std::min<uint32_t>(tiles, (uint32_t)(per_sm * sm_count()));
}

re_status alloc_train(re_nsdf* s, uint32_t batch) {
  if (s->batch == batch) return RE_OK;
  free_train(s);
  // the whole shared-memory carveout, so that 2-3 of these 75 KB CTAs fit on
  // an SM (measured: the default carveout held one, 4 warps per SM)
  RE_CUDA(cudaFuncSetAttribute(k_tc_train_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kTrFwdSmemBytes));
  RE_CUDA(cudaFuncSetAttribute(k_tc_train_fwd, cudaFuncAttributePreferredSharedMemoryCarveout,
                               100));
  RE_CUDA(cudaFuncSetAttribute(k_tc_train_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)kTrBwdSmemBytes));
  RE_CUDA(cudaFuncSetAttribute(k_tc_train_bwd, cudaFuncAttributePreferredSharedMemoryCarveout,
                               100));
  size_t B = batch;
  uint32_t tiles = batch / kTrRows;
  s->fwd_grid = train_grid(k_tc_train_fwd, kTrFwdSmemBytes, 64, tiles);
  s->bwd_grid = train_grid(k_tc_train_bwd, kTrBwdSmemBytes, 128, tiles);
  RE_CUDA(cudaMalloc(&s->tb.x0, B * kIn * 2));
  for (int l = 0; l < 4; ++l) RE_CUDA(cudaMalloc(&s->tb.z[l], B * kHidden * 4));
  for (int l = 0; l < 3; ++l) RE_CUDA(cudaMalloc(&s->tb.a[l], B * kHidden * 2));
  RE_CUDA(cudaMalloc(&s->tb.da, B * kHidden * 4));
  RE_CUDA(cudaMalloc(&s->tb.da2, B * kHidden * 4));
  RE_CUDA(cudaMalloc(&s->tb.part, (size_t)s->bwd_grid * kNumParams * 4));
  RE_CUDA(cudaMalloc(&s->tb.part_head, (size_t)tiles * (kHidden + 2) * 4));
  RE_CUDA(cudaMalloc(&s->train_pack, kTrPackBytes));
  s->batch = batch;
  return RE_OK;
}

re_status check(const re_nsdf* s, const char* fn) {
  if (!s) return fail(RE_ERR_INVALID_ARG, "%s: null model", fn);
  int dev = -1;
  RE_CUDA(cudaGetDevice(&dev));
  if (dev != s->device)
    return fail(RE_ERR_INVALID_ARG, "%s: model lives on device %d, current device is %d", fn,
                s->device, dev);
  return RE_OK;
}

// One optimisation step on a batch (sampled from s->data, or given points
// when direct): pack, forward + L1 loss, backward, reduction, optional Adam.
re_status enqueue_step(re_nsdf* s, const float4* data, uint32_t npts, int direct, float lr,
                       bool adam, float* pred, cudaStream_t st) {
  uint32_t B = s->batch;
  uint32_t nfwd = B / kTrRows, nbwd = (uint32_t)s->bwd_grid;
  k_pack_train<<<(3 * kHidden * kHidden + 255) / 256, 256, 0, st>>>(s->params, s->train_pack);
  k_tc_train_fwd<<<s->fwd_grid, kTrRows, kTrFwdSmemBytes, st>>>(
      s->map, data, npts, s->step_ctr, s->seed, direct, s->train_pack, s->params, s->tb, B, pred,
      s->err);
  // backward: da holds dA4; alternate da / da2
  float* din = s->tb.da;
  float* dout = s->tb.da2;
  for (int l = 3; l >= 0; --l) {
    k_tc_train_bwd<<<s->bwd_grid, kTrRows, kTrBwdSmemBytes, st>>>(l, s->train_pack, s->tb, din,
                                                                  l > 0 ? dout : nullptr, B,
                                                                  s->err);
    std::swap(din, dout);
  }
  k_reduce<<<(kNumParams + 2 + 255) / 256, 256, 0, st>>>(s->tb, nbwd, nfwd, s->grad,
                                                         adam ? s->loss_hist : nullptr,
                                                         s->step_ctr, B);
  if (adam) {
    k_adam<<<(kNumParams + 255) / 256, 256, 0, st>>>(s->params, s->grad, s->adam_m, s->adam_v,
                                                     s->step_ctr, lr);
    k_step_inc<<<1, 1, 0, st>>>(s->step_ctr);
  }
  RE_CHECK_LAUNCH("nsdf training step launch");
  return RE_OK;
}

re_status ensure_pack(re_nsdf* s, cudaStream_t st) {
  if (s->pack_valid) return RE_OK;
  // one thread per element of the largest section (W2..W4: 3 x 64 x 64)
  constexpr int kPackThreads = 3 * kHidden * kHidden > kHidden * kIn ? 3 * kHidden * kHidden
                                                                      : kHidden * kIn;
  k_pack<<<(kPackThreads + 255) / 256, 256, 0, st>>>(s->params, s->pack);
  RE_CHECK_LAUNCH("nsdf pack launch");
  s->pack_valid = true;
  return RE_OK;
}

constexpr size_t kTcSmemBytes = sizeof(TcSmem) + 1024;

template <typename K>
int tc_grid(K kernel) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTcThreads, kTcSmemBytes) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  per_sm = std::min(per_sm, 2);  // 2 x 256 TMEM columns of 512
  return per_sm * sm_count();
}

CamDev cam_dev(const re_camera& c) {
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

PermTable perm_of(uint32_t seed) {
  uint32_t full[512];
  perlin_permutation(seed, full);
  PermTable t;
  for (int i = 0; i < 512; ++i) t.p[i] = (uint8_t)full[i];
  return t;
}

FieldDev field_of(const re_sdf_params& p) {
  FieldDev f;
  f.octaves = p.octaves;
  f.max_steps = p.max_steps;
  f.scale = p.scale;
  f.amp = p.amplitude;
  f.step_factor = p.step_factor;
  f.eps = p.eps;
  f.tmax = p.tmax;
  return f;
}

re_status check_field(const re_sdf_params* p, const char* fn) {
  if (!p) return fail(RE_ERR_INVALID_ARG, "%s: null field", fn);
  if (p->octaves > 32) return fail(RE_ERR_LIMIT, "%s: octaves > 32", fn);
  if (p->max_steps == 0 || p->max_steps > (1u << 20))
    return fail(RE_ERR_LIMIT, "%s: max_steps must be in [1, 2^20]", fn);
  return RE_OK;
}

}  // namespace
}  // namespace re

extern "C" {

RE_API uint32_t re_nsdf_num_params(void) { return (uint32_t)re::nsdf::kNumParams; }

RE_API re_status re_nsdf_box_for_camera(const re_camera* cam, uint32_t w, uint32_t h, float tmax,
                                        float y_lo, float y_hi, float* box_min, float* box_max) {
  if (!cam || !box_min || !box_max || w < 2 || h < 2 || !(tmax > 0.f) || !(y_hi > y_lo))
    return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_box_for_camera: bad arguments");
  re::CamBasis b;
  re::camera_basis(*cam, b);
  double lo[3], hi[3];
  for (int k = 0; k < 3; ++k) lo[k] = hi[k] = b.campos[k];
  for (int cx = -1; cx <= 1; cx += 2)
    for (int cy = -1; cy <= 1; cy += 2) {
      double dir[3], n = 0;
      for (int k = 0; k < 3; ++k) {
        dir[k] = (b.middle[k] + cx * b.horizontal[k] + cy * b.vertical[k] - b.campos[k]) * b.focal;
        n += dir[k] * dir[k];
      }
      n = std::sqrt(n);
      for (int k = 0; k < 3; ++k) {
        double e = b.campos[k] + dir[k] / n * tmax;
        lo[k] = std::min(lo[k], e);
        hi[k] = std::max(hi[k], e);
      }
    }
  lo[1] = std::max(lo[1], (double)y_lo);
  hi[1] = std::min(hi[1], (double)y_hi);
  if (!(hi[1] > lo[1])) {
    lo[1] = y_lo;
    hi[1] = y_hi;
  }
  for (int k = 0; k < 3; ++k) {
    box_min[k] = (float)lo[k];
    box_max[k] = (float)hi[k];
  }
  return RE_OK;
}

RE_API re_status re_nsdf_create(const re_nsdf_config* cfg, re_nsdf** out) {
  using namespace re::nsdf;
  if (!cfg || !out) return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_create: null argument");
  for (int k = 0; k < 3; ++k)
    if (!(cfg->box_max[k] > cfg->box_min[k]))
      return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_create: empty box");
  if (!(cfg->f0 > 0.f)) return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_create: f0 must be > 0");
  re_nsdf* s = new (std::nothrow) re_nsdf();
  if (!s) return re::fail(RE_ERR_OUT_OF_MEMORY, "re_nsdf_create: host allocation");
  cudaError_t e = cudaGetDevice(&s->device);
  for (int k = 0; k < 3; ++k) {
    s->map.center[k] = 0.5f * (cfg->box_min[k] + cfg->box_max[k]);
    s->map.inv_half[k] = 2.0f / (cfg->box_max[k] - cfg->box_min[k]);
  }
  s->map.f0 = cfg->f0;
  s->seed = cfg->seed;
  if (e == cudaSuccess) e = cudaMalloc(&s->params, kNumParams * 4);
  if (e == cudaSuccess) e = cudaMalloc(&s->grad, kNumParams * 4);
  if (e == cudaSuccess) e = cudaMalloc(&s->adam_m, kNumParams * 4);
  if (e == cudaSuccess) e = cudaMalloc(&s->adam_v, kNumParams * 4);
  if (e == cudaSuccess) e = cudaMalloc(&s->pack, re::nsdf::kPackBytes);
  if (e == cudaSuccess) e = cudaMalloc(&s->step_ctr, 16);
  if (e == cudaSuccess) e = cudaMalloc(&s->counters, 64);
  if (e == cudaSuccess) e = cudaMalloc(&s->err, 4);
  if (e == cudaSuccess) e = cudaMemset(s->adam_m, 0, kNumParams * 4);
  if (e == cudaSuccess) e = cudaMemset(s->adam_v, 0, kNumParams * 4);
  if (e == cudaSuccess) e = cudaMemset(s->step_ctr, 0, 16);
  if (e == cudaSuccess) e = cudaMemset(s->err, 0, 4);
  if (e == cudaSuccess) {
    // Glorot-uniform weights, zero biases (std::mt19937 seeded by cfg->seed)
    std::vector<float> h(kNumParams, 0.f);
    std::mt19937 gen(cfg->seed);
    auto fill = [&](int off, int fan_out, int fan_in) {
      float a = std::sqrt(6.0f / (float)(fan_in + fan_out));
      std::uniform_real_distribution<float> U(-a, a);
      for (int i = 0; i < fan_out * fan_in; ++i) h[off + i] = U(gen);
    };
    fill(OFF_W1, kHidden, kIn);
    fill(OFF_W2, kHidden, kHidden);
    fill(OFF_W3, kHidden, kHidden);
    fill(OFF_W4, kHidden, kHidden);
    fill(OFF_W5, 1, kHidden);
    e = cudaMemcpy(s->params, h.data(), kNumParams * 4, cudaMemcpyHostToDevice);
  }
  if (e != cudaSuccess) {
    re_status st = re::cuda_fail(e, "re_nsdf_create");
    re_nsdf_destroy(s);
    return st;
  }
  *out = s;
  return RE_OK;
}

RE_API re_status re_nsdf_destroy(re_nsdf* s) {
  if (!s) return RE_OK;
  re::free_train(s);
  cudaFree(s->params);
  cudaFree(s->grad);
  cudaFree(s->adam_m);
  cudaFree(s->adam_v);
  cudaFree(s->pack);
  cudaFree(s->step_ctr);
  cudaFree(s->data);
  cudaFree(s->loss_hist);
  cudaFree(s->counters);
  cudaFree(s->queue);
  cudaFree(s->cone_t);
  cudaFree(s->err);
  delete s;
  return RE_OK;
}

RE_API re_status re_nsdf_get_params(const re_nsdf* s, float* host) {
  re_status st = re::check(s, "re_nsdf_get_params");
  if (st != RE_OK) return st;
  if (!host) return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_get_params: null output");
  RE_CUDA(cudaMemcpy(host, s->params, re::nsdf::kNumParams * 4, cudaMemcpyDeviceToHost));
  return RE_OK;
}

RE_API re_status re_nsdf_set_params(re_nsdf* s, const float* host) {
  re_status st = re::check(s, "re_nsdf_set_params");
  if (st != RE_OK) return st;
  if (!host) return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_set_params: null input");
  RE_CUDA(cudaMemcpy(s->params, host, re::nsdf::kNumParams * 4, cudaMemcpyHostToDevice));
  s->pack_valid = false;
  s->lipschitz = 0.f;
  return RE_OK;
}

RE_API re_status re_nsdf_generate(re_nsdf* s, const re_sdf_params* field, const re_camera* cam,
                                  uint32_t w, uint32_t h, uint32_t num_points, uint32_t seed,
                                  void* stream) {
  re_status st = re::check(s, "re_nsdf_generate");
  if (st != RE_OK) return st;
  st = re::check_field(field, "re_nsdf_generate");
  if (st != RE_OK) return st;
  if (!cam || w < 2 || h < 2 || num_points < 2)
    return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_generate: bad arguments");
  if (num_points > (1u << 28)) return re::fail(RE_ERR_LIMIT, "re_nsdf_generate: > 2^28 points");
  cudaStream_t cs = (cudaStream_t)stream;
  if (s->npts != num_points) {
    RE_CUDA(cudaStreamSynchronize(cs));
    cudaFree(s->data);
    s->data = nullptr;
    s->npts = 0;
    RE_CUDA(cudaMalloc(&s->data, (size_t)num_points * sizeof(float4)));
    s->npts = num_points;
  }
  float3 bmin, bmax;
  bmin.x = s->map.center[0] - 1.f / s->map.inv_half[0];
  bmin.y = s->map.center[1] - 1.f / s->map.inv_half[1];
  bmin.z = s->map.center[2] - 1.f / s->map.inv_half[2];
  bmax.x = s->map.center[0] + 1.f / s->map.inv_half[0];
  bmax.y = s->map.center[1] + 1.f / s->map.inv_half[1];
  bmax.z = s->map.center[2] + 1.f / s->map.inv_half[2];
  RE_CUDA(cudaFuncSetAttribute(re::nsdf::k_nsdf_data, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)re::kPermSmemBytes));
  re::nsdf::k_nsdf_data<<<re::sm_count() * 3, 256, re::kPermSmemBytes, cs>>>(
      re::perm_of(field->seed), re::field_of(*field), re::cam_dev(*cam), w, h, bmin, bmax,
      num_points, seed, s->data);
  RE_CHECK_LAUNCH("re_nsdf_generate: launch");
  return RE_OK;
}

RE_API re_status re_nsdf_get_data(const re_nsdf* s, float* host_xyzl, uint32_t max_points) {
  re_status st = re::check(s, "re_nsdf_get_data");
  if (st != RE_OK) return st;
  if (!host_xyzl) return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_get_data: null output");
  uint32_t n = std::min(max_points, s->npts);
  RE_CUDA(cudaMemcpy(host_xyzl, s->data, (size_t)n * 16, cudaMemcpyDeviceToHost));
  return RE_OK;
}

RE_API re_status re_nsdf_train(re_nsdf* s, uint32_t steps, uint32_t batch, float lr,
                               float* loss_out, void* stream) {
  re_status st = re::check(s, "re_nsdf_train");
  if (st != RE_OK) return st;
  if (!s->data || s->npts == 0) return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_train: no data (call re_nsdf_generate)");
  if (batch == 0 || batch % re::nsdf::kRowsBwd != 0 || batch > (1u << 22))
    return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_train: batch must be a positive multiple of %d up to 2^22",
                    re::nsdf::kRowsBwd);
  if (steps == 0) return RE_OK;
  cudaStream_t cs = (cudaStream_t)stream;
  st = re::alloc_train(s, batch);
  if (st != RE_OK) return st;
  uint32_t done = s->total_steps_done;
  if (s->loss_cap < done + steps) {
    RE_CUDA(cudaStreamSynchronize(cs));
    float* nh = nullptr;
    uint32_t cap = std::max(done + steps, 2 * s->loss_cap);
    RE_CUDA(cudaMalloc(&nh, (size_t)cap * 4));
    if (s->loss_hist) {
      RE_CUDA(cudaMemcpy(nh, s->loss_hist, (size_t)s->loss_cap * 4, cudaMemcpyDeviceToDevice));
      cudaFree(s->loss_hist);
    }
    s->loss_hist = nh;
    s->loss_cap = cap;
    if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    s->graph_exec = nullptr;
    s->graph = nullptr;
  }
  if (!s->graph_exec || s->graph_lr != lr) {
    if (s->graph_exec) cudaGraphExecDestroy(s->graph_exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    s->graph_exec = nullptr;
    s->graph = nullptr;
    cudaStream_t cap_stream;
    RE_CUDA(cudaStreamCreateWithFlags(&cap_stream, cudaStreamNonBlocking));
    cudaError_t e = cudaStreamBeginCapture(cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e == cudaSuccess) {
      st = re::enqueue_step(s, s->data, s->npts, 0, lr, true, nullptr, cap_stream);
      e = cudaStreamEndCapture(cap_stream, &s->graph);
    }
    if (e == cudaSuccess && st == RE_OK) e = cudaGraphInstantiate(&s->graph_exec, s->graph, 0);
    cudaStreamDestroy(cap_stream);
    if (st != RE_OK) return st;
    if (e != cudaSuccess) return re::cuda_fail(e, "re_nsdf_train: graph capture");
    s->graph_lr = lr;
  }
  RE_CUDA(cudaMemsetAsync(s->err, 0, 4, cs));
  for (uint32_t i = 0; i < steps; ++i) RE_CUDA(cudaGraphLaunch(s->graph_exec, cs));
  s->pack_valid = false;
  s->lipschitz = 0.f;
  if (loss_out)
    RE_CUDA(cudaMemcpyAsync(loss_out, s->loss_hist + done, (size_t)steps * 4,
                            cudaMemcpyDeviceToHost, cs));
  int herr = 0;
  RE_CUDA(cudaMemcpyAsync(&herr, s->err, 4, cudaMemcpyDeviceToHost, cs));
  RE_CUDA(cudaStreamSynchronize(cs));
  s->total_steps_done = done + steps;
  if (herr) return re::fail(RE_ERR_INTERNAL, "re_nsdf_train: tensor-core wait bound reached");
  return RE_OK;
}

// Loss gradient of a given batch (points + labels as float4), no update.
RE_API re_status re_nsdf_loss_grad(re_nsdf* s, const float* d_xyzl, uint32_t n, float* d_grad,
                                   float* d_pred, void* stream) {
  re_status st = re::check(s, "re_nsdf_loss_grad");
  if (st != RE_OK) return st;
  if (!d_xyzl || !d_grad || n == 0 || n % re::nsdf::kRowsBwd != 0)
    return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_loss_grad: n must be a positive multiple of %d",
                    re::nsdf::kRowsBwd);
  cudaStream_t cs = (cudaStream_t)stream;
  st = re::alloc_train(s, n);
  if (st != RE_OK) return st;
  RE_CUDA(cudaMemsetAsync(s->err, 0, 4, cs));
  st = re::enqueue_step(s, reinterpret_cast<const float4*>(d_xyzl), n, 1, 0.f, false, d_pred, cs);
  if (st != RE_OK) return st;
  RE_CUDA(cudaMemcpyAsync(d_grad, s->grad, re::nsdf::kNumParams * 4, cudaMemcpyDeviceToDevice, cs));
  int herr = 0;
  RE_CUDA(cudaMemcpyAsync(&herr, s->err, 4, cudaMemcpyDeviceToHost, cs));
  RE_CUDA(cudaStreamSynchronize(cs));
  if (herr) return re::fail(RE_ERR_INTERNAL, "re_nsdf_loss_grad: tensor-core wait bound reached");
  return RE_OK;
}

RE_API re_status re_nsdf_eval(re_nsdf* s, const float* d_pts, uint32_t n, float* d_out,
                              void* stream) {
  re_status st = re::check(s, "re_nsdf_eval");
  if (st != RE_OK) return st;
  if (!d_pts || !d_out) return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_eval: null buffer");
  if (n == 0) return RE_OK;
  cudaStream_t cs = (cudaStream_t)stream;
  st = re::ensure_pack(s, cs);
  if (st != RE_OK) return st;
  auto k = re::nsdf::k_tc_eval;
  RE_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)re::kTcSmemBytes));
  int grid = std::min<int>(re::tc_grid(k), (int)((n + 511) / 512));
  RE_CUDA(cudaMemsetAsync(s->err, 0, 4, cs));
  k<<<grid, re::nsdf::kTcThreads, re::kTcSmemBytes, cs>>>(s->map, s->pack, d_pts, n, d_out, s->err);
  RE_CHECK_LAUNCH("re_nsdf_eval: launch");
  int herr = 0;
  RE_CUDA(cudaMemcpyAsync(&herr, s->err, 4, cudaMemcpyDeviceToHost, cs));
  RE_CUDA(cudaStreamSynchronize(cs));
  if (herr) return re::fail(RE_ERR_INTERNAL, "re_nsdf_eval: tensor-core wait bound reached");
  return RE_OK;
}

RE_API re_status re_nsdf_eval_reference(re_nsdf* s, const float* d_pts, uint32_t n, float* d_out,
                                        void* stream) {
  re_status st = re::check(s, "re_nsdf_eval_reference");
  if (st != RE_OK) return st;
  if (!d_pts || !d_out) return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_eval_reference: null buffer");
  if (n == 0) return RE_OK;
  re::nsdf::k_ref_eval<<<(n + 127) / 128, 128, 0, (cudaStream_t)stream>>>(s->map, s->params, d_pts,
                                                                            n, d_out);
  RE_CHECK_LAUNCH("re_nsdf_eval_reference: launch");
  return RE_OK;
}

// Lipschitz estimate of the network over `samples` training points: the
// `quantile` (1 = the maximum) of the forward-difference gradient norms
// with step h.
RE_API re_status re_nsdf_lipschitz(re_nsdf* s, uint32_t samples, float h, float quantile,
                                   float* out, void* stream) {
  re_status st = re::check(s, "re_nsdf_lipschitz");
  if (st != RE_OK) return st;
  if (!out || samples == 0 || !(h > 0.f) || !(quantile > 0.f && quantile <= 1.f) || !s->data)
    return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_lipschitz: bad arguments or no data");
  cudaStream_t cs = (cudaStream_t)stream;
  uint32_t n = std::min(samples, s->npts);
  std::vector<float4> pts(n);
  RE_CUDA(cudaMemcpy(pts.data(), s->data, (size_t)n * 16, cudaMemcpyDeviceToHost));
  std::vector<float> q(12 * (size_t)n);
  for (uint32_t i = 0; i < n; ++i) {
    float p[3] = {pts[i].x, pts[i].y, pts[i].z};
    for (int k = 0; k < 4; ++k)
      for (int a = 0; a < 3; ++a) q[12 * (size_t)i + 3 * k + a] = p[a] + ((k == a + 1) ? h : 0.f);
  }
  float *dq = nullptr, *dv = nullptr, *dn = nullptr;
  std::vector<float> norms(n);
  RE_CUDA(cudaMalloc(&dq, q.size() * 4));
  cudaError_t e = cudaMalloc(&dv, (size_t)n * 4 * 4);
  if (e == cudaSuccess) e = cudaMalloc(&dn, (size_t)n * 4);
  if (e == cudaSuccess) e = cudaMemcpy(dq, q.data(), q.size() * 4, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    st = re_nsdf_eval(s, dq, 4 * n, dv, stream);
    if (st == RE_OK) {
      re::nsdf::k_grad_norm<<<(n + 255) / 256, 256, 0, cs>>>(dv, n, h, dn);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaMemcpyAsync(norms.data(), dn, (size_t)n * 4, cudaMemcpyDeviceToHost, cs);
      if (e == cudaSuccess) e = cudaStreamSynchronize(cs);
    }
  }
  cudaFree(dq);
  cudaFree(dv);
  cudaFree(dn);
  if (st != RE_OK) return st;
  if (e != cudaSuccess) return re::cuda_fail(e, "re_nsdf_lipschitz");
  size_t k = std::min<size_t>(n - 1, (size_t)std::ceil((double)quantile * n) - 1);
  std::nth_element(norms.begin(), norms.begin() + k, norms.end());
  *out = norms[k];
  s->lipschitz = norms[k];
  return RE_OK;
}

namespace re {
namespace {
re_status trace_check(re_nsdf* s, const re_sdf_params* field, const re_nsdf_trace_params* tp,
                      const re_camera* cam, uint32_t w, uint32_t h, re_sdf_hit* d_out,
                      const char* fn) {
  re_status st = check(s, fn);
  if (st != RE_OK) return st;
  st = check_field(field, fn);
  if (st != RE_OK) return st;
  if (!tp || !cam || !d_out || w < 2 || h < 2) return fail(RE_ERR_INVALID_ARG, "%s: bad arguments", fn);
  if ((uint64_t)w * h > (1ull << 28)) return fail(RE_ERR_LIMIT, "%s: image > 2^28 pixels", fn);
  if (!(tp->flags & RE_NSDF_EXACT_ONLY) && !(tp->lipschitz > 0.f && tp->safety > 0.f))
    return fail(RE_ERR_INVALID_ARG, "%s: lipschitz and safety must be > 0", fn);
  if (tp->cone_tile > 256 ||
      (tp->cone_coarse && (tp->cone_tile == 0 || tp->cone_coarse > 1024 ||
                           tp->cone_coarse <= tp->cone_tile || tp->cone_coarse % tp->cone_tile)))
    return fail(RE_ERR_INVALID_ARG,
                "%s: cone_tile <= 256; cone_coarse 0 or a multiple of cone_tile above it, <= 1024",
                fn);
  if (tp->normal_taps != 0 && tp->normal_taps != 1 && tp->normal_taps != 4 &&
      tp->normal_taps != 6)
    return fail(RE_ERR_INVALID_ARG, "%s: normal_taps 0, 1, 4 or 6", fn);
  if (tp->cone_lanes > 16 || (tp->cone_lanes & (tp->cone_lanes - 1u)))
    return fail(RE_ERR_INVALID_ARG, "%s: cone_lanes 0, 1, 2, 4, 8 or 16", fn);
  return RE_OK;
}
}  // namespace
}  // namespace re

RE_API re_status re_nsdf_trace_network(re_nsdf* s, const re_sdf_params* field,
                                       const re_nsdf_trace_params* tp, const re_camera* cam,
                                       uint32_t w, uint32_t h, re_sdf_hit* d_out, void* stream) {
  re_status st = re::trace_check(s, field, tp, cam, w, h, d_out, "re_nsdf_trace_network");
  if (st != RE_OK) return st;
  cudaStream_t cs = (cudaStream_t)stream;
  const bool exact_only = (tp->flags & RE_NSDF_EXACT_ONLY) != 0u;
  const bool cone = !exact_only && tp->cone_tile > 0;
  size_t need = (size_t)w * h;
  const uint32_t T = tp->cone_tile, C = tp->cone_coarse;
  const uint32_t ctx = cone ? (w + T - 1) / T : 0, cty = cone ? (h + T - 1) / T : 0;
  const uint32_t pcx = cone && C ? (w + C - 1) / C : 0, pcy = cone && C ? (h + C - 1) / C : 0;
  const size_t cone_need = (size_t)ctx * cty + (size_t)pcx * pcy;
  if (cone && s->cone_cap < cone_need) {
    RE_CUDA(cudaStreamSynchronize(cs));
    cudaFree(s->cone_t);
    s->cone_t = nullptr;
    s->cone_cap = 0;
    RE_CUDA(cudaMalloc(&s->cone_t, cone_need * sizeof(float)));
    s->cone_cap = cone_need;
  }
  s->cone_w = s->cone_h = s->cone_tile = s->cone_tiles_x = 0;
  if (!exact_only && !cone && s->queue_cap < need) {
    RE_CUDA(cudaStreamSynchronize(cs));
    cudaFree(s->queue);
    s->queue = nullptr;
    s->queue_cap = 0;
    RE_CUDA(cudaMalloc(&s->queue, need * sizeof(uint4)));
    s->queue_cap = need;
  }
  RE_CUDA(cudaMemsetAsync(s->counters, 0, 64, cs));
  RE_CUDA(cudaMemsetAsync(s->err, 0, 4, cs));
  if (exact_only) return RE_OK;
  st = re::ensure_pack(s, cs);
  if (st != RE_OK) return st;
  unsigned long long* totals = reinterpret_cast<unsigned long long*>(s->counters + 4);
  re::nsdf::MarchDev md;
  md.alpha = tp->safety / tp->lipschitz;
  md.switch_dist = tp->switch_dist;
  md.min_step = tp->min_step;
  md.tmax = field->tmax;
  md.max_steps = tp->max_network_steps ? tp->max_network_steps : 256;
  for (int k = 0; k < 3; ++k) {
    float half = 1.0f / s->map.inv_half[k];
    md.bmin[k] = s->map.center[k] - half;
    md.bmax[k] = s->map.center[k] + half;
  }
  if (cone) {
    const uint32_t K = tp->cone_lanes ? tp->cone_lanes : 1u;
    auto kc = K == 16u  ? re::nsdf::k_nsdf_cone<16>
              : K == 8u ? re::nsdf::k_nsdf_cone<8>
              : K == 4u ? re::nsdf::k_nsdf_cone<4>
              : K == 2u ? re::nsdf::k_nsdf_cone<2>
                        : re::nsdf::k_nsdf_cone<1>;
    RE_CUDA(cudaFuncSetAttribute(kc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)re::kTcSmemBytes));
    float* fine = s->cone_t;
    float* coarse = s->cone_t + (size_t)ctx * cty;
    re::nsdf::ConeDev cd{};
    if (C) {
      // coarse level from the box entry (cursor counters[0])
      cd.tile = C;
      cd.tiles_x = pcx;
      cd.tiles_y = pcy;
      cd.parent = nullptr;
      const int grid = std::min<int>(re::tc_grid(kc),
                                     (int)((pcx * pcy * K + re::nsdf::kTcThreads - 1) /
                                           re::nsdf::kTcThreads));
      kc<<<grid, re::nsdf::kTcThreads, re::kTcSmemBytes, cs>>>(
          s->map, s->pack, md, cd, re::cam_dev(*cam), w, h, s->counters, totals, coarse, s->err);
      RE_CHECK_LAUNCH("re_nsdf_trace_network: coarse cone launch");
    }
    // fine level, from the coarse tiles' starts (cursor counters[3])
    cd.tile = T;
    cd.tiles_x = ctx;
    cd.tiles_y = cty;
    cd.parent = C ? coarse : nullptr;
    cd.parent_tile = C;
    cd.parent_tiles_x = pcx;
    const int grid = std::min<int>(
        re::tc_grid(kc), (int)((ctx * cty * K + re::nsdf::kTcThreads - 1) / re::nsdf::kTcThreads));
    kc<<<grid, re::nsdf::kTcThreads, re::kTcSmemBytes, cs>>>(
        s->map, s->pack, md, cd, re::cam_dev(*cam), w, h, s->counters + 3, totals, fine, s->err);
    RE_CHECK_LAUNCH("re_nsdf_trace_network: cone launch");
    s->cone_w = w;
    s->cone_h = h;
    s->cone_tile = T;
    s->cone_tiles_x = ctx;
    return RE_OK;
  }
  auto k = re::nsdf::k_nsdf_march;
  RE_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)re::kTcSmemBytes));
  k<<<re::tc_grid(k), re::nsdf::kTcThreads, re::kTcSmemBytes, cs>>>(
      s->map, s->pack, md, re::cam_dev(*cam), w, h, s->counters, totals, s->queue,
      reinterpret_cast<float4*>(d_out), s->err);
  RE_CHECK_LAUNCH("re_nsdf_trace_network: march launch");
  return RE_OK;
}

RE_API re_status re_nsdf_trace_exact(re_nsdf* s, const re_sdf_params* field,
                                     const re_nsdf_trace_params* tp, const re_camera* cam,
                                     uint32_t w, uint32_t h, re_sdf_hit* d_out, void* stream) {
  re_status st = re::trace_check(s, field, tp, cam, w, h, d_out, "re_nsdf_trace_exact");
  if (st != RE_OK) return st;
  const bool exact_only = (tp->flags & RE_NSDF_EXACT_ONLY) != 0u;
  const bool cone = !exact_only && tp->cone_tile > 0;
  if (cone && !(s->cone_w == w && s->cone_h == h && s->cone_tile == tp->cone_tile))
    return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_trace_exact: no cone phase for this image");
  if (!exact_only && !cone && s->queue_cap < (size_t)w * h)
    return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_trace_exact: no network phase for this image");
  cudaStream_t cs = (cudaStream_t)stream;
  unsigned long long* totals = reinterpret_cast<unsigned long long*>(s->counters + 4);
  auto kr = tp->normal_taps == 1u   ? re::nsdf::k_sdf_refine<1u>
            : tp->normal_taps == 4u ? re::nsdf::k_sdf_refine<4u>
                                    : re::nsdf::k_sdf_refine<6u>;
  RE_CUDA(cudaFuncSetAttribute(kr, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int)re::kPermSmemBytes));
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kr, 256, re::kPermSmemBytes) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  re::nsdf::RefineDev rd;
  rd.max_steps = tp->max_exact_steps ? tp->max_exact_steps : field->max_steps;
  rd.root_steps = tp->root_steps ? tp->root_steps : 4;
  rd.relax = tp->relax;
  rd.root_tol = tp->root_tol > 0.f ? tp->root_tol : 0.f;
  // |Perlin| <= 2 (each corner term |g . r| <= |r_x| + |r_y| <= 2 and the
  // interpolation is convex), so fBm <= 2 (2 - 2^(1 - octaves)) and the
  // density is positive above this height
  rd.ceiling =
      2.0f * std::fabs(field->amplitude) * (2.0f - std::ldexp(1.0f, 1 - (int)field->octaves)) + 1e-3f;
  rd.normal_taps = tp->normal_taps == 4u || tp->normal_taps == 1u ? tp->normal_taps : 6u;
  rd.tile_t = cone ? s->cone_t : nullptr;
  rd.cone_tile = cone ? s->cone_tile : 1u;
  rd.cone_tiles_x = cone ? s->cone_tiles_x : 0u;
  kr<<<per_sm * re::sm_count(), 256, re::kPermSmemBytes, cs>>>(
      re::perm_of(field->seed), re::field_of(*field), rd, re::cam_dev(*cam), w, h,
      exact_only || cone ? 1 : 0, s->queue, s->counters, totals, reinterpret_cast<float4*>(d_out));
  RE_CHECK_LAUNCH("re_nsdf_trace_exact: refine launch");
  if (rd.normal_taps == 1u) {
    auto kg = re::nsdf::k_sdf_grad_normal;
    int gper_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&gper_sm, kg, 256, re::kPermSmemBytes) !=
            cudaSuccess ||
        gper_sm < 1)
      gper_sm = 1;
    kg<<<gper_sm * re::sm_count(), 256, re::kPermSmemBytes, cs>>>(
        re::perm_of(field->seed), re::field_of(*field), w * h, reinterpret_cast<float4*>(d_out),
        totals);
    RE_CHECK_LAUNCH("re_nsdf_trace_exact: normal launch");
  }
  return RE_OK;
}

RE_API re_status re_nsdf_trace(re_nsdf* s, const re_sdf_params* field,
                               const re_nsdf_trace_params* tp, const re_camera* cam, uint32_t w,
                               uint32_t h, re_sdf_hit* d_out, void* stream) {
  re_status st = re_nsdf_trace_network(s, field, tp, cam, w, h, d_out, stream);
  if (st != RE_OK) return st;
  return re_nsdf_trace_exact(s, field, tp, cam, w, h, d_out, stream);
}

RE_API re_status re_nsdf_trace_status(re_nsdf* s, uint32_t* num_refined, int* error,
                                      uint64_t* evals) {
  re_status st = re::check(s, "re_nsdf_trace_status");
  if (st != RE_OK) return st;
  uint32_t c[16] = {};
  int e = 0;
  RE_CUDA(cudaMemcpy(c, s->counters, 64, cudaMemcpyDeviceToHost));
  RE_CUDA(cudaMemcpy(&e, s->err, 4, cudaMemcpyDeviceToHost));
  if (num_refined) *num_refined = c[1];
  if (error) *error = e;
  if (evals) std::memcpy(evals, c + 4, 4 * sizeof(uint64_t));
  return RE_OK;
}

// Checkpoint: 16-byte header ("RENSDF01", parameter count, steps done),
// the input map, then parameters and both Adam moments as FP32.
RE_API re_status re_nsdf_save(const re_nsdf* s, const char* path) {
  using namespace re::nsdf;
  re_status st = re::check(s, "re_nsdf_save");
  if (st != RE_OK) return st;
  if (!path) return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_save: null path");
  std::vector<float> buf(3 * (size_t)kNumParams);
  RE_CUDA(cudaMemcpy(buf.data(), s->params, kNumParams * 4, cudaMemcpyDeviceToHost));
  RE_CUDA(cudaMemcpy(buf.data() + kNumParams, s->adam_m, kNumParams * 4, cudaMemcpyDeviceToHost));
  RE_CUDA(cudaMemcpy(buf.data() + 2 * kNumParams, s->adam_v, kNumParams * 4, cudaMemcpyDeviceToHost));
  uint32_t steps = 0;
  RE_CUDA(cudaMemcpy(&steps, s->step_ctr, 4, cudaMemcpyDeviceToHost));
  FILE* f = std::fopen(path, "wb");
  if (!f) return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_save: cannot open %s", path);
  uint32_t hdr[4] = {0x534E4552u, 0x31304653u, (uint32_t)kNumParams, steps};
  bool ok = std::fwrite(hdr, 4, 4, f) == 4 && std::fwrite(&s->map, sizeof(s->map), 1, f) == 1 &&
            std::fwrite(buf.data(), 4, buf.size(), f) == buf.size();
  std::fclose(f);
  if (!ok) return re::fail(RE_ERR_INTERNAL, "re_nsdf_save: write failed");
  return RE_OK;
}

RE_API re_status re_nsdf_load(re_nsdf* s, const char* path) {
  using namespace re::nsdf;
  re_status st = re::check(s, "re_nsdf_load");
  if (st != RE_OK) return st;
  if (!path) return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_load: null path");
  FILE* f = std::fopen(path, "rb");
  if (!f) return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_load: cannot open %s", path);
  uint32_t hdr[4];
  InputMap m;
  std::vector<float> buf(3 * (size_t)kNumParams);
  bool ok = std::fread(hdr, 4, 4, f) == 4 && hdr[0] == 0x534E4552u && hdr[1] == 0x31304653u &&
            hdr[2] == (uint32_t)kNumParams && std::fread(&m, sizeof(m), 1, f) == 1 &&
            std::fread(buf.data(), 4, buf.size(), f) == buf.size();
  std::fclose(f);
  if (!ok) return re::fail(RE_ERR_INVALID_ARG, "re_nsdf_load: %s is not a checkpoint of this network", path);
  RE_CUDA(cudaMemcpy(s->params, buf.data(), kNumParams * 4, cudaMemcpyHostToDevice));
  RE_CUDA(cudaMemcpy(s->adam_m, buf.data() + kNumParams, kNumParams * 4, cudaMemcpyHostToDevice));
  RE_CUDA(cudaMemcpy(s->adam_v, buf.data() + 2 * kNumParams, kNumParams * 4, cudaMemcpyHostToDevice));
  RE_CUDA(cudaMemcpy(s->step_ctr, &hdr[3], 4, cudaMemcpyHostToDevice));
  s->map = m;
  s->total_steps_done = hdr[3];
  s->pack_valid = false;
  s->lipschitz = 0.f;
  return RE_OK;
}

}  // extern "C"
