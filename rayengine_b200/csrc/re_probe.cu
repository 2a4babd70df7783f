// Measurement probes: the denominators the benchmark uses where the hardware
// peaks supplied with the pool have no figure.
//   L2 read bandwidth  the traversal kernels' L2 roofline (their node, leaf
//                      and triangle reads mostly hit L2)
//   FP32 FMA rate      the SIMT field kernels (noise, sphere tracing)
#include <cuda_runtime.h>

#include "re_common.hpp"

namespace re {
namespace {

// Every thread streams its share of an L2-resident buffer `passes` times
// with 16-byte L2-only loads (ld.global.cg); the XOR of everything read
// goes to `sink` so the loads cannot be removed.
__global__ void k_l2_read(const uint4* __restrict__ buf, size_t n, uint32_t passes,
                          uint4* __restrict__ sink) {
  uint4 acc = make_uint4(0u, 0u, 0u, 0u);
  size_t stride = (size_t)gridDim.x * blockDim.x;
  for (uint32_t p = 0; p < passes; ++p)
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += stride) {
      uint4 v = __ldcg(buf + i);
      acc.x ^= v.x;
      acc.y ^= v.y;
      acc.z ^= v.z;
      acc.w ^= v.w;
    }
  if ((acc.x ^ acc.y ^ acc.z ^ acc.w) == 0x9E3779B9u) sink[0] = acc;
}

// Every thread runs 8 independent FMA chains of `iters` steps; the operands
// come from the arguments so nothing folds, and the sum goes to `sink` only
// if it equals an impossible value.
__global__ void __launch_bounds__(256) k_fma(uint32_t iters, float a, float b, float* sink) {
  float x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = (float)(threadIdx.x + k);
  for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 8; ++k) x[k] = __fmaf_rn(x[k], a, b);
  }
  float acc = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) acc += x[k];
  if (acc == -1.2345e-30f) sink[0] = acc;
}

}  // namespace
}  // namespace re

extern "C" {

// Reads a `bytes` buffer (<= 64 MB so it stays in L2) `passes` times in one
// launch after a warm-up launch; *gbs = bytes * passes / kernel time.
RE_API re_status re_measure_l2_read(size_t bytes, uint32_t passes, float* gbs, void* stream) {
  if (!gbs || bytes < (1u << 20) || bytes > (64u << 20) || passes == 0 || passes > 1000)
    return re::fail(RE_ERR_INVALID_ARG, "re_measure_l2_read: bytes in [1 MB, 64 MB], passes in [1, 1000]");
  cudaStream_t st = (cudaStream_t)stream;
  uint4* buf = nullptr;
  uint4* sink = nullptr;
  RE_CUDA(cudaMalloc(&buf, bytes));
  cudaError_t e = cudaMalloc(&sink, sizeof(uint4));
  cudaEvent_t a = nullptr, b = nullptr;
  if (e == cudaSuccess) e = cudaMemsetAsync(buf, 1, bytes, st);
  if (e == cudaSuccess) e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  size_t n = bytes / sizeof(uint4);
  int grid = 4 * re::sm_count();
  if (e == cudaSuccess) {
    re::k_l2_read<<<grid, 512, 0, st>>>(buf, n, 2, sink);  // warm-up: bring the buffer into L2
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(a, st);
  if (e == cudaSuccess) {
    re::k_l2_read<<<grid, 512, 0, st>>>(buf, n, passes, sink);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(b, st);
  if (e == cudaSuccess) e = cudaEventSynchronize(b);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  cudaFree(buf);
  cudaFree(sink);
  if (e != cudaSuccess) return re::cuda_fail(e, "re_measure_l2_read");
  *gbs = (float)((double)bytes * passes / (ms / 1e3) / 1e9);
  return RE_OK;
}

// FP32 fused multiply-add rate: one launch of 8 blocks of 256 threads per
// SM, each thread 8 independent chains of `iters` FMAs, after a warm-up
// launch; *tops = FMAs (one operation each) / kernel time, in 10^12/s.
RE_API re_status re_measure_fp32_fma(uint32_t iters, float* tops, void* stream) {
  if (!tops || iters < 1024 || iters > (1u << 20))
    return re::fail(RE_ERR_INVALID_ARG, "re_measure_fp32_fma: iters in [1024, 2^20]");
  cudaStream_t st = (cudaStream_t)stream;
  float* sink = nullptr;
  RE_CUDA(cudaMalloc(&sink, sizeof(float)));
  cudaEvent_t a = nullptr, b = nullptr;
  cudaError_t e = cudaEventCreate(&a);
  if (e == cudaSuccess) e = cudaEventCreate(&b);
  const int grid = 8 * re::sm_count(), block = 256;
  // a = 1 - 2^-20 keeps the chains finite and away from denormals
  const float fa = 0.99999905f, fb = 0.5f;
  if (e == cudaSuccess) {
    re::k_fma<<<grid, block, 0, st>>>(iters / 8u, fa, fb, sink);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(a, st);
  if (e == cudaSuccess) {
    re::k_fma<<<grid, block, 0, st>>>(iters, fa, fb, sink);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(b, st);
  if (e == cudaSuccess) e = cudaEventSynchronize(b);
  float ms = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
  if (a) cudaEventDestroy(a);
  if (b) cudaEventDestroy(b);
  cudaFree(sink);
  if (e != cudaSuccess) return re::cuda_fail(e, "re_measure_fp32_fma");
  *tops = (float)((double)grid * block * 8.0 * iters / (ms / 1e3) / 1e12);
  return RE_OK;
}

}  // extern "C"
