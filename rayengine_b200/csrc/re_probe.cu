// L2 read-bandwidth probe: the denominator the benchmark uses for the
// traversal kernels' L2 roofline (their node, leaf and triangle reads mostly
// hit L2; no measured L2 figure is supplied with the hardware peaks).
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

}  // extern "C"
