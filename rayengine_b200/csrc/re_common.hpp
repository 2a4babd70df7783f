// Shared host-side helpers: error reporting and CUDA status checks.
#pragma once
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/rayengine_b200.h"

namespace re {

void set_error(const char* fmt, ...);
re_status fail(re_status s, const char* fmt, ...);
// Empties this thread's last-error message (entry points whose only error
// channel is re_last_error clear it first).
void clear_error();

inline re_status cuda_fail(cudaError_t e, const char* what) {
  return fail(e == cudaErrorMemoryAllocation ? RE_ERR_OUT_OF_MEMORY : RE_ERR_CUDA,
              "%s: %s", what, cudaGetErrorString(e));
}

#define RE_CUDA(call)                                   \
  do {                                                  \
    cudaError_t _e = (call);                            \
    if (_e != cudaSuccess) return ::re::cuda_fail(_e, #call); \
  } while (0)

#define RE_CHECK_LAUNCH(what)                             \
  do {                                                    \
    cudaError_t _e = cudaGetLastError();                  \
    if (_e != cudaSuccess) return ::re::cuda_fail(_e, what); \
  } while (0)

// Per-frame camera constants (generate_ray, ray_functions.cuh:26-37).
struct CamBasis {
  float campos[3], middle[3], horizontal[3], vertical[3];
  float focal;
};
void camera_basis(const re_camera& cam, CamBasis& out);

// RPerlinNoise(seed).permutationTable (PerlinNoise.h:16-52).
void perlin_permutation(uint32_t seed, uint32_t out[512]);

int sm_count();

}  // namespace re
