// The scene handle behind re_scene* (internal): the host tree and its
// device copy.  Shared by the frame kernels (re_trace.cu) and the batched
// renderer (re_batch.cu), which reads a scene's device arrays in place.
#pragma once
#include <cuda_runtime.h>

#include "kd_build.hpp"
#include "../../include/rayengine_b200.h"

struct re_scene {
  int device = 0;
  re::FlatTree host;
  uint2* d_nodes = nullptr;
  float4* d_leaves = nullptr;
  float4* d_tris = nullptr;
  uint32_t* d_counters = nullptr;  // [0] tiles, [1] queue size, [2] queue chunks
  float4* d_queue = nullptr;
  size_t queue_cap = 0;  // rays
  uint32_t max_visits = 16384;
  uint32_t stage = 0;
  int blocks_per_sm = 0;
  float ao_length = 1.0f;    // AO ray length of the last primary pass
  uint32_t queue_stride = 0;  // record capacity per ray kind in d_queue
  re_tuning tune = {0, 0, 32, 32};
};
