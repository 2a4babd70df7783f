// The scene handle behind re_scene* (internal): the host tree and its
// device copy.  Shared by the frame kernels (re_trace.cu) and the batched
// renderer (re_batch.cu), which reads a scene's device arrays in place.
#pragma once
#include <cuda_runtime.h>

#include "kd_build.hpp"
#include "../../include/rayengine_b200.h"

// 16 32-bit counters per scene (64 bytes)
#define RE_SCENE_TRUNC_SLOT 8
#define RE_SCENE_RESET_BYTES (4 * (RE_SCENE_TRUNC_SLOT + 1))

struct re_scene {
  int device = 0;
  re::FlatTree host;
  uint2* d_nodes = nullptr;
  float4* d_leaves = nullptr;
  float4* d_tris = nullptr;
  uint32_t* d_entry = nullptr;  // the host's entry table (FlatTree::entry)
  // [0] tile cursor, [1] queue size, [2] queue cursor, [3] secondary rays,
  // [RE_SCENE_TRUNC_SLOT] rays of the last trace call stopped at the
  // leaf-visit cap; every trace call clears the first RE_SCENE_RESET_BYTES
  uint32_t* d_counters = nullptr;
  float4* d_queue = nullptr;
  size_t queue_cap = 0;  // rays
  uint32_t max_visits = 16384;
  uint32_t stage = 0;
  int blocks_per_sm = 0;
  float ao_length = 1.0f;    // AO ray length of the last primary pass
  uint32_t queue_stride = 0;  // record capacity per ray kind in d_queue
  re_tuning tune = {0, 0, 32, 32, 1};
};
