// Multi-object scenes: instances of built meshes, each with a yaw rotation
// and a location, traced together (closest hit over the instances).
//
// Replaces, in the reference (hadalhw17/RayEngine, "RE/" = RayEngine/src/):
//   per-object ray transform   RE/cuda-src/ray_functions.cuh:236-267
//     d' = normalize(Ry d), o' = Ry o + location, with
//     Ry v = (v.x cos y + v.z sin y, v.y, -v.x sin y + v.z cos y)
//   trace_scene                RE/cuda-src/ray_functions.cuh:377-396: an
//     object's hit replaces the current one only if strictly closer
//   per-object roots / offsets RE/World/RTScene.cpp:40-62 (each instance
//     keeps its own tree here; the concatenated arrays are not needed)
// The reference's "is_character" special case (a different transform for
// secondary rays of the player object) is not reproduced.
#include <cuda_runtime.h>

#include <cmath>

#include "re_common.hpp"
#include "re_kd.cuh"
#include "re_math.cuh"
#include "re_scene.hpp"

namespace re {
namespace inst {

constexpr uint32_t kMaxInstances = 64;

struct InstDev {
  KdDev kd;
  float c, s;  // cos / sin of the yaw, from the host
  V3 loc;
};

struct InstTable {
  InstDev i[kMaxInstances];
  uint32_t n;
};

template <int MODE>
__global__ void __launch_bounds__(256) k_instances(const InstTable* __restrict__ tab, CamDev cam,
                                                   uint32_t w, uint32_t h, re_hit* __restrict__ out,
                                                   int32_t* __restrict__ inst_out) {
  uint32_t pix = blockIdx.x * blockDim.x + threadIdx.x;
  if (pix >= w * h) return;
  V3 o, d;
  generate_ray(cam, w, h, pix % w, pix / w, o, d);
  float best_t = __int_as_float(0x7f800000);
  int32_t best_id = -1, best_inst = -1;
  float best_u = 0.f, best_v = 0.f;
  Counters c = {0, 0, 0, 0};
  const uint32_t n = tab->n;
  for (uint32_t k = 0; k < n; ++k) {
    const InstDev& I = tab->i[k];
    V3 nd = normalize(v3(d.x * I.c + d.z * I.s, d.y, -d.x * I.s + d.z * I.c));
    V3 no = v3(o.x * I.c + o.z * I.s + I.loc.x, o.y + I.loc.y, -o.x * I.s + o.z * I.c + I.loc.z);
    HitState hs;
    traverse<MODE, false, false>(I.kd, nullptr, no, nd, best_t, 0u, hs, c);
    if (hs.id >= 0 && hs.t < best_t) {
      best_t = hs.t;
      best_id = hs.id;
      best_u = hs.u;
      best_v = hs.v;
      best_inst = (int32_t)k;
    }
  }
  reinterpret_cast<int4*>(out)[pix] =
      make_int4(best_id, __float_as_int(best_id >= 0 ? best_t : K_INF), __float_as_int(best_u),
                __float_as_int(best_v));
  inst_out[pix] = best_inst;
}

}  // namespace inst
}  // namespace re

namespace re {
namespace {

CamDev cam_of_inst(const re_camera& c) {
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

}  // namespace
}  // namespace re

extern "C" {

RE_API re_status re_trace_instances(const re_instance* instances, uint32_t n, const re_camera* cam,
                                    uint32_t w, uint32_t h, uint32_t flags, re_hit* d_out,
                                    int32_t* d_instance, void* stream) {
  using namespace re::inst;
  if (!instances || n == 0 || !cam || !d_out || !d_instance || w == 0 || h == 0)
    return re::fail(RE_ERR_INVALID_ARG, "re_trace_instances: bad arguments");
  if (n > kMaxInstances) return re::fail(RE_ERR_LIMIT, "re_trace_instances: more than %u instances", kMaxInstances);
  if ((uint64_t)w * h > (1ull << 30)) return re::fail(RE_ERR_LIMIT, "re_trace_instances: image too large");
  InstTable tab;
  tab.n = n;
  for (uint32_t k = 0; k < n; ++k) {
    const re_scene* s = instances[k].mesh;
    if (!s || !s->d_nodes) return re::fail(RE_ERR_INVALID_ARG, "re_trace_instances: instance %u has no device scene", k);
    InstDev& I = tab.i[k];
    I.kd.nodes = s->d_nodes;
    I.kd.leaves = s->d_leaves;
    I.kd.tris = s->d_tris;
    I.kd.bmin = {s->host.bmin[0], s->host.bmin[1], s->host.bmin[2]};
    I.kd.bmax = {s->host.bmax[0], s->host.bmax[1], s->host.bmax[2]};
    I.kd.max_visits = s->max_visits;
    I.kd.stage = 0;
    I.kd.trunc = nullptr;
    re_instance_trig(instances[k].yaw, &I.c, &I.s);
    I.loc = {instances[k].location[0], instances[k].location[1], instances[k].location[2]};
  }
  cudaStream_t st = (cudaStream_t)stream;
  InstTable* d_tab = nullptr;
  RE_CUDA(cudaMallocAsync(&d_tab, sizeof(InstTable), st));
  cudaError_t e = cudaMemcpyAsync(d_tab, &tab, sizeof(InstTable), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) {
    uint32_t total = w * h;
    if (flags & RE_TRACE_ONE_SIDED)
      k_instances<1><<<(total + 255) / 256, 256, 0, st>>>(d_tab, re::cam_of_inst(*cam), w, h, d_out, d_instance);
    else
      k_instances<0><<<(total + 255) / 256, 256, 0, st>>>(d_tab, re::cam_of_inst(*cam), w, h, d_out, d_instance);
    e = cudaGetLastError();
  }
  // the table is freed in stream order after the kernel; the host copy
  // must stay valid until the copy ran
  cudaError_t e2 = cudaStreamSynchronize(st);
  cudaFreeAsync(d_tab, st);
  if (e == cudaSuccess) e = e2;
  if (e != cudaSuccess) return re::cuda_fail(e, "re_trace_instances");
  return RE_OK;
}

// The yaw's cosine and sine as the tracer uses them (host sinf / cosf).
RE_API void re_instance_trig(float yaw, float* c, float* s) {
  *c = std::cos(yaw);
  *s = std::sin(yaw);
}

}  // extern "C"
