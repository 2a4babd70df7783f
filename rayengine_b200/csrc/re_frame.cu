// The frame step behind the reference's render call: primary rays, Phong
// shading with one shadow ray per light, sky for misses, RGBA8 pack into a
// headless device buffer.
//
// Replaces, in the reference (hadalhw17/RayEngine, "RE/" = RayEngine/src/):
//   cuda_render_frame      RE/cuda-src/renderer.cu:702-738 (frame driver,
//                          light animation Craze :288-300)
//   trace_secondary_rays   RE/cuda-src/renderer.cu:435-492 (per-pixel shading)
//   phong_light / shade    RE/cuda-src/material_functions.cuh:69-119
//   illuminate             RE/cuda-src/cuda_helper_functions.h:90-102
//   rgbaFloatToInt         RE/cuda-src/cuda_helper_functions.h:61-68
//
// Shading of a hit (material colour c, geometric normal n facing the ray,
// view direction v, per light at position L with intensity I):
//   l  = (p - L) / |p - L|,  r2 = |p - L|^2
//   Li = (0.86, 0.80, 0.45) * I / (4 pi r2)
//   visible: no triangle on the shadow ray from p + 1e-4 n toward L
//   diffuse  = Li * 0.18 * max(0, n . -l)
//   specular = Li * max(0, R . -v)^10,  R = l - 2 (n . l) n
//   colour  += visible * (0.8 diffuse + 0.2 specular)
// Deviations from the reference, on purpose: the light direction and 1/r^2
// use the distance from p to the light (illuminate uses |L|, the light's
// distance from the origin); visibility is "shadow ray unoccluded" as in
// shade() (phong_light multiplies by the shadow ray's hit flag, which lights
// occluded points); the pixel is written once (trace_secondary_rays adds the
// packed colour into the buffer five times, carrying between channels); a
// miss gets a two-colour sky gradient instead of the atmosphere integral.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "re_common.hpp"
#include "re_kd.cuh"
#include "re_math.cuh"
#include "re_scene.hpp"

namespace re {
namespace frame {

constexpr uint32_t kMaxLights = 8;

struct ShadeDev {
  V3 albedo, sky_zenith, sky_horizon;
  V3 light_pos[kMaxLights];
  float light_int[kMaxLights];
  uint32_t num_lights;
};

// rgbaFloatToInt (cuda_helper_functions.h:61-68): saturate, scale by 255,
// truncate, alpha 255, R in the low byte
__device__ __forceinline__ uint32_t pack_rgba(V3 c) {
  float r = __saturatef(c.x), g = __saturatef(c.y), b = __saturatef(c.z);
  return (255u << 24) | ((uint32_t)(b * 255.0f) << 16) | ((uint32_t)(g * 255.0f) << 8) |
         (uint32_t)(r * 255.0f);
}

template <int MODE>
__device__ __forceinline__ void shade_pixel(const KdDev& kd, const uint2* snodes, const CamDev& cam,
                                            const ShadeDev& sh, uint32_t w, uint32_t h, uint32_t x,
                                            uint32_t y, uint32_t* __restrict__ out, Counters& c);

template <int MODE>
__global__ void __launch_bounds__(256) k_frame(KdDev kd, CamDev cam, ShadeDev sh, uint32_t w,
                                               uint32_t h, uint32_t* __restrict__ out,
                                               uint32_t* __restrict__ tile_counter) {
  extern __shared__ uint2 snodes[];
  stage_nodes(kd, snodes);
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t tiles_x = (w + 7) / 8, tiles = tiles_x * ((h + 3) / 4);
  Counters c = {0, 0, 0, 0};
  for (;;) {
    uint32_t tile = warp_fetch(tile_counter);
    if (tile >= tiles) break;
    uint32_t x = (tile % tiles_x) * 8 + (lane & 7u), y = (tile / tiles_x) * 4 + (lane >> 3);
    if (x < w && y < h) shade_pixel<MODE>(kd, snodes, cam, sh, w, h, x, y, out, c);
  }
}

template <int MODE>
__device__ __forceinline__ void shade_pixel(const KdDev& kd, const uint2* snodes, const CamDev& cam,
                                            const ShadeDev& sh, uint32_t w, uint32_t h, uint32_t x,
                                            uint32_t y, uint32_t* __restrict__ out, Counters& c) {
  {
    V3 o, d;
    generate_ray(cam, w, h, x, y, o, d);
    HitState hs;
    traverse<MODE, false, false>(kd, snodes, o, d, __int_as_float(0x7f800000), 0u, hs, c);
    V3 col;
    if (hs.id < 0) {
      float s = fmaxf(d.y, 0.0f);
      col = v3(__fmaf_rn(s, sh.sky_zenith.x - sh.sky_horizon.x, sh.sky_horizon.x),
               __fmaf_rn(s, sh.sky_zenith.y - sh.sky_horizon.y, sh.sky_horizon.y),
               __fmaf_rn(s, sh.sky_zenith.z - sh.sky_horizon.z, sh.sky_horizon.z));
    } else {
      const float4* T = kd.tris + 3 * (size_t)hs.ref;
      float4 T1 = __ldg(T + 1), T2 = __ldg(T + 2);
      V3 n = normalize(cross(v3(T1.x, T1.y, T1.z), v3(T2.x, T2.y, T2.z)));
      if (dot(n, d) > 0.0f) n = v3(-n.x, -n.y, -n.z);
      V3 p = v3(__fmaf_rn(hs.t, d.x, o.x), __fmaf_rn(hs.t, d.y, o.y), __fmaf_rn(hs.t, d.z, o.z));
      V3 org = v3(__fmaf_rn(n.x, 1e-4f, p.x), __fmaf_rn(n.y, 1e-4f, p.y), __fmaf_rn(n.z, 1e-4f, p.z));
      col = sh.albedo;
      for (uint32_t i = 0; i < sh.num_lights; ++i) {
        V3 L = sh.light_pos[i];
        V3 pl = sub(p, L);
        float r2 = dot(pl, pl);
        float dist = sqrtf(r2);
        V3 l = v3(pl.x / dist, pl.y / dist, pl.z / dist);
        float k = sh.light_int[i] / (4.0f * 3.14159265358979f * r2);
        V3 li = v3(0.86f * k, 0.80f * k, 0.45f * k);
        V3 toward = v3(-l.x, -l.y, -l.z);
        HitState sv;
        traverse<0, true, false>(kd, snodes, org, toward, dist, 0u, sv, c);
        if (sv.id >= 0) continue;  // occluded
        float nl = fmaxf(0.0f, dot(n, toward));
        float dn = dot(n, l);
        V3 R = v3(__fmaf_rn(-2.0f * dn, n.x, l.x), __fmaf_rn(-2.0f * dn, n.y, l.y),
                  __fmaf_rn(-2.0f * dn, n.z, l.z));
        float rv = fmaxf(0.0f, -dot(R, d));
        float r2v = rv * rv, r4 = r2v * r2v, r8 = r4 * r4;
        float spec = r8 * r2v;
        float dfac = 0.8f * (0.18f * nl), sfac = 0.2f * spec;
        col = v3(__fmaf_rn(li.x, sfac, __fmaf_rn(li.x, dfac, col.x)),
                 __fmaf_rn(li.y, sfac, __fmaf_rn(li.y, dfac, col.y)),
                 __fmaf_rn(li.z, sfac, __fmaf_rn(li.z, dfac, col.z)));
      }
    }
    out[(size_t)y * w + x] = pack_rgba(col);
  }
}

}  // namespace frame
}  // namespace re

namespace re {
// SDF mode of cuda_render_frame (re_sdf_frame.cu)
bool sdf_render_bound(unsigned int* output, unsigned int width, unsigned int height);
void sdf_unbind();

namespace {

using namespace frame;

KdDev kd_of_scene(const re_scene* s) {
  KdDev kd;
  kd.nodes = s->d_nodes;
  kd.leaves = s->d_leaves;
  kd.tris = s->d_tris;
  kd.bmin = {s->host.bmin[0], s->host.bmin[1], s->host.bmin[2]};
  kd.bmax = {s->host.bmax[0], s->host.bmax[1], s->host.bmax[2]};
  kd.max_visits = s->max_visits;
  kd.stage = s->stage;
  kd.trunc = s->d_counters + RE_SCENE_TRUNC_SLOT;
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

CamDev cam_of_frame(const re_camera& c) {
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

// State bound for the reference-style entry point cuda_render_frame(), which
// takes only the output buffer and its size (the reference keeps the scene,
// camera and lights in globals set by copy_memory).
struct Bound {
  std::mutex mu;
  re_scene* scene = nullptr;
  re_camera cam{};
  re_light lights[kMaxLights]{};
  uint32_t num_lights = 0;
  re_shade_params sp{};
  uint32_t flags = 0;
  int animate = 0;
  float angle = 0.f;
  uint32_t* d_tiles = nullptr;
};
Bound& bound() {
  static Bound b;
  return b;
}

}  // namespace
}  // namespace re

extern "C" {

RE_API re_status re_render_frame(re_scene* s, const re_camera* cam, const re_light* lights,
                                 uint32_t num_lights, const re_shade_params* sp, uint32_t w,
                                 uint32_t h, uint32_t* d_rgba, void* stream) {
  using namespace re::frame;
  if (!s || !cam || !sp || !d_rgba || w == 0 || h == 0 || (num_lights && !lights))
    return re::fail(RE_ERR_INVALID_ARG, "re_render_frame: bad arguments");
  if (!s->d_nodes) return re::fail(RE_ERR_INVALID_ARG, "re_render_frame: scene has no device copy");
  if (num_lights > kMaxLights) return re::fail(RE_ERR_LIMIT, "re_render_frame: more than %u lights", kMaxLights);
  if ((uint64_t)w * h > (1ull << 30)) return re::fail(RE_ERR_LIMIT, "re_render_frame: image too large");
  ShadeDev sh;
  std::memset(&sh, 0, sizeof(sh));
  sh.albedo = {sp->albedo[0], sp->albedo[1], sp->albedo[2]};
  sh.sky_zenith = {sp->sky_zenith[0], sp->sky_zenith[1], sp->sky_zenith[2]};
  sh.sky_horizon = {sp->sky_horizon[0], sp->sky_horizon[1], sp->sky_horizon[2]};
  sh.num_lights = num_lights;
  for (uint32_t i = 0; i < num_lights; ++i) {
    sh.light_pos[i] = {lights[i].pos[0], lights[i].pos[1], lights[i].pos[2]};
    sh.light_int[i] = lights[i].intensity;
  }
  cudaStream_t st = (cudaStream_t)stream;
  RE_CUDA(cudaMemsetAsync(s->d_counters, 0, RE_SCENE_RESET_BYTES, st));
  re::KdDev kd = re::kd_of_scene(s);
  size_t smem = (size_t)kd.stage * sizeof(uint2);
  int grid = 0;
  if (sp->flags & RE_TRACE_ONE_SIDED) {
    RE_CUDA(cudaFuncSetAttribute(k_frame<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    RE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_frame<1>, 256, smem));
    grid = std::max(per_sm, 1) * re::sm_count();
    k_frame<1><<<grid, 256, smem, st>>>(kd, re::cam_of_frame(*cam), sh, w, h, d_rgba, s->d_counters);
  } else {
    RE_CUDA(cudaFuncSetAttribute(k_frame<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    RE_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_frame<0>, 256, smem));
    grid = std::max(per_sm, 1) * re::sm_count();
    k_frame<0><<<grid, 256, smem, st>>>(kd, re::cam_of_frame(*cam), sh, w, h, d_rgba, s->d_counters);
  }
  RE_CHECK_LAUNCH("re_render_frame: launch");
  return RE_OK;
}

RE_API re_status re_frame_bind(re_scene* s, const re_camera* cam, const re_light* lights,
                               uint32_t num_lights, const re_shade_params* sp, int animate_light) {
  using namespace re::frame;
  if (!s || !cam || !sp || (num_lights && !lights))
    return re::fail(RE_ERR_INVALID_ARG, "re_frame_bind: bad arguments");
  if (num_lights > kMaxLights) return re::fail(RE_ERR_LIMIT, "re_frame_bind: more than %u lights", kMaxLights);
  re::sdf_unbind();
  re::Bound& b = re::bound();
  std::lock_guard<std::mutex> lk(b.mu);
  b.scene = s;
  b.cam = *cam;
  b.num_lights = num_lights;
  for (uint32_t i = 0; i < num_lights; ++i) b.lights[i] = lights[i];
  b.sp = *sp;
  b.animate = animate_light;
  b.angle = 0.f;
  return RE_OK;
}

}  // extern "C"

// The reference's render call (renderer.cu:701-738), same C++ signature:
// renders the bound scene into the W x H RGBA8 device buffer `output` on the
// default stream and waits for it, then advances the light animation as
// Craze does (light 0 at x = z = 20 cos(angle), angle += 0.001, wrapping
// past 1.1) when enabled in re_frame_bind.  Errors are reported through
// re_last_error() (the reference exits the process).
__attribute__((visibility("default"))) void cuda_render_frame(unsigned int* output,
                                                              const unsigned int& width,
                                                              const unsigned int& heigth) {
  re::clear_error();
  if (re::sdf_render_bound(output, width, heigth)) return;
  re::Bound& b = re::bound();
  std::lock_guard<std::mutex> lk(b.mu);
  if (!b.scene) {
    re::fail(RE_ERR_INVALID_ARG,
             "cuda_render_frame: nothing bound (re_sdf_frame_bind or re_frame_bind)");
    return;
  }
  if (re_render_frame(b.scene, &b.cam, b.lights, b.num_lights, &b.sp, width, heigth, output,
                      nullptr) != RE_OK)
    return;
  cudaError_t e = cudaStreamSynchronize(nullptr);
  if (e != cudaSuccess) {
    re::cuda_fail(e, "cuda_render_frame");
    return;
  }
  if (b.animate && b.num_lights > 0) {
    float x = std::cos(b.angle) * 20.f;
    b.lights[0].pos[0] = x;
    b.lights[0].pos[2] = x;
    b.angle += 0.001f;
    if (b.angle > 1.1f) b.angle = 0.f;
  }
}
