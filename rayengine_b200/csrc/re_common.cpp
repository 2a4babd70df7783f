// Status strings, per-thread error text, host generators and the camera
// set-up shared by the kernels.
#include "re_common.hpp"

#include <cmath>
#include <cstring>
#include <random>

namespace re {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

void clear_error() { g_last_error.clear(); }

re_status fail(re_status s, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return s;
}

namespace {
inline float dot3(const float a[3], const float b[3]) {
  return std::fma(a[2], b[2], std::fma(a[1], b[1], a[0] * b[0]));
}
inline void cross3(const float a[3], const float b[3], float r[3]) {
  r[0] = std::fma(a[1], b[2], -(a[2] * b[1]));
  r[1] = std::fma(a[2], b[0], -(a[0] * b[2]));
  r[2] = std::fma(a[0], b[1], -(a[1] * b[0]));
}
inline void normalize3(float v[3]) {
  float inv = 1.0f / std::sqrt(dot3(v, v));
  v[0] *= inv;
  v[1] *= inv;
  v[2] *= inv;
}
}  // namespace

// generate_ray's frame constants (RayEngine/src/cuda-src/ray_functions.cuh:26-37),
// hoisted out of the per-pixel kernel.  The reference evaluates
// fov * 0.5 * (M_PI / 180) in double and passes it to tanf.
void camera_basis(const re_camera& cam, CamBasis& out) {
  float view[3] = {cam.view[0], cam.view[1], cam.view[2]};
  float down[3] = {cam.camdown[0], cam.camdown[1], cam.camdown[2]};
  float h[3], v[3];
  normalize3(view);
  normalize3(down);
  cross3(view, down, h);
  normalize3(h);
  cross3(h, view, v);
  normalize3(v);
  float th = std::tan((float)(cam.fov[0] * 0.5 * (3.14159265358979323846 / 180.0)));
  float tv = std::tan((float)(cam.fov[1] * 0.5 * (3.14159265358979323846 / 180.0)));
  for (int k = 0; k < 3; ++k) {
    out.campos[k] = cam.campos[k];
    out.middle[k] = cam.campos[k] + view[k];
    out.horizontal[k] = h[k] * th;
    out.vertical[k] = v[k] * tv;
  }
  out.focal = cam.focial_distance;
}

// RPerlinNoise (RayEngine/src/World/PerlinNoise.h:16-52): identity table,
// 256 swaps with raw std::mt19937 draws masked to 8 bits (the float draws
// before them advance a copy of the engine held by std::bind), duplicated.
void perlin_permutation(uint32_t seed, uint32_t out[512]) {
  std::mt19937 gen(seed);
  for (uint32_t i = 0; i < 256; ++i) out[i] = i;
  for (uint32_t i = 0; i < 256; ++i) std::swap(out[i], out[gen() & 255u]);
  for (uint32_t i = 0; i < 256; ++i) out[256 + i] = out[i];
}

int sm_count() {
  static int cached = 0;
  if (!cached) {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess)
      cached = n;
    else
      return 148;
  }
  return cached;
}

}  // namespace re

extern "C" {

RE_API int re_abi_version(void) { return RE_ABI_VERSION; }

RE_API const char* re_status_string(re_status s) {
  switch (s) {
    case RE_OK: return "ok";
    case RE_ERR_INVALID_ARG: return "invalid argument";
    case RE_ERR_CUDA: return "CUDA error";
    case RE_ERR_OUT_OF_MEMORY: return "out of memory";
    case RE_ERR_LIMIT: return "size limit exceeded";
    case RE_ERR_NO_DEVICE: return "no CUDA device";
    default: return "internal error";
  }
}

RE_API const char* re_last_error(void) { return re::g_last_error.c_str(); }

RE_API re_status re_perlin_permutation(uint32_t seed, uint32_t* out512) {
  if (!out512) return re::fail(RE_ERR_INVALID_ARG, "re_perlin_permutation: null output");
  re::perlin_permutation(seed, out512);
  return RE_OK;
}

// Seeded triangle soup: centroid ~ U[-1,1]^3, vertices = centroid +
// N(0, 0.02) per axis; std::mt19937_64, 53-bit uniforms, Box-Muller pairs.
RE_API re_status re_gen_soup(uint64_t seed, uint32_t n, float* verts) {
  if (!verts) return re::fail(RE_ERR_INVALID_ARG, "re_gen_soup: null output");
  std::mt19937_64 g(seed);
  auto u01 = [&]() { return (double)(g() >> 11) * 0x1.0p-53; };
  for (uint32_t i = 0; i < n; ++i) {
    double c[3], nz[10];
    for (int k = 0; k < 3; ++k) c[k] = -1.0 + 2.0 * u01();
    for (int p = 0; p < 5; ++p) {
      double u1 = 1.0 - u01();
      double u2 = u01();
      double r = std::sqrt(-2.0 * std::log(u1));
      nz[2 * p] = r * std::cos(6.283185307179586 * u2);
      nz[2 * p + 1] = r * std::sin(6.283185307179586 * u2);
    }
    for (int j = 0; j < 3; ++j)
      for (int k = 0; k < 3; ++k)
        verts[9 * (size_t)i + 3 * j + k] = (float)(c[k] + 0.02 * nz[3 * j + k]);
  }
  return RE_OK;
}

// Two triangles per grid cell, vertex (i, j) at index j*(cells+1)+i.
RE_API re_status re_gen_grid_faces(uint32_t cells, uint32_t* faces) {
  if (!faces || cells == 0) return re::fail(RE_ERR_INVALID_ARG, "re_gen_grid_faces: bad args");
  if (cells > 16384) return re::fail(RE_ERR_LIMIT, "re_gen_grid_faces: cells > 16384");
  uint32_t nv = cells + 1;
  for (uint32_t j = 0; j < cells; ++j)
    for (uint32_t i = 0; i < cells; ++i) {
      uint32_t a = j * nv + i, b = a + 1, c = a + 1 + nv, d = a + nv;
      uint32_t* F = faces + 6 * ((size_t)j * cells + i);
      F[0] = a; F[1] = b; F[2] = c;
      F[3] = a; F[4] = c; F[5] = d;
    }
  return RE_OK;
}

}  // extern "C"
