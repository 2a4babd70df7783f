// A C++ program that drives the library on the GPU through its header only,
// the way the reference's engine would: it uploads a triangle soup
// (re_scene_create_packed), traces primary rays into caller-owned device
// memory (re_trace_primary), then binds the shaded SDF terrain
// (re_sdf_frame_bind) and renders it with the reference's own render call
// (cuda_render_frame).  Device memory comes from the CUDA runtime directly.
//
// Input file: uint32 n, n x 12 floats (packed triangles), re_camera (mesh
// view), uint32 w, h, re_sdf_params, re_sdf_shade_params, re_camera
// (terrain view), uint32 fw, fh.  Output file: w x h re_hit, then fw x fh
// RGBA8 words.  Prints "ok" on success.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstring>
#include <vector>

#include "rayengine_b200.h"

#define CHECK(cond, what)                                               \
  do {                                                                  \
    if (!(cond)) {                                                      \
      std::fprintf(stderr, "%s failed: %s\n", what, re_last_error());  \
      return 1;                                                         \
    }                                                                   \
  } while (0)

template <class T>
static bool read_one(std::FILE* f, T* v) {
  return std::fread(v, sizeof(T), 1, f) == 1;
}

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: gpu_caller <input> <output>\n");
    return 2;
  }
  std::FILE* in = std::fopen(argv[1], "rb");
  CHECK(in, "open input");
  uint32_t n = 0, w = 0, h = 0, fw = 0, fh = 0;
  CHECK(read_one(in, &n) && n > 0, "read triangle count");
  std::vector<float> tris((size_t)n * 12);
  CHECK(std::fread(tris.data(), sizeof(float), tris.size(), in) == tris.size(), "read triangles");
  re_camera cam, tcam;
  re_sdf_params field;
  re_sdf_shade_params shade;
  CHECK(read_one(in, &cam) && read_one(in, &w) && read_one(in, &h), "read mesh view");
  CHECK(read_one(in, &field) && read_one(in, &shade) && read_one(in, &tcam) &&
            read_one(in, &fw) && read_one(in, &fh),
        "read terrain view");
  std::fclose(in);

  re_scene* scene = nullptr;
  CHECK(re_scene_create_packed(tris.data(), n, nullptr, &scene) == RE_OK, "re_scene_create_packed");
  re_hit* d_hits = nullptr;
  CHECK(cudaMalloc(&d_hits, (size_t)w * h * sizeof(re_hit)) == cudaSuccess, "cudaMalloc hits");
  cudaStream_t stream;
  CHECK(cudaStreamCreate(&stream) == cudaSuccess, "cudaStreamCreate");
  CHECK(re_trace_primary(scene, &cam, w, h, RE_TRACE_TWO_SIDED, d_hits, stream) == RE_OK,
        "re_trace_primary");
  std::vector<re_hit> hits((size_t)w * h);
  CHECK(cudaMemcpyAsync(hits.data(), d_hits, hits.size() * sizeof(re_hit), cudaMemcpyDeviceToHost,
                        stream) == cudaSuccess &&
            cudaStreamSynchronize(stream) == cudaSuccess,
        "read back hits");

  unsigned int* d_rgba = nullptr;
  CHECK(cudaMalloc(&d_rgba, (size_t)fw * fh * 4) == cudaSuccess, "cudaMalloc frame");
  CHECK(re_sdf_frame_bind(&field, &shade, &tcam, 0) == RE_OK, "re_sdf_frame_bind");
  const unsigned int width = fw, height = fh;
  cuda_render_frame(d_rgba, width, height);
  CHECK(re_last_error()[0] == '\0', "cuda_render_frame");
  std::vector<unsigned int> rgba((size_t)fw * fh);
  CHECK(cudaMemcpy(rgba.data(), d_rgba, rgba.size() * 4, cudaMemcpyDeviceToHost) == cudaSuccess,
        "read back frame");

  std::FILE* out = std::fopen(argv[2], "wb");
  CHECK(out, "open output");
  std::fwrite(hits.data(), sizeof(re_hit), hits.size(), out);
  std::fwrite(rgba.data(), 4, rgba.size(), out);
  std::fclose(out);

  cudaFree(d_rgba);
  cudaFree(d_hits);
  cudaStreamDestroy(stream);
  CHECK(re_scene_destroy(scene) == RE_OK, "re_scene_destroy");
  std::printf("ok\n");
  return 0;
}
