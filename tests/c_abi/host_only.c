/* A plain C11 caller of the library's C ABI (no GPU needed): the header
 * must compile as C, and the host-only entry points must work through it.
 * Prints "ok" and exits 0 on success; prints the failing step otherwise. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "rayengine_b200.h"

#define CHECK(cond, what)                                  \
  do {                                                     \
    if (!(cond)) {                                         \
      printf("fail: %s (%s)\n", what, re_last_error());    \
      return 1;                                            \
    }                                                      \
  } while (0)

int main(void) {
  CHECK(re_abi_version() > 0, "abi version");
  CHECK(re_status_string(RE_ERR_INVALID_ARG) != NULL, "status string");

  /* RPerlinNoise table: 256 entries, second half a copy of the first */
  uint32_t perm[512];
  CHECK(re_perlin_permutation(2016, perm) == RE_OK, "permutation");
  for (int i = 0; i < 256; ++i) CHECK(perm[i + 256] == perm[i] && perm[i] < 256, "perm doubled");

  /* a small grid of triangles in the packed {v0, e1, e2} form */
  enum { N = 16 * 16 * 2 };
  float* tris = calloc((size_t)N * 12, sizeof(float));
  CHECK(tris != NULL, "alloc");
  int t = 0;
  for (int z = 0; z < 16; ++z)
    for (int x = 0; x < 16; ++x)
      for (int k = 0; k < 2; ++k, ++t) {
        float* T = tris + 12 * t;
        T[0] = (float)x; T[1] = 0.1f * (float)((x + z) % 3); T[2] = (float)z;
        T[4] = 1.0f; T[6] = (float)k;
        T[8] = (float)(1 - k); T[10] = 1.0f;
      }

  re_kd_params p;
  re_kd_params_default(&p);
  re_scene* s = NULL;
  CHECK(re_scene_build_host(tris, N, &p, &s) == RE_OK && s != NULL, "build host");
  re_scene_stats st;
  CHECK(re_scene_stats_get(s, &st) == RE_OK, "stats");
  CHECK(st.num_tris == N && st.num_leaves > 1 && st.num_nodes == 2 * st.num_leaves - 1, "tree shape");
  uint32_t* nodes = malloc((size_t)st.num_nodes * 2 * sizeof(uint32_t));
  uint32_t* leaves = malloc((size_t)st.num_leaves * 16 * sizeof(uint32_t));
  CHECK(nodes && leaves, "alloc");
  CHECK(re_scene_export(s, nodes, leaves, NULL) == RE_OK, "export");
  /* every leaf node's record index is in range */
  for (uint32_t i = 0; i < st.num_nodes; ++i)
    if ((nodes[2 * i + 1] & 3u) == 3u) CHECK((nodes[2 * i + 1] >> 2) < st.num_leaves, "leaf index");

  /* a host-only scene refuses device work with a status, not a crash */
  re_camera cam;
  memset(&cam, 0, sizeof cam);
  CHECK(re_trace_primary(s, &cam, 8, 8, RE_TRACE_TWO_SIDED, NULL, NULL) != RE_OK, "host-only trace");
  CHECK(re_scene_build_host(NULL, N, &p, &s) == RE_ERR_INVALID_ARG, "null triangles");
  CHECK(re_scene_destroy(s) == RE_OK, "destroy");
  free(nodes);
  free(leaves);
  free(tris);
  printf("ok\n");
  return 0;
}
