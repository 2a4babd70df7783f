/*
 * TEST INFRASTRUCTURE ONLY -- reads a PLY file the way the reference's
 * RStaticMesh::LoadFromFile (RayEngine/src/Objects/RStaticMesh.cpp:19-128)
 * does, through the reference's own vendored rply reader compiled from its
 * sources (oracle/Makefile.ref): x, y, z of every vertex and the first three
 * entries of every face's vertex_indices.  Used by tests to check the
 * library's PLY loader; never linked into the product.
 */
#include <stdint.h>
#include <stdlib.h>

#include "rply.h"

typedef struct {
  float* v;
  long nv, cap_v;
  uint32_t* f;
  long nf, cap_f;
} ply_ctx;

static int push_v(ply_ctx* c, float x) {
  if (c->nv == c->cap_v) {
    long cap = c->cap_v ? 2 * c->cap_v : 1024;
    float* p = (float*)realloc(c->v, (size_t)cap * sizeof(float));
    if (!p) return 0;
    c->v = p;
    c->cap_v = cap;
  }
  c->v[c->nv++] = x;
  return 1;
}

static int push_f(ply_ctx* c, uint32_t i) {
  if (c->nf == c->cap_f) {
    long cap = c->cap_f ? 2 * c->cap_f : 1024;
    uint32_t* p = (uint32_t*)realloc(c->f, (size_t)cap * sizeof(uint32_t));
    if (!p) return 0;
    c->f = p;
    c->cap_f = cap;
  }
  c->f[c->nf++] = i;
  return 1;
}

static int vertex_cb(p_ply_argument a) {
  void* ud;
  long which;
  ply_get_argument_user_data(a, &ud, &which);
  return push_v((ply_ctx*)ud, (float)ply_get_argument_value(a));
}

static int face_cb(p_ply_argument a) {
  void* ud;
  long which, length, value_index;
  ply_get_argument_user_data(a, &ud, &which);
  ply_get_argument_property(a, NULL, &length, &value_index);
  if (value_index >= 0 && value_index < 3)
    return push_f((ply_ctx*)ud, (uint32_t)ply_get_argument_value(a));
  return 1;
}

/* Returns 1 on success; *v = 3 * nv floats, *f = 3 * nf indices (free with
 * ref_ply_free). */
int ref_ply_load(const char* path, float** v, long* nv, uint32_t** f, long* nf) {
  ply_ctx c = {0};
  p_ply ply = ply_open(path, NULL, 0, NULL);
  if (!ply) return 0;
  if (!ply_read_header(ply)) {
    ply_close(ply);
    return 0;
  }
  ply_set_read_cb(ply, "vertex", "x", vertex_cb, &c, 0);
  ply_set_read_cb(ply, "vertex", "y", vertex_cb, &c, 1);
  ply_set_read_cb(ply, "vertex", "z", vertex_cb, &c, 2);
  ply_set_read_cb(ply, "face", "vertex_indices", face_cb, &c, 0);
  int ok = ply_read(ply);
  ply_close(ply);
  *v = c.v;
  *nv = c.nv / 3;
  *f = c.f;
  *nf = c.nf / 3;
  return ok;
}

void ref_ply_free(void* p) { free(p); }
