/*
 * TEST INFRASTRUCTURE ONLY -- an SAH kd-tree builder for the benchmark's
 * reference arm.
 *
 * The reference's own builder ships with MAX_DEPTH = 1 (one leaf,
 * RayEngine/src/Primitives/KDTree.cpp:12,347) and its SAH code commented out
 * (KDTree.cpp:392-547), so it cannot build the tree the configurations name
 * (SAH, depth <= 24, leaves of <= 8 references).  This builder makes such a
 * tree on the host so that the reference's compiled CPU ray query
 * (RKDTreeCPU::singleRayStacklessIntersect, KDTree.cpp:993-1066, driven
 * through oracle/ref_shim.cpp) can run over it.  It is not the product's
 * builder (rayengine_b200/csrc/kd_build.cpp) and shares no code with it:
 *
 *   * cost model: C_t + C_i (N_L A_L + N_R A_R) / A, the leaf cost C_i N,
 *     an empty side's cost scaled by (1 - empty_bonus);
 *   * candidate planes: 32 uniform bins per axis over the node box, counted
 *     on the bounding boxes of the triangles clipped to the node box
 *     (Sutherland-Hodgman against its six planes, the box then widened by a
 *     relative 1e-6 so that rounding never drops a triangle that touches
 *     the node); a triangle whose clipped box straddles the plane goes to
 *     both children, one whose clipped part is empty to neither;
 *   * a node becomes a leaf at max_depth, at <= leaf_size references, when
 *     no plane beats the leaf cost, or when a split would not shrink
 *     either side.
 *
 * Nodes are stored in pre-order: {axis (3 = leaf), split, left, right,
 * first, count}; leaves list their triangles in `index[first..first+count)`.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define KB_BINS 32

typedef struct {
  o_kdb_node* nodes;
  int32_t n_nodes, cap_nodes;
  int32_t* index;
  int64_t n_index, cap_index;
  const float* verts;
  const uint32_t* faces;
  int max_depth, leaf_size;
  float ci, ct, bonus;
  int failed;
} kb_state;

/* Bounding box of triangle t clipped to the box [lo, hi]; 0 if empty. */
static int kb_clip(const kb_state* s, int32_t t, const float lo[3], const float hi[3], float clo[3],
                   float chi[3]) {
  float poly[2][12][3];
  int n = 3, cur = 0;
  for (int v = 0; v < 3; ++v)
    for (int k = 0; k < 3; ++k) poly[0][v][k] = s->verts[3 * s->faces[3 * t + v] + k];
  for (int ax = 0; ax < 3 && n > 0; ++ax) {
    for (int side = 0; side < 2 && n > 0; ++side) {
      const float plane = side ? hi[ax] : lo[ax];
      int m = 0;
      for (int i = 0; i < n; ++i) {
        const float* a = poly[cur][i];
        const float* b = poly[cur][(i + 1) % n];
        float da = side ? plane - a[ax] : a[ax] - plane;
        float db = side ? plane - b[ax] : b[ax] - plane;
        if (da >= 0.0f) {
          memcpy(poly[cur ^ 1][m++], a, sizeof(float) * 3);
        }
        if ((da >= 0.0f) != (db >= 0.0f) && m < 12) {
          float f = da / (da - db);
          for (int k = 0; k < 3; ++k) poly[cur ^ 1][m][k] = a[k] + f * (b[k] - a[k]);
          poly[cur ^ 1][m][ax] = plane;
          ++m;
        }
      }
      n = m;
      cur ^= 1;
    }
  }
  if (n == 0) return 0;
  for (int k = 0; k < 3; ++k) {
    clo[k] = 1e30f;
    chi[k] = -1e30f;
  }
  for (int i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      float x = poly[cur][i][k];
      if (x < clo[k]) clo[k] = x;
      if (x > chi[k]) chi[k] = x;
    }
  for (int k = 0; k < 3; ++k) {
    float pad = 1e-6f * (fabsf(clo[k]) + fabsf(chi[k]) + (hi[k] - lo[k])) + 1e-30f;
    clo[k] -= pad;
    chi[k] += pad;
    if (clo[k] < lo[k]) clo[k] = lo[k];
    if (chi[k] > hi[k]) chi[k] = hi[k];
  }
  return 1;
}

static float kb_area(const float lo[3], const float hi[3]) {
  float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
  return 2.0f * (dx * dy + dy * dz + dz * dx);
}

static int32_t kb_new_node(kb_state* s) {
  if (s->n_nodes == s->cap_nodes) {
    int32_t cap = s->cap_nodes ? 2 * s->cap_nodes : 1024;
    o_kdb_node* p = (o_kdb_node*)realloc(s->nodes, (size_t)cap * sizeof(o_kdb_node));
    if (!p) {
      s->failed = 1;
      return -1;
    }
    s->nodes = p;
    s->cap_nodes = cap;
  }
  return s->n_nodes++;
}

static void kb_make_leaf(kb_state* s, int32_t id, const int32_t* tris, int32_t n) {
  if (s->n_index + n > s->cap_index) {
    int64_t cap = s->cap_index ? 2 * s->cap_index : 4096;
    while (cap < s->n_index + n) cap *= 2;
    int32_t* p = (int32_t*)realloc(s->index, (size_t)cap * sizeof(int32_t));
    if (!p) {
      s->failed = 1;
      return;
    }
    s->index = p;
    s->cap_index = cap;
  }
  memcpy(s->index + s->n_index, tris, (size_t)n * sizeof(int32_t));
  o_kdb_node* nd = &s->nodes[id];
  nd->axis = 3;
  nd->split = 0.0f;
  nd->left = nd->right = -1;
  nd->first = (int32_t)s->n_index;
  nd->count = n;
  s->n_index += n;
}

static void kb_build(kb_state* s, int32_t id, int32_t* tris, int32_t n, const float lo[3],
                     const float hi[3], int depth) {
  if (s->failed) return;
  /* clipped boxes of the node's triangles; triangles that miss the node are dropped */
  float* cb = (float*)malloc((size_t)(n > 0 ? n : 1) * 6 * sizeof(float));
  if (!cb) {
    s->failed = 1;
    return;
  }
  {
    int32_t m = 0;
    for (int32_t i = 0; i < n; ++i) {
      if (kb_clip(s, tris[i], lo, hi, cb + 6 * m, cb + 6 * m + 3)) tris[m++] = tris[i];
    }
    n = m;
  }
  float leaf_cost = s->ci * (float)n;
  float area = kb_area(lo, hi);
  int best_axis = -1;
  float best_split = 0.0f, best_cost = leaf_cost;
  if (n > s->leaf_size && depth < s->max_depth && area > 0.0f) {
    for (int ax = 0; ax < 3; ++ax) {
      float ext = hi[ax] - lo[ax];
      if (!(ext > 0.0f)) continue;
      int32_t cmin[KB_BINS], cmax[KB_BINS];
      memset(cmin, 0, sizeof(cmin));
      memset(cmax, 0, sizeof(cmax));
      float scale = (float)KB_BINS / ext;
      for (int32_t i = 0; i < n; ++i) {
        float a = cb[6 * i + ax], b = cb[6 * i + 3 + ax];
        int ba = (int)((a - lo[ax]) * scale), bb = (int)((b - lo[ax]) * scale);
        ba = ba < 0 ? 0 : (ba >= KB_BINS ? KB_BINS - 1 : ba);
        bb = bb < 0 ? 0 : (bb >= KB_BINS ? KB_BINS - 1 : bb);
        cmin[ba]++;
        cmax[bb]++;
      }
      /* plane k sits between bins k-1 and k: N_L = triangles starting in a
       * bin below k, N_R = triangles ending in bin k or above */
      int32_t nl = 0, nr = n;
      for (int k = 1; k < KB_BINS; ++k) {
        nl += cmin[k - 1];
        nr -= cmax[k - 1];
        float plane = lo[ax] + ext * (float)k / (float)KB_BINS;
        float llo[3] = {lo[0], lo[1], lo[2]}, lhi[3] = {hi[0], hi[1], hi[2]};
        float rlo[3] = {lo[0], lo[1], lo[2]}, rhi[3] = {hi[0], hi[1], hi[2]};
        lhi[ax] = plane;
        rlo[ax] = plane;
        float cost = s->ct + s->ci * ((float)nl * kb_area(llo, lhi) + (float)nr * kb_area(rlo, rhi)) / area;
        if (nl == 0 || nr == 0) cost *= 1.0f - s->bonus;
        if (cost < best_cost && !(nl == n && nr == n)) {
          best_cost = cost;
          best_axis = ax;
          best_split = plane;
        }
      }
    }
  }
  if (best_axis < 0) {
    free(cb);
    kb_make_leaf(s, id, tris, n);
    return;
  }
  int32_t* left = (int32_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
  int32_t* right = (int32_t*)malloc((size_t)(n > 0 ? n : 1) * sizeof(int32_t));
  if (!left || !right) {
    free(left);
    free(right);
    free(cb);
    s->failed = 1;
    return;
  }
  int32_t nl = 0, nr = 0;
  for (int32_t i = 0; i < n; ++i) {
    int32_t t = tris[i];
    float a = cb[6 * i + best_axis], b = cb[6 * i + 3 + best_axis];
    if (a <= best_split) left[nl++] = t;
    if (b >= best_split) right[nr++] = t;
  }
  free(cb);
  float llo[3] = {lo[0], lo[1], lo[2]}, lhi[3] = {hi[0], hi[1], hi[2]};
  float rlo[3] = {lo[0], lo[1], lo[2]}, rhi[3] = {hi[0], hi[1], hi[2]};
  lhi[best_axis] = best_split;
  rlo[best_axis] = best_split;
  int32_t l = kb_new_node(s);
  int32_t r = kb_new_node(s);
  if (s->failed) {
    free(left);
    free(right);
    return;
  }
  s->nodes[id].axis = best_axis;
  s->nodes[id].split = best_split;
  s->nodes[id].left = l;
  s->nodes[id].right = r;
  s->nodes[id].first = 0;
  s->nodes[id].count = 0;
  kb_build(s, l, left, nl, llo, lhi, depth + 1);
  free(left);
  kb_build(s, r, right, nr, rlo, rhi, depth + 1);
  free(right);
}

int o_kdb_build(const float* verts, int32_t nv, const uint32_t* faces, int32_t nf,
                int max_depth, int leaf_size, float ci, float ct, float empty_bonus,
                o_kdb_tree* out) {
  memset(out, 0, sizeof(*out));
  if (nf <= 0 || nv <= 0) return -1;
  int32_t* all = (int32_t*)malloc((size_t)nf * sizeof(int32_t));
  if (!all) return -1;
  float blo[3] = {1e30f, 1e30f, 1e30f}, bhi[3] = {-1e30f, -1e30f, -1e30f};
  for (int32_t i = 0; i < nf; ++i) {
    all[i] = i;
    for (int v = 0; v < 3; ++v)
      for (int k = 0; k < 3; ++k) {
        float x = verts[3 * faces[3 * i + v] + k];
        if (x < blo[k]) blo[k] = x;
        if (x > bhi[k]) bhi[k] = x;
      }
  }
  (void)nv;
  kb_state s;
  memset(&s, 0, sizeof(s));
  s.verts = verts;
  s.faces = faces;
  s.max_depth = max_depth;
  s.leaf_size = leaf_size;
  s.ci = ci;
  s.ct = ct;
  s.bonus = empty_bonus;
  int32_t root = kb_new_node(&s);
  if (root >= 0) kb_build(&s, root, all, nf, blo, bhi, 0);
  free(all);
  if (s.failed) {
    free(s.nodes);
    free(s.index);
    return -1;
  }
  out->nodes = s.nodes;
  out->n_nodes = s.n_nodes;
  out->index = s.index;
  out->n_index = s.n_index;
  for (int k = 0; k < 3; ++k) {
    out->bmin[k] = blo[k];
    out->bmax[k] = bhi[k];
  }
  return 0;
}

void o_kdb_free(o_kdb_tree* t) {
  if (!t) return;
  free(t->nodes);
  free(t->index);
  memset(t, 0, sizeof(*t));
}
