// Test infrastructure: a thin extern "C" wrapper around the reference's own
// host code, compiled from the reference's unmodified sources (see
// oracle/Makefile.ref).  It is only used by tests and by the generator of the
// golden fixtures to pin the CPU restatement in oracle/oracle.c:
//
//   * RKDTreeCPU + RKDThreeGPU (RayEngine/src/Primitives/KDTree.cpp:117-173,
//     RayEngine/src/Primitives/KDThreeGPU.cpp:9-54,155-194): the tree the
//     reference actually builds (MAX_DEPTH = 1 as shipped -> one leaf), its
//     flattened 128-byte RKDTreeNodeGPU records and obj_index_list.
//   * RPerlinNoise (RayEngine/src/World/PerlinNoise.h:16-52): the 512-entry
//     permutation table for a seed.
//   * RKDTreeCPU::singleRayStacklessIntersect (KDTree.cpp:993-1066): the
//     reference's own CPU ray query (closest hit: t and the interpolated
//     vertex normal, two-sided triIntersect, KDTree.cpp:909-949) over its
//     own tree, run over many rays with OpenMP `parallel for
//     schedule(dynamic)` as RRayTracer::trace does
//     (RayEngine/src/Engine/RayTracer.cpp:154).  The benchmark's reference
//     arm times this, over the reference's own one-leaf tree and over an SAH
//     tree of the configured parameters (oracle_kdbuild.c) turned into the
//     reference's KDNodeCPU objects (ref_tree_from_kd).
//
// Nothing in the product links this file.
#include "repch.h"
#include "Primitives/KDThreeGPU.h"
#include "Primitives/Ray.h"
#include "World/PerlinNoise.h"

#include <omp.h>

#include <cmath>
#include <cstdint>
#include <cstring>

extern "C" {

int ref_sizeof_node(void) { return (int)sizeof(RKDTreeNodeGPU); }

// Builds the reference kd-tree over an indexed mesh and copies out the
// flattened node array (raw RKDTreeNodeGPU bytes) and the leaf index list.
// Returns the number of nodes, or -1 if the caller's buffers are too small.
// On return *out_root = root vid, *out_nidx = obj_index_list size,
// *out_levels = numLevels, *out_leaves = numLeaves.
int ref_build_kdtree(const float* verts, int num_verts, const uint32_t* faces,
                     int num_faces, void* out_nodes, int max_nodes,
                     int32_t* out_index_list, int max_index, int* out_root,
                     int* out_nidx, int* out_levels, int* out_leaves) {
  std::vector<float3> v(num_verts), n(num_verts);
  for (int i = 0; i < num_verts; ++i) {
    v[i] = make_float3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
    n[i] = make_float3(0.f, 1.f, 0.f);
  }
  std::vector<uint3> f(num_faces);
  for (int i = 0; i < num_faces; ++i)
    f[i] = make_uint3(faces[3 * i], faces[3 * i + 1], faces[3 * i + 2]);
  RKDTreeCPU* cpu = new RKDTreeCPU(v.data(), f.data(), n.data(), nullptr,
                                   num_verts, num_faces, num_verts, 0);
  RKDThreeGPU* gpu = new RKDThreeGPU(cpu);
  int nn = (int)gpu->GetNumNodes();
  std::vector<int> idx = gpu->GetIndexList();
  int rc = nn;
  if (nn > max_nodes || (int)idx.size() > max_index) {
    rc = -1;
  } else {
    std::memcpy(out_nodes, gpu->GetNodes(), sizeof(RKDTreeNodeGPU) * nn);
    for (size_t i = 0; i < idx.size(); ++i) out_index_list[i] = idx[i];
  }
  *out_root = (int)gpu->get_root_index();
  *out_nidx = (int)idx.size();
  *out_levels = cpu->numLevels;
  *out_leaves = cpu->numLeaves;
  // The reference destructors free the mesh copies; the node array of
  // RKDThreeGPU is freed by its destructor as well.
  delete gpu;
  delete cpu;
  return rc;
}

// The reference's CPU tree (RKDTreeCPU) over an indexed mesh, kept for ray
// queries.  Vertex normals: the normalised sum of the adjacent faces'
// normals (the reference's mesh loaders supply per-vertex normals).
void* ref_tree_create(const float* verts, int num_verts, const uint32_t* faces, int num_faces) {
  std::vector<float3> v(num_verts), n(num_verts, make_float3(0.f, 0.f, 0.f));
  for (int i = 0; i < num_verts; ++i)
    v[i] = make_float3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
  std::vector<uint3> f(num_faces);
  for (int i = 0; i < num_faces; ++i) {
    f[i] = make_uint3(faces[3 * i], faces[3 * i + 1], faces[3 * i + 2]);
    float3 a = v[f[i].x], b = v[f[i].y], c = v[f[i].z];
    float3 e1 = make_float3(b.x - a.x, b.y - a.y, b.z - a.z);
    float3 e2 = make_float3(c.x - a.x, c.y - a.y, c.z - a.z);
    float3 fn = make_float3(e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z,
                            e1.x * e2.y - e1.y * e2.x);
    for (uint32_t k : {f[i].x, f[i].y, f[i].z}) {
      n[k].x += fn.x;
      n[k].y += fn.y;
      n[k].z += fn.z;
    }
  }
  for (auto& x : n) {
    float l = std::sqrt(x.x * x.x + x.y * x.y + x.z * x.z);
    x = l > 0.f ? make_float3(x.x / l, x.y / l, x.z / l) : make_float3(0.f, 1.f, 0.f);
  }
  return new RKDTreeCPU(v.data(), f.data(), n.data(), nullptr, num_verts, num_faces, num_verts, 0);
}

// An SAH tree made elsewhere (oracle_kdbuild.c: pre-order nodes {axis (3 =
// leaf), split, left, right, first, count} and the leaves' triangle lists)
// turned into the reference's own KDNodeCPU objects inside an RKDTreeCPU, so
// that its CPU query runs over a tree of the configured parameters instead
// of the one leaf its builder makes.  Node boxes are the root box cut at
// the splits; the query (singleRayStacklessIntersect) tests each node's box
// and recurses into both children, testing every leaf the ray's box test
// reaches.
struct RefKdbNode {
  int32_t axis;
  float split;
  int32_t left, right, first, count;
};

static KDNodeCPU* ref_make_node(const RefKdbNode* nodes, const int32_t* index, int32_t id,
                                float3 lo, float3 hi) {
  const RefKdbNode& src = nodes[id];
  KDNodeCPU* n = new KDNodeCPU();
  n->box = RBoundingVolume(lo, hi);
  n->numFaces = 0;
  n->numVerts = 0;
  n->objIndeces = nullptr;
  n->split_val = src.split;
  n->axis = src.axis == 0 ? X_Axis : (src.axis == 1 ? Y_Axis : Z_Axis);
  if (src.axis == 3) {
    n->isLeaf = true;
    n->numFaces = src.count;
    if (src.count > 0) {
      n->objIndeces = new int[src.count];
      for (int32_t i = 0; i < src.count; ++i) n->objIndeces[i] = index[src.first + i];
    }
    return n;
  }
  float3 lhi = hi, rlo = lo;
  if (src.axis == 0) {
    lhi.x = src.split;
    rlo.x = src.split;
  } else if (src.axis == 1) {
    lhi.y = src.split;
    rlo.y = src.split;
  } else {
    lhi.z = src.split;
    rlo.z = src.split;
  }
  n->isLeaf = false;
  n->LeftNode = ref_make_node(nodes, index, src.left, lo, lhi);
  n->RightNode = ref_make_node(nodes, index, src.right, rlo, hi);
  return n;
}

void* ref_tree_from_kd(const float* verts, int num_verts, const uint32_t* faces, int num_faces,
                       const void* kd_nodes, const int32_t* kd_index, const float* bmin,
                       const float* bmax) {
  RKDTreeCPU* t = new RKDTreeCPU();
  t->num_verts = num_verts;
  t->num_norms = num_verts;
  t->num_faces = num_faces;
  t->num_uvs = 0;
  t->uvs = nullptr;
  t->verts = new float3[num_verts];
  t->norms = new float3[num_verts];
  t->faces = new uint3[num_faces];
  for (int i = 0; i < num_verts; ++i) {
    t->verts[i] = make_float3(verts[3 * i], verts[3 * i + 1], verts[3 * i + 2]);
    t->norms[i] = make_float3(0.f, 0.f, 0.f);
  }
  for (int i = 0; i < num_faces; ++i) {
    t->faces[i] = make_uint3(faces[3 * i], faces[3 * i + 1], faces[3 * i + 2]);
    float3 a = t->verts[t->faces[i].x], b = t->verts[t->faces[i].y], c = t->verts[t->faces[i].z];
    float3 e1 = make_float3(b.x - a.x, b.y - a.y, b.z - a.z);
    float3 e2 = make_float3(c.x - a.x, c.y - a.y, c.z - a.z);
    float3 fn = make_float3(e1.y * e2.z - e1.z * e2.y, e1.z * e2.x - e1.x * e2.z,
                            e1.x * e2.y - e1.y * e2.x);
    for (uint32_t k : {t->faces[i].x, t->faces[i].y, t->faces[i].z}) {
      t->norms[k].x += fn.x;
      t->norms[k].y += fn.y;
      t->norms[k].z += fn.z;
    }
  }
  for (int i = 0; i < num_verts; ++i) {
    float3& x = t->norms[i];
    float l = std::sqrt(x.x * x.x + x.y * x.y + x.z * x.z);
    x = l > 0.f ? make_float3(x.x / l, x.y / l, x.z / l) : make_float3(0.f, 1.f, 0.f);
  }
  t->root = ref_make_node(static_cast<const RefKdbNode*>(kd_nodes), kd_index, 0,
                          make_float3(bmin[0], bmin[1], bmin[2]),
                          make_float3(bmax[0], bmax[1], bmax[2]));
  return t;
}

void ref_tree_destroy(void* tree) { delete static_cast<RKDTreeCPU*>(tree); }

// rays: n x 6 floats {origin, direction}.  out_t: closest hit distance
// (K_INFINITY where the query reports no hit), out_n: n x 3 normal.
// Returns the number of rays that hit.
int64_t ref_tree_trace(void* tree, const float* rays, int64_t n, float* out_t, float* out_n,
                       int threads) {
  RKDTreeCPU* t = static_cast<RKDTreeCPU*>(tree);
  int64_t hits = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : hits) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < n; ++i) {
    const float* r = rays + 6 * i;
    RRay ray(make_float3(r[0], r[1], r[2]), make_float3(r[3], r[4], r[5]));
    float th = K_INFINITY;
    float3 nrm = make_float3(0.f, 0.f, 0.f);
    bool hit = t->singleRayStacklessIntersect(ray, th, nrm);
    out_t[i] = hit ? th : K_INFINITY;
    out_n[3 * i] = nrm.x;
    out_n[3 * i + 1] = nrm.y;
    out_n[3 * i + 2] = nrm.z;
    hits += hit ? 1 : 0;
  }
  return hits;
}

int ref_max_threads(void) { return omp_get_max_threads(); }

// Writes RPerlinNoise(seed).permutationTable (512 entries) to out.
void ref_perlin_permutation(uint32_t seed, uint32_t* out) {
  RayEngine::RPerlinNoise noise(seed);
  for (unsigned i = 0; i < 2 * RayEngine::RPerlinNoise::tableSize; ++i)
    out[i] = noise.permutationTable[i];
}

}  // extern "C"
