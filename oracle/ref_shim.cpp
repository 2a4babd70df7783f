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
//
// Nothing in the product links this file.
#include "repch.h"
#include "Primitives/KDThreeGPU.h"
#include "World/PerlinNoise.h"

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

// Writes RPerlinNoise(seed).permutationTable (512 entries) to out.
void ref_perlin_permutation(uint32_t seed, uint32_t* out) {
  RayEngine::RPerlinNoise noise(seed);
  for (unsigned i = 0; i < 2 * RayEngine::RPerlinNoise::tableSize; ++i)
    out[i] = noise.permutationTable[i];
}

}  // extern "C"
