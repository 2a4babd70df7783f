// Host-side SAH kd-tree builder with ropes and the flattened device layout.
//
// Replaces RKDTreeCPU::build / buildRopeStructure / optimizeRopes
// (RayEngine/src/Primitives/KDTree.cpp:335-834) and RKDThreeGPU::buildTree
// (RayEngine/src/Primitives/KDThreeGPU.cpp:155-194).
//
// Flattened layout (all 32-bit words, little endian):
//   node  (8 B):  { float split, uint32 meta }
//                 meta & 3 = split axis (0..2) or 3 for a leaf;
//                 meta >> 2 = index of the left child (right = left + 1) for
//                 inner nodes, index of the leaf record for leaves.
//   leaf (64 B):  { min.xyz, max.x | max.yz, first, count |
//                   rope[0..3] | rope[4..5], depth, 0 }
//                 rope[2k] / rope[2k+1] = node reached through the -k / +k
//                 face of the leaf's region (-1 = outside the scene).
//   tri  (48 B):  { v0.xyz, id | e1.xyz, 0 | e2.xyz, 0 } one per leaf
//                 reference, stored in leaf order (straddling triangles are
//                 duplicated into every leaf they overlap).
#pragma once
#include <cstdint>
#include <vector>

#include "../../include/rayengine_b200.h"

namespace re {

// Entry table: for each face of the root box (axis k, side 0 = the -k face,
// 1 = the +k face) a kEntryRes x kEntryRes grid of cells over the face's
// other two axes (a < b, cell i along a, j along b), each holding the
// deepest node whose region contains the whole cell grown by a margin of
// 1e-4 x the box's largest extent.  A ray that enters the root box through
// that cell of that face starts its first descent there: at every node
// above, its entry point lies farther from the split plane than rounding
// can move it, so the root descent takes the same path to that node.
// Entry (k, side, i, j) is at ((k * 2 + side) * kEntryRes + i) * kEntryRes + j.
constexpr uint32_t kEntryRes = 128;

struct FlatTree {
  std::vector<uint32_t> nodes;   // 2 words per node
  std::vector<uint32_t> leaves;  // 16 words per leaf
  std::vector<float> tris;       // 12 words per reference
  std::vector<uint32_t> entry;   // 6 * kEntryRes^2 start nodes
  float bmin[3], bmax[3];
  uint32_t num_tris = 0, num_nodes = 0, num_leaves = 0, num_refs = 0;
  uint32_t max_depth = 0, max_leaf_size = 0, bfs_nodes = 0;
  double build_seconds = 0.0;
};

// tris: num_tris x 12 floats {v0,_, e1,_, e2,_}; the builder bounds each
// triangle by v0, v0+e1, v0+e2 evaluated in double.
bool build_kdtree(const float* tris, uint32_t num_tris, const re_kd_params& p,
                  FlatTree& out, const char** err);

}  // namespace re
