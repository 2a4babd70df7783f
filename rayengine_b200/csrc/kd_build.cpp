// SAH kd-tree with ropes, built on the host.  See kd_build.hpp for the layout.
//
// Differences from the reference builder (RayEngine/src/Primitives/KDTree.cpp):
//  * split choice: surface-area heuristic (exact event sweep for small nodes,
//    binned for large ones) instead of the spatial median of the longest axis
//    (:367-389; the reference's SAH code at :392-547 is commented out);
//  * children share the split plane exactly (no +-K_EPSILON padding, :376-387)
//    and straddling triangles are clipped to each child region ("perfect
//    splits") instead of being sent whole to both sides (:561-601);
//  * ropes follow the neighbour links of buildRopeStructure (:636-686) and are
//    pushed down as in optimizeRopes (:694-834) with the split-axis test the
//    reference meant (it compares split_val against the axis enum, :757-805).
#include "kd_build.hpp"

#include <omp.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstring>
#include <deque>
#include <memory>

namespace re {
namespace {

struct Box {
  float lo[3], hi[3];
};

struct Ref {
  uint32_t tri;
  float lo[3], hi[3];
};

struct BNode {
  int axis = -1;  // -1: leaf
  float split = 0.f;
  BNode* child[2] = {nullptr, nullptr};
  std::vector<uint32_t> tris;  // leaves only
  Box box;
  int depth = 0;
  BNode* ropes[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  uint32_t flat = 0;
  uint32_t leaf_index = 0;
};

inline double surface_area(const Box& b) {
  double dx = (double)b.hi[0] - b.lo[0], dy = (double)b.hi[1] - b.lo[1],
         dz = (double)b.hi[2] - b.lo[2];
  return 2.0 * (dx * dy + dx * dz + dy * dz);
}

inline float round_down(double x) {
  float f = (float)x;
  if ((double)f > x) f = std::nextafter(f, -INFINITY);
  return f;
}
inline float round_up(double x) {
  float f = (float)x;
  if ((double)f < x) f = std::nextafter(f, INFINITY);
  return f;
}

struct Ctx {
  const float* tris;
  uint32_t num_tris;
  re_kd_params p;
  std::atomic<uint64_t> total_refs{0};
  std::atomic<uint32_t> nodes{0};

  void vertices(uint32_t t, double v[3][3]) const {
    const float* T = tris + 12 * (size_t)t;
    for (int k = 0; k < 3; ++k) {
      v[0][k] = T[k];
      v[1][k] = (double)T[k] + (double)T[4 + k];
      v[2][k] = (double)T[k] + (double)T[8 + k];
    }
  }

  // Bounds of the part of triangle t inside box (Sutherland-Hodgman in
  // double, rounded outward).  false if they do not overlap.
  bool clip(uint32_t t, const Box& box, Ref& r) const {
    double a[12][3], b[12][3];
    int na = 3;
    vertices(t, reinterpret_cast<double(*)[3]>(a));
    for (int k = 0; k < 3; ++k) {
      for (int side = 0; side < 2; ++side) {
        double c = side == 0 ? box.lo[k] : box.hi[k];
        int nb = 0;
        for (int i = 0; i < na; ++i) {
          const double* P = a[i];
          const double* Q = a[(i + 1) % na];
          bool pin = side == 0 ? P[k] >= c : P[k] <= c;
          bool qin = side == 0 ? Q[k] >= c : Q[k] <= c;
          if (pin) {
            std::memcpy(b[nb++], P, sizeof(double) * 3);
          }
          if (pin != qin) {
            double s = (c - P[k]) / (Q[k] - P[k]);
            for (int m = 0; m < 3; ++m) b[nb][m] = P[m] + s * (Q[m] - P[m]);
            b[nb][k] = c;
            ++nb;
          }
        }
        na = nb;
        if (na == 0) return false;
        std::memcpy(a, b, sizeof(double) * 3 * na);
      }
    }
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int i = 0; i < na; ++i)
      for (int k = 0; k < 3; ++k) {
        lo[k] = std::min(lo[k], a[i][k]);
        hi[k] = std::max(hi[k], a[i][k]);
      }
    r.tri = t;
    for (int k = 0; k < 3; ++k) {
      r.lo[k] = std::max(round_down(lo[k]), box.lo[k]);
      r.hi[k] = std::min(round_up(hi[k]), box.hi[k]);
      if (r.lo[k] > r.hi[k]) return false;
    }
    return true;
  }

  double cost(const Box& box, int k, float s, double nl, double nr) const {
    Box L = box, R = box;
    L.hi[k] = s;
    R.lo[k] = s;
    double sa = surface_area(box);
    double pl = sa > 0 ? surface_area(L) / sa : 0.5, pr = sa > 0 ? surface_area(R) / sa : 0.5;
    double bonus = (nl == 0 || nr == 0) ? (double)p.empty_bonus : 0.0;
    return p.cost_traversal + p.cost_intersect * (1.0 - bonus) * (pl * nl + pr * nr);
  }

  struct Split {
    double cost = INFINITY;
    int axis = -1;
    float pos = 0.f;
    bool planar_left = true;
    size_t nl = 0, nr = 0;
  };

  void sweep_exact(const std::vector<Ref>& refs, const Box& box, Split& best) const {
    struct Ev {
      float pos;
      int type;  // 0 end, 1 planar, 2 start
    };
    std::vector<Ev> ev;
    ev.reserve(refs.size() * 2);
    size_t n = refs.size();
    for (int k = 0; k < 3; ++k) {
      if (!(box.hi[k] > box.lo[k])) continue;
      ev.clear();
      for (const Ref& r : refs) {
        if (r.lo[k] == r.hi[k]) {
          ev.push_back({r.lo[k], 1});
        } else {
          ev.push_back({r.lo[k], 2});
          ev.push_back({r.hi[k], 0});
        }
      }
      std::sort(ev.begin(), ev.end(), [](const Ev& a, const Ev& b) {
        return a.pos < b.pos || (a.pos == b.pos && a.type < b.type);
      });
      size_t nl = 0, nr = n;
      for (size_t i = 0; i < ev.size();) {
        float pos = ev[i].pos;
        size_t pe = 0, pp = 0, ps = 0;
        while (i < ev.size() && ev[i].pos == pos && ev[i].type == 0) { ++pe; ++i; }
        while (i < ev.size() && ev[i].pos == pos && ev[i].type == 1) { ++pp; ++i; }
        while (i < ev.size() && ev[i].pos == pos && ev[i].type == 2) { ++ps; ++i; }
        nr -= pp + pe;
        if (pos > box.lo[k] && pos < box.hi[k]) {
          double cl = cost(box, k, pos, (double)(nl + pp), (double)nr);
          double cr = cost(box, k, pos, (double)nl, (double)(nr + pp));
          if (cl < best.cost) {
            best = {cl, k, pos, true, nl + pp, nr};
          }
          if (cr < best.cost) {
            best = {cr, k, pos, false, nl, nr + pp};
          }
        }
        nl += ps + pp;
      }
    }
  }

  void sweep_binned(const std::vector<Ref>& refs, const Box& box, Split& best) const {
    constexpr int NB = 256;
    size_t n = refs.size();
    for (int k = 0; k < 3; ++k) {
      double ext = (double)box.hi[k] - box.lo[k];
      if (!(ext > 0)) continue;
      double scale = NB / ext;
      std::vector<uint32_t> starts(NB, 0), ends(NB, 0);
      auto bin = [&](float x) {
        int b = (int)(((double)x - box.lo[k]) * scale);
        return std::min(std::max(b, 0), NB - 1);
      };
      for (const Ref& r : refs) {
        starts[bin(r.lo[k])]++;
        ends[bin(r.hi[k])]++;
      }
      size_t nl = 0, nr = n;
      for (int b = 1; b < NB; ++b) {
        nl += starts[b - 1];
        nr -= ends[b - 1];
        float pos = (float)((double)box.lo[k] + ext * b / NB);
        if (!(pos > box.lo[k] && pos < box.hi[k])) continue;
        double c = cost(box, k, pos, (double)nl, (double)nr);
        if (c < best.cost) best = {c, k, pos, true, nl, nr};
      }
    }
  }

  BNode* make_leaf(std::vector<Ref>& refs, const Box& box, int depth) {
    BNode* node = new BNode();
    node->box = box;
    node->depth = depth;
    node->tris.reserve(refs.size());
    for (const Ref& r : refs) node->tris.push_back(r.tri);
    std::sort(node->tris.begin(), node->tris.end());
    refs.clear();
    refs.shrink_to_fit();
    nodes.fetch_add(1, std::memory_order_relaxed);
    return node;
  }

  BNode* build(std::vector<Ref>& refs, const Box& box, int depth) {
    size_t n = refs.size();
    if (n <= p.leaf_size || depth >= (int)p.max_depth) return make_leaf(refs, box, depth);
    Split best;
    if (n <= 1024)
      sweep_exact(refs, box, best);
    else
      sweep_binned(refs, box, best);
    if (best.axis < 0) return make_leaf(refs, box, depth);
    double leaf_cost = p.cost_intersect * (double)n;
    if (best.cost >= leaf_cost) {
      // The SAH prefers a leaf; the leaf-size bound still asks for a split
      // as long as both sides shrink and duplication stays bounded.
      bool progress = best.nl < n && best.nr < n;
      bool budget = total_refs.load(std::memory_order_relaxed) < 8ull * num_tris + 1024;
      if (!progress || !budget) return make_leaf(refs, box, depth);
    }
    int k = best.axis;
    float s = best.pos;
    Box lb = box, rb = box;
    lb.hi[k] = s;
    rb.lo[k] = s;
    std::vector<Ref> left, right;
    left.reserve(best.nl + 16);
    right.reserve(best.nr + 16);
    for (const Ref& r : refs) {
      if (r.lo[k] == s && r.hi[k] == s) {
        (best.planar_left ? left : right).push_back(r);
      } else if (r.hi[k] <= s) {
        left.push_back(r);
      } else if (r.lo[k] >= s) {
        right.push_back(r);
      } else {
        Ref c;
        if (clip(r.tri, lb, c)) left.push_back(c);
        if (clip(r.tri, rb, c)) right.push_back(c);
      }
    }
    if (left.size() == n && right.size() == n) return make_leaf(refs, box, depth);
    refs.clear();
    refs.shrink_to_fit();
    total_refs.fetch_add(left.size() + right.size() - n, std::memory_order_relaxed);
    BNode* node = new BNode();
    node->axis = k;
    node->split = s;
    node->box = box;
    node->depth = depth;
    nodes.fetch_add(1, std::memory_order_relaxed);
    size_t work = left.size() + right.size();
    if (work > 4096) {
#pragma omp task shared(left, lb, node) firstprivate(depth)
      node->child[0] = build(left, lb, depth + 1);
#pragma omp task shared(right, rb, node) firstprivate(depth)
      node->child[1] = build(right, rb, depth + 1);
#pragma omp taskwait
    } else {
      node->child[0] = build(left, lb, depth + 1);
      node->child[1] = build(right, rb, depth + 1);
    }
    return node;
  }
};

void free_tree(BNode* n) {
  if (!n) return;
  free_tree(n->child[0]);
  free_tree(n->child[1]);
  delete n;
}

void link_ropes(BNode* n, BNode* const r[6]) {
  if (n->axis < 0) {
    for (int f = 0; f < 6; ++f) {
      BNode* t = r[f];
      int fk = f >> 1;
      bool positive = (f & 1) != 0;
      while (t && t->axis >= 0) {
        int k = t->axis;
        if (k == fk) {
          t = positive ? t->child[0] : t->child[1];
        } else if (t->split <= n->box.lo[k]) {
          t = t->child[1];
        } else if (t->split >= n->box.hi[k]) {
          t = t->child[0];
        } else {
          break;
        }
      }
      n->ropes[f] = t;
    }
    return;
  }
  int k = n->axis;
  BNode* rl[6];
  BNode* rr[6];
  for (int f = 0; f < 6; ++f) rl[f] = rr[f] = r[f];
  rl[2 * k + 1] = n->child[1];
  rr[2 * k] = n->child[0];
  link_ropes(n->child[0], rl);
  link_ropes(n->child[1], rr);
}

}  // namespace

// The entry table of FlatTree (kd_build.hpp): per face cell, descend from
// the root while the cell, grown by the margin, lies strictly on one side of
// the split (on the face's own axis the cell is the face plane itself).
void build_entry_table(FlatTree& t) {
  const uint32_t R = kEntryRes;
  t.entry.assign(6u * R * R, 0u);
  double lo_box[3], ext[3], emax = 0.0;
  for (int k = 0; k < 3; ++k) {
    lo_box[k] = t.bmin[k];
    ext[k] = (double)t.bmax[k] - (double)t.bmin[k];
    emax = std::max(emax, ext[k]);
  }
  const double m = 1e-4 * emax;
  auto split_of = [&](uint32_t n) {
    float f;
    std::memcpy(&f, &t.nodes[2 * (size_t)n], 4);
    return (double)f;
  };
#pragma omp parallel for schedule(static)
  for (int face = 0; face < 6; ++face) {
    const int k = face >> 1, side = face & 1;
    const int a = k == 0 ? 1 : 0, b = k == 2 ? 1 : 2;
    const double f = side ? (double)t.bmax[k] : (double)t.bmin[k];
    for (uint32_t i = 0; i < R; ++i) {
      for (uint32_t j = 0; j < R; ++j) {
        double lo[3], hi[3];
        lo[a] = lo_box[a] + ext[a] * i / R - m;
        hi[a] = lo_box[a] + ext[a] * (i + 1) / R + m;
        lo[b] = lo_box[b] + ext[b] * j / R - m;
        hi[b] = lo_box[b] + ext[b] * (j + 1) / R + m;
        lo[k] = f - m;
        hi[k] = f + m;
        uint32_t node = 0;
        for (;;) {
          const uint32_t meta = t.nodes[2 * (size_t)node + 1];
          const uint32_t axis = meta & 3u;
          if (axis == 3u) break;
          const double s = split_of(node);
          if (hi[axis] < s) {
            node = meta >> 2;
          } else if (lo[axis] > s) {
            node = (meta >> 2) + 1u;
          } else {
            break;
          }
        }
        t.entry[((size_t)face * R + i) * R + j] = node;
      }
    }
  }
}

bool build_kdtree(const float* tris, uint32_t num_tris, const re_kd_params& params,
                  FlatTree& out, const char** err) {
  auto t0 = std::chrono::steady_clock::now();
  if (num_tris == 0) {
    *err = "build_kdtree: no triangles";
    return false;
  }
  Ctx ctx;
  ctx.tris = tris;
  ctx.num_tris = num_tris;
  ctx.p = params;

  // Root box: the bounding box of the triangles' float vertices, as
  // RKDTreeCPU's generateBox computes it (KDTree.cpp:837-888).
  Box root;
  for (int k = 0; k < 3; ++k) {
    root.lo[k] = INFINITY;
    root.hi[k] = -INFINITY;
  }
  for (uint32_t t = 0; t < num_tris; ++t) {
    const float* T = tris + 12 * (size_t)t;
    for (int k = 0; k < 3; ++k) {
      float a = T[k], b = T[k] + T[4 + k], c = T[k] + T[8 + k];
      root.lo[k] = std::min(root.lo[k], std::min(a, std::min(b, c)));
      root.hi[k] = std::max(root.hi[k], std::max(a, std::max(b, c)));
    }
  }
  for (int k = 0; k < 3; ++k) {
    if (!std::isfinite(root.lo[k]) || !std::isfinite(root.hi[k])) {
      *err = "build_kdtree: non-finite vertex";
      return false;
    }
  }

  std::vector<Ref> refs;
  refs.reserve(num_tris);
  for (uint32_t t = 0; t < num_tris; ++t) {
    Ref r;
    double v[3][3];
    ctx.vertices(t, v);
    r.tri = t;
    for (int k = 0; k < 3; ++k) {
      double lo = std::min(v[0][k], std::min(v[1][k], v[2][k]));
      double hi = std::max(v[0][k], std::max(v[1][k], v[2][k]));
      r.lo[k] = std::max(round_down(lo), root.lo[k]);
      r.hi[k] = std::min(round_up(hi), root.hi[k]);
    }
    refs.push_back(r);
  }
  ctx.total_refs = num_tris;

  int threads = params.threads ? (int)params.threads : omp_get_max_threads();
  BNode* tree = nullptr;
#pragma omp parallel num_threads(threads)
  {
#pragma omp single
    tree = ctx.build(refs, root, 0);
  }

  BNode* none[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  link_ropes(tree, none);

  // Flat order: breadth-first for the top levels (a prefix of the node array
  // the kernels can stage in shared memory), then depth-first subtrees with
  // sibling pairs adjacent.
  std::vector<BNode*> order;
  order.reserve(ctx.nodes.load());
  std::vector<BNode*> deferred;
  std::deque<BNode*> q;
  tree->flat = 0;
  order.push_back(tree);
  q.push_back(tree);
  while (!q.empty()) {
    BNode* n = q.front();
    q.pop_front();
    if (n->axis < 0) continue;
    if (n->depth < (int)params.bfs_levels) {
      for (int c = 0; c < 2; ++c) {
        n->child[c]->flat = (uint32_t)order.size();
        order.push_back(n->child[c]);
        q.push_back(n->child[c]);
      }
    } else {
      deferred.push_back(n);
    }
  }
  uint32_t bfs_nodes = (uint32_t)order.size();
  // iterative DFS per deferred subtree
  std::vector<BNode*> stack;
  for (BNode* d : deferred) {
    stack.push_back(d);
    while (!stack.empty()) {
      BNode* n = stack.back();
      stack.pop_back();
      if (n->axis < 0) continue;
      for (int c = 0; c < 2; ++c) {
        n->child[c]->flat = (uint32_t)order.size();
        order.push_back(n->child[c]);
      }
      stack.push_back(n->child[1]);
      stack.push_back(n->child[0]);
    }
  }

  uint32_t nn = (uint32_t)order.size();
  if (nn >= (1u << 30)) {
    free_tree(tree);
    *err = "build_kdtree: tree exceeds 2^30 nodes";
    return false;
  }
  uint32_t nl = 0;
  uint64_t nrefs = 0;
  uint32_t maxd = 0, maxleaf = 0;
  for (BNode* n : order) {
    if (n->axis < 0) {
      n->leaf_index = nl++;
      nrefs += n->tris.size();
      maxleaf = std::max<uint32_t>(maxleaf, (uint32_t)n->tris.size());
    }
    maxd = std::max<uint32_t>(maxd, (uint32_t)n->depth);
  }
  if (nrefs >= (1ull << 31)) {
    free_tree(tree);
    *err = "build_kdtree: too many triangle references";
    return false;
  }
  out.nodes.assign(2 * (size_t)nn, 0);
  out.leaves.assign(16 * (size_t)nl, 0);
  out.tris.assign(12 * (size_t)nrefs, 0.f);
  uint32_t ref = 0;
  for (BNode* n : order) {
    uint32_t* N = &out.nodes[2 * (size_t)n->flat];
    if (n->axis >= 0) {
      std::memcpy(&N[0], &n->split, 4);
      N[1] = (uint32_t)n->axis | (n->child[0]->flat << 2);
      continue;
    }
    // first triangle reference, so traversal can fetch it with the leaf
    // record; bit 31 marks an empty leaf (references stay below 2^31)
    N[0] = n->tris.empty() ? (ref | 0x80000000u) : ref;
    N[1] = 3u | (n->leaf_index << 2);
    uint32_t* L = &out.leaves[16 * (size_t)n->leaf_index];
    std::memcpy(&L[0], n->box.lo, 12);
    std::memcpy(&L[3], n->box.hi, 12);
    L[6] = ref;
    L[7] = (uint32_t)n->tris.size();
    for (int f = 0; f < 6; ++f) L[8 + f] = n->ropes[f] ? n->ropes[f]->flat : 0xFFFFFFFFu;
    L[14] = (uint32_t)n->depth;
    L[15] = 0;
    for (uint32_t t : n->tris) {
      float* D = &out.tris[12 * (size_t)ref];
      const float* S = tris + 12 * (size_t)t;
      D[0] = S[0];
      D[1] = S[1];
      D[2] = S[2];
      std::memcpy(&D[3], &t, 4);
      D[4] = S[4];
      D[5] = S[5];
      D[6] = S[6];
      D[7] = 0.f;
      D[8] = S[8];
      D[9] = S[9];
      D[10] = S[10];
      D[11] = 0.f;
      ++ref;
    }
  }
  for (int k = 0; k < 3; ++k) {
    out.bmin[k] = root.lo[k];
    out.bmax[k] = root.hi[k];
  }
  out.num_tris = num_tris;
  out.num_nodes = nn;
  out.num_leaves = nl;
  out.num_refs = (uint32_t)nrefs;
  out.max_depth = maxd;
  out.max_leaf_size = maxleaf;
  out.bfs_nodes = bfs_nodes;
  free_tree(tree);
  build_entry_table(out);
  out.build_seconds =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  return true;
}

}  // namespace re
