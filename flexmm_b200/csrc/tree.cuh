// Quadtree data on the device.  Nodes of all levels live in one level-major
// array; inside a level they are in Morton order, and the four children of a
// box are consecutive (digit = 2*[x > xmid] + [y > ymid]).
#pragma once
#include "common.cuh"

namespace fmmb {

enum NodeFlag : uint8_t {
  NF_LEAF = 1,      // real leaf (targets stop here); X-list leaves included
  NF_FAKE = 2,      // fake leaf: child of an X-list leaf, source-only
  NF_XLIST = 4,     // real leaf with a non-leaf colleague; owns 4 fake children
  NF_CHILDREN = 8,  // has 4 children on the next level
};

constexpr int N_OFFSETS = 40;  // far-field offsets (-3..3)^2 minus (-1..1)^2

// offset id 0..39 <-> (ox, oy); ids walk ox = -3..3 (outer), oy = -3..3 (inner)
__host__ __device__ inline void offset_of(int id, int &ox, int &oy) {
  int k = 0;
  for (int a = -3; a <= 3; ++a)
    for (int b = -3; b <= 3; ++b) {
      if (a >= -1 && a <= 1 && b >= -1 && b <= 1) continue;
      if (k == id) {
        ox = a;
        oy = b;
        return;
      }
      ++k;
    }
  ox = oy = 0;
}

struct TreeDev {
  // points (sorted by key)
  DevBuf<uint64_t> pkeys;
  DevBuf<int> ordv;       // sorted position -> original index
  DevBuf<double> sx, sy;  // sorted source coordinates
  // nodes
  DevBuf<uint64_t> code;  // morton code at the node's level
  DevBuf<double> xmin, ymin, xmid, ymid;
  DevBuf<int> bot, top, parent, child;
  DevBuf<uint8_t> flags;
  DevBuf<int> coll;  // [n_total x 9], -1 padded
  DevBuf<int> il;    // [n_total x 40] source node per offset, -1 if none
  DevBuf<int> dev_off;  // level offsets [L+1]
  DevBuf<int> rg;       // first node of every real sibling group, level-major
  DevBuf<int> ix, iy;   // integer box coordinates at the node's level
  // nodes at levels >= 2 whose multipoles come from their own points (S2M):
  // real leaves that are not X-list leaves, and fake leaves, holding points;
  // in node order (so level-major).  Count on the device.
  DevBuf<int> uplist, n_up;
  // set to 1 by a radix sort of this tree (the build's or a target sort)
  // whose grid barrier wait ran out; the sorted outputs are then invalid
  DevBuf<int> sort_fail;
};

struct TreeHost {
  int L = 0;
  int64_t n_points = 0;
  int ppl = 0;
  double x0 = 0, y0 = 0, w0 = 0;
  std::vector<int> off;       // L+1 (after finalize_tree)
  std::vector<double> width;  // per level
  std::vector<int> rg_lo, rg_hi;  // per level: range of its real groups in rg (after finalize_tree)
  int n_total() const { return off.empty() ? 0 : off.back(); }
  // build_tree returns before the per-level counts reach the host: they
  // come back by an asynchronous copy into pinned memory, `ready` marks its
  // completion, and finalize_tree() fills off / rg_lo / rg_hi from them.
  bool pending = false;
  int *pending_counts = nullptr;  // pinned, 2 (L+1) ints
  cudaEvent_t ready = nullptr;
  TreeHost() = default;
  TreeHost(const TreeHost &) = delete;
  TreeHost &operator=(const TreeHost &) = delete;
  ~TreeHost();
};

// Wait for the per-level counts of the last build_tree and fill the host
// offsets (a no-op once done).  Every use of off, rg_lo, rg_hi or n_total()
// after build_tree comes after this.
void finalize_tree(TreeHost &th);

// Build the tree over device coordinates x, y (n points) on `stream`;
// boxes of levels >= max_split are never split (default: no floor).
void build_tree(TreeDev &td, TreeHost &th, const double *x, const double *y, int64_t n, int ppl,
                const double bbox[4], cudaStream_t stream, int max_split = 64);

// Sort arbitrary points by the same descent key on its top `sorted_digits`
// quadrant digits (enough to place them in boxes of levels <= sorted_digits);
// returns the keys in that order and the permutation sorted -> original,
// and (if sx, sy are given) the coordinates in that order.
// The sort is stable (points with equal digits keep their input order).
// fail (optional, device int) is set to 1 if the sort's grid barrier wait
// ran out (the outputs are then invalid but hold valid indices).
void sort_points(const double *x, const double *y, int64_t n, const TreeHost &th,
                 DevBuf<uint64_t> &keys, DevBuf<int> &perm, cudaStream_t stream,
                 int sorted_digits = MAXD, double *sx = nullptr, double *sy = nullptr,
                 int *fail = nullptr);

// The same into caller-provided memory: keys [n], perm [n], optional sx, sy
// [n], and scratch of sort_points_scratch_bytes(n, sorted_digits) bytes.
size_t sort_points_scratch_bytes(int64_t n, int sorted_digits);

// Points into the tree's leaves without a sort: leaf_of[i] (the real leaf
// holding point i, -1 for none) and slot[i] (its place among the leaf's
// points, in no particular order); count[node] (zeroed by the caller) gets
// the points per leaf.  scatter_binned then writes the points leaf by leaf
// (first[node]: the exclusive scan of count) with perm (position -> point).
void bin_points(const double *x, const double *y, int64_t m, const TreeDev &td, const TreeHost &th,
                int *count, int *leaf_of, int *slot, cudaStream_t s);
void scatter_binned(const double *x, const double *y, int64_t m, const int *leaf_of,
                    const int *slot, const int *first, double *xs, double *ys, int *perm,
                    cudaStream_t s);
void sort_points_scratch(const double *x, const double *y, int64_t n, const TreeHost &th,
                         int sorted_digits, uint64_t *keys, int *perm, double *sx, double *sy,
                         void *scratch, size_t scratch_bytes, int *fail, cudaStream_t stream);

}  // namespace fmmb
