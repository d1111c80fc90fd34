// GPU quadtree build, reproducing the reference tree (flexmm/tree.py) box for box.
//
// The reference refines level by level, splitting every node with more than
// `ppl` points (flexmm/tree.py:191-220), then enforces a 2:1 rule by
// repeatedly splitting leaves with a colleague of subtree depth >= 2
// (flexmm/tree.py:371-383, 529-541), then gives every leaf with a non-leaf
// colleague four "fake" children (flexmm/tree.py:385-397, 542-553).
//
// Here the same tree is computed without sequential partitioning:
//  1. every point gets a key of 29 quadrant digits equal to descending from
//     the root with the reference's own float64 midpoint arithmetic
//     (xmid = xmin + half_width, child xmin = xmid - half_width or xmid,
//     class = 2*(x > xmid) + (y > ymid)): the bits of the fixed-point cell
//     index where a point is clear of every split line, the descent itself
//     near one, so every comparison is bit-identical;
//  2. keys are radix-sorted (on 32-bit prefixes while 16 digits suffice):
//     every box is a contiguous run of sorted keys;
//  3. the initially split boxes S0 are the key prefixes with more than `ppl`
//     points, read off the sorted keys (a run starting at i is longer than
//     ppl iff key i and key i+ppl share the prefix);
//  4. the 2:1 closure is computed bottom-up as a set: a box is split iff it
//     is initially split or it neighbours (incl. diagonally) a box with a
//     split child; the set is grown level by level in a GPU hash set.  This
//     least fixpoint is the same one the reference's iteration reaches;
//  5. X-list leaves are the real leaves adjacent to a split box;
//  6. the parent boxes (split boxes and X-list leaves) are sorted by
//     (level, morton); each contributes 4 consecutive children, so node
//     arrays, ranges, colleagues and interaction lists follow from binary
//     searches in sorted arrays.
// The host waits twice (for the split-box count and depth, then for the
// balance closure's size); the per-level node counts come back without a
// wait (finalize_tree).
#include <cmath>

#include <memory>
#include <mutex>

#include "radix.cuh"
#include "scan.cuh"
#include "timing.cuh"
#include "tree.cuh"

namespace fmmb {
namespace {

constexpr int TPB = 256;

struct Counters {
  unsigned long long s0_count;
  unsigned long long f_count;
  unsigned long long x_count;
  int max_level;
  int too_deep;
  int overflow;
  int need_full_sort;
  unsigned int bar_count;  // grid barrier of the cooperative balance kernel
  unsigned int bar_gen;
  int bar_timeout;
  int sort_fail;  // copy of the tree's sort failure flag, read back with the counts
};

// The source keys are first sorted on their top SORT_DIGITS digits only; that
// fixes every box of levels <= SORT_DIGITS.  A tree that would split a box of
// level >= SORT_DIGITS is redone with a full sort.  12 digits are 24 bits of
// the 32-bit sort keys: three radix passes (16 digits took four), enough for
// trees up to 14 levels (the 1M clustered headline tree has 13).
constexpr int SORT_DIGITS = 12;

__device__ __forceinline__ int common_digits(uint64_t a, uint64_t b) {
  uint64_t d = a ^ b;
  if (d == 0) return MAXD;
  return (__clzll((long long)d) - (64 - 2 * MAXD)) >> 1;
}

__device__ __forceinline__ uint64_t mix64(uint64_t k) {
  k ^= k >> 33;
  k *= 0xff51afd7ed558ccdULL;
  k ^= k >> 33;
  k *= 0xc4ceb9fe1a85ec53ULL;
  k ^= k >> 33;
  return k;
}

// insert; returns 1 if newly inserted, 0 if present, -1 if the table is full
__device__ int hash_insert(uint64_t *tab, uint64_t mask, uint64_t key) {
  uint64_t h = mix64(key) & mask;
  for (uint64_t probe = 0; probe <= mask; ++probe) {
    unsigned long long cur =
        atomicCAS((unsigned long long *)&tab[h], (unsigned long long)EMPTY_SLOT,
                  (unsigned long long)key);
    if (cur == EMPTY_SLOT) return 1;
    if (cur == key) return 0;
    h = (h + 1) & mask;
  }
  return -1;
}

// reads through L2: the table is filled by atomics from every SM
__device__ bool hash_contains(const uint64_t *tab, uint64_t mask, uint64_t key) {
  uint64_t h = mix64(key) & mask;
  for (uint64_t probe = 0; probe <= mask; ++probe) {
    const uint64_t cur = __ldcg(&tab[h]);
    if (cur == key) return true;
    if (cur == EMPTY_SLOT) return false;
    h = (h + 1) & mask;
  }
  return false;
}

template <class T>
__device__ __forceinline__ int64_t lower_bound(const T *a, int64_t lo, int64_t hi, T v) {
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if (a[mid] < v)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

// --- 1. point keys -----------------------------------------------------------
// The reference locates a point by descending the tree: at each level it
// compares the point with the box midpoint xmin + w/2, computed level by
// level in FP64.  key_descent restates that descent digit by digit.
__device__ __forceinline__ uint64_t key_descent(double px, double py, double x0, double y0,
                                                double w0) {
  double xmin = x0, ymin = y0, w = w0;
  uint64_t key = 0;
#pragma unroll 1
  for (int l = 0; l < MAXD; ++l) {
    const double hw = 0.5 * w;
    const double xm = __dadd_rn(xmin, hw);
    const double ym = __dadd_rn(ymin, hw);
    const int hx = px > xm, hy = py > ym;
    key = (key << 2) | uint64_t(2 * hx + hy);
    xmin = hx ? xm : __dsub_rn(xm, hw);
    ymin = hy ? ym : __dsub_rn(ym, hw);
    w = hw;
  }
  return key;
}

// bits 0..28 of v to the even bit positions 0..56
__device__ __forceinline__ uint64_t spread_bits(uint64_t v) {
  v &= (uint64_t(1) << MAXD) - 1;
  v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
  v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
  v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
  v = (v | (v << 2)) & 0x3333333333333333ull;
  v = (v | (v << 1)) & 0x5555555555555555ull;
  return v;
}

// Every midpoint of the descent lies on a line x0 + k w0 / 2^MAXD, off by
// its accumulated FP64 rounding at most.  A point whose scaled coordinate
// q = (p - x0) 2^MAXD / w0 is farther than `margin` from every integer is on
// the same side of all of them as floor(q) says, so its digits are the bits
// of floor(q) (interleaved x, y); points within the margin (and NaN or
// infinite ones) take the descent itself.  The margin covers both roundings
// with a wide factor; the host sets it.
__device__ __forceinline__ uint64_t point_key(double px, double py, double x0, double y0,
                                               double w0, double scale, double margin) {
  const double qmax = double(uint64_t(1) << MAXD);
  const double qx = (px - x0) * scale, qy = (py - y0) * scale;
  const bool clear = fabs(qx - rint(qx)) > margin && fabs(qy - rint(qy)) > margin;
  if (!clear) return key_descent(px, py, x0, y0, w0);
  const double fx = fmin(fmax(floor(qx), 0.0), qmax - 1.0);
  const double fy = fmin(fmax(floor(qy), 0.0), qmax - 1.0);
  return (spread_bits(uint64_t(fx)) << 1) | spread_bits(uint64_t(fy));
}

// The top KEY32_DIGITS digits of the key as a 32-bit sort key: a sort on at
// most that many digits moves 8-byte pairs instead of 12-byte ones.
constexpr int KEY32_DIGITS = 16;

// Radix sort source of the point sort: the key of point i computed from its
// coordinates (its top KEY32_DIGITS digits for 32-bit sort keys), value i.
template <class K>
struct SrcPoints {
  const double *x, *y;
  double x0, y0, w0, scale, margin;
  __device__ K key(int i) const {
    const uint64_t k = point_key(__ldg(x + i), __ldg(y + i), x0, y0, w0, scale, margin);
    if constexpr (sizeof(K) == 8)
      return k;
    else
      return K(k >> (2 * (MAXD - KEY32_DIGITS)));
  }
  __device__ int val(int i) const { return int(i); }
};

// Radix sort emit of the point sort: the permutation (sorted -> input), the
// full 64-bit keys (computed again from the point for 32-bit sort keys) and,
// if sx is given, the coordinates in sorted order.
template <class K>
struct EmitPoints {
  struct Pre {
    double x, y;
  };
  const double *x, *y;
  double x0, y0, w0, scale, margin;
  uint64_t *keys;
  int *perm;
  double *sx, *sy;
  __device__ void init(int i) const { perm[i] = int(i); }
  __device__ Pre fetch(int v) const { return Pre{__ldg(x + v), __ldg(y + v)}; }
  __device__ void operator()(int pos, K k, int v, Pre q) const {
    perm[pos] = v;
    if (sx) {
      sx[pos] = q.x;
      sy[pos] = q.y;
    }
    if constexpr (sizeof(K) == 8)
      keys[pos] = k;
    else
      keys[pos] = point_key(q.x, q.y, x0, y0, w0, scale, margin);
  }
};

namespace {
// scale and margin of point_key for a tree box (x0, y0, w0)
void key_params(double x0, double y0, double w0, double &scale, double &margin) {
  scale = std::ldexp(1.0, MAXD) / w0;
  // A descent midpoint is off its line by at most two roundings per level,
  // each within half an ulp of the box's largest coordinate X: MAXD 2^-51 X,
  // i.e. 29 2^-22 X / w0 < 7e-6 X / w0 in units of q.  q itself is within
  // 3 2^-53 of its value relative, 2e-7 absolute.  2^-14 (6.1e-5) times
  // max(1, X / w0) covers both about 8 times over.
  const double big = std::fmax(std::fmax(std::fabs(x0), std::fabs(x0 + w0)),
                               std::fmax(std::fabs(y0), std::fabs(y0 + w0)));
  margin = std::ldexp(1.0, -14) * std::fmax(1.0, big / w0);
}
}  // namespace

// --- 3. initially split boxes ------------------------------------------------
// With keys sorted on their top `sorted_digits` digits, point i starts a box
// of every level in (cprev, cnext] that holds more than ppl points: the run
// from i is longer than ppl iff key i and key i+ppl share that prefix.
// Boxes of levels >= max_split stay leaves whatever their point count (the
// local evaluator's width floor, flexmm/local_tree.py:191-222).
__device__ __forceinline__ void split_range(const uint64_t *__restrict__ keys, int64_t n, int ppl,
                                            int64_t i, int &cprev, int &cnext, int max_split) {
  const uint64_t k = keys[i];
  cprev = (i == 0) ? -1 : common_digits(keys[i - 1], k);
  cnext = (i + ppl < n) ? common_digits(k, keys[i + ppl]) : -1;
  if (cnext >= max_split) cnext = max_split - 1;
}

// number of split boxes each point starts; flags trees too deep for the key
// or for the partial sort; deepest split level
__global__ void k_split_counts(const uint64_t *__restrict__ keys, int64_t n, int ppl,
                               int sorted_digits, unsigned long long *__restrict__ counts,
                               Counters *cnt, int max_split) {
  int lmax = -1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    int cprev, cnext;
    split_range(keys, n, ppl, i, cprev, cnext, max_split);
    unsigned long long c = 0;
    if (cnext > cprev) {
      if (cnext >= MAXD) {
        atomicExch(&cnt->too_deep, 1);
      } else if (sorted_digits < MAXD && cnext >= sorted_digits) {
        atomicExch(&cnt->need_full_sort, 1);
      } else {
        c = (unsigned long long)(cnext - cprev);
        lmax = max(lmax, cnext);
      }
    }
    counts[i] = c;
  }
  for (int o = 16; o >= 1; o >>= 1) lmax = max(lmax, __shfl_xor_sync(0xffffffffu, lmax, o));
  if ((threadIdx.x & 31) == 0 && lmax >= 0) atomicMax(&cnt->max_level, lmax);
}

// writes the split boxes at their scanned positions: point-major, so every
// level's boxes come out in increasing morton order
__global__ void k_split_emit(const uint64_t *__restrict__ keys, int64_t n, int ppl,
                             const unsigned long long *__restrict__ counts,
                             const unsigned long long *__restrict__ pos, uint64_t *__restrict__ out,
                             unsigned long long cap, Counters *cnt, int max_split,
                             const int *__restrict__ sort_fail) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (i == n - 1) {
      cnt->s0_count = pos[i] + counts[i];
      cnt->sort_fail = *sort_fail;  // the point sort and the scan ran before
    }
    if (!counts[i]) continue;
    int cprev, cnext;
    split_range(keys, n, ppl, i, cprev, cnext, max_split);
    const uint64_t k = keys[i];
    for (int m = cprev + 1; m <= cnext; ++m) {
      const unsigned long long p = pos[i] + (unsigned long long)(m - cprev - 1);
      if (p < cap)
        out[p] = box_code(m, k >> (2 * (MAXD - m)));
      else
        atomicExch(&cnt->overflow, 1);
    }
  }
}

// split-box count and level count of a tree from its split counters
// (n0 = 0: the root alone, one level)
__device__ __forceinline__ int64_t split_boxes(const Counters *split, unsigned long long cap) {
  return (int64_t)min(__ldcg(&split->s0_count), cap);
}
__device__ __forceinline__ int split_levels(const Counters *split, int64_t n0) {
  return n0 > 0 ? __ldcg(&split->max_level) + 2 : 1;
}

// bounds[l] = first index of a code of level >= l, l = 0..L + 1 (codes sorted
// by level; n and the tree's L from its split counters, bounds [MAXD + 3])
__global__ void k_level_starts(const uint64_t *__restrict__ codes, const Counters *split,
                               unsigned long long cap, int *__restrict__ bounds) {
  const int64_t n = split_boxes(split, cap);
  const int L = split_levels(split, n) + 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int lv = min(code_level(codes[i]), L + 1);
    const int prev = (i == 0) ? -1 : min(code_level(codes[i - 1]), L + 1);
    for (int l = prev + 1; l <= min(lv, L); ++l) bounds[l] = int(i);
    if (i == n - 1)
      for (int l = lv + 1; l <= L; ++l) bounds[l] = int(n);
  }
}

// --- 4-5. balance closure and X-list: one cooperative launch ------------------
// Grid-wide barrier for a cooperative launch.  Every wait is bounded: after
// BARRIER_TRIES polls the block flags bar_timeout and every block returns.
// The last block to arrive stores f_count to *snap (if given) before it
// releases the others.
constexpr unsigned int BARRIER_TRIES = 1u << 22;

__device__ bool grid_sync(Counters *cnt, unsigned long long *snap) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int g, old;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(g) : "l"(&cnt->bar_gen) : "memory");
    asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], 1;"
                 : "=r"(old) : "l"(&cnt->bar_count) : "memory");
    int good = 1;
    if (old == gridDim.x - 1) {
      // last to arrive: reset the count and take the snapshot, then release
      cnt->bar_count = 0u;
      if (snap) *snap = atomicAdd(&cnt->f_count, 0ull);
      asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&cnt->bar_gen), "r"(g + 1u) : "memory");
    } else {
      unsigned int tries = 0, cur = g;
      while (cur == g) {
        if (++tries > BARRIER_TRIES) {
          atomicExch(&cnt->bar_timeout, 1);
          good = 0;
          break;
        }
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(cur) : "l"(&cnt->bar_gen) : "memory");
      }
    }
    ok = good;
  }
  __syncthreads();
  return ok;
}

// 4: S_m gains every box neighbouring the parent of a box of S_{m+1}, for
//    m = mtop..1, with S = S0 (sorted, bounds s0b) plus the boxes forced so
//    far; forced[fb[m+1], fb[m]) are the boxes forced at level m+1.
// 5: X-list leaves: real leaves (parent split, self not split) next to a
//    split box.
// Boxes written by other blocks are read through L2 (__ldcg).
__global__ void __launch_bounds__(TPB) k_balance_xlist(
    const uint64_t *__restrict__ s0, const int *__restrict__ s0b,
    uint64_t *forced, unsigned long long *fb, unsigned long long capf, uint64_t *xl,
    unsigned long long capx, uint64_t *tab, uint64_t mask, Counters *cnt,
    const int *sort_fail, const Counters *split, unsigned long long cap0) {
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t nthr = (int64_t)gridDim.x * blockDim.x;
  // the split boxes' count and the tree's levels, from the split pass's
  // counters (the host has not read them: it waits once, after this kernel)
  const int64_t n0 = split_boxes(split, cap0);
  const int L = split_levels(split, n0), mtop = L - 3;
  if (tid == 0) cnt->sort_fail = __ldcg(sort_fail);  // the split-box sort ran before
  for (int64_t i = tid; i < n0; i += nthr)
    if (hash_insert(tab, mask, s0[i]) < 0) atomicExch(&cnt->overflow, 1);
  if (!grid_sync(cnt, nullptr)) return;
  for (int m = mtop; m >= 1; --m) {
    const int64_t a0 = s0b[m + 1], na = s0b[m + 2] - a0;
    const int64_t f0 = (int64_t)min(__ldcg(&fb[m + 1]), capf);
    const int64_t f1 = (int64_t)min(__ldcg(&fb[m]), capf);
    const int64_t work = 9 * (na + (f1 - f0));
    const int64_t side = int64_t(1) << m;
    for (int64_t w = tid; w < work; w += nthr) {
      const int64_t i = w / 9;
      const int d = int(w - 9 * i);
      const uint64_t c = (i < na) ? s0[a0 + i] : __ldcg(&forced[f0 + (i - na)]);
      uint32_t px, py;
      morton_xy(code_morton(c) >> 2, m, px, py);
      const int64_t qx = int64_t(px) + d / 3 - 1, qy = int64_t(py) + d % 3 - 1;
      if (qx < 0 || qy < 0 || qx >= side || qy >= side) continue;
      const uint64_t q = box_code(m, morton_of(uint32_t(qx), uint32_t(qy), m));
      const int r = hash_insert(tab, mask, q);
      if (r < 0) {
        atomicExch(&cnt->overflow, 1);
      } else if (r == 1) {
        const unsigned long long pos = atomicAdd(&cnt->f_count, 1ULL);
        if (pos < capf)
          forced[pos] = q;
        else
          atomicExch(&cnt->overflow, 1);
      }
    }
    if (!grid_sync(cnt, &fb[m - 1])) return;
  }
  const int64_t nf = (int64_t)min(__ldcg(&fb[0]), capf);
  const int64_t work = 8 * (n0 + nf);
  for (int64_t w = tid; w < work; w += nthr) {
    const int64_t i = w / 8;
    int d = int(w - 8 * i);
    d += (d >= 4);  // skip the centre of the 3x3 block
    const uint64_t c = (i < n0) ? s0[i] : __ldcg(&forced[i - n0]);
    const int m = code_level(c);
    if (m < 1 || m > L - 2) continue;
    uint32_t px, py;
    morton_xy(code_morton(c), m, px, py);
    const int64_t side = int64_t(1) << m;
    const int64_t qx = int64_t(px) + d / 3 - 1, qy = int64_t(py) + d % 3 - 1;
    if (qx < 0 || qy < 0 || qx >= side || qy >= side) continue;
    const uint64_t qm = morton_of(uint32_t(qx), uint32_t(qy), m);
    const uint64_t q = box_code(m, qm);
    if (hash_contains(tab, mask, q)) continue;                        // split: not a leaf
    if (!hash_contains(tab, mask, box_code(m - 1, qm >> 2))) continue;  // does not exist
    const int r = hash_insert(tab, mask, q | XLIST_TAG);
    if (r < 0) {
      atomicExch(&cnt->overflow, 1);
    } else if (r == 1) {
      const unsigned long long pos = atomicAdd(&cnt->x_count, 1ULL);
      if (pos < capx)
        xl[pos] = q;
      else
        atomicExch(&cnt->overflow, 1);
    }
  }
}

// --- 6. parent boxes ------------------------------------------------------------
// Parent boxes (split boxes, then X-list leaves) as compact sort keys:
// ((level << mb) | morton) << 1 | is_xlist, mb = 2 * (deepest parent level).
__global__ void k_parent_keys(const uint64_t *__restrict__ s0, int64_t n0,
                              const uint64_t *__restrict__ f, int64_t nf,
                              const uint64_t *__restrict__ xl, int64_t nx, int mb,
                              uint64_t *__restrict__ keys) {
  const int64_t total = n0 + nf + nx;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t c = (i < n0) ? s0[i] : (i < n0 + nf) ? f[i - n0] : xl[i - n0 - nf];
    const uint64_t v = (uint64_t(code_level(c)) << mb) | code_morton(c);
    keys[i] = (v << 1) | uint64_t(i >= n0 + nf);
  }
}

// sorted compact keys -> box codes, X-list flags, real flags (children of
// split boxes form real sibling groups) and level starts pb[0..L]
__global__ void k_parent_decode(const uint64_t *__restrict__ keys, int64_t n, int mb, int L,
                                uint64_t *__restrict__ codes, uint8_t *__restrict__ isx,
                                int *__restrict__ real, int *__restrict__ pb) {
  const uint64_t mmask = (uint64_t(1) << mb) - 1;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const uint64_t k = keys[i];
    const int x = int(k & 1);
    const int lv = int((k >> 1) >> mb);
    codes[i] = box_code(lv, (k >> 1) & mmask);
    isx[i] = uint8_t(x);
    real[i] = 1 - x;
    const int prev = (i == 0) ? -1 : int((keys[i - 1] >> 1) >> mb);
    for (int l = prev + 1; l <= min(lv, L); ++l) pb[l] = int(i);
    if (i == n - 1)
      for (int l = lv + 1; l <= L; ++l) pb[l] = int(n);
  }
}

// real sibling groups: the children of split boxes (not of X-list leaves)
// (rgb[L + 1]: the tree's sort failure flag, read back with the bounds;
// the last thread of the block writes the level offsets, as k_level_offsets)
__device__ __forceinline__ void level_offsets(const int *__restrict__ pb, int L, int *__restrict__ off) {
  off[0] = 0;
  if (L >= 1) off[1] = 1;
  for (int m = 1; m < L; ++m) off[m + 1] = off[m] + 4 * (pb[m] - pb[m - 1]);
}

__global__ void k_real_bounds(const int *__restrict__ pos, const int *__restrict__ real, int64_t n,
                              const int *__restrict__ pb, int L, int *__restrict__ rgb,
                              const int *__restrict__ sort_fail, int *__restrict__ off) {
  int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l == (int)blockDim.x - 1) level_offsets(pb, L, off);  // blockDim.x > L + 1
  if (l == L + 1) rgb[l] = *sort_fail;
  if (l > L) return;
  const int total = n ? pos[n - 1] + real[n - 1] : 0;
  rgb[l] = (pb[l] < n) ? pos[pb[l]] : total;
}

__global__ void k_real_groups(const uint64_t *__restrict__ pkeys, const int *__restrict__ real,
                              const int *__restrict__ pos, int64_t n, const int *__restrict__ pb,
                              const int *__restrict__ off, int *__restrict__ rg) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n;
       e += (int64_t)gridDim.x * blockDim.x) {
    if (!real[e]) continue;
    const int l = code_level(pkeys[e]);
    rg[pos[e]] = off[l + 1] + 4 * int(e - pb[l]);
  }
}

__device__ __forceinline__ int level_of(const int *__restrict__ off, int L, int g) {
  int lo = 0, hi = L;  // find largest l with off[l] <= g
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (off[mid] <= g)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// --- 6. node arrays -----------------------------------------------------------
// level offsets from the per-level parent-box bounds (one thread; a tree
// without split boxes, else k_real_bounds writes them)
__global__ void k_level_offsets(const int *__restrict__ pb, int L, int *__restrict__ off) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  level_offsets(pb, L, off);
}

// The node kernels are launched for an upper bound of the node count (the
// host does not wait for it); the count itself is off[L] in device memory.
__global__ void k_node_codes(const int *__restrict__ off, int L, int total_ub,
                             const uint64_t *__restrict__ pkeys, const uint8_t *__restrict__ pisx,
                             const int *__restrict__ pb, uint64_t *__restrict__ code,
                             uint8_t *__restrict__ flags) {
  const int total = min(off[L], total_ub);
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    const int m = level_of(off, L, g);
    if (m == 0) {
      code[g] = 0;
      flags[g] = 0;
      continue;
    }
    const int j = g - off[m];
    const int e = pb[m - 1] + (j >> 2);
    code[g] = (code_morton(pkeys[e]) << 2) | uint64_t(j & 3);
    flags[g] = pisx[e] ? NF_FAKE : 0;
  }
}

// Per node: 12 binary searches (8 colleagues, point range bot / top,
// parent, children), run as one branchless loop: a search over a range of n
// keys takes ceil(log2 n) steps whatever it looks for, so the searches of
// each step issue their loads together and the dependent chain is as long
// as the longest search (~20 loads for 1M points), not the sum of all.
constexpr int NA_SEARCH = 12;

__global__ void k_node_attrs(const int *__restrict__ off, int L, int total_ub, double x0, double y0,
                             double w0, const uint64_t *__restrict__ pts, int64_t npts,
                             const uint64_t *__restrict__ pkeys, const uint8_t *__restrict__ pisx,
                             const int *__restrict__ pb, const uint64_t *__restrict__ code,
                             uint8_t *__restrict__ flags, double *__restrict__ xmin,
                             double *__restrict__ ymin, double *__restrict__ xmid,
                             double *__restrict__ ymid, int *__restrict__ bot,
                             int *__restrict__ top, int *__restrict__ parent,
                             int *__restrict__ child, int *__restrict__ coll,
                             int *__restrict__ nix, int *__restrict__ niy) {
  const int total = min(off[L], total_ub);
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    const int m = level_of(off, L, g);
    const uint64_t c = code[g];
    uint32_t ix, iy;
    morton_xy(c, m, ix, iy);
    nix[g] = int(ix);
    niy[g] = int(iy);
    // searches: 0-7 colleagues (offsets (-1..1)^2 without the centre, in
    // offset order), 8 bot, 9 top, 10 parent, 11 children.  Every step of
    // every search is taken (a finished or empty one steps by 0 and reloads
    // a valid element), so each step's 12 loads issue together.
    auto arr = [&](int k) -> const uint64_t * {
      return (k == 8 || k == 9) ? pts : (k == 11 ? pkeys : code);
    };
    uint64_t val[NA_SEARCH];
    int base[NA_SEARCH], len[NA_SEARCH];
    const uint32_t side = 1u << m;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int d = k + (k >= 4);
      const int64_t qx = int64_t(ix) + d / 3 - 1, qy = int64_t(iy) + d % 3 - 1;
      const bool in = qx >= 0 && qy >= 0 && qx < side && qy < side;
      val[k] = in ? morton_of(uint32_t(qx), uint32_t(qy), m) : 0;
      base[k] = off[m];  // level m holds this node: a valid index
      len[k] = in ? off[m + 1] - off[m] : 0;
    }
    const int sh = 2 * (MAXD - m);
    val[8] = c << sh, base[8] = 0, len[8] = int(npts);
    val[9] = (c + 1) << sh, base[9] = 0, len[9] = int(npts);
    val[10] = c >> 2, base[10] = m > 0 ? off[m - 1] : 0, len[10] = m > 0 ? off[m] - off[m - 1] : 0;
    const bool has_pb = m < L - 1 && pb[m + 1] > pb[m];
    val[11] = box_code(m, c), base[11] = has_pb ? pb[m] : 0;  // pkeys[0] exists
    len[11] = has_pb ? pb[m + 1] - pb[m] : 0;
    // bot / top (k = 8, 9) want the lower bound: the last element below the
    // key moves the window; the others look the key itself up: the last
    // element not above it does, and the window ends on the key if present
    auto lower = [](int k) { return k == 8 || k == 9; };
    for (bool more = true; more;) {
      uint64_t a[NA_SEARCH];
#pragma unroll
      for (int k = 0; k < NA_SEARCH; ++k) a[k] = __ldg(arr(k) + base[k] + (len[k] >> 1));
      more = false;
#pragma unroll
      for (int k = 0; k < NA_SEARCH; ++k) {
        const int half = len[k] >> 1;
        base[k] += (lower(k) ? a[k] < val[k] : a[k] <= val[k]) ? half : 0;
        len[k] -= half;
        more |= len[k] > 1;
      }
    }
    int lb[NA_SEARCH];  // lower bound (k = 8, 9) or the key's index (others, if eq)
    bool eq[NA_SEARCH];
#pragma unroll
    for (int k = 0; k < NA_SEARCH; ++k) {
      const uint64_t v = __ldg(arr(k) + base[k]);
      lb[k] = base[k] + (lower(k) && len[k] == 1 && v < val[k] ? 1 : 0);
      eq[k] = len[k] == 1 && v == val[k];
    }
    bot[g] = lb[8];
    top[g] = lb[9];
    parent[g] = m == 0 ? -1 : lb[10];
    // children: is this box a parent box?
    uint8_t f = flags[g];
    int ch = -1;
    if (eq[11]) {
      ch = off[m + 1] + 4 * (lb[11] - pb[m]);
      f |= NF_CHILDREN;
      if (pisx[lb[11]]) f |= NF_XLIST;
    }
    if (!(f & NF_FAKE) && (ch < 0 || (f & NF_XLIST))) f |= NF_LEAF;
    flags[g] = f;
    child[g] = ch;
    // colleagues: existing same-level boxes at offsets (-1..1)^2, self
    // included, first in offset order, then -1
    int kc = 0;
#pragma unroll
    for (int d = 0; d < 9; ++d) {
      int found;
      if (d == 4) {
        found = g;
      } else {
        const int k = d - (d > 4);
        found = eq[k] ? lb[k] : -1;
      }
      if (found >= 0) coll[int64_t(g) * 9 + (kc++)] = found;
    }
    for (; kc < 9; ++kc) coll[int64_t(g) * 9 + kc] = -1;
    // geometry: replay the descent along the node's digits (bit-exact with the reference)
    double xm0 = x0, ym0 = y0, w = w0;
    for (int l = 0; l < m; ++l) {
      const int d = int((c >> (2 * (m - 1 - l))) & 3u);
      const double hw = 0.5 * w;
      const double xm = __dadd_rn(xm0, hw), ym = __dadd_rn(ym0, hw);
      xm0 = (d >> 1) ? xm : __dsub_rn(xm, hw);
      ym0 = (d & 1) ? ym : __dsub_rn(ym, hw);
      w = hw;
    }
    const double hw = 0.5 * w;
    xmin[g] = xm0;
    ymin[g] = ym0;
    xmid[g] = __dadd_rn(xm0, hw);
    ymid[g] = __dadd_rn(ym0, hw);
  }
}

// offset id (0..39) of a 7x7 cell (ox+3)*7 + (oy+3); -1 for the (-1..1)^2 centre
__constant__ int8_t c_cell_to_offset[49] = {
    0,  1,  2,  3,  4,  5,  6,  7,  8,  9,  10, 11, 12, 13, 14, 15, -1,
    -1, -1, 16, 17, 18, 19, -1, -1, -1, 20, 21, 22, 23, -1, -1, -1, 24,
    25, 26, 27, 28, 29, 30, 31, 32, 33, 34, 35, 36, 37, 38, 39};

// far-field interaction lists of real nodes at levels >= 2: the children of
// the parent's colleagues (parent excluded) that are not adjacent
// (build_interaction_list, flexmm/tree.py:399-435), keeping only sources
// that hold points
__global__ void k_interactions(const int *__restrict__ off, int L, int total_ub,
                               const uint8_t *__restrict__ flags, const int *__restrict__ parent,
                               const int *__restrict__ child, const int *__restrict__ coll,
                               const int *__restrict__ ix, const int *__restrict__ iy,
                               const int *__restrict__ bot, const int *__restrict__ top,
                               int *__restrict__ il) {
  // 8 lanes per node: lane j takes the parent's colleague j (and 8), with
  // its four children
  const int total = min(off[L], total_ub);
  const int sub = threadIdx.x & 7;
  const unsigned gmask = 0xffu << (threadIdx.x & 24);
  const int64_t stride = (int64_t)gridDim.x * blockDim.x / 8;
  for (int64_t gg = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 8; gg < total;
       gg += stride) {
    const int g = int(gg);
    int *row = il + int64_t(g) * N_OFFSETS;
    for (int o = sub; o < N_OFFSETS; o += 8) row[o] = -1;
    if (g < off[min(2, L)] || (flags[g] & NF_FAKE)) continue;  // the same for the whole group
    __syncwarp(gmask);  // the -1 row before the entries
    const int P = parent[g];
    const int tx = ix[g], ty = iy[g];
    for (int j = sub; j < 9; j += 8) {
      const int c = coll[int64_t(P) * 9 + j];
      if (c < 0 || c == P) continue;
      const int ch = child[c];
      if (ch < 0) continue;
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int cc = ch + k;
        const int ox = ix[cc] - tx, oy = iy[cc] - ty;
        if (ox < -3 || ox > 3 || oy < -3 || oy > 3) continue;
        const int o = c_cell_to_offset[(ox + 3) * 7 + (oy + 3)];
        if (o >= 0 && top[cc] > bot[cc]) row[o] = cc;  // distinct boxes: distinct offsets
      }
    }
  }
}

// S2M nodes: see TreeDev::uplist
__global__ void k_up_flags(const int *__restrict__ off, int L, int total_ub,
                           const uint8_t *__restrict__ flags, const int *__restrict__ bot,
                           const int *__restrict__ top, int *__restrict__ f) {
  const int total = min(off[L], total_ub);
  const int g0 = L > 2 ? off[2] : total;
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total_ub; g += gridDim.x * blockDim.x) {
    if (g >= total) {
      f[g] = 0;
      continue;
    }
    const uint8_t fl = flags[g];
    const bool up = (((fl & NF_LEAF) && !(fl & NF_XLIST)) || (fl & NF_FAKE)) && top[g] > bot[g];
    f[g] = (g >= g0 && up) ? 1 : 0;
  }
}

__global__ void k_up_scatter(const int *__restrict__ off, int L, int total_ub,
                             const int *__restrict__ f, const int *__restrict__ pos,
                             int *__restrict__ list, int *__restrict__ count) {
  const int total = min(off[L], total_ub);
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    if (f[g]) list[pos[g]] = g;
    if (g == total - 1) *count = pos[g] + f[g];
  }
}

uint64_t next_pow2(uint64_t v) {
  uint64_t p = 1;
  while (p < v) p <<= 1;
  return p;
}

// stable sort of keys on bits [begin_bit, end_bit)
template <class K>
void sort_keys(const K *kin, K *kout, int64_t n, int begin_bit, int end_bit, int *fail,
               cudaStream_t s, const unsigned long long *n_dev = nullptr) {
  radix_sort<K, false>(SrcKeys<K>{kin, nullptr}, EmitPairs<K>{kout, nullptr}, n, begin_bit, end_bit,
                       fail, s, n_dev);
}

template <class T>
void exclusive_sum(const T *in, T *out, int64_t n, int *fail, bool offsets, cudaStream_t s) {
  prefix_sum<T, false>(in, out, n, fail, offsets, s);
}

// blocks of a cooperative launch: all co-resident, one per SM (the grid
// barriers' cost grows with the block count; the per-level work is small)
int cooperative_grid(const void *kernel, int threads) {
  int dev = 0, coop = 0, sms = 0, per = 0;
  FMMB_CUDA(cudaGetDevice(&dev));
  FMMB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  FMMB_CHECK(coop, ERR_UNSUPPORTED, "the device does not support cooperative launches");
  FMMB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  FMMB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, threads, 0));
  FMMB_CHECK(per >= 1, ERR_CUDA, "cooperative kernel does not fit on an SM");
  return sms;
}

}  // namespace

// Small pinned host blocks for the per-level counts, kept for reuse: pinned
// allocation is slow, and a plan is built per step in many loops.
namespace {
constexpr int PINNED_INTS = 64;  // >= 2 (MAXD + 2) + 1
std::mutex g_pinned_mu;
std::vector<int *> g_pinned_free;

int *pinned_acquire() {
  {
    std::lock_guard<std::mutex> g(g_pinned_mu);
    if (!g_pinned_free.empty()) {
      int *p = g_pinned_free.back();
      g_pinned_free.pop_back();
      return p;
    }
  }
  // pinned allocation can take milliseconds: 16 blocks at a time (never freed)
  constexpr int CHUNK = 16;
  int *p = nullptr;
  FMMB_CUDA(cudaHostAlloc((void **)&p, CHUNK * PINNED_INTS * sizeof(int), cudaHostAllocDefault));
  std::lock_guard<std::mutex> g(g_pinned_mu);
  for (int i = 1; i < CHUNK; ++i) g_pinned_free.push_back(p + i * PINNED_INTS);
  return p;
}

void pinned_release(int *p) {
  if (!p) return;
  std::lock_guard<std::mutex> g(g_pinned_mu);
  g_pinned_free.push_back(p);
}

// the counts and, after them (dev_counts[count]), the tree's sort failure flag
void begin_pending_counts(TreeHost &th, const int *dev_counts, int count, cudaStream_t s) {
  FMMB_CHECK(count + 1 <= PINNED_INTS, ERR_INVALID_ARGUMENT, "too many levels");
  if (!th.pending_counts) th.pending_counts = pinned_acquire();
  if (!th.ready) FMMB_CUDA(cudaEventCreateWithFlags(&th.ready, cudaEventDisableTiming));
  FMMB_CUDA(cudaMemcpyAsync(th.pending_counts, dev_counts, (count + 1) * sizeof(int),
                            cudaMemcpyDeviceToHost, s));
  FMMB_CUDA(cudaEventRecord(th.ready, s));
  th.pending = true;
  th.off.clear();
  th.rg_lo.clear();
  th.rg_hi.clear();
}
}  // namespace

void finalize_tree(TreeHost &th) {
  if (!th.pending) return;
  FMMB_CUDA(cudaEventSynchronize(th.ready));
  const int L = th.L;
  const int *hpb = th.pending_counts;  // [0, L]: parent-box bounds; [L+1, 2L+1]: real groups
  // (stays pending: every later use reports the failure again)
  FMMB_CHECK(!hpb[2 * (L + 1)], ERR_CUDA, "tree sort: a grid barrier wait ran out of time");
  th.off.assign(L + 1, 0);
  if (L >= 1) th.off[1] = 1;
  for (int m = 1; m < L; ++m) th.off[m + 1] = th.off[m] + 4 * (hpb[m] - hpb[m - 1]);
  th.rg_lo.assign(L + 1, 0);
  th.rg_hi.assign(L + 1, 0);
  for (int m = 1; m < L; ++m) {
    th.rg_lo[m] = hpb[L + 1 + m - 1];
    th.rg_hi[m] = hpb[L + 1 + m];
  }
  th.pending = false;
}

TreeHost::~TreeHost() {
  // a copy still in flight writes into the pinned block: let it land first
  if (pending && ready) cudaEventSynchronize(ready);
  if (ready) cudaEventDestroy(ready);
  pinned_release(pending_counts);
}

namespace {
int clamp_digits(int d) { return d < 1 ? 1 : (d > MAXD ? MAXD : d); }

template <class K>
using PointSortKernel = decltype(&k_radix_sort<K, SrcPoints<K>, EmitPoints<K>, true>);

template <class K>
PointSortKernel<K> point_sort_kernel() {
  return &k_radix_sort<K, SrcPoints<K>, EmitPoints<K>, true>;
}

// bit range of the sort keys for `digits` top digits
void point_sort_bits(int digits, int &begin_bit, int &end_bit) {
  if (digits <= KEY32_DIGITS) {
    begin_bit = 2 * (KEY32_DIGITS - digits);
    end_bit = 2 * KEY32_DIGITS;
  } else {
    begin_bit = 2 * (MAXD - digits);
    end_bit = 2 * MAXD;
  }
}

template <class K>
size_t point_sort_bytes(int64_t n, int digits) {
  int b0, b1;
  point_sort_bits(digits, b0, b1);
  return radix_scratch_bytes<K, true>(n, (b1 - b0 + 7) / 8);
}

template <class K>
void point_sort_run(const double *x, const double *y, int64_t n, const TreeHost &th, int digits,
                    uint64_t *keys, int *perm, double *sx, double *sy, void *scratch,
                    size_t bytes, int *fail, cudaStream_t s) {
  double scale, margin;
  key_params(th.x0, th.y0, th.w0, scale, margin);
  int b0, b1;
  point_sort_bits(digits, b0, b1);
  const SrcPoints<K> src{x, y, th.x0, th.y0, th.w0, scale, margin};
  const EmitPoints<K> emit{x, y, th.x0, th.y0, th.w0, scale, margin, keys, perm, sx, sy};
  radix_sort_run<K, true>(src, emit, n, b0, b1, scratch, bytes,
                          radix_grid<K, true>(point_sort_kernel<K>(), n), fail, s);
}
}  // namespace

size_t sort_points_scratch_bytes(int64_t n, int sorted_digits) {
  if (n <= 0) return 0;
  const int digits = clamp_digits(sorted_digits);
  return digits <= KEY32_DIGITS ? point_sort_bytes<uint32_t>(n, digits)
                                : point_sort_bytes<uint64_t>(n, digits);
}

void sort_points_scratch(const double *x, const double *y, int64_t n, const TreeHost &th,
                         int sorted_digits, uint64_t *keys, int *perm, double *sx, double *sy,
                         void *scratch, size_t scratch_bytes, int *fail, cudaStream_t s) {
  if (n <= 0) return;
  const int digits = clamp_digits(sorted_digits);
  if (digits <= KEY32_DIGITS)
    point_sort_run<uint32_t>(x, y, n, th, digits, keys, perm, sx, sy, scratch, scratch_bytes, fail,
                             s);
  else
    point_sort_run<uint64_t>(x, y, n, th, digits, keys, perm, sx, sy, scratch, scratch_bytes, fail,
                             s);
}

void sort_points(const double *x, const double *y, int64_t n, const TreeHost &th,
                 DevBuf<uint64_t> &keys, DevBuf<int> &perm, cudaStream_t s, int sorted_digits,
                 double *sx, double *sy, int *fail) {
  keys.alloc(n, s);
  perm.alloc(n, s);
  if (n == 0) return;
  const size_t bytes = sort_points_scratch_bytes(n, sorted_digits);
  DevBuf<unsigned char> tmp;
  tmp.alloc(bytes, s);
  sort_points_scratch(x, y, n, th, sorted_digits, keys.get(), perm.get(), sx, sy, tmp.get(), bytes,
                      fail, s);
}

// --- targets into leaves without a sort ---------------------------------------
// Each point's key digits lead from the root down the tree to the first real
// leaf (NF_LEAF, X-list leaves included): the leaf whose code is a prefix of
// the key, the same leaf a lower-bound search of the sorted keys finds.  Its
// slot inside the leaf is taken by an atomic count per leaf and warp (any
// order).
__global__ void k_bin_points(const double *__restrict__ x, const double *__restrict__ y, int64_t m,
                             double x0, double y0, double w0, double scale, double margin, int L,
                             const uint8_t *__restrict__ flags, const int *__restrict__ child,
                             int *__restrict__ leaf_of, int *__restrict__ slot,
                             int *__restrict__ count) {
  const int lane = threadIdx.x & 31;
  unsigned lt;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(lt));
  // whole warps step together (the slot count below is per warp)
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i0 = blockIdx.x * (int64_t)blockDim.x + (threadIdx.x & ~31); i0 < m; i0 += stride) {
    const int64_t i = i0 + lane;
    int g = -2;  // past m
    if (i < m) {
      const uint64_t key = point_key(__ldg(x + i), __ldg(y + i), x0, y0, w0, scale, margin);
      g = 0;
      for (int l = 0;; ++l) {
        const uint8_t f = __ldg(flags + g);
        if (f & NF_LEAF) break;
        if (!(f & NF_CHILDREN) || l >= L - 1) {  // (never in a built tree)
          g = -1;
          break;
        }
        g = __ldg(child + g) + int((key >> (2 * (MAXD - 1 - l))) & 3u);
      }
    }
    // one atomic per leaf met by the warp (neighbouring points share leaves)
    const unsigned peers = __match_any_sync(0xffffffffu, g);
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (lane == leader && g >= 0) base = atomicAdd(count + g, __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (i < m) {
      leaf_of[i] = g;
      slot[i] = g >= 0 ? base + __popc(peers & lt) : -1;
    }
  }
}

__global__ void k_scatter_binned(const double *__restrict__ x, const double *__restrict__ y,
                                 int64_t m, const int *__restrict__ leaf_of,
                                 const int *__restrict__ slot, const int *__restrict__ first,
                                 double *__restrict__ xs, double *__restrict__ ys,
                                 int *__restrict__ perm) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int g = leaf_of[i];
    if (g < 0) continue;
    const int pos = first[g] + slot[i];
    xs[pos] = x[i];
    ys[pos] = y[i];
    perm[pos] = int(i);
  }
}

void bin_points(const double *x, const double *y, int64_t m, const TreeDev &td, const TreeHost &th,
                int *count, int *leaf_of, int *slot, cudaStream_t s) {
  if (m <= 0) return;
  double scale, margin;
  key_params(th.x0, th.y0, th.w0, scale, margin);
  k_bin_points<<<grid_for(m, TPB), TPB, 0, s>>>(x, y, m, th.x0, th.y0, th.w0, scale, margin, th.L,
                                                td.flags.get(), td.child.get(), leaf_of, slot, count);
  FMMB_CUDA(cudaGetLastError());
}

void scatter_binned(const double *x, const double *y, int64_t m, const int *leaf_of,
                    const int *slot, const int *first, double *xs, double *ys, int *perm,
                    cudaStream_t s) {
  if (m <= 0) return;
  k_scatter_binned<<<grid_for(m, TPB), TPB, 0, s>>>(x, y, m, leaf_of, slot, first, xs, ys, perm);
  FMMB_CUDA(cudaGetLastError());
}

void build_tree(TreeDev &td, TreeHost &th, const double *x, const double *y, int64_t n, int ppl,
                const double bbox[4], cudaStream_t s, int max_split) {
  FMMB_CHECK(n > 0, ERR_INVALID_ARGUMENT, "tree needs at least one point");
  FMMB_CHECK(ppl >= 1, ERR_INVALID_ARGUMENT, "Ncutoff must be >= 1");
  FMMB_CHECK(n < (int64_t(1) << 31) - 1, ERR_INVALID_ARGUMENT, "more than 2^31-2 points");
  th.n_points = n;
  th.ppl = ppl;
  th.x0 = bbox[0];
  th.y0 = bbox[2];
  th.w0 = bbox[1] - bbox[0];
  FMMB_CHECK(th.w0 > 0, ERR_INVALID_ARGUMENT, "bbox has non-positive width");

  // counters: [0] the split pass's (box count, deepest level, flags), [1] the
  // balance kernel's; both come back through a pinned block in one copy, at
  // the tree build's one host wait (after the balance kernel: the level sort
  // and the balance kernel read the split counts on the device)
  DevBuf<Counters> cnt;
  cnt.alloc(2, s);
  Counters *csplit = cnt.get(), *cbal = cnt.get() + 1;
  static_assert(2 * sizeof(Counters) <= PINNED_INTS * sizeof(int), "pinned block too small");
  std::unique_ptr<int, void (*)(int *)> hblk(pinned_acquire(), pinned_release);
  Counters *hcs = reinterpret_cast<Counters *>(hblk.get());
  const Counters &hc = hcs[0], &hb = hcs[1];
  auto read_counters = [&] {
    FMMB_CUDA(cudaMemcpyAsync(hcs, cnt.get(), 2 * sizeof(Counters), cudaMemcpyDeviceToHost, s));
    FMMB_CUDA(cudaStreamSynchronize(s));
  };
  const unsigned long long cap0 = (unsigned long long)MAXD * (n / (ppl + 1) + 1) + 64;
  DevBuf<uint64_t> s0raw, s0;
  DevBuf<unsigned long long> scount, spos;
  s0raw.alloc(cap0, s);
  s0.alloc(cap0, s);
  scount.alloc(n, s);
  spos.alloc(n, s);
  DevBuf<int> s0b;            // split boxes' level starts
  s0b.alloc(MAXD + 3, s);
  // balance buffers: first sized from an estimate of the split-box count
  // (the true one is known only after the wait); an overflow is retried
  // with capacities from the true count
  const unsigned long long n0_est = 2ull * (unsigned long long)(n / (ppl + 1)) + 64;
  unsigned long long capf = 8ull * n0_est + 4096, capx = 8ull * n0_est + 4096;
  DevBuf<uint64_t> tab, forced, xl;
  DevBuf<unsigned long long> fb;
  uint64_t hcap = 0;
  auto launch_balance = [&] {
    hcap = next_pow2(2 * (n0_est + capf + capx));
    tab.alloc(hcap, s);
    FMMB_CUDA(cudaMemsetAsync(tab.get(), 0xff, hcap * sizeof(uint64_t), s));
    forced.alloc(capf, s);
    xl.alloc(capx, s);
    fb.alloc(MAXD + 2, s);
    fb.zero(s);
    FMMB_CUDA(cudaMemsetAsync(cbal, 0, sizeof(Counters), s));
    const uint64_t *s0p = s0.get();
    const int *s0bp = s0b.get();
    uint64_t *fp = forced.get(), *xp = xl.get(), *tp = tab.get();
    unsigned long long *fbp = fb.get();
    uint64_t mask = hcap - 1;
    Counters *cp = cbal;
    const Counters *sp = csplit;
    const int *sfp = td.sort_fail.get();
    unsigned long long c0 = cap0;
    void *args[] = {&s0p, &s0bp, &fp, &fbp, &capf, &xp, &capx, &tp, &mask, &cp, &sfp, &sp, &c0};
    FMMB_CUDA(cudaLaunchCooperativeKernel((const void *)k_balance_xlist,
                                          cooperative_grid((const void *)k_balance_xlist, TPB), TPB,
                                          args, 0, s));
  };
  // 1-5: keys, sort (top digits first), initial splits in point order, the
  // split boxes by (level, morton) -- a stable sort on the level bits keeps
  // the morton order every level already has -- and the balance closure
  // with the X-list in one cooperative launch over a hash set
  std::unique_ptr<PhaseTimer> t_split(new PhaseTimer(PH_TREE_SPLITS, s));
  std::unique_ptr<PhaseTimer> t_bal;
  td.sx.alloc(n, s);
  td.sy.alloc(n, s);
  td.sort_fail.alloc(1, s);
  td.sort_fail.zero(s);
  for (int digits = SORT_DIGITS;; digits = MAXD) {
    sort_points(x, y, n, th, td.pkeys, td.ordv, s, digits, td.sx.get(), td.sy.get(),
                td.sort_fail.get());
    FMMB_CUDA(cudaMemsetAsync(csplit, 0, sizeof(Counters), s));
    k_split_counts<<<grid_for(n, TPB), TPB, 0, s>>>(td.pkeys.get(), n, ppl, digits, scount.get(),
                                                     csplit, max_split);
    FMMB_CUDA(cudaGetLastError());
    // (k_split_emit checks its writes against the capacity)
    exclusive_sum(scount.get(), spos.get(), n, td.sort_fail.get(), false, s);
    k_split_emit<<<grid_for(n, TPB), TPB, 0, s>>>(td.pkeys.get(), n, ppl, scount.get(), spos.get(),
                                                   s0raw.get(), cap0, csplit, max_split,
                                                   td.sort_fail.get());
    FMMB_CUDA(cudaGetLastError());
    t_split.reset();
    t_bal.reset(new PhaseTimer(PH_TREE_BALANCE, s));
    sort_keys(s0raw.get(), s0.get(), (int64_t)cap0, LEVEL_SHIFT, LEVEL_SHIFT + 5,
              td.sort_fail.get(), s, &csplit->s0_count);
    k_level_starts<<<grid_for((int64_t)cap0, TPB), TPB, 0, s>>>(s0.get(), csplit, cap0, s0b.get());
    FMMB_CUDA(cudaGetLastError());
    launch_balance();
    read_counters();
    FMMB_CHECK(!hc.sort_fail, ERR_CUDA, "point sort: a grid barrier wait ran out of time");
    FMMB_CHECK(!hc.too_deep, ERR_TREE_TOO_DEEP,
               "more than Ncutoff points share a box of width bbox/2^29 (coincident points?)");
    FMMB_CHECK(!hc.overflow, ERR_CAPACITY, "initial split buffer overflow");
    if (!hc.need_full_sort || digits == MAXD) break;
    t_bal.reset();
    t_split.reset(new PhaseTimer(PH_TREE_SPLITS, s));
  }
  scount.release();
  spos.release();
  const int64_t n0 = (int64_t)hc.s0_count;
  const int L = (n0 > 0) ? hc.max_level + 2 : 1;
  th.L = L;

  DevBuf<uint64_t> pk, pkc, pks;  // parent boxes: compact keys (unsorted, sorted), codes
  DevBuf<uint8_t> pxs;
  DevBuf<int> pb, preal, ppos;
  int64_t np = 0;
  const int mb = 2 * (L - 2);  // morton bits of the deepest parent level
  if (n0 > 0) {
    for (int attempt = 0;; ++attempt) {
      FMMB_CHECK(!hb.bar_timeout, ERR_CUDA, "tree balance: a grid barrier wait ran out of time");
      FMMB_CHECK(!hb.sort_fail, ERR_CUDA, "split-box sort: a grid barrier wait ran out of time");
      if (!hb.overflow) break;
      // capacities grow on overflow (from the true split-box count now)
      FMMB_CHECK(attempt < 6, ERR_CAPACITY, "tree balance buffers overflow");
      capf = std::max(4 * capf, 8ull * n0 + 4096);
      capx = std::max(4 * capx, 8ull * n0 + 4096);
      launch_balance();
      read_counters();
    }
    const int64_t nf = (int64_t)hb.f_count, nx = (int64_t)hb.x_count;
    np = n0 + nf + nx;
    pk.alloc(np, s);
    k_parent_keys<<<grid_for(np, TPB), TPB, 0, s>>>(s0.get(), n0, forced.get(), nf, xl.get(), nx,
                                                     mb, pk.get());
    FMMB_CUDA(cudaGetLastError());
    // 6: sorted parent boxes, per-level bounds, real sibling groups
    t_bal.reset();
    pkc.alloc(np, s);
    sort_keys(pk.get(), pkc.get(), np, 0, 1 + mb + 5, td.sort_fail.get(), s);
    pks.alloc(np, s);
    pxs.alloc(np, s);
    preal.alloc(np, s);
    ppos.alloc(np, s);
    // pb[0..L], the real-group bounds rgb[0..L] and the sort failure flag
    // share one buffer: one copy back
    pb.alloc(2 * (L + 1) + 1, s);
    k_parent_decode<<<grid_for(np, TPB), TPB, 0, s>>>(pkc.get(), np, mb, L, pks.get(), pxs.get(),
                                                       preal.get(), pb.get());
    FMMB_CUDA(cudaGetLastError());
    exclusive_sum(preal.get(), ppos.get(), np, td.sort_fail.get(), true, s);
    td.dev_off.alloc(L + 1, s);
    k_real_bounds<<<1, 64, 0, s>>>(ppos.get(), preal.get(), np, pb.get(), L, pb.get() + L + 1,
                                   td.sort_fail.get(), td.dev_off.get());
    FMMB_CUDA(cudaGetLastError());
  } else {
    pb.alloc(2 * (L + 1) + 1, s);
    pb.zero(s);
    pks.alloc(1, s);
    pxs.alloc(1, s);
  }

  t_bal.reset();
  PhaseTimer t_nodes(PH_TREE_NODES, s);
  th.width.assign(L, 0.0);
  double w = th.w0;
  for (int m = 0; m < L; ++m) {
    th.width[m] = w;
    w = 0.5 * w;
  }
  // level offsets on the device; their host copy (with the real-group
  // bounds) travels back without a wait (finalize_tree)
  if (n0 == 0) {  // (otherwise k_real_bounds wrote them)
    td.dev_off.alloc(L + 1, s);
    k_level_offsets<<<1, 1, 0, s>>>(pb.get(), L, td.dev_off.get());
    FMMB_CUDA(cudaGetLastError());
  }
  begin_pending_counts(th, pb.get(), 2 * (L + 1), s);
  // every parent box has 4 children: at most 1 + 4 np nodes, np real groups
  const int total_ub = 1 + 4 * int(np);
  td.rg.alloc(np > 0 ? np : 1, s);
  if (np > 0) {
    k_real_groups<<<grid_for(np, TPB), TPB, 0, s>>>(pks.get(), preal.get(), ppos.get(), np, pb.get(),
                                                     td.dev_off.get(), td.rg.get());
    FMMB_CUDA(cudaGetLastError());
  }
  td.code.alloc(total_ub, s);
  td.flags.alloc(total_ub, s);
  td.xmin.alloc(total_ub, s);
  td.ymin.alloc(total_ub, s);
  td.xmid.alloc(total_ub, s);
  td.ymid.alloc(total_ub, s);
  td.bot.alloc(total_ub, s);
  td.top.alloc(total_ub, s);
  td.parent.alloc(total_ub, s);
  td.child.alloc(total_ub, s);
  td.coll.alloc(int64_t(total_ub) * 9, s);
  td.il.alloc(int64_t(total_ub) * N_OFFSETS, s);
  td.ix.alloc(total_ub, s);
  td.iy.alloc(total_ub, s);
  k_node_codes<<<grid_for(total_ub, TPB), TPB, 0, s>>>(td.dev_off.get(), L, total_ub, pks.get(),
                                                         pxs.get(), pb.get(), td.code.get(),
                                                         td.flags.get());
  FMMB_CUDA(cudaGetLastError());
  k_node_attrs<<<grid_for(total_ub, TPB), TPB, 0, s>>>(
      td.dev_off.get(), L, total_ub, th.x0, th.y0, th.w0, td.pkeys.get(), n, pks.get(), pxs.get(),
      pb.get(), td.code.get(), td.flags.get(), td.xmin.get(), td.ymin.get(), td.xmid.get(),
      td.ymid.get(), td.bot.get(), td.top.get(), td.parent.get(), td.child.get(), td.coll.get(),
      td.ix.get(), td.iy.get());
  FMMB_CUDA(cudaGetLastError());
  k_interactions<<<grid_for(int64_t(total_ub) * 8, TPB), TPB, 0, s>>>(
      td.dev_off.get(), L, total_ub, td.flags.get(), td.parent.get(), td.child.get(), td.coll.get(),
      td.ix.get(), td.iy.get(), td.bot.get(), td.top.get(), td.il.get());
  FMMB_CUDA(cudaGetLastError());
  // S2M node list
  {
    DevBuf<int> f, pos;
    f.alloc(total_ub, s);
    pos.alloc(total_ub, s);
    td.uplist.alloc(total_ub, s);
    td.n_up.alloc(1, s);
    k_up_flags<<<grid_for(total_ub, TPB), TPB, 0, s>>>(td.dev_off.get(), L, total_ub,
                                                         td.flags.get(), td.bot.get(), td.top.get(),
                                                         f.get());
    FMMB_CUDA(cudaGetLastError());
    exclusive_sum(f.get(), pos.get(), total_ub, td.sort_fail.get(), true, s);
    k_up_scatter<<<grid_for(total_ub, TPB), TPB, 0, s>>>(td.dev_off.get(), L, total_ub, f.get(),
                                                           pos.get(), td.uplist.get(),
                                                           td.n_up.get());
    FMMB_CUDA(cudaGetLastError());
  }
}

}  // namespace fmmb
