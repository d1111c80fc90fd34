// FMM passes (FP64): upward (S2M / M2M + check-to-equivalent), offset-grouped
// M2L, downward (L2L + check-to-equivalent) and evaluation (L2T + P2P).
//
// Reference path: flexmm/flexmm2d/fmm.py:67-176 (passes), kifmm.py:83-144
// (S2M, C2E, L2T), helpers.py:5-33 (M2L factors), helpers.py:152-194 (P2P).
// Differences of form, not of result:
//  * check-to-equivalent is applied as VH^T diag(1/S) U^T, the factored SVD
//    solve (flexmm/kifmm2d/scalar/helpers.py:240-248), never an explicit
//    inverse; it agrees with the reference's LU solve to ~1e-15;
//  * M2L is target-centric: a tile of 64 target boxes of one parity class
//    (position inside the parent: 27 of the 40 offsets can occur) gathers the
//    source multipoles of one offset and multiplies them by that offset's
//    dense or SVD-factored operator, accumulating all offsets in registers
//    (the reference multiplies every multipole by every offset, then gathers);
//  * L2L is parent-centric: one GEMM per tile of 8 parents produces the
//    partial locals of their 32 children;
//  * fake leaves (source-only boxes) get no local expansions: they are never
//    evaluated and never pass anything down;
//  * the GEMMs run on the FP64 tensor cores (mma.sync m8n8k4 f64); the
//    activations sit in shared memory with padded rows (stride 4 mod 16
//    doubles: conflict-free fragment loads), the operators are read through
//    the read-only cache.

#include <algorithm>
#include <type_traits>

#include "fmm.cuh"
#include "gemm.cuh"
#include "scan.cuh"
#include "timing.cuh"

namespace fmmb {
namespace {

constexpr int TN = 32;      // nodes per upward / downward tile
constexpr int TM = 64;      // targets per M2L tile
constexpr int NT = 256;     // threads per tile CTA
constexpr int TCH = 128;    // targets per evaluation work item (= threads)
// callers size the work-item array as total + m / EVAL_CHUNK + 1 entries
static_assert(TCH == EVAL_CHUNK, "evaluation work items hold EVAL_CHUNK targets");
constexpr int SMAX = 896;   // sources staged per evaluation pass (8 blocks of 128 per SM
                            // with the log2 table beside them)

// the 27 offsets a target can see, by its parity class 2*(ix&1) + (iy&1)
// (offset ids walk ox = -3..3 outer, oy = -3..3 inner, skipping (-1..1)^2)
__constant__ int8_t c_class_off[4][27] = {
    {8, 9, 10, 11, 12, 13, 15, 16, 17, 19, 20, 21, 23, 24, 25, 27, 28, 29, 30, 31, 32, 34, 35, 36, 37, 38, 39},
    {7, 8, 9, 10, 11, 12, 14, 15, 16, 18, 19, 20, 22, 23, 24, 26, 27, 28, 29, 30, 31, 33, 34, 35, 36, 37, 38},
    {1, 2, 3, 4, 5, 6, 8, 9, 10, 11, 12, 13, 15, 16, 17, 19, 20, 21, 23, 24, 25, 27, 28, 29, 30, 31, 32},
    {0, 1, 2, 3, 4, 5, 7, 8, 9, 10, 11, 12, 14, 15, 16, 18, 19, 20, 22, 23, 24, 26, 27, 28, 29, 30, 31}};

// the factor a kernel's loops fold into their staged charges and locals
template <class KF, bool kFolded>
__device__ __forceinline__ double fold_of() {
  if constexpr (kFolded)
    return KF::kFold;
  else
    return 1.0;
}

// ---------------------------------------------------------------- upward ----
__device__ __forceinline__ int level_of_node(const int *__restrict__ off, int L, int g) {
  int lo = 0, hi = L;  // largest l with off[l] <= g
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (off[mid] <= g)
      lo = mid;
    else
      hi = mid;
  }
  return lo;
}

// kernel value at the difference (ax, ay) = target - source; raw log2 for
// the table-driven Laplace functor (its factor folded into the charges)
template <class KF>
__device__ __forceinline__ double kernel_at(const KF &K, double ax, double ay) {
  if constexpr (KF::kLogTable)
    return K.raw(ax, ay);
  else
    return K(0.0, 0.0, ax, ay);
}

// S2M + C2E of every S2M node (leaves holding points, levels >= 2) of every
// level in one launch (flexmm/flexmm2d/kifmm.py:96-105, then fmm.py:86-90):
// a tile is TN consecutive entries of the level-major S2M node list, a warp
// sums one node's sources into its check potentials (lanes over check
// points, the node's sources staged 32 at a time, four independent sums
// per lane); C2E runs once for each level the tile holds.
constexpr double INV_2PI = 1.0 / (2.0 * M_PI);

// double-layer kernel of the Laplace kernel -log(r^2)/(4 pi): the field at
// offset (ax, ay) = target - source of a dipole (dx, dy) = strength * normal,
// (d . a) / (2 pi |a|^2) (Laplace_Both_Eval, examples/pure_kifmm_laplace_dipoles.py:31-40)
__device__ __forceinline__ double dipole_at(double dx, double dy, double ax, double ay) {
  return fma(dx, ax, dy * ay) / fma(ax, ax, ay * ay) * INV_2PI;
}

template <class KF, bool DIP = false>
__global__ void __launch_bounds__(NT) k_s2m(KernelParams kp, int neq, int np, int L,
                                            const int *__restrict__ off,
                                            const int *__restrict__ uplist,
                                            const int *__restrict__ n_up_ptr,
                                            const int *__restrict__ bot,
                                            const int *__restrict__ top,
                                            const double *__restrict__ xmid,
                                            const double *__restrict__ ymid,
                                            const double *__restrict__ sx,
                                            const double *__restrict__ sy,
                                            const double *__restrict__ tau,
                                            const LevelOpsDev *__restrict__ ops,
                                            double *__restrict__ mult,
                                            const double *__restrict__ dvx = nullptr,
                                            const double *__restrict__ dvy = nullptr,
                                            int64_t tstride = 0, int64_t cstride = 0) {
  // charge column blockIdx.y (multi-RHS: column strides tstride / cstride)
  tau += blockIdx.y * tstride;
  mult += blockIdx.y * cstride;
  extern __shared__ double smem[];
  const int ldp = pad_ld(np);
  double *P = smem;          // [TN][ldp] check potentials
  double *T = P + TN * ldp;  // [TN][ldp] C2E scratch
  double *Bs = T + TN * ldp;  // C2E operators streamed through (gemm_stage_doubles(np))
  __shared__ double srcx[NT / 32][32], srcy[NT / 32][32], srct[NT / 32][32];
  __shared__ double srcdx[DIP ? NT / 32 : 1][32], srcdy[DIP ? NT / 32 : 1][32];
  __shared__ int node[TN], nlev[TN];
  __shared__ double *orow[TN];
  __shared__ FunctorSmem<KF> fsm;
  KF K(kp);
  fsm.bind(K);
  const double fold = fold_of<KF, KF::kLogTable>();
  const int n_up = *n_up_ptr;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int tile = blockIdx.x; tile * TN < n_up; tile += gridDim.x) {
    const int i0 = tile * TN, nloc = min(TN, n_up - i0);
    for (int i = threadIdx.x; i < TN * ldp; i += NT) P[i] = 0.0;
    if (threadIdx.x < TN) {
      const int g = (int)threadIdx.x < nloc ? uplist[i0 + threadIdx.x] : -1;
      node[threadIdx.x] = g;
      nlev[threadIdx.x] = g >= 0 ? level_of_node(off, L, g) : -1;
    }
    __syncthreads();
    const int mlo = nlev[0], mhi = nlev[nloc - 1];
    for (int t = warp; t < nloc; t += NT / 32) {
      const int g = node[t];
      const LevelOpsDev &op = ops[nlev[t]];
      const int b = bot[g], e = top[g];
      const double cx = xmid[g], cy = ymid[g];
      const bool k0 = lane < neq, k1 = lane + 32 < neq;
      const double lx0 = k0 ? op.lx[lane] : 0.0, ly0 = k0 ? op.ly[lane] : 0.0;
      const double lx1 = k1 ? op.lx[lane + 32] : 0.0, ly1 = k1 ? op.ly[lane + 32] : 0.0;
      double a0 = 0.0, b0 = 0.0, a1 = 0.0, b1 = 0.0;
      for (int j0 = b; j0 < e; j0 += 32) {
        const int nj = min(32, e - j0);
        if (lane < nj) {
          srcx[warp][lane] = sx[j0 + lane] - cx;
          srcy[warp][lane] = sy[j0 + lane] - cy;
          srct[warp][lane] = tau[j0 + lane] * fold;
          if constexpr (DIP) {
            srcdx[warp][lane] = dvx[j0 + lane];
            srcdy[warp][lane] = dvy[j0 + lane];
          }
        } else {  // padding pairs: zero charge at a harmless distance
          srcx[warp][lane] = 0.0;
          srcy[warp][lane] = 0.0;
          srct[warp][lane] = 0.0;
          if constexpr (DIP) {
            srcdx[warp][lane] = 0.0;
            srcdy[warp][lane] = 0.0;
          }
        }
        __syncwarp();
        const int nj2 = (nj + 1) & ~1;
        // one source's contribution at check point (lx, ly)
        auto term = [&](double lx, double ly, int j) -> double {
          const double ax = lx - srcx[warp][j], ay = ly - srcy[warp][j];
          double v = kernel_at(K, ax, ay) * srct[warp][j];
          if constexpr (DIP) v += dipole_at(srcdx[warp][j], srcdy[warp][j], ax, ay);
          return v;
        };
        if (k0)
          for (int j = 0; j < nj2; j += 2) {
            a0 += term(lx0, ly0, j);
            b0 += term(lx0, ly0, j + 1);
          }
        if (k1)
          for (int j = 0; j < nj2; j += 2) {
            a1 += term(lx1, ly1, j);
            b1 += term(lx1, ly1, j + 1);
          }
        __syncwarp();
      }
      if (k0) P[t * ldp + lane] = a0 + b0;
      if (k1) P[t * ldp + lane + 32] = a1 + b1;
    }
    for (int m = mlo; m <= mhi; ++m) {
      __syncthreads();
      if (threadIdx.x < TN)
        orow[threadIdx.x] = nlev[threadIdx.x] == m ? mult + (size_t)node[threadIdx.x] * np : nullptr;
      __syncthreads();
      c2e_tile_staged(ops[m], np, P, T, orow, Bs);
    }
    __syncthreads();
  }
}

// M2M + C2E of the parent boxes of level m (flexmm/flexmm2d/fmm.py:91-98):
// TN parent groups per tile; their children are the contiguous node rows
// c_first + 4e .. c_first + 4e + 3 of level m+1.  P[t] = M2MC . children.
__global__ void __launch_bounds__(NT) k_m2m(int m, int np, int c_first, int n_groups,
                                            const int *__restrict__ parent,
                                            const LevelOpsDev *__restrict__ ops,
                                            double *__restrict__ mult, int64_t cstride) {
  mult += blockIdx.y * cstride;  // charge column blockIdx.y
  extern __shared__ double smem[];
  const int ldp = pad_ld(np), lda = pad_ld(4 * np);
  double *P = smem;           // [TN][ldp] check potentials
  double *T = P + TN * ldp;   // [TN][ldp] C2E scratch
  double *A = T + TN * ldp;   // [TN][lda] children multipoles
  double *Bs = A + TN * lda;  // operators streamed through (gemm_stage_doubles(np))
  __shared__ double *orow[TN];
  const LevelOpsDev &op = ops[m];
  const int e0 = blockIdx.x * TN, nloc = min(TN, n_groups - e0);
  for (int i = threadIdx.x; i < TN * ldp; i += NT) P[i] = T[i] = 0.0;
  for (int i = threadIdx.x + nloc * lda; i < TN * lda; i += NT) A[i] = 0.0;
  pdl_wait();  // the children's multipoles come from the kernels before
  pdl_trigger();
  stage_rows(A, lda, mult + (size_t)(c_first + 4 * e0) * np, nloc, 4 * np);
  if (threadIdx.x < TN) {
    const int t = threadIdx.x;
    orow[t] = t < nloc ? mult + (size_t)parent[c_first + 4 * (e0 + t)] * np : nullptr;
  }
  cp_async_wait_all();
  __syncthreads();
  {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
    const int r0 = 8 * (warp & 3), c0 = 8 * (warp >> 2);
    double acc[1][4][2];
    zero_acc(acc);
    warp_gemm_staged<1, 4>(A, lda, op.m2mct, np, 4 * np, r0, c0, 2, np, acc, Bs);
    const int t = r0 + g;
#pragma unroll
    for (int cb = 0; cb < 4; ++cb) {
      const int col = c0 + 16 * cb + 2 * q;
      if (col < np) {
        P[t * ldp + col] = acc[0][cb][0];
        P[t * ldp + col + 1] = acc[0][cb][1];
      }
    }
  }
  __syncthreads();
  c2e_tile_staged(op, np, P, T, orow, Bs);
}

// ------------------------------------------------------------------- M2L ----
struct M2LTiles {
  int n_levels;
  int tile_start[4 * FMM_MAX_LEVELS_DEV + 1];  // first tile of each (level, parity class)
  int rg_lo[FMM_MAX_LEVELS_DEV];               // real groups of each level
  int rg_cnt[FMM_MAX_LEVELS_DEV];
};

// One tile = 64 targets of one parity class of one level (the 27 offsets
// that class can see).  The active offsets (an operator, and a source for
// some target) are pipelined: the gathered source multipoles and the
// offset's operators of offset a + 1 are copied into the second of two
// shared buffers (cp.async) while the DMMA GEMMs of offset a run, so
// neither the gather nor the operator reads wait on L2 inside the GEMM.
// Dense offsets: acc += G . D^T; SVD offsets: W = G . M1^T, acc += W . M2^T.
__host__ __device__ inline int m2l_op_doubles(int np) {
  const int dense = np * pad_ld(np), svd = np * pad_ld(32) + 32 * pad_ld(np);
  return dense > svd ? dense : svd;
}
__host__ __device__ inline size_t m2l_smem_doubles(int np) {
  return (size_t)2 * TM * pad_ld(np) + (size_t)TM * pad_ld(32) + 2 * (size_t)m2l_op_doubles(np);
}

__global__ void __launch_bounds__(NT) k_m2l(M2LTiles tiles, int np, const int *__restrict__ rg,
                                            const int *__restrict__ il,
                                            const LevelOpsDev *__restrict__ ops,
                                            const double *__restrict__ mult,
                                            double *__restrict__ ple, int64_t cstride) {
  mult += blockIdx.y * cstride;  // charge column blockIdx.y
  ple += blockIdx.y * cstride;
  extern __shared__ double smem[];
  const int ldp = pad_ld(np), ldw = pad_ld(32), ldb = pad_ld(np);
  double *Gb[2] = {smem, smem + TM * ldp};   // [TM][ldp] gathered source multipoles
  double *W = smem + 2 * TM * ldp;           // [TM][ldw] SVD intermediate (rank <= 32)
  double *Ob[2] = {W + TM * ldw, W + TM * ldw + m2l_op_doubles(np)};  // the offset's operators
  __shared__ int tgt[TM];
  __shared__ int s_src[27][TM];  // source node per class offset and target row
  __shared__ int s_act[27];      // active class offsets, in order
  __shared__ int s_nact;
  __shared__ unsigned int s_mask;
  // this block's (level, parity class, range of real groups)
  int slot = 0;
  while (slot + 1 < 4 * tiles.n_levels && tiles.tile_start[slot + 1] <= (int)blockIdx.x) ++slot;
  const int m = slot >> 2, cls = slot & 3;
  const int q0 = TM * (blockIdx.x - tiles.tile_start[slot]);
  const int nloc = min(TM, tiles.rg_cnt[m] - q0);
  const LevelOpsDev &op = ops[m];
  if (threadIdx.x == 0) s_mask = 0u;
  __syncthreads();
  if (threadIdx.x < TM) {
    const int tg = (threadIdx.x < nloc) ? rg[tiles.rg_lo[m] + q0 + threadIdx.x] + cls : -1;
    tgt[threadIdx.x] = tg;
    int sidx[27];  // all loads issued together
#pragma unroll
    for (int oi = 0; oi < 27; ++oi) {
      const int o = c_class_off[cls][oi];
      sidx[oi] = (tg >= 0 && op.kind[o] != M2L_NULL) ? __ldg(il + (size_t)tg * N_OFFSETS + o) : -1;
    }
    unsigned int mask = 0;
#pragma unroll
    for (int oi = 0; oi < 27; ++oi) {
      s_src[oi][threadIdx.x] = sidx[oi];
      if (sidx[oi] >= 0) mask |= 1u << oi;
    }
    mask = __reduce_or_sync(0xffffffffu, mask);
    if ((threadIdx.x & 31) == 0) atomicOr(&s_mask, mask);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int n = 0;
    for (int oi = 0; oi < 27; ++oi)
      if ((s_mask >> oi) & 1u) s_act[n++] = oi;
    s_nact = n;
  }
  __syncthreads();
  const int nact = s_nact;
  // copies of active offset a into buffer set b (one cp.async group)
  auto prefetch = [&](int a, int b) {
    const int oi = s_act[a], o = c_class_off[cls][oi];
    double *G = Gb[b], *O = Ob[b];
    const int h = np / 2;
    for (int i = threadIdx.x; i < TM * h; i += NT) {
      const int t = i / h, k2 = 2 * (i - t * h);
      const int src = s_src[oi][t];
      if (src >= 0) {
        cp_async16(G + t * ldp + k2, mult + (size_t)src * np + k2);
      } else {
        G[t * ldp + k2] = 0.0;
        G[t * ldp + k2 + 1] = 0.0;
      }
    }
    const double *B = op.m2l[o];
    if (op.kind[o] == M2L_DENSE) {
      for (int i = threadIdx.x; i < np * h; i += NT) {
        const int r = i / h, c2 = 2 * (i - r * h);
        cp_async16(O + r * ldb + c2, B + (size_t)r * np + c2);
      }
    } else {
      const int rp = op.rp[o], hr = rp / 2, ld1 = pad_ld(rp);
      for (int i = threadIdx.x; i < np * hr; i += NT) {  // M1^T [np][rp]
        const int r = i / hr, c2 = 2 * (i - r * hr);
        cp_async16(O + r * ld1 + c2, B + (size_t)r * rp + c2);
      }
      const double *B2 = B + (size_t)np * rp;
      double *O2 = O + np * ld1;
      for (int i = threadIdx.x; i < rp * h; i += NT) {  // M2^T [rp][np]
        const int r = i / h, c2 = 2 * (i - r * h);
        cp_async16(O2 + r * ldb + c2, B2 + (size_t)r * np + c2);
      }
    }
    cp_async_commit_group();
  };
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  // dense / stage-2 mapping: rows 16*(warp&3) + [0,16), column blocks 8*(warp>>2) + 16*cb
  const int r0 = 16 * (warp & 3), c0 = 8 * (warp >> 2);
  double acc[2][4][2];
  zero_acc(acc);
  if (nact > 0) prefetch(0, 0);
  for (int a = 0; a < nact; ++a) {
    const int b = a & 1;
    if (a + 1 < nact) {
      prefetch(a + 1, b ^ 1);
      cp_async_wait_group<1>();
    } else {
      cp_async_wait_group<0>();
    }
    __syncthreads();
    const int o = c_class_off[cls][s_act[a]];
    if (op.kind[o] == M2L_DENSE) {
      warp_gemm<2, 4, true>(Gb[b], ldp, Ob[b], ldb, np, r0, c0, 2, np, acc);
    } else {
      const int rp = op.rp[o], ld1 = pad_ld(rp);
      // stage 1: W[64][rp] = G . M1^T ; warp -> rows 8*warp + [0,8), column blocks 0..3
      double w[1][4][2];
      zero_acc(w);
      warp_gemm<1, 4, true>(Gb[b], ldp, Ob[b], ld1, np, 8 * warp, 0, 1, rp, w);
#pragma unroll
      for (int cb = 0; cb < 4; ++cb) {
        const int col = 8 * cb + 2 * q;
        if (col < rp) {
          W[(8 * warp + g) * ldw + col] = w[0][cb][0];
          W[(8 * warp + g) * ldw + col + 1] = w[0][cb][1];
        }
      }
      __syncthreads();
      // stage 2: acc += W . M2^T
      warp_gemm<2, 4, true>(W, ldw, Ob[b] + np * ld1, ldb, rp, r0, c0, 2, np, acc);
    }
    __syncthreads();  // buffer set b is refilled by the next iteration's copies
  }
#pragma unroll
  for (int rb = 0; rb < 2; ++rb) {
    const int t = r0 + 8 * rb + g;
    if (t < nloc) {
#pragma unroll
      for (int cb = 0; cb < 4; ++cb) {
        const int col = c0 + 16 * cb + 2 * q;
        if (col < np)
          *reinterpret_cast<double2 *>(ple + (size_t)tgt[t] * np + col) =
              make_double2(acc[rb][cb][0], acc[rb][cb][1]);
      }
    }
  }
}

// -------------------------------------------------------------- downward ----
// One tile = 8 real sibling groups of level m (32 nodes): L2L from their
// parents (m >= 3), plus the M2L partial locals, then check-to-equivalent.
__global__ void __launch_bounds__(NT) k_downward(int m, int np, int rg_lo, int rg_cnt,
                                                 const int *__restrict__ rg,
                                                 const int *__restrict__ parent,
                                                 const LevelOpsDev *__restrict__ ops,
                                                 const double *__restrict__ ple,
                                                 double *__restrict__ loc, int64_t cstride) {
  ple += blockIdx.y * cstride;  // charge column blockIdx.y
  loc += blockIdx.y * cstride;
  extern __shared__ double smem[];
  const int ldp = pad_ld(np);
  double *P = smem;           // [32][ldp] partial locals
  double *T = P + TN * ldp;   // [32][ldp] parent locals, then C2E scratch
  double *Bs = T + TN * ldp;  // operators streamed through (gemm_stage_doubles(4 np))
  __shared__ int node[TN];
  __shared__ double *orow[TN];
  const LevelOpsDev &op = ops[m];
  const int q0 = 8 * blockIdx.x;
  const int ngrp = min(8, rg_cnt - q0);
  if (threadIdx.x < TN) {
    const int grp = threadIdx.x >> 2;
    const int n = (grp < ngrp) ? rg[rg_lo + q0 + grp] + int(threadIdx.x & 3) : -1;
    node[threadIdx.x] = n;
    orow[threadIdx.x] = n >= 0 ? loc + (size_t)n * np : nullptr;
  }
  pdl_wait();  // partial locals (M2L) and the parents' locals come from the kernels before
  pdl_trigger();
  __syncthreads();
  for (int i = threadIdx.x; i < TN * np; i += NT) {
    const int t = i / np, k = i % np;
    P[t * ldp + k] = (node[t] >= 0) ? ple[(size_t)node[t] * np + k] : 0.0;
    T[t * ldp + k] = 0.0;
  }
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  if (m >= 3) {
    const LevelOpsDev &opp = ops[m - 1];
    for (int i = threadIdx.x; i < 8 * np; i += NT) {
      const int grp = i / np, k = i % np;
      const int n0 = node[4 * grp];
      T[grp * ldp + k] = (n0 >= 0) ? loc[(size_t)parent[n0] * np + k] : 0.0;
    }
    __syncthreads();
    // L2L: [8 parents][4np] = Lp . M2MC (flexmm/flexmm2d/fmm.py:140-147);
    // warp -> column blocks warp + 8*cb of the 4np columns
    double acc[1][4][2];
    zero_acc(acc);
    warp_gemm_staged<1, 4>(T, ldp, opp.m2mc, 4 * np, np, 0, 8 * warp, 8, 4 * np, acc, Bs);
#pragma unroll
    for (int cb = 0; cb < 4; ++cb) {
      const int col = 8 * warp + 64 * cb + 2 * q;  // column of the 4np-wide parent row
      if (col < 4 * np) {
        const int c = col / np, i = col % np;
        P[(4 * g + c) * ldp + i] += acc[0][cb][0];
        P[(4 * g + c) * ldp + i + 1] += acc[0][cb][1];
      }
    }
    __syncthreads();
  }
  c2e_tile_staged(op, np, P, T, orow, Bs);
}

// ------------------------------------------------------------ evaluation ----
__global__ void k_leaf_targets(int total, int L, const int *__restrict__ off,
                               const uint64_t *__restrict__ code, const uint8_t *__restrict__ flags,
                               const uint64_t *__restrict__ tkeys, int64_t m,
                               int *__restrict__ tb, int *__restrict__ te,
                               int *__restrict__ nchunk) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    int lo = 0, hi = L;
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (off[mid] <= g)
        lo = mid;
      else
        hi = mid;
    }
    const int lev = lo;
    int b = 0, e = 0;
    if ((flags[g] & NF_LEAF) && m > 0) {
      // both ends of the leaf's key range: two branchless lower-bound
      // searches over [0, m) in step (same length, same step count), so each
      // step's two loads are issued together
      const int sh = 2 * (MAXD - lev);
      const uint64_t c = code[g];
      const uint64_t vlo = c << sh, vhi = (c + 1) << sh;
      int64_t b0 = 0, b1 = 0, len = m;
      while (len > 1) {
        const int64_t half = len >> 1;
        const uint64_t k0 = __ldg(tkeys + b0 + half), k1 = __ldg(tkeys + b1 + half);
        b0 += k0 < vlo ? half : 0;
        b1 += k1 < vhi ? half : 0;
        len -= half;
      }
      b = int(b0 + (__ldg(tkeys + b0) < vlo ? 1 : 0));
      e = int(b1 + (__ldg(tkeys + b1) < vhi ? 1 : 0));
    }
    tb[g] = b;
    te[g] = e;
    nchunk[g] = (e - b + TCH - 1) / TCH;
  }
}

// expand the per-leaf chunk counts into a flat item list
__global__ void k_make_items(int total, int L, const int *__restrict__ off, const int *__restrict__ tb,
                             const int *__restrict__ te, const int *__restrict__ nch,
                             const int *__restrict__ choff, int4 *__restrict__ items,
                             int *__restrict__ n_items, int mark_multi) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    if (g == total - 1) *n_items = choff[g] + nch[g];
    const int n = nch[g];
    if (n == 0) continue;
    int lo = 0, hi = L;
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (off[mid] <= g) lo = mid; else hi = mid;
    }
    const int y = lo | (mark_multi && n > 1 ? EVAL_MULTI : 0);
    for (int c = 0; c < n; ++c) {
      const int t0 = tb[g] + c * TCH;
      items[choff[g] + c] = make_int4(g, y, t0, min(TCH, te[g] - t0));
    }
  }
}

// One work item = (leaf, up to 128 of its targets).  G = 128 / targets
// (rounded down to a power of two) threads share a target: they split the
// circle points of L2T and the colleague sources of P2P, then reduce with
// warp shuffles (and shared memory when G > 32).
// NOUT = 1: potential; NOUT = 3: potential and its gradient in the target
// position (rows of out, stride ld_out).
// PART: EVAL_FULL (L2T + P2P), EVAL_NEAR (P2P only, into near[], caller's
// point order) or EVAL_FAR (L2T only, plus near[]: out = far + near).
// DIP: the sources also carry dipoles (dvx, dvy: strength * normal, sorted);
// Laplace (table-driven functor), potential only.
// CAT (near field only): a source whose category scat[] (sorted order)
// equals the target's tcat[] (caller's order) is left out
// (flexmm/flexmm2d/local_evaluator_category.py:33-38).
template <class KF, int NOUT, int PART = EVAL_FULL, bool DIP = false, bool CAT = false>
__global__ void __launch_bounds__(TCH) k_evaluate(KernelParams kp, int neq, int np,
                                                  const int4 *__restrict__ items,
                                                  const int *__restrict__ n_items_ptr,
                                                  const int *__restrict__ coll,
                                                  const int *__restrict__ bot,
                                                  const int *__restrict__ top,
                                                  const double *__restrict__ xmid,
                                                  const double *__restrict__ ymid,
                                                  const double *__restrict__ sx,
                                                  const double *__restrict__ sy,
                                                  const double *__restrict__ tau,
                                                  const LevelOpsDev *__restrict__ ops,
                                                  const double *__restrict__ loc,
                                                  const double *__restrict__ txs,
                                                  const double *__restrict__ tys,
                                                  const int *__restrict__ tperm, int check,
                                                  double *__restrict__ out, int64_t ld_out,
                                                  double *__restrict__ near = nullptr,
                                                  const double *__restrict__ dvx = nullptr,
                                                  const double *__restrict__ dvy = nullptr,
                                                  const int64_t *__restrict__ scat = nullptr,
                                                  const int64_t *__restrict__ tcat = nullptr) {
  static_assert(PART == EVAL_FULL || NOUT == 1, "split evaluation: potential only");
  static_assert(!CAT || (PART == EVAL_NEAR && !DIP), "categories: near field of charges only");
  static_assert(!DIP || (KF::kLogTable && NOUT == 1), "dipoles: table Laplace, potential only");
  __shared__ double Ls[64], lxs[64], lys[64];
  __shared__ double ssx[SMAX], ssy[SMAX], stau[SMAX];
  __shared__ double sdx[DIP ? SMAX : 1], sdy[DIP ? SMAX : 1];
  __shared__ long long scs[CAT ? SMAX : 1];
  __shared__ int rb[9], rs[10];  // colleague range begins and prefix sizes
  __shared__ double red[NOUT][TCH / 32];
  __shared__ FunctorSmem<KF> fsm;
  KF K(kp);
  fsm.bind(K);
  // table-driven Laplace (potential only): the kernel's constant factor is
  // folded into the staged locals and charges, the loops sum raw log2 values
  constexpr bool kFolded = KF::kLogTable && NOUT == 1;
  const double fold = fold_of<KF, kFolded>();
  const int n_items = *n_items_ptr;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int4 it = items[item];
    const int g = it.x, lev = it.y & EVAL_LEVEL_MASK, t0 = it.z, cnt = it.w;
    int G = 1;
    if (!(it.y & EVAL_MULTI))
      while (2 * G * cnt <= TCH) G *= 2;
    const int t = threadIdx.x / G, sub = threadIdx.x % G;
    const bool valid = t < cnt;
    const double x = valid ? txs[t0 + t] : 0.0, y = valid ? tys[t0 + t] : 0.0;
    long long tc = 0;
    if constexpr (CAT) tc = valid ? (long long)tcat[tperm[t0 + t]] : 0;
    if (threadIdx.x < 9) {
      const int cg = PART == EVAL_FAR ? -1 : coll[(size_t)g * 9 + threadIdx.x];
      rb[threadIdx.x] = cg >= 0 ? bot[cg] : 0;
      rs[threadIdx.x + 1] = cg >= 0 ? top[cg] - bot[cg] : 0;
    }
    if (threadIdx.x == 0) rs[0] = 0;
    // L2T (flexmm/flexmm2d/kifmm.py:106-120); locals of levels 0-1 are zero
    const bool l2t = lev >= 2 && PART != EVAL_NEAR;
    if (l2t)
      for (int k = threadIdx.x; k < neq; k += TCH) {
        Ls[k] = loc[(size_t)g * np + k] * fold;
        lxs[k] = ops[lev].lx[k];
        lys[k] = ops[lev].ly[k];
      }
    __syncthreads();
    if (threadIdx.x == 0)
      for (int c = 1; c <= 9; ++c) rs[c] += rs[c - 1];
    double u0 = 0.0, u1 = 0.0, u2 = 0.0, u3 = 0.0;
    double gu = 0.0, gx = 0.0, gy = 0.0;  // NOUT = 3
    if (l2t && valid) {
      const double dx = x - xmid[g], dy = y - ymid[g];
      if constexpr (NOUT == 1) {
        auto kv = [&](int k) -> double {
          if constexpr (kFolded)
            return K.raw(dx - lxs[k], dy - lys[k]);
          else
            return K(lxs[k], lys[k], dx, dy);
        };
        int k = sub;
        for (; k + 3 * G < neq; k += 4 * G) {
          u0 = fma(kv(k), Ls[k], u0);
          u1 = fma(kv(k + G), Ls[k + G], u1);
          u2 = fma(kv(k + 2 * G), Ls[k + 2 * G], u2);
          u3 = fma(kv(k + 3 * G), Ls[k + 3 * G], u3);
        }
        for (; k < neq; k += G) u0 = fma(kv(k), Ls[k], u0);
      } else {
        for (int k = sub; k < neq; k += G) K.grad(lxs[k], lys[k], dx, dy, Ls[k], gu, gx, gy);
      }
    }
    __syncthreads();
    // P2P over the colleagues' sorted source ranges (flexmm/flexmm2d/helpers.py:152-194);
    // a coincident pair is skipped when check is set (helpers.py:99-107)
    auto pair = [&](int j) -> double {
      const double qx = ssx[j], qy = ssy[j];
      if constexpr (DIP) {  // single plus double layer; coincident pairs skipped when check
        const double ax = x - qx, ay = y - qy;
        if (check && ax == 0.0 && ay == 0.0) return 0.0;
        return K.raw(ax, ay) * stau[j] + dipole_at(sdx[j], sdy[j], ax, ay);
      } else if constexpr (CAT) {  // a source of the target's own category adds nothing
        if (scs[j] == tc) return 0.0;
        if constexpr (kFolded) {
          return K.raw_checked(qx, qy, x, y, check) * stau[j];
        } else {
          const double v = K(qx, qy, x, y) * stau[j];
          return (check && x - qx == 0.0 && y - qy == 0.0) ? 0.0 : v;
        }
      } else if constexpr (kFolded) {
        return K.raw_checked(qx, qy, x, y, check) * stau[j];
      } else {
        const double v = K(qx, qy, x, y) * stau[j];
        return (check && x - qx == 0.0 && y - qy == 0.0) ? 0.0 : v;
      }
    };
    const int ns = rs[9];
    for (int base = 0; base < ns; base += SMAX) {
      const int nb = min(SMAX, ns - base);
      for (int i = threadIdx.x; i < nb; i += TCH) {
        const int idx = base + i;
        int c = 0;
        while (idx >= rs[c + 1]) ++c;
        const int j = rb[c] + (idx - rs[c]);
        ssx[i] = sx[j];
        ssy[i] = sy[j];
        stau[i] = tau[j] * fold;
        if constexpr (DIP) {
          sdx[i] = dvx[j];
          sdy[i] = dvy[j];
        }
        if constexpr (CAT) scs[i] = (long long)scat[j];
      }
      __syncthreads();
      if (valid) {
        if constexpr (NOUT == 1) {
          int j = sub;
          for (; j + 3 * G < nb; j += 4 * G) {
            u0 += pair(j);
            u1 += pair(j + G);
            u2 += pair(j + 2 * G);
            u3 += pair(j + 3 * G);
          }
          for (; j < nb; j += G) u0 += pair(j);
        } else {
          for (int j = sub; j < nb; j += G) {
            const double qx = ssx[j], qy = ssy[j];
            if (!(check && x - qx == 0.0 && y - qy == 0.0)) K.grad(qx, qy, x, y, stau[j], gu, gx, gy);
          }
        }
      }
      __syncthreads();
    }
    // reduce over the G threads of each target
    double r[NOUT];
    if constexpr (NOUT == 1) {
      r[0] = (u0 + u1) + (u2 + u3);
    } else {
      r[0] = gu;
      r[1] = gx;
      r[2] = gy;
    }
#pragma unroll
    for (int o = 0; o < NOUT; ++o) {
      double u = r[o];
      for (int w = min(G, 32) >> 1; w >= 1; w >>= 1) u += __shfl_xor_sync(0xffffffffu, u, w);
      if (G > 32) {
        if ((threadIdx.x & 31) == 0) red[o][threadIdx.x >> 5] = u;
        __syncthreads();
        if (sub == 0) {
          u = 0.0;
          for (int w = 0; w < G / 32; ++w) u += red[o][(threadIdx.x >> 5) + w];
        }
      }
      if (valid && sub == 0) {
        const int i = tperm[t0 + t];
        if constexpr (PART == EVAL_NEAR)
          near[i] = u;
        else if constexpr (PART == EVAL_FAR)
          out[i] = u + near[i];
        else
          out[o * ld_out + i] = u;
      }
    }
    __syncthreads();
  }
}

// FP64 direct sum (kernel_apply / kernel_apply_single_check,
// flexmm/flexmm2d/helpers.py:91-116): all sources, one target per thread,
// Several charge columns on one tree (multi-RHS): columns r0 .. r0 + R - 1
// of the charges (stride n_src) and locals (stride col_stride); each kernel
// value (L2T and P2P) is computed once and applied to the R columns.  Output
// row r of out (stride ld_out).  One work item = (leaf, up to 128 targets).
constexpr int SMAX_MR = 256;
template <class KF, int R>
__global__ void __launch_bounds__(TCH) k_evaluate_multi(KernelParams kp, int neq, int np, int ncol,
                                                        const int4 *__restrict__ items,
                                                        const int *__restrict__ n_items_ptr,
                                                        const int *__restrict__ coll,
                                                        const int *__restrict__ bot,
                                                        const int *__restrict__ top,
                                                        const double *__restrict__ xmid,
                                                        const double *__restrict__ ymid,
                                                        const double *__restrict__ sx,
                                                        const double *__restrict__ sy,
                                                        const double *__restrict__ tau, int64_t n_src,
                                                        const LevelOpsDev *__restrict__ ops,
                                                        const double *__restrict__ loc,
                                                        int64_t col_stride,
                                                        const double *__restrict__ txs,
                                                        const double *__restrict__ tys,
                                                        const int *__restrict__ tperm, int check,
                                                        double *__restrict__ out, int64_t ld_out) {
  __shared__ double ssx[SMAX_MR], ssy[SMAX_MR], stau[R][SMAX_MR];
  __shared__ int rb[9], rs[10];
  __shared__ double red[R][TCH / 32];
  __shared__ FunctorSmem<KF> fsm;
  KF K(kp);
  fsm.bind(K);
  const int n_items = *n_items_ptr;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int4 it = items[item];
    const int g = it.x, lev = it.y & EVAL_LEVEL_MASK, t0 = it.z, cnt = it.w;
    int G = 1;
    if (!(it.y & EVAL_MULTI))
      while (2 * G * cnt <= TCH) G *= 2;
    const int t = threadIdx.x / G, sub = threadIdx.x % G;
    const bool valid = t < cnt;
    const double x = valid ? txs[t0 + t] : 0.0, y = valid ? tys[t0 + t] : 0.0;
    if (threadIdx.x < 9) {
      const int cg = coll[(size_t)g * 9 + threadIdx.x];
      rb[threadIdx.x] = cg >= 0 ? bot[cg] : 0;
      rs[threadIdx.x + 1] = cg >= 0 ? top[cg] - bot[cg] : 0;
    }
    if (threadIdx.x == 0) rs[0] = 0;
    __syncthreads();
    if (threadIdx.x == 0)
      for (int c = 1; c <= 9; ++c) rs[c] += rs[c - 1];
    double u[R];
#pragma unroll
    for (int c = 0; c < R; ++c) u[c] = 0.0;
    if (lev >= 2 && valid) {  // L2T, one kernel value per circle point for all columns
      const double dx = x - xmid[g], dy = y - ymid[g];
      const double *lx = ops[lev].lx, *ly = ops[lev].ly;
      for (int k = sub; k < neq; k += G) {
        const double kv = K(lx[k], ly[k], dx, dy);
#pragma unroll
        for (int c = 0; c < R; ++c)
          if (c < ncol) u[c] = fma(kv, loc[c * col_stride + (size_t)g * np + k], u[c]);
      }
    }
    __syncthreads();
    const int ns = rs[9];
    for (int base = 0; base < ns; base += SMAX_MR) {
      const int nb = min(SMAX_MR, ns - base);
      for (int i = threadIdx.x; i < nb; i += TCH) {
        const int idx = base + i;
        int c = 0;
        while (idx >= rs[c + 1]) ++c;
        const int j = rb[c] + (idx - rs[c]);
        ssx[i] = sx[j];
        ssy[i] = sy[j];
#pragma unroll
        for (int q = 0; q < R; ++q) stau[q][i] = q < ncol ? tau[q * n_src + j] : 0.0;
      }
      __syncthreads();
      if (valid)
        for (int j = sub; j < nb; j += G) {
          const double qx = ssx[j], qy = ssy[j];
          if (check && x - qx == 0.0 && y - qy == 0.0) continue;
          const double kv = K(qx, qy, x, y);
#pragma unroll
          for (int c = 0; c < R; ++c) u[c] = fma(kv, stau[c][j], u[c]);
        }
      __syncthreads();
    }
#pragma unroll
    for (int c = 0; c < R; ++c) {
      double w = u[c];
      for (int q = min(G, 32) >> 1; q >= 1; q >>= 1) w += __shfl_xor_sync(0xffffffffu, w, q);
      if (G > 32) {
        if ((threadIdx.x & 31) == 0) red[c][threadIdx.x >> 5] = w;
        __syncthreads();
        if (sub == 0) {
          w = 0.0;
          for (int q = 0; q < G / 32; ++q) w += red[c][(threadIdx.x >> 5) + q];
        }
      }
      if (valid && sub == 0 && c < ncol) out[c * ld_out + tperm[t0 + t]] = w;
    }
    __syncthreads();
  }
}

// sources staged through shared memory
template <class KF>
__global__ void __launch_bounds__(256) k_direct(KernelParams kp, const double *__restrict__ sx,
                                                const double *__restrict__ sy,
                                                const double *__restrict__ tau, int64_t ns,
                                                const double *__restrict__ tx,
                                                const double *__restrict__ ty, int64_t nt,
                                                int check, double *__restrict__ out) {
  __shared__ double qx[256], qy[256], qt[256];
  const KF K(kp);
  for (int64_t base = (int64_t)blockIdx.x * 256; base < nt; base += (int64_t)gridDim.x * 256) {
    const int64_t i = base + threadIdx.x;
    const bool valid = i < nt;
    const double x = valid ? tx[i] : 0.0, y = valid ? ty[i] : 0.0;
    double u = 0.0;
    for (int64_t j0 = 0; j0 < ns; j0 += 256) {
      const int nj = (int)(ns - j0 < 256 ? ns - j0 : 256);
      __syncthreads();
      if (threadIdx.x < nj) {
        qx[threadIdx.x] = sx[j0 + threadIdx.x];
        qy[threadIdx.x] = sy[j0 + threadIdx.x];
        qt[threadIdx.x] = tau[j0 + threadIdx.x];
      }
      __syncthreads();
      if (valid)
        for (int j = 0; j < nj; ++j) {
          if (check && x - qx[j] == 0.0 && y - qy[j] == 0.0) continue;
          u = fma(K(qx[j], qy[j], x, y), qt[j], u);
        }
    }
    if (valid) out[i] = u;
  }
}

__global__ void k_gather_sorted(const double *__restrict__ v, const int *__restrict__ perm,
                                int64_t n, double *__restrict__ o) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    o[i] = v[perm[i]];
}

template <class KF>
void upward_impl(const PassArgs &a, const double *tau_s, double *mult, cudaStream_t s, int n_rhs,
                 int64_t tstride, int64_t cstride) {
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  const int np = a.np;
  if (th.L < 3) return;
  const size_t s2m_bytes = sizeof(double) * ((size_t)TN * pad_ld(np) * 2 + gemm_stage_doubles(np));
  smem_limit(k_s2m<KF>, s2m_bytes);
  // persistent over the S2M nodes; at most one block per TN nodes of the tree
  // (small trees launch small grids)
  const int s2m_grid = std::max(1, std::min(148 * 4, (th.n_total() + TN - 1) / TN));
  PhaseTimer timer(PH_UPWARD, s);
  if (a.dvx) {
    if constexpr (std::is_same<KF, LaplaceF64T>::value) {
      smem_limit(k_s2m<KF, true>, s2m_bytes);
      k_s2m<KF, true><<<dim3(s2m_grid, n_rhs), NT, s2m_bytes, s>>>(
          a.kp, a.neq, np, th.L, td.dev_off.get(), td.uplist.get(), td.n_up.get(), td.bot.get(),
          td.top.get(), td.xmid.get(), td.ymid.get(), td.sx.get(), td.sy.get(), tau_s, a.ops_dev,
          mult, a.dvx, a.dvy, tstride, cstride);
    } else {
      throw Error(ERR_UNSUPPORTED, "dipole sources: Laplace kernel only");
    }
  } else {
    k_s2m<KF><<<dim3(s2m_grid, n_rhs), NT, s2m_bytes, s>>>(
        a.kp, a.neq, np, th.L, td.dev_off.get(), td.uplist.get(), td.n_up.get(), td.bot.get(),
        td.top.get(), td.xmid.get(), td.ymid.get(), td.sx.get(), td.sy.get(), tau_s, a.ops_dev,
        mult, nullptr, nullptr, tstride, cstride);
  }
  FMMB_CUDA(cudaGetLastError());
  const size_t m2m_bytes =
      sizeof(double) * ((size_t)TN * (2 * pad_ld(np) + pad_ld(4 * np)) + gemm_stage_doubles(np));
  smem_limit(k_m2m, m2m_bytes);
  for (int m = th.L - 2; m >= 2; --m) {
    const int c_first = th.off[m + 1];
    const int n_groups = (th.off[m + 2] - th.off[m + 1]) / 4;
    if (n_groups == 0) continue;
    launch_pdl(k_m2m, dim3((n_groups + TN - 1) / TN, n_rhs), dim3(NT), m2m_bytes, s, m, np,
               c_first, n_groups, td.parent.get(), a.ops_dev, mult, cstride);
  }
}

}  // namespace

// the tree's own sources: each leaf's range is its [bot, top) (the same
// lower-bound searches of the same sorted keys, done by the node pass)
__global__ void k_leaf_sources(int total, const uint8_t *__restrict__ flags,
                               const int *__restrict__ bot, const int *__restrict__ top,
                               int *__restrict__ tb, int *__restrict__ te, int *__restrict__ nchunk) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    const bool leaf = flags[g] & NF_LEAF;
    const int b = leaf ? bot[g] : 0, e = leaf ? top[g] : 0;
    tb[g] = b;
    te[g] = e;
    nchunk[g] = (e - b + TCH - 1) / TCH;
  }
}

void eval_items(const PassArgs &a, const uint64_t *tkeys, int64_t m, EvalItems &it, cudaStream_t s) {
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  const int total = th.n_total();
  it.tb.alloc(total, s);
  it.te.alloc(total, s);
  it.nch.alloc(total, s);
  it.choff.alloc(total, s);
  if (tkeys == td.pkeys.get() && m == th.n_points)
    k_leaf_sources<<<grid_for(total, 256), 256, 0, s>>>(total, td.flags.get(), td.bot.get(),
                                                        td.top.get(), it.tb.get(), it.te.get(),
                                                        it.nch.get());
  else
    k_leaf_targets<<<grid_for(total, 256), 256, 0, s>>>(total, th.L, td.dev_off.get(), td.code.get(),
                                                        td.flags.get(), tkeys, m, it.tb.get(),
                                                        it.te.get(), it.nch.get());
  FMMB_CUDA(cudaGetLastError());
  prefix_sum<int, false>(it.nch.get(), it.choff.get(), total, td.sort_fail.get(), true, s);
  it.items.alloc(total + m / TCH + 1, s);
  it.n_items.alloc(1, s);
  k_make_items<<<grid_for(total, 256), 256, 0, s>>>(total, th.L, td.dev_off.get(), it.tb.get(),
                                                    it.te.get(), it.nch.get(), it.choff.get(),
                                                    it.items.get(), it.n_items.get(), 0);
  FMMB_CUDA(cudaGetLastError());
}

// per leaf: end of its target range and its item count (counts from binning)
__global__ void k_leaf_ranges(int total, const int *__restrict__ count, const int *__restrict__ tb,
                              int *__restrict__ te, int *__restrict__ nch) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x) {
    te[g] = tb[g] + count[g];
    nch[g] = (count[g] + TCH - 1) / TCH;
  }
}

void eval_items_binned(const PassArgs &a, const double *tx, const double *ty, int64_t m,
                       EvalItems &it, double *txs, double *tys, int *tperm, cudaStream_t s) {
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  const int total = th.n_total();
  DevBuf<int> count, leaf_of, slot;
  count.alloc(total, s);
  count.zero(s);
  leaf_of.alloc(m, s);
  slot.alloc(m, s);
  bin_points(tx, ty, m, td, th, count.get(), leaf_of.get(), slot.get(), s);
  it.tb.alloc(total, s);
  it.te.alloc(total, s);
  it.nch.alloc(total, s);
  it.choff.alloc(total, s);
  prefix_sum<int, false>(count.get(), it.tb.get(), total, td.sort_fail.get(), true, s);
  scatter_binned(tx, ty, m, leaf_of.get(), slot.get(), it.tb.get(), txs, tys, tperm, s);
  k_leaf_ranges<<<grid_for(total, 256), 256, 0, s>>>(total, count.get(), it.tb.get(), it.te.get(),
                                                     it.nch.get());
  FMMB_CUDA(cudaGetLastError());
  prefix_sum<int, false>(it.nch.get(), it.choff.get(), total, td.sort_fail.get(), true, s);
  it.items.alloc(total + m / TCH + 1, s);
  it.n_items.alloc(1, s);
  k_make_items<<<grid_for(total, 256), 256, 0, s>>>(total, th.L, td.dev_off.get(), it.tb.get(),
                                                    it.te.get(), it.nch.get(), it.choff.get(),
                                                    it.items.get(), it.n_items.get(), 1);
  FMMB_CUDA(cudaGetLastError());
}

namespace {
template <class KF>
void evaluate_impl(const PassArgs &a, const double *tau_s, const double *loc, const double *txs,
                   const double *tys, const uint64_t *tkeys, const int *tperm, int64_t m, int check,
                   int nout, double *out, int64_t ld_out, cudaStream_t s, const EvalItems *pre) {
  const TreeDev &td = *a.td;
  EvalItems own;
  if (!pre) eval_items(a, tkeys, m, own, s);
  const EvalItems &it = pre ? *pre : own;
  const int64_t units = a.th->n_total() + m / TCH + 1;  // work items, upper bound
  PhaseTimer timer(PH_EVAL, s);
  if (a.dvx) {
    FMMB_CHECK(nout == 1, ERR_UNSUPPORTED, "dipole sources: potential only");
    if constexpr (std::is_same<KF, LaplaceF64T>::value) {
      k_evaluate<KF, 1, EVAL_FULL, true><<<work_grid(units, 5), TCH, 0, s>>>(
          a.kp, a.neq, a.np, it.items.get(), it.n_items.get(), td.coll.get(), td.bot.get(),
          td.top.get(), td.xmid.get(), td.ymid.get(), td.sx.get(), td.sy.get(), tau_s, a.ops_dev,
          loc, txs, tys, tperm, check, out, ld_out, nullptr, a.dvx, a.dvy);
    } else {
      throw Error(ERR_UNSUPPORTED, "dipole sources: Laplace kernel only");
    }
  } else {
    auto kern = nout == 3 ? k_evaluate<KF, 3> : k_evaluate<KF, 1>;
    kern<<<work_grid(units, 8), TCH, 0, s>>>(a.kp, a.neq, a.np, it.items.get(), it.n_items.get(),
                                 td.coll.get(), td.bot.get(), td.top.get(), td.xmid.get(),
                                 td.ymid.get(), td.sx.get(), td.sy.get(), tau_s, a.ops_dev, loc,
                                 txs, tys, tperm, check, out, ld_out, nullptr, nullptr, nullptr,
                                 nullptr, nullptr);
  }
  FMMB_CUDA(cudaGetLastError());
}
}  // namespace

void run_upward(const PassArgs &a, const double *tau_s, double *mult, cudaStream_t s, int n_rhs,
                int64_t tstride, int64_t cstride) {
  FMMB_CHECK(n_rhs >= 1 && n_rhs <= 65535, ERR_INVALID_ARGUMENT, "1..65535 charge columns");
  switch (a.kernel_id) {
    case KERNEL_LAPLACE: upward_impl<LaplaceF64T>(a, tau_s, mult, s, n_rhs, tstride, cstride); break;
    case KERNEL_MOD_HELMHOLTZ:
      upward_impl<ModHelmholtzF64>(a, tau_s, mult, s, n_rhs, tstride, cstride);
      break;
    case KERNEL_RADIAL_TABLE:
      upward_impl<RadialTableF64>(a, tau_s, mult, s, n_rhs, tstride, cstride);
      break;
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
}

void run_m2l(const PassArgs &a, const double *mult, double *ple, cudaStream_t s, int n_rhs,
             int64_t cstride) {
  const TreeHost &th = *a.th;
  if (th.L < 3) return;
  FMMB_CHECK(th.L <= FMM_MAX_LEVELS_DEV, ERR_INVALID_ARGUMENT, "too many levels");
  M2LTiles tl{};
  tl.n_levels = th.L;
  int tiles = 0;
  for (int m = 0; m < th.L; ++m) {
    tl.rg_lo[m] = th.rg_lo[m];
    tl.rg_cnt[m] = th.rg_hi[m] - th.rg_lo[m];
    for (int c = 0; c < 4; ++c) {
      tl.tile_start[4 * m + c] = tiles;
      if (m >= 2) tiles += (tl.rg_cnt[m] + TM - 1) / TM;
    }
  }
  tl.tile_start[4 * th.L] = tiles;
  if (tiles == 0) return;
  const size_t sm = sizeof(double) * m2l_smem_doubles(a.np);
  smem_limit(k_m2l, sizeof(double) * m2l_smem_doubles(64));
  PhaseTimer timer(PH_M2L, s);
  k_m2l<<<dim3(tiles, n_rhs), NT, sm, s>>>(tl, a.np, a.td->rg.get(), a.td->il.get(), a.ops_dev,
                                           mult, ple, cstride);
  FMMB_CUDA(cudaGetLastError());
}

void run_downward(const PassArgs &a, const double *ple, double *loc, cudaStream_t s, int n_rhs,
                  int64_t cstride) {
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  const size_t sm =
      sizeof(double) * ((size_t)TN * pad_ld(a.np) * 2 + gemm_stage_doubles(4 * a.np));
  smem_limit(k_downward, sm);
  for (int m = 2; m < th.L; ++m) {
    const int lo = th.rg_lo[m], cnt = th.rg_hi[m] - th.rg_lo[m];
    if (cnt <= 0) continue;
    const int tiles = (cnt + 7) / 8;
    PhaseTimer timer(PH_DOWNWARD, s);
    launch_pdl(k_downward, dim3(tiles, n_rhs), dim3(NT), sm, s, m, a.np, lo, cnt, td.rg.get(),
               td.parent.get(), a.ops_dev, ple, loc, cstride);
    FMMB_CUDA(cudaGetLastError());
  }
}

void run_evaluate(const PassArgs &a, const double *tau_s, const double *loc, const double *txs,
                  const double *tys, const uint64_t *tkeys, const int *tperm, int64_t m, int check,
                  int nout, double *out, int64_t ld_out, cudaStream_t s, const EvalItems *pre) {
  if (m == 0) return;
  switch (a.kernel_id) {
    case KERNEL_LAPLACE:
      evaluate_impl<LaplaceF64T>(a, tau_s, loc, txs, tys, tkeys, tperm, m, check, nout, out, ld_out,
                                 s, pre);
      break;
    case KERNEL_MOD_HELMHOLTZ:
      evaluate_impl<ModHelmholtzF64>(a, tau_s, loc, txs, tys, tkeys, tperm, m, check, nout, out,
                                     ld_out, s, pre);
      break;
    case KERNEL_RADIAL_TABLE:
      FMMB_CHECK(nout == 1, ERR_UNSUPPORTED, "tabulated kernels evaluate potentials only");
      evaluate_impl<RadialTableF64>(a, tau_s, loc, txs, tys, tkeys, tperm, m, check, nout, out,
                                    ld_out, s, pre);
      break;
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
}

namespace {
template <class KF, bool DIP>
void evaluate_split_impl(const PassArgs &a, const double *tau_s, const double *loc, int check,
                         double *out, cudaStream_t s, const SplitEval &se) {
  const TreeDev &td = *a.td;
  const int64_t m = a.th->n_points;
  FMMB_CUDA(cudaStreamWaitEvent(se.side, se.ready, 0));
  EvalItems it;
  eval_items(a, td.pkeys.get(), m, it, se.side);
  DevBuf<double> near;
  near.alloc(m, se.side);
  const int64_t units = a.th->n_total() + m / TCH + 1;  // work items, upper bound
  {
    // the SMs keep their largest shared-memory carveout while near-field
    // blocks sit on them, so the level passes' CTAs still fit beside them
    static const bool carveout_set = [] {
      FMMB_CUDA(cudaFuncSetAttribute(k_evaluate<KF, 1, EVAL_NEAR, DIP>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared));
      return true;
    }();
    (void)carveout_set;
    PhaseTimer timer(PH_EVAL, se.side);
    k_evaluate<KF, 1, EVAL_NEAR, DIP><<<work_grid(units, NEAR_BLOCKS_PER_SM), TCH, 0, se.side>>>(
        a.kp, a.neq, a.np, it.items.get(), it.n_items.get(), td.coll.get(), td.bot.get(),
        td.top.get(), td.xmid.get(), td.ymid.get(), td.sx.get(), td.sy.get(), tau_s, a.ops_dev,
        loc, td.sx.get(), td.sy.get(), td.ordv.get(), check, out, 0, near.get(), a.dvx, a.dvy);
    FMMB_CUDA(cudaGetLastError());
  }
  FMMB_CUDA(cudaEventRecord(se.near_done, se.side));
  FMMB_CUDA(cudaStreamWaitEvent(s, se.near_done, 0));
  {
    PhaseTimer timer(PH_EVAL, s);
    k_evaluate<KF, 1, EVAL_FAR><<<work_grid(units, 8), TCH, 0, s>>>(
        a.kp, a.neq, a.np, it.items.get(), it.n_items.get(), td.coll.get(), td.bot.get(),
        td.top.get(), td.xmid.get(), td.ymid.get(), td.sx.get(), td.sy.get(), tau_s, a.ops_dev,
        loc, td.sx.get(), td.sy.get(), td.ordv.get(), check, out, 0, near.get(), nullptr,
        nullptr);
    FMMB_CUDA(cudaGetLastError());
  }
  // the scratch (allocated on the side stream) is freed there once the plan
  // stream is done with it
  FMMB_CUDA(cudaEventRecord(se.far_done, s));
  FMMB_CUDA(cudaStreamWaitEvent(se.side, se.far_done, 0));
}

template <class KF>
void evaluate_multi_impl(const PassArgs &a, const double *tau_s, int64_t n_src, int n_rhs,
                         const double *loc, int64_t col_stride, const double *txs,
                         const double *tys, const uint64_t *tkeys, const int *tperm, int64_t m,
                         int check, double *out, int64_t ld_out, cudaStream_t s) {
  const TreeDev &td = *a.td;
  EvalItems it;
  eval_items(a, tkeys, m, it, s);
  PhaseTimer timer(PH_EVAL, s);
  constexpr int R = 8;
  for (int r0 = 0; r0 < n_rhs; r0 += R) {
    const int ncol = std::min(R, n_rhs - r0);
    k_evaluate_multi<KF, R><<<work_grid(a.th->n_total() + m / TCH + 1, 8), TCH, 0, s>>>(
        a.kp, a.neq, a.np, ncol, it.items.get(), it.n_items.get(), td.coll.get(), td.bot.get(),
        td.top.get(), td.xmid.get(), td.ymid.get(), td.sx.get(), td.sy.get(), tau_s + r0 * n_src,
        n_src, a.ops_dev, loc + r0 * col_stride, col_stride, txs, tys, tperm, check,
        out + r0 * ld_out, ld_out);
    FMMB_CUDA(cudaGetLastError());
  }
}
}  // namespace

void run_evaluate_multi(const PassArgs &a, const double *tau_s, int64_t n_src, int n_rhs,
                        const double *loc, int64_t col_stride, const double *txs, const double *tys,
                        const uint64_t *tkeys, const int *tperm, int64_t m, int check, double *out,
                        int64_t ld_out, cudaStream_t s) {
  if (m == 0 || n_rhs == 0) return;
  switch (a.kernel_id) {
    case KERNEL_LAPLACE:
      evaluate_multi_impl<LaplaceF64T>(a, tau_s, n_src, n_rhs, loc, col_stride, txs, tys, tkeys,
                                      tperm, m, check, out, ld_out, s);
      break;
    case KERNEL_MOD_HELMHOLTZ:
      evaluate_multi_impl<ModHelmholtzF64>(a, tau_s, n_src, n_rhs, loc, col_stride, txs, tys, tkeys,
                                           tperm, m, check, out, ld_out, s);
      break;
    case KERNEL_RADIAL_TABLE:
      evaluate_multi_impl<RadialTableF64>(a, tau_s, n_src, n_rhs, loc, col_stride, txs, tys, tkeys,
                                          tperm, m, check, out, ld_out, s);
      break;
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
}

void run_evaluate_sources_split(const PassArgs &a, const double *tau_s, const double *loc,
                                int check, double *out, cudaStream_t s, const SplitEval &se) {
  if (a.th->n_points == 0) return;
  switch (a.kernel_id) {
    case KERNEL_LAPLACE:
      if (a.dvx)
        evaluate_split_impl<LaplaceF64T, true>(a, tau_s, loc, check, out, s, se);
      else
        evaluate_split_impl<LaplaceF64T, false>(a, tau_s, loc, check, out, s, se);
      break;
    case KERNEL_MOD_HELMHOLTZ:
      FMMB_CHECK(!a.dvx, ERR_UNSUPPORTED, "dipole sources: Laplace kernel only");
      evaluate_split_impl<ModHelmholtzF64, false>(a, tau_s, loc, check, out, s, se);
      break;
    case KERNEL_RADIAL_TABLE:
      FMMB_CHECK(!a.dvx, ERR_UNSUPPORTED, "dipole sources: Laplace kernel only");
      evaluate_split_impl<RadialTableF64, false>(a, tau_s, loc, check, out, s, se);
      break;
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
}

namespace {
template <class KF>
void local_impl(const PassArgs &a, const double *tau_s, const double *txs, const double *tys,
                const uint64_t *tkeys, const int *tperm, int64_t m, int check,
                const int64_t *scat, const int64_t *tcat, double *out, cudaStream_t s) {
  const TreeDev &td = *a.td;
  EvalItems it;
  eval_items(a, tkeys, m, it, s);
  const int grid = work_grid(a.th->n_total() + m / TCH + 1, 8);
  PhaseTimer timer(PH_EVAL, s);
  if (scat)
    k_evaluate<KF, 1, EVAL_NEAR, false, true><<<grid, TCH, 0, s>>>(
        a.kp, a.neq, a.np, it.items.get(), it.n_items.get(), td.coll.get(), td.bot.get(),
        td.top.get(), td.xmid.get(), td.ymid.get(), td.sx.get(), td.sy.get(), tau_s, a.ops_dev,
        nullptr, txs, tys, tperm, check, out, 0, out, nullptr, nullptr, scat, tcat);
  else
    k_evaluate<KF, 1, EVAL_NEAR><<<grid, TCH, 0, s>>>(
        a.kp, a.neq, a.np, it.items.get(), it.n_items.get(), td.coll.get(), td.bot.get(),
        td.top.get(), td.xmid.get(), td.ymid.get(), td.sx.get(), td.sy.get(), tau_s, a.ops_dev,
        nullptr, txs, tys, tperm, check, out, 0, out, nullptr, nullptr, nullptr, nullptr);
  FMMB_CUDA(cudaGetLastError());
}
}  // namespace

void run_local_evaluate(const PassArgs &a, const double *tau_s, const double *txs,
                        const double *tys, const uint64_t *tkeys, const int *tperm, int64_t m,
                        int check, const int64_t *scat, const int64_t *tcat, double *out,
                        cudaStream_t s) {
  if (m == 0) return;
  switch (a.kernel_id) {
    case KERNEL_LAPLACE:
      local_impl<LaplaceF64T>(a, tau_s, txs, tys, tkeys, tperm, m, check, scat, tcat, out, s);
      break;
    case KERNEL_MOD_HELMHOLTZ:
      local_impl<ModHelmholtzF64>(a, tau_s, txs, tys, tkeys, tperm, m, check, scat, tcat, out, s);
      break;
    case KERNEL_RADIAL_TABLE:
      local_impl<RadialTableF64>(a, tau_s, txs, tys, tkeys, tperm, m, check, scat, tcat, out, s);
      break;
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
}

__global__ void k_gather_i64(const int64_t *__restrict__ v, const int *__restrict__ perm, int64_t n,
                             int64_t *__restrict__ o) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    o[i] = v[perm[i]];
}

void gather_sorted_i64(const int64_t *v, const int *perm, int64_t n, int64_t *o, cudaStream_t s) {
  if (n == 0) return;
  k_gather_i64<<<grid_for(n, 256), 256, 0, s>>>(v, perm, n, o);
  FMMB_CUDA(cudaGetLastError());
}

void run_direct(int kernel_id, const KernelParams &kp, const double *sx, const double *sy,
                const double *tau, int64_t ns, const double *tx, const double *ty, int64_t nt,
                int check, double *out, cudaStream_t s) {
  if (nt == 0) return;
  PhaseTimer timer(PH_DIRECT, s);
  const int grid = grid_for(nt, 256, 148 * 64);
  switch (kernel_id) {
    case KERNEL_LAPLACE:
      k_direct<LaplaceF64><<<grid, 256, 0, s>>>(kp, sx, sy, tau, ns, tx, ty, nt, check, out);
      break;
    case KERNEL_MOD_HELMHOLTZ:
      k_direct<ModHelmholtzF64><<<grid, 256, 0, s>>>(kp, sx, sy, tau, ns, tx, ty, nt, check, out);
      break;
    case KERNEL_RADIAL_TABLE:
      k_direct<RadialTableF64><<<grid, 256, 0, s>>>(kp, sx, sy, tau, ns, tx, ty, nt, check, out);
      break;
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
  FMMB_CUDA(cudaGetLastError());
}

size_t evaluate_scratch_bytes(int total_nodes) { return scan_scratch_bytes<int>(total_nodes); }

void run_evaluate_scratch(const PassArgs &a, const double *tau_s, const double *loc,
                          const double *txs, const double *tys, const uint64_t *tkeys,
                          const int *tperm, int64_t m, int check, double *out, int *tb, int *te,
                          int *nch, int *choff, int4 *items, int *n_items, void *temp,
                          size_t temp_bytes, cudaStream_t s) {
  if (m == 0) return;
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  const int total = th.n_total();
  k_leaf_targets<<<grid_for(total, 256), 256, 0, s>>>(total, th.L, td.dev_off.get(), td.code.get(),
                                                      td.flags.get(), tkeys, m, tb, te, nch);
  FMMB_CUDA(cudaGetLastError());
  prefix_sum_run<int, false>(nch, choff, total, temp, temp_bytes, td.sort_fail.get(), true, s);
  k_make_items<<<grid_for(total, 256), 256, 0, s>>>(total, th.L, td.dev_off.get(), tb, te, nch, choff,
                                                    items, n_items, 0);
  FMMB_CUDA(cudaGetLastError());
  PhaseTimer timer(PH_EVAL, s);
  auto launch = [&](auto kern) {
    kern<<<work_grid(total + m / TCH + 1, 8), TCH, 0, s>>>(a.kp, a.neq, a.np, items, n_items,
                                                             td.coll.get(), td.bot.get(),
                                 td.top.get(), td.xmid.get(), td.ymid.get(), td.sx.get(),
                                 td.sy.get(), tau_s, a.ops_dev, loc, txs, tys, tperm, check, out, 0,
                                 nullptr, nullptr, nullptr, nullptr, nullptr);
  };
  switch (a.kernel_id) {
    case KERNEL_LAPLACE: launch(k_evaluate<LaplaceF64T, 1>); break;
    case KERNEL_MOD_HELMHOLTZ: launch(k_evaluate<ModHelmholtzF64, 1>); break;
    case KERNEL_RADIAL_TABLE: launch(k_evaluate<RadialTableF64, 1>); break;
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
  FMMB_CUDA(cudaGetLastError());
}

namespace {
__global__ void k_diag_log2(const double *__restrict__ x, int64_t n, double *__restrict__ out_tab,
                            double *__restrict__ out_lib) {
  __shared__ FunctorSmem<LaplaceF64T> fsm;
  LaplaceF64T K(KernelParams{});
  fsm.bind(K);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double d = x[i];
    out_tab[i] = log2_tab_rare(d) ? log2(d) : log2_tab(d, K.lt);
    out_lib[i] = log2(d);
  }
}
}  // namespace

void run_diag_log2(const double *x, int64_t n, double *out_tab, double *out_lib, cudaStream_t s) {
  if (n == 0) return;
  k_diag_log2<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(x, n, out_tab, out_lib);
  FMMB_CUDA(cudaGetLastError());
}

void gather_sorted(const double *v, const int *perm, int64_t n, double *o, cudaStream_t s) {
  if (n == 0) return;
  k_gather_sorted<<<grid_for(n, 256), 256, 0, s>>>(v, perm, n, o);
  FMMB_CUDA(cudaGetLastError());
}

}  // namespace fmmb
