// Row GEMMs on the FP64 tensor cores for the dense-operator FMM forms
// (black-box, Stokes): every translation there maps node rows of np doubles
// to node rows through a fixed operator,
//
//   Y[row] (=, +=) sum_b X_b(row) . W_b,
//
// with X_b(row) the row's b-th input block (kb doubles: a contiguous row, a
// gathered parent row, or for M2L the source multipole at offset b) and W_b
// rows b kb .. (b+1) kb - 1 of the operator W, row-major [K][ldw].  A block
// computes a 64 x 64 tile of Y with mma.sync.m8n8k4.f64 (FP64 DMMA), staging
// 16-deep K chunks of X and W in shared memory with cp.async, double buffered
// (the next chunk in flight while the current one is multiplied).  An input block
// that no row of the tile reads (an M2L offset absent for the whole tile) is
// skipped: M2L tiles hold rows of one parity class (position inside the
// parent), so the 13 offsets that class never sees cost nothing.
//
// Loaders (row ids of a tile, source of a row's block) and stores (how a
// row's outputs land) are small structs passed by value.
#pragma once
#include "gemm.cuh"

namespace fmmb {
namespace {

constexpr int RG_TM = 64;       // output rows per block
constexpr int RG_TN = 64;       // output columns per block
constexpr int RG_KC = 16;       // K chunk staged per step (4 mma k-steps)
constexpr int RG_THREADS = 256;
constexpr int RG_LDX = 20;      // shared row stride of the X chunk (conflict-free fragments)
constexpr int RG_LDW = 72;      // shared row stride of the W chunk

// ---- loaders ----
// X rows contiguous: row r at base + r * ldx, one input block of kb doubles
struct RowsContig {
  const double *base;
  int64_t ldx;
  int n_rows, kb;
  __device__ int nblk() const { return 1; }
  __device__ int row(int tile, int i) const {
    const int r = tile * RG_TM + i;
    return r < n_rows ? r : -1;
  }
  __device__ const double *src(int r, int) const { return base + r * ldx; }
};

// X row e = the local of the parent of real group e: src[parent[rg[lo + e]]]
struct ParentRows {
  const int *rg, *parent;
  const double *rows;
  int lo, n_groups, np;
  __device__ int nblk() const { return 1; }
  __device__ int row(int tile, int i) const {
    const int e = tile * RG_TM + i;
    return e < n_groups ? e : -1;
  }
  __device__ const double *src(int e, int) const {
    return rows + (size_t)parent[rg[lo + e]] * np;
  }
};

// M2L of one level: row 4 g + c is child c of real group g (node rg[lo+g]+c);
// its input block o is the source multipole at offset o (il), or none.
// Tiles hold one class c: tile = c * tpc + (g / 64).
struct M2LRows {
  const int *rg, *il;
  const double *mult;
  int lo, n_groups, np, tpc;
  __device__ int nblk() const { return N_OFFSETS; }
  __device__ int row(int tile, int i) const {
    const int c = tile / tpc, g = (tile - c * tpc) * RG_TM + i;
    return g < n_groups ? 4 * g + c : -1;
  }
  __device__ const double *src(int r, int o) const {
    const int node = rg[lo + (r >> 2)] + (r & 3);
    const int s = il[(size_t)node * N_OFFSETS + o];
    return s >= 0 ? mult + (size_t)s * np : nullptr;
  }
};

// ---- stores (two consecutive columns) ----
struct StoreRows {  // Y row r at base + r * ld, overwritten
  double *base;
  int64_t ld;
  __device__ void put2(int r, int col, double a, double b) const {
    *reinterpret_cast<double2 *>(base + r * ld + col) = make_double2(a, b);
  }
};

struct StoreParents {  // row e -> dst[parent[c_first + 4 e]], overwritten (M2M)
  const int *parent;
  double *dst;
  int c_first, np;
  __device__ void put2(int e, int col, double a, double b) const {
    *reinterpret_cast<double2 *>(dst + (size_t)parent[c_first + 4 * e] * np + col) =
        make_double2(a, b);
  }
};

struct AddChildRows {  // row e (4 np wide) -> ple rows rg[lo+e] .. +3, added (L2L)
  const int *rg;
  double *ple;
  int lo, np;
  __device__ void put2(int e, int col, double a, double b) const {
    double2 *p = reinterpret_cast<double2 *>(ple + (size_t)rg[lo + e] * np + col);
    const double2 v = *p;
    *p = make_double2(v.x + a, v.y + b);
  }
};

struct AddGroupRows {  // row 4 g + c -> ple[rg[lo+g] + c], added (M2L)
  const int *rg;
  double *ple;
  int lo, np;
  __device__ void put2(int r, int col, double a, double b) const {
    double2 *p =
        reinterpret_cast<double2 *>(ple + (size_t)(rg[lo + (r >> 2)] + (r & 3)) * np + col);
    const double2 v = *p;
    *p = make_double2(v.x + a, v.y + b);
  }
};

template <class Load, class Store>
__global__ void __launch_bounds__(RG_THREADS) k_rowgemm(Load ld, Store st,
                                                       const double *__restrict__ W, int ldw,
                                                       int M, int kb) {
  // two buffers of each chunk: chunk c + 1 of an input block is copied while
  // chunk c is multiplied
  __shared__ __align__(16) double Xs[2][RG_TM * RG_LDX];
  __shared__ __align__(16) double Ws[2][RG_KC * RG_LDW];
  __shared__ int rid[RG_TM];
  __shared__ const double *rsrc[RG_TM];
  const int tile = blockIdx.x, c0 = blockIdx.y * RG_TN;
  if (threadIdx.x < RG_TM) rid[threadIdx.x] = ld.row(tile, threadIdx.x);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  const int r0 = 16 * (warp & 3), cw = 32 * (warp >> 2);
  double acc[2][4][2];
  zero_acc(acc);
  const int nb = ld.nblk(), nch = (kb + RG_KC - 1) / RG_KC;
  for (int blk = 0; blk < nb; ++blk) {
    const double *p = nullptr;
    __syncthreads();  // rid written; rsrc of the previous block read
    if (threadIdx.x < RG_TM) {
      const int r = rid[threadIdx.x];
      p = r >= 0 ? ld.src(r, blk) : nullptr;
      rsrc[threadIdx.x] = p;
    }
    if (!__syncthreads_or(p != nullptr)) continue;  // no row of the tile reads this block
    auto stage = [&](int c) {  // chunk c of this block into buffer c & 1 (one copy group)
      const int k0 = c * RG_KC, bf = c & 1, kn = min(RG_KC, kb - k0);
      // X chunk: 64 rows x RG_KC doubles (rows past kb or without a source: 0)
      for (int i = threadIdx.x; i < RG_TM * (RG_KC / 2); i += RG_THREADS) {
        const int r = i / (RG_KC / 2), pr = 2 * (i - r * (RG_KC / 2));
        const double *s = rsrc[r];
        if (s && pr < kn) {
          cp_async16(&Xs[bf][r * RG_LDX + pr], s + k0 + pr);
        } else {
          Xs[bf][r * RG_LDX + pr] = 0.0;
          Xs[bf][r * RG_LDX + pr + 1] = 0.0;
        }
      }
      // W chunk: RG_KC rows x 64 columns
      for (int i = threadIdx.x; i < RG_KC * (RG_TN / 2); i += RG_THREADS) {
        const int kr = i / (RG_TN / 2), cc = 2 * (i - kr * (RG_TN / 2));
        if (kr < kn && c0 + cc < M) {
          cp_async16(&Ws[bf][kr * RG_LDW + cc], W + (size_t)(blk * kb + k0 + kr) * ldw + c0 + cc);
        } else {
          Ws[bf][kr * RG_LDW + cc] = 0.0;
          Ws[bf][kr * RG_LDW + cc + 1] = 0.0;
        }
      }
      cp_async_commit_group();
    };
    stage(0);
    for (int c = 0; c < nch; ++c) {
      if (c + 1 < nch) {
        stage(c + 1);
        cp_async_wait_group<1>();
      } else {
        cp_async_wait_group<0>();
      }
      __syncthreads();
      const double *X = Xs[c & 1], *Wc = Ws[c & 1];
#pragma unroll
      for (int ks = 0; ks < RG_KC; ks += 4) {
        double a[2], b[4];
#pragma unroll
        for (int rb = 0; rb < 2; ++rb) a[rb] = X[(r0 + 8 * rb + g) * RG_LDX + ks + q];
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) b[cb] = Wc[(ks + q) * RG_LDW + cw + 8 * cb + g];
#pragma unroll
        for (int rb = 0; rb < 2; ++rb)
#pragma unroll
          for (int cb = 0; cb < 4; ++cb) dmma(acc[rb][cb], a[rb], b[cb]);
      }
      __syncthreads();  // buffer c & 1 is refilled by the next iteration's copies
    }
  }
#pragma unroll
  for (int rb = 0; rb < 2; ++rb) {
    const int r = rid[r0 + 8 * rb + g];
    if (r < 0) continue;
#pragma unroll
    for (int cb = 0; cb < 4; ++cb) {
      const int col = c0 + cw + 8 * cb + 2 * q;
      if (col < M) st.put2(r, col, acc[rb][cb][0], acc[rb][cb][1]);
    }
  }
}

// Launch over n_tiles row tiles and all M output columns (M, kb multiples of
// 8; W rows of ldw doubles, 16-byte aligned; every X source 16-byte aligned).
template <class Load, class Store>
void rowgemm(const Load &ld, const Store &st, int n_tiles, const double *W, int ldw, int M, int kb,
             cudaStream_t s) {
  if (n_tiles <= 0 || M <= 0) return;
  FMMB_CHECK(M % 8 == 0 && kb % 8 == 0 && ldw % 2 == 0, ERR_INVALID_ARGUMENT,
             "row GEMM shapes must be multiples of 8");
  k_rowgemm<<<dim3(n_tiles, (M + RG_TN - 1) / RG_TN), RG_THREADS, 0, s>>>(ld, st, W, ldw, M, kb);
  FMMB_CUDA(cudaGetLastError());
}

inline int row_tiles(int n_rows) { return (n_rows + RG_TM - 1) / RG_TM; }

}  // namespace
}  // namespace fmmb
