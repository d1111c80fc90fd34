// Mixed-precision FMM passes: the same tree, operators and pass structure as
// fmm.cu, with FP32 kernel evaluations and split-precision tensor-core GEMMs.
//
//  * S2M, L2T and P2P evaluate the kernel in FP32 on coordinates taken
//    relative to the box centre and divided by its width (the subtraction is
//    done in FP64, so no absolute position error enters; a scale-invariant
//    kernel's constant offset times the charge sum is added in FP64); P2P
//    sums FP32 partials of a few terms into FP64, and a pair that coincides
//    in FP32 is redone in FP64 (so coincident points are
//    skipped exactly as in the reference, flexmm/flexmm2d/helpers.py:99-107);
//  * M2M, M2L and L2L are 3xTF32 tensor-core GEMMs (hi*hi + hi*lo + lo*hi,
//    FP32 accumulate per k-step, partial sums added in FP64) on operators
//    with their mean removed: for an operator
//    B = c*1*1^T + B', B.x = B'.x + c*sum(x), where sum(x) is carried in FP64
//    per box.  The log kernel's operators are dominated by a per-level
//    constant (-log(w^2)/4pi); without the deflation the TF32 rounding of
//    that constant costs an order of magnitude of accuracy;
//  * multipoles and locals are stored as FP32 plus their FP64 component sum;
//  * check-to-equivalent stays FP64 (the FP64 tensor-core tiles of fmm.cu).
// Error against FP64 direct summation on the 1M clustered workload at
// Nequiv 24: ~4e-7 relative L2 (the FP64 path at Nequiv 24: ~2e-7).

#include <cstdlib>
#include <string>

#include "fmm.cuh"
#include "gemm.cuh"
#include "scan.cuh"
#include "tcgen05.cuh"
#include "timing.cuh"

namespace fmmb {
namespace {

constexpr int TN = 32;      // nodes per upward / downward tile
constexpr int TM = 64;      // targets per M2L tile
constexpr int NT = 256;     // threads per tile CTA
constexpr int TCH = 128;    // targets per evaluation work item (= threads)
static_assert(TCH == EVAL_CHUNK, "work items (built in fmm.cu) hold EVAL_CHUNK targets");
constexpr int SMAX = 1024;  // sources staged per evaluation pass
constexpr int EVAL_BLOCKS_PER_SM = 12;  // 40 registers, 17 KB shared memory per block

__constant__ int8_t c_class_off_mx[4][27] = {
    {8, 9, 10, 11, 12, 13, 15, 16, 17, 19, 20, 21, 23, 24, 25, 27, 28, 29, 30, 31, 32, 34, 35, 36, 37, 38, 39},
    {7, 8, 9, 10, 11, 12, 14, 15, 16, 18, 19, 20, 22, 23, 24, 26, 27, 28, 29, 30, 31, 33, 34, 35, 36, 37, 38},
    {1, 2, 3, 4, 5, 6, 8, 9, 10, 11, 12, 13, 15, 16, 17, 19, 20, 21, 23, 24, 25, 27, 28, 29, 30, 31, 32},
    {0, 1, 2, 3, 4, 5, 7, 8, 9, 10, 11, 12, 14, 15, 16, 18, 19, 20, 22, 23, 24, 26, 27, 28, 29, 30, 31}};

// the inverse: class position of offset o in class cls, or -1
__constant__ int8_t c_oi_of_mx[4][40] = {
    {-1, -1, -1, -1, -1, -1, -1, -1, 0, 1, 2, 3, 4, 5, -1, 6, 7, 8, -1, 9, 10, 11, -1, 12, 13, 14, -1, 15, 16, 17, 18, 19, 20, -1, 21, 22, 23, 24, 25, 26},
    {-1, -1, -1, -1, -1, -1, -1, 0, 1, 2, 3, 4, 5, -1, 6, 7, 8, -1, 9, 10, 11, -1, 12, 13, 14, -1, 15, 16, 17, 18, 19, 20, -1, 21, 22, 23, 24, 25, 26, -1},
    {-1, 0, 1, 2, 3, 4, 5, -1, 6, 7, 8, 9, 10, 11, -1, 12, 13, 14, -1, 15, 16, 17, -1, 18, 19, 20, -1, 21, 22, 23, 24, 25, 26, -1, -1, -1, -1, -1, -1, -1},
    {0, 1, 2, 3, 4, 5, -1, 6, 7, 8, 9, 10, 11, -1, 12, 13, 14, -1, 15, 16, 17, -1, 18, 19, 20, -1, 21, 22, 23, 24, 25, 26, -1, -1, -1, -1, -1, -1, -1, -1}};

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// D[16x8] += A[16x8] . B[8x8], TF32 inputs, FP32 accumulate
__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// 3xTF32 warp tile: C[r0 + g (+8)][n0 + 8*cb*nstride + 2q (+1)] += A . B for the
// column blocks below ncols.  A: shared float [.][lda] (split to hi/lo here);
// B: hi/lo float [K][ldb] (pre-split), in global memory or, with SB, staged
// in shared memory.  K multiple of 8.
// The tensor cores' FP32 accumulation does not round to nearest (it behaves
// like truncation, which biases long sums), so every k-step's three products
// go into a fresh zero fragment and the partial sums are accumulated in FP64.
template <int CB, bool SB = false>
__device__ __forceinline__ void warp_gemm_x3(const float *A, int lda, const float *Bh,
                                             const float *Bl, int ldb, int K, int r0,
                                             int n0, int nstride, int ncols, double (&acc)[CB][4]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  for (int k0 = 0; k0 < K; k0 += 8) {
    const float a[4] = {A[(r0 + g) * lda + k0 + q], A[(r0 + g + 8) * lda + k0 + q],
                        A[(r0 + g) * lda + k0 + q + 4], A[(r0 + g + 8) * lda + k0 + q + 4]};
    uint32_t ah[4], al[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      ah[i] = to_tf32(a[i]);
      al[i] = to_tf32(a[i] - __uint_as_float(ah[i]));
    }
#pragma unroll
    for (int cb = 0; cb < CB; ++cb) {
      const int n = n0 + 8 * cb * nstride;
      if (n < ncols) {
        const size_t i0 = (size_t)(k0 + q) * ldb + n + g, i1 = i0 + (size_t)4 * ldb;
        const uint32_t bh0 = __float_as_uint(SB ? Bh[i0] : __ldg(Bh + i0));
        const uint32_t bh1 = __float_as_uint(SB ? Bh[i1] : __ldg(Bh + i1));
        const uint32_t bl0 = __float_as_uint(SB ? Bl[i0] : __ldg(Bl + i0));
        const uint32_t bl1 = __float_as_uint(SB ? Bl[i1] : __ldg(Bl + i1));
        float part[4] = {0.f, 0.f, 0.f, 0.f};
        mma_tf32(part, al, bh0, bh1);
        mma_tf32(part, ah, bl0, bl1);
        mma_tf32(part, ah, bh0, bh1);
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[cb][i] += (double)part[i];
      }
    }
  }
}

__host__ __device__ inline int pad_f(int n) { return n + 4; }  // float rows: stride 4 mod 32 words

// FP64 C2E result rows in shared memory -> FP32 rows + FP64 component sums
// out_tc (optional): the same rows split as TF32 hi, lo ([node][hi np | lo np]),
// the operand format of the tcgen05 M2L
__device__ __forceinline__ void store_mixed(const double *P, int ldp, int np, int neq,
                                            const int *node, int ntile, float *out32,
                                            double *outsum, float *out_tc = nullptr) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int t = warp; t < ntile; t += NT / 32) {
    const int n = node[t];
    if (n < 0) continue;
    double s = 0.0;
    for (int k = lane; k < np; k += 32) {
      const double v = k < neq ? P[t * ldp + k] : 0.0;
      const float f = (float)v;
      out32[(size_t)n * np + k] = f;
      if (out_tc) {
        const float h = __uint_as_float(to_tf32(f));
        out_tc[(size_t)n * 2 * np + k] = h;
        out_tc[(size_t)n * 2 * np + np + k] = __uint_as_float(to_tf32(f - h));
      }
      s += v;
    }
    for (int w = 16; w >= 1; w >>= 1) s += __shfl_xor_sync(0xffffffffu, s, w);
    if (lane == 0) outsum[n] = s;
  }
}

// ---------------------------------------------------------------- upward ----
__device__ __forceinline__ int node_level(const int *__restrict__ off, int L, int g) {
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

// S2M + C2E of every S2M node (leaves holding points) of every level, in one
// launch (flexmm/flexmm2d/kifmm.py:96-105 then fmm.py:86-90).  A tile is TN
// consecutive entries of the level-major node list; C2E runs once for each
// level the tile holds.
template <class KF32>
__global__ void __launch_bounds__(NT) k_s2m_mx(KernelParams kp, int neq, int np, int L,
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
                                               const double *__restrict__ tsum,
                                               const LevelOpsDev *__restrict__ ops,
                                               float *__restrict__ mult32,
                                               double *__restrict__ msum,
                                               float *__restrict__ mult_tc) {
  extern __shared__ double smem[];
  const int ldp = pad_ld(np);
  double *P = smem;          // [TN][ldp] check potentials
  double *T = P + TN * ldp;  // [TN][ldp] C2E scratch
  double *Cs = T + TN * ldp;  // staged C2E operators of one level
  __shared__ float srcx[NT / 32][32], srcy[NT / 32][32], srct[NT / 32][32];
  __shared__ int node[TN], nlev[TN];
  __shared__ double *orow[TN];
  const KF32 K(kp);
  const int n_up = *n_up_ptr;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  for (int i = threadIdx.x; i < TN * ldp; i += NT) T[i] = 0.0;
  for (int tile = blockIdx.x; tile * TN < n_up; tile += gridDim.x) {
    const int i0 = tile * TN, nloc = min(TN, n_up - i0);
    for (int i = threadIdx.x; i < TN * ldp; i += NT) P[i] = 0.0;
    if (threadIdx.x < TN) {
      const int g = (int)threadIdx.x < nloc ? uplist[i0 + threadIdx.x] : -1;
      node[threadIdx.x] = g;
      nlev[threadIdx.x] = g >= 0 ? node_level(off, L, g) : -1;
    }
    __syncthreads();
    const int mlo = nlev[0], mhi = nlev[nloc - 1];
    C2EView cv = c2e_stage(ops[mlo], np, Cs);  // in flight during S2M
    for (int t = warp; t < nloc; t += NT / 32) {
      const int g = node[t];
      const LevelOpsDev &op = ops[nlev[t]];
      const int b = bot[g], e = top[g];
      const double cx = xmid[g], cy = ymid[g], iw = op.inv_w;
      float acc0 = 0.f, acc1 = 0.f;
      const float lx0 = lane < neq ? op.lx32[lane] : 0.f, ly0 = lane < neq ? op.ly32[lane] : 0.f;
      const float lx1 = lane + 32 < neq ? op.lx32[lane + 32] : 0.f;
      const float ly1 = lane + 32 < neq ? op.ly32[lane + 32] : 0.f;
      for (int j0 = b; j0 < e; j0 += 32) {
        const int nj = min(32, e - j0);
        if (lane < nj) {
          srcx[warp][lane] = (float)((sx[j0 + lane] - cx) * iw);
          srcy[warp][lane] = (float)((sy[j0 + lane] - cy) * iw);
          srct[warp][lane] = (float)tau[j0 + lane];
        }
        __syncwarp();
        if (lane < neq)
          for (int j = 0; j < nj; ++j) acc0 = fmaf(K(lx0 - srcx[warp][j], ly0 - srcy[warp][j]), srct[warp][j], acc0);
        if (lane + 32 < neq)
          for (int j = 0; j < nj; ++j) acc1 = fmaf(K(lx1 - srcx[warp][j], ly1 - srcy[warp][j]), srct[warp][j], acc1);
        __syncwarp();
      }
      const double c0 = op.kofs * tsum[g];  // kernel offset times the box's charge, FP64
      if (lane < neq) P[t * ldp + lane] = c0 + (double)acc0;
      if (lane + 32 < neq) P[t * ldp + lane + 32] = c0 + (double)acc1;
    }
    for (int m = mlo; m <= mhi; ++m) {
      __syncthreads();
      if (m > mlo) cv = c2e_stage(ops[m], np, Cs);
      if (threadIdx.x < TN) orow[threadIdx.x] = nlev[threadIdx.x] == m ? P + threadIdx.x * ldp : nullptr;
      cp_async_wait_all();
      __syncthreads();
      c2e_tile<true>(cv, np, P, T, orow);
    }
    __syncthreads();
    store_mixed(P, ldp, np, neq, node, TN, mult32, msum, mult_tc);
    __syncthreads();
  }
}

// M2M + C2E of the parent boxes of level m (flexmm/flexmm2d/fmm.py:91-98):
// TN parent groups per tile; their children are the contiguous node rows
// c_first + 4e .. c_first + 4e + 3 of level m+1.
// P[t] = (M2MC - c) . children + c * sum(children)
template <bool kStageB>
__global__ void __launch_bounds__(NT) k_m2m_mx(int m, int neq, int np, int c_first, int n_groups,
                                               const int *__restrict__ parent,
                                               const LevelOpsDev *__restrict__ ops, float *mult32,
                                               double *msum, float *mult_tc) {
  extern __shared__ double smem[];
  const int ldp = pad_ld(np), lda = pad_f(4 * np), ldb = ldb_f(np);
  double *P = smem;                                    // [TN][ldp] check potentials
  double *T = P + TN * ldp;                            // [TN][ldp] C2E scratch
  double *Cs = T + TN * ldp;                           // staged C2E operators
  float *A = reinterpret_cast<float *>(Cs + c2e_stage_doubles(np));  // [TN][lda] children (FP32)
  float *Bh = A + TN * lda, *Bl = Bh + 4 * np * ldb;  // staged (M2MC - c)^T hi / lo [4np][ldb]
  __shared__ double csum[TN];
  __shared__ int node[TN];
  __shared__ double *orow[TN];
  const LevelOpsDev &op = ops[m];
  const int e0 = blockIdx.x * TN, nloc = min(TN, n_groups - e0);
  // operators and the tile's children multipoles (contiguous rows) in flight together
  const C2EView cv = c2e_stage(op, np, Cs);
  if (kStageB) {
    stage_rows(Bh, ldb, op.m2mct_hi, 4 * np, np);
    stage_rows(Bl, ldb, op.m2mct_lo, 4 * np, np);
  }
  pdl_wait();  // the children's multipoles come from the kernels before
  pdl_trigger();
  const float *Ag = mult32 + (size_t)(c_first + 4 * e0) * np;
  stage_rows(A, lda, Ag, nloc, 4 * np);
  const int rowlen = 4 * np;
  for (int i = threadIdx.x + nloc * rowlen; i < TN * rowlen; i += NT) {
    const int t = i / rowlen, k = i - t * rowlen;
    A[t * lda + k] = 0.f;
  }
  for (int i = threadIdx.x; i < TN * ldp; i += NT) P[i] = T[i] = 0.0;
  if (threadIdx.x < TN) {
    const int t = threadIdx.x;
    const int c0 = c_first + 4 * (e0 + t);
    node[t] = t < nloc ? parent[c0] : -1;
    csum[t] = t < nloc ? (msum[c0] + msum[c0 + 1]) + (msum[c0 + 2] + msum[c0 + 3]) : 0.0;
    orow[t] = P + t * ldp;
  }
  cp_async_wait_all();
  __syncthreads();
  {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, q = lane & 3;
    const int r0 = 16 * (warp & 1), n0 = 8 * (warp >> 1);
    double acc[2][4] = {};
    if (kStageB)
      warp_gemm_x3<2, true>(A, lda, Bh, Bl, ldb, 4 * np, r0, n0, 4, np, acc);
    else
      warp_gemm_x3<2, false>(A, lda, op.m2mct_hi, op.m2mct_lo, np, 4 * np, r0, n0, 4, np, acc);
#pragma unroll
    for (int cb = 0; cb < 2; ++cb)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int t = r0 + g + 8 * h, col = n0 + 32 * cb + 2 * q;
        if (t < nloc && col < np) {
          const double r1 = op.c_m2m * csum[t];
          if (col < neq) P[t * ldp + col] = acc[cb][2 * h] + r1;
          if (col + 1 < neq) P[t * ldp + col + 1] = acc[cb][2 * h + 1] + r1;
        }
      }
  }
  __syncthreads();
  c2e_tile<true>(cv, np, P, T, orow);
  __syncthreads();
  store_mixed(P, ldp, np, neq, node, TN, mult32, msum, mult_tc);
}

// shared memory of k_m2m_mx
size_t m2m_mx_smem(int np, bool stage_b) {
  return sizeof(double) * ((size_t)2 * TN * pad_ld(np) + c2e_stage_doubles(np)) +
         sizeof(float) * ((size_t)TN * pad_f(4 * np) + (stage_b ? (size_t)2 * 4 * np * ldb_f(np) : 0));
}

// largest dynamic shared memory a block may request on this device
size_t smem_optin() {
  int dev = 0, v = 0;
  FMMB_CUDA(cudaGetDevice(&dev));
  FMMB_CUDA(cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  return size_t(v);
}

// ------------------------------------------------------------------- M2L ----
struct M2LTilesMx {
  int n_levels;
  int tile_start[4 * FMM_MAX_LEVELS_DEV + 1];
  int rg_lo[FMM_MAX_LEVELS_DEV];
  int rg_cnt[FMM_MAX_LEVELS_DEV];
};

// 64 targets of one parity class per CTA, 4 warps x 16 target rows; output
// FP64 partial locals = FP32 tensor-core sum + FP64 rank-one terms
__global__ void __launch_bounds__(128) k_m2l_mx(M2LTilesMx tiles, int neq, int np,
                                                const int *__restrict__ rg,
                                                const int *__restrict__ il,
                                                const LevelOpsDev *__restrict__ ops,
                                                const float *__restrict__ mult32,
                                                const double *__restrict__ msum,
                                                double *__restrict__ ple) {
  extern __shared__ float smf[];
  const int ldg = pad_f(np);
  float *G = smf;  // [TM][ldg]
  __shared__ int tgt[TM], srow[TM];
  __shared__ double r1s[TM];
  int slot = 0;
  while (slot + 1 < 4 * tiles.n_levels && tiles.tile_start[slot + 1] <= (int)blockIdx.x) ++slot;
  const int m = slot >> 2, cls = slot & 3;
  const int q0 = TM * (blockIdx.x - tiles.tile_start[slot]);
  const int nloc = min(TM, tiles.rg_cnt[m] - q0);
  if (threadIdx.x < TM)
    tgt[threadIdx.x] = (threadIdx.x < nloc) ? rg[tiles.rg_lo[m] + q0 + threadIdx.x] + cls : -1;
  __syncthreads();
  const LevelOpsDev &op = ops[m];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  double acc[8][4] = {};
  double r1 = 0.0;  // rank-one FP64 sum of target threadIdx.x
  for (int oi = 0; oi < 27; ++oi) {
    const int o = c_class_off_mx[cls][oi];
    if (op.kind[o] == M2L_NULL) continue;
    int src = -1;
    if (threadIdx.x < TM && tgt[threadIdx.x] >= 0) src = il[(size_t)tgt[threadIdx.x] * N_OFFSETS + o];
    if (threadIdx.x < TM) {
      srow[threadIdx.x] = src;
      if (src >= 0) r1 += op.c_m2l[o] * msum[src];
    }
    if (!__syncthreads_or(src >= 0)) continue;
    for (int i = threadIdx.x; i < TM * (np / 4); i += 128) {
      const int t = i / (np / 4), k4 = 4 * (i % (np / 4));
      const int s = srow[t];
      float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
      if (s >= 0) v = *reinterpret_cast<const float4 *>(mult32 + (size_t)s * np + k4);
      *reinterpret_cast<float4 *>(G + t * ldg + k4) = v;
    }
    __syncthreads();
    warp_gemm_x3<8>(G, ldg, op.m2l_hi[o], op.m2l_lo[o], np, np, 16 * warp, 0, 1, np, acc);
    __syncthreads();
  }
  if (threadIdx.x < TM) r1s[threadIdx.x] = r1;
  __syncthreads();
#pragma unroll
  for (int cb = 0; cb < 8; ++cb)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int t = 16 * warp + g + 8 * h, col = 8 * cb + 2 * q;
      if (t < nloc && col < np) {
        double *o = ple + (size_t)tgt[t] * np + col;
        o[0] = col < neq ? acc[cb][2 * h] + r1s[t] : 0.0;
        o[1] = col + 1 < neq ? acc[cb][2 * h + 1] + r1s[t] : 0.0;
      }
    }
}

// ---------------------------------------------------- M2L on tcgen05 ----
// Tiles of 128 targets of one parity class (MMA M = 128).  Per offset, the
// gathered source multipoles (A: 128 x K, read pre-split as TF32 hi / lo
// from the upward pass's mult_tc rows) and the deflated operator (B: N x K,
// N = NP rounded up to 16) sit in shared memory in the K-major 128-byte
// swizzle layout (one 128-byte row per target or operator row, 16-byte
// chunk c of row r at chunk c ^ (r & 7), 8-row groups 1024 bytes apart) and
// are multiplied by tcgen05.mma kind::tf32 into tensor memory.  Producer
// thread r copies target row r's gathered chunks; the swizzle puts a warp's
// 32 rows' chunk k in distinct banks.
//
// Measured at 1M (clustered, Nequiv 24; M2L phase): 0.158 ms with the
// unswizzled core-matrix layout, 0.152 swizzled, 0.131 with the per-tile
// set-up loading whole interaction rows and the operator table once and the
// epilogue reading its k-step slots in one TMEM load.  Per-role clock
// counters show the producers issuing ~1600 cycles per offset (the copies'
// issue, not their waits), with the MMA lane waiting on them ~25% of the
// time.  Tried without gain: copies ordered so consecutive threads take
// consecutive chunks of one row (0.150), sources read from a small hot
// window (same time: not an L2 cost), tile::gather4 TMA loads of the rows
// (0.24), 4 TMEM buffers, a copy lag of 3, per-tile rotation of the offset
// order (0.138), per-warp instead of per-thread mbarrier arrivals (0.138).  Each k-step's three split
// products (lo.hi, hi.lo, hi.hi) go to their own 32 TMEM columns (the tensor
// cores truncate their FP32 accumulation); the k-step slots are added in
// FP32 (round to nearest) and the result into FP64 registers.
//
// Persistent and warp specialised, one CTA per SM walking its tiles:
//   warps 0-3  epilogue: one target row per thread (TMEM lanes 0-127)
//   warps 4-7  producers: cp.async of the operands into a 5-stage ring, a
//              stage announced once the copies 2 offsets later are issued
//   warp 8     lane 0 issues the MMAs
// and they hand over through mbarriers instead of CTA barriers:
//   full[s]   stage s loaded        (128 producer arrivals)
//   sfree[s]  MMAs reading s done   (tcgen05.commit)
//   mdone[b]  TMEM buffer b written (tcgen05.commit)
//   tfree[b]  TMEM buffer b read    (128 epilogue arrivals)
// Use u of the pipeline (a running count of offsets over the CTA's tiles)
// takes stage u % 5 and buffer u % TC_NBUF; each barrier's k-th completion has
// parity k & 1.  Every wait is bounded: one that runs out sets the plan's
// error flag and the CTA stops, after letting its copies and MMAs land.
constexpr int TCM = 128;       // targets per tile = MMA M
constexpr int TC_MAX_NP = 32;  // up to 4 k-steps x 32 TMEM columns per buffer
constexpr int TC_NBUF = 2;     // TMEM accumulator buffers (128 columns each)
constexpr int TC_COLS = 128 * TC_NBUF;  // TMEM columns per CTA (a power of 2)
constexpr int TC_STAGES = 5;   // operand stages in shared memory
// producer: an offset is announced once the copies TC_LAG offsets later are
// issued; a stage is refilled TC_STAGES - TC_LAG - 1 offsets after its MMAs
// could start
constexpr int TC_LAG = 2;
constexpr int TC_EPI = 128, TC_PROD = 128;
constexpr int TC_THREADS = TC_EPI + TC_PROD + 32;
constexpr uint32_t TC_MAX_TRIES = 1u << 20;

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_lag() {
  static_assert(TC_LAG >= 1 && TC_LAG <= 4, "wait_group takes the lag as an immediate");
  if (TC_LAG == 1) asm volatile("cp.async.wait_group 1;\n" ::: "memory");
  if (TC_LAG == 2) asm volatile("cp.async.wait_group 2;\n" ::: "memory");
  if (TC_LAG == 3) asm volatile("cp.async.wait_group 3;\n" ::: "memory");
  if (TC_LAG == 4) asm volatile("cp.async.wait_group 4;\n" ::: "memory");
}

// sum of a TMEM buffer's NK k-step slots (32 columns each), in k order
template <int NK>
__device__ __forceinline__ void tmem_slot_sum(uint32_t taddr, float (&sum)[32]) {
  float v[NK][32];
  tc::tmem_ld32_slots<NK>(taddr, v);
#pragma unroll
  for (int c = 0; c < 32; ++c) {
    float t = v[0][c];
#pragma unroll
    for (int k = 1; k < NK; ++k) t += v[k][c];
    sum[c] = t;
  }
}

// shared memory of one operand stage: A hi, A lo, B hi, B lo (128-byte
// rows, each part 1024-byte aligned)
__host__ __device__ inline uint32_t m2l_tc_a_bytes() { return uint32_t(TCM) * 128u; }
__host__ __device__ inline uint32_t m2l_tc_b_bytes(int np) {
  return ((uint32_t((np + 15) & ~15) * 128u) + 1023u) & ~1023u;
}
// dynamic shared memory: the stages and slack to align them to 1024 bytes
size_t m2l_tc_smem_bytes(int np) {
  return size_t(TC_STAGES) * (2 * m2l_tc_a_bytes() + 2 * m2l_tc_b_bytes(np)) + 1024;
}

__global__ void __launch_bounds__(TC_THREADS, 1) k_m2l_tc(M2LTilesMx tiles, int n_tiles, int neq,
                                                         int np, const int *__restrict__ rg,
                                                         const int *__restrict__ il,
                                                         const LevelOpsDev *__restrict__ ops,
                                                         const float *__restrict__ mult_tc,
                                                         const double *__restrict__ msum,
                                                         double *__restrict__ ple, int *err,
                                                         int *tile_counter) {
  extern __shared__ __align__(1024) unsigned char smraw[];
  __shared__ __align__(8) uint64_t bar_full[TC_STAGES], bar_sfree[TC_STAGES];
  __shared__ __align__(8) uint64_t bar_mdone[TC_NBUF], bar_tfree[TC_NBUF], bar_drain;
  __shared__ uint32_t tmem_base;
  __shared__ int s_src[27][TCM];  // source node per class offset and target row
  __shared__ int s_act[27];       // offsets with work, in class order
  __shared__ const float *s_bop[2][N_OFFSETS];  // the level's operators (hi, lo) per offset
  __shared__ double s_c[N_OFFSETS];             // and their means
  __shared__ int s_nact;
  __shared__ unsigned int s_mask;
  __shared__ volatile int s_abort;
  __shared__ int s_tile;
  const int tid = threadIdx.x, warp = tid >> 5;
  const int ntc = (np + 15) & ~15;
  const int nks = np / 8, nk4 = np / 4;
  const uint32_t a_sz = m2l_tc_a_bytes(), b_sz = m2l_tc_b_bytes(np);
  const uint32_t st_sz = 2 * a_sz + 2 * b_sz;
  // the stages, 1024-byte aligned (the swizzle follows address bits 4-9)
  unsigned char *const stages = smraw + ((1024u - (tc::smem_u32(smraw) & 1023u)) & 1023u);
  if (warp == 0) tc::tmem_alloc(tc::smem_u32(&tmem_base), TC_COLS);
  if (tid == 0) {
    for (int st = 0; st < TC_STAGES; ++st) {
      tc::mbar_init(tc::smem_u32(&bar_full[st]), TC_PROD);
      tc::mbar_init(tc::smem_u32(&bar_sfree[st]), 1);
    }
    for (int b = 0; b < TC_NBUF; ++b) {
      tc::mbar_init(tc::smem_u32(&bar_mdone[b]), 1);
      tc::mbar_init(tc::smem_u32(&bar_tfree[b]), TC_EPI);
    }
    tc::mbar_init(tc::smem_u32(&bar_drain), 1);
    tc::fence_mbar_init();
    s_mask = 0u;
    s_abort = 0;
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = tmem_base;
  const uint32_t idesc = tc::idesc_tf32(TCM, ntc);
  const int units = ntc * nk4;  // 16-byte chunks of one B part
  auto fail = [&] {
    s_abort = 1;
    atomicExch(err, 1);
  };
  uint32_t gu = 0;  // pipeline uses before the current tile
  // tiles handed out dynamically (their offset counts differ): the first
  // one is blockIdx.x, the next ones come from a counter
  for (int tile = blockIdx.x; tile < n_tiles;) {
    int slot = 0;
    while (slot + 1 < 4 * tiles.n_levels && tiles.tile_start[slot + 1] <= tile) ++slot;
    const int m = slot >> 2, cls = slot & 3;
    const int q0 = TCM * (tile - tiles.tile_start[slot]);
    const int nloc = min(TCM, tiles.rg_cnt[m] - q0);
    const LevelOpsDev &op = ops[m];
    int tg = -1;
    if (tid < TC_EPI) {
      // this tile's offsets that have an operator and a source for some
      // target, and every target's source per offset: the target's whole
      // interaction row in ten 16-byte loads, the class's 27 kept
      tg = tid < nloc ? rg[tiles.rg_lo[m] + q0 + tid] + cls : -1;
      if (tid < 2 * N_OFFSETS) {  // the operators' addresses and means, beside the loads
        const int o = tid % N_OFFSETS;
        s_bop[tid / N_OFFSETS][o] = tid < N_OFFSETS ? op.m2l_tc_hi[o] : op.m2l_tc_lo[o];
        if (tid < N_OFFSETS) s_c[o] = op.c_m2l[o];
      }
      const int4 *ilr = reinterpret_cast<const int4 *>(il + (size_t)max(tg, 0) * N_OFFSETS);
      unsigned int mask = 0;
#pragma unroll
      for (int i = 0; i < N_OFFSETS / 4; ++i) {
        const int4 q4 = tg >= 0 ? __ldg(ilr + i) : make_int4(-1, -1, -1, -1);
        const int q[4] = {q4.x, q4.y, q4.z, q4.w};
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int o = 4 * i + j, oi = c_oi_of_mx[cls][o];
          if (oi >= 0) {
            const int v = __ldg(&op.kind[o]) != M2L_NULL ? q[j] : -1;
            s_src[oi][tid] = v;
            if (v >= 0) mask |= 1u << oi;
          }
        }
      }
      mask = __reduce_or_sync(0xffffffffu, mask);
      if ((tid & 31) == 0) atomicOr(&s_mask, mask);
    }
    __syncthreads();
    if (tid == 0) {
      int n = 0;
      for (int oi = 0; oi < 27; ++oi)
        if ((s_mask >> oi) & 1u) s_act[n++] = oi;
      s_nact = n;
      s_mask = 0u;
    }
    __syncthreads();
    const int nact = s_nact;
    if (tid < TC_EPI) {
      // ---- epilogue: TMEM -> FP32 slot sum -> FP64 ----
      double acc[32];
#pragma unroll
      for (int c = 0; c < 32; ++c) acc[c] = 0.0;
      // charge-sum terms c_o * sum(source) first: independent loads, off the
      // TMEM loop's path
      double r1 = 0.0;
#pragma unroll 4
      for (int a = 0; a < nact; ++a) {
        const int oi = s_act[a], src = s_src[oi][tid];
        if (src >= 0) r1 += s_c[c_class_off_mx[cls][oi]] * __ldg(msum + src);
      }
      for (int a = 0; a < nact; ++a) {
        if (__any_sync(0xffffffffu, s_abort)) break;
        const uint32_t u = gu + a, b = u % TC_NBUF;
        const bool ok = tc::mbar_wait(tc::smem_u32(&bar_mdone[b]), (u / TC_NBUF) & 1u, TC_MAX_TRIES);
        if (!__all_sync(0xffffffffu, ok)) {
          fail();
          break;
        }
        tc::fence_after_sync();
        float sum[32];
        const uint32_t ta = tmem + (uint32_t(32 * warp) << 16) + b * 128u;
        if (nks == 3) {  // Nequiv 21-24: the three k-step slots in one load
          tmem_slot_sum<3>(ta, sum);
        } else {  // added in k order either way
          for (int ks = 0; ks < nks; ++ks) {
            float v[32];
            tc::tmem_ld32(ta + uint32_t(ks * 32), v);
#pragma unroll
            for (int c = 0; c < 32; ++c) sum[c] = ks == 0 ? v[c] : sum[c] + v[c];
          }
        }
        tc::fence_before_sync();
        tc::mbar_arrive(tc::smem_u32(&bar_tfree[b]));
#pragma unroll
        for (int c = 0; c < 32; ++c) acc[c] += (double)sum[c];
      }
      if (tg >= 0) {
        double *o = ple + (size_t)tg * np;
#pragma unroll
        for (int c = 0; c < 32; ++c)
          if (c < np) o[c] = c < neq ? acc[c] + r1 : 0.0;
      }
    } else if (tid < TC_EPI + TC_PROD) {
      // ---- producers: row r of A (hi, lo) and a share of B per offset ----
      const int r = tid - TC_EPI;
      int a = 0;
      for (; a < nact; ++a) {
        if (s_abort) break;
        const uint32_t u = gu + a, st = u % TC_STAGES;
        if (u >= TC_STAGES &&
            !tc::mbar_wait(tc::smem_u32(&bar_sfree[st]), ((u / TC_STAGES) - 1) & 1u, TC_MAX_TRIES)) {
          fail();
          break;
        }
        const int oi = s_act[a], o = c_class_off_mx[cls][oi];
        unsigned char *sp = stages + st * st_sz;
        // row r of A (hi, lo): its 16-byte chunks to swizzled positions
        const int src = s_src[oi][r];
        for (int k4 = 0; k4 < nk4; ++k4) {
          unsigned char *dh = sp + tc::sw128_offset(r, k4), *dl = dh + a_sz;
          if (src >= 0) {
            cp_async16(dh, mult_tc + (size_t)src * 2 * np + 4 * k4);
            cp_async16(dl, mult_tc + (size_t)src * 2 * np + np + 4 * k4);
          } else {
            *reinterpret_cast<float4 *>(dh) = make_float4(0.f, 0.f, 0.f, 0.f);
            *reinterpret_cast<float4 *>(dl) = make_float4(0.f, 0.f, 0.f, 0.f);
          }
        }
        for (int q = r; q < 2 * units; q += TC_PROD) {
          const int part = q >= units, qq = part ? q - units : q;
          const int n = qq / nk4, k4 = qq - (qq / nk4) * nk4;
          const float *bsrc = s_bop[part][o];
          cp_async16(sp + 2 * a_sz + part * b_sz + tc::sw128_offset(n, k4), bsrc + (size_t)n * np + 4 * k4);
        }
        cp_async_commit();
        if (a >= TC_LAG) {  // the copies of offset a - TC_LAG have landed: announce them
          cp_async_wait_lag();
          tc::fence_proxy_async();
          tc::mbar_arrive(tc::smem_u32(&bar_full[(u - TC_LAG) % TC_STAGES]));
        }
      }
      cp_async_wait_all();
      if (a == nact) {  // announce the offsets still unannounced
        tc::fence_proxy_async();
        for (int b = max(0, nact - TC_LAG); b < nact; ++b)
          tc::mbar_arrive(tc::smem_u32(&bar_full[(gu + uint32_t(b)) % TC_STAGES]));
      }
    } else if (tid == TC_EPI + TC_PROD) {
      // ---- MMA issue ----
      for (int a = 0; a < nact; ++a) {
        if (s_abort) break;
        const uint32_t u = gu + a, st = u % TC_STAGES, b = u % TC_NBUF;
        if (!tc::mbar_wait(tc::smem_u32(&bar_full[st]), (u / TC_STAGES) & 1u, TC_MAX_TRIES)) {
          fail();
          break;
        }
        if (u >= uint32_t(TC_NBUF) &&
            !tc::mbar_wait(tc::smem_u32(&bar_tfree[b]), ((u / TC_NBUF) - 1) & 1u, TC_MAX_TRIES)) {
          fail();
          break;
        }
        tc::fence_after_sync();
        unsigned char *sp = stages + st * st_sz;
        for (int ks = 0; ks < nks; ++ks) {
          const uint32_t d = tmem + b * 128u + uint32_t(ks * 32);
#pragma unroll
          for (int p = 0; p < 3; ++p) {  // lo.hi, hi.lo, hi.hi
            const int apart = p == 0 ? 1 : 0, bpart = p == 1 ? 1 : 0;
            const uint64_t ad = tc::desc_sw128(tc::smem_u32(sp + apart * a_sz) + ks * 32u);
            const uint64_t bd = tc::desc_sw128(tc::smem_u32(sp + 2 * a_sz + bpart * b_sz) + ks * 32u);
            tc::mma_tf32(d, ad, bd, idesc, p > 0 ? 1u : 0u);
          }
        }
        tc::commit(tc::smem_u32(&bar_mdone[b]));
        tc::commit(tc::smem_u32(&bar_sfree[st]));
      }
    }
    gu += uint32_t(nact);
    if (tid == 0) s_tile = int(gridDim.x) + atomicAdd(tile_counter, 1);
    __syncthreads();
    if (s_abort) break;
    tile = s_tile;
  }
  // every MMA issued has completed before the tensor memory is freed (the
  // epilogue waited for each one; after a run-out this drains them)
  if (tid == TC_EPI + TC_PROD) {
    tc::commit(tc::smem_u32(&bar_drain));
    tc::mbar_wait(tc::smem_u32(&bar_drain), 0u, TC_MAX_TRIES);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, TC_COLS);
}

// -------------------------------------------------------------- downward ----
template <bool kStageB>
__global__ void __launch_bounds__(NT) k_downward_mx(int m, int neq, int np, int rg_lo, int rg_cnt,
                                                    const int *__restrict__ rg,
                                                    const int *__restrict__ parent,
                                                    const LevelOpsDev *__restrict__ ops,
                                                    const double *__restrict__ ple,
                                                    float *__restrict__ loc32,
                                                    double *__restrict__ lsum) {
  extern __shared__ double smem[];
  const int ldp = pad_ld(np), ldl = pad_f(np), ldb = ldb_f(4 * np);
  double *P = smem;                                      // [32][ldp] partial locals
  double *T = P + TN * ldp;                              // [32][ldp] C2E scratch
  double *Cs = T + TN * ldp;                             // staged C2E operators
  float *Lp = reinterpret_cast<float *>(Cs + c2e_stage_doubles(np));  // [16][ldl] parent locals
  float *Bh = Lp + 16 * ldl, *Bl = Bh + np * ldb;       // staged (M2MC - c) hi / lo [np][ldb]
  __shared__ int node[TN];
  __shared__ double *orow[TN];
  __shared__ double psum[8];
  const LevelOpsDev &op = ops[m];
  const int q0 = 8 * blockIdx.x;
  const int ngrp = min(8, rg_cnt - q0);
  // operators in flight while the node indices and locals are read
  const C2EView cv = c2e_stage(op, np, Cs);
  if (kStageB && m >= 3) {
    stage_rows(Bh, ldb, ops[m - 1].m2mc_hi, np, 4 * np);
    stage_rows(Bl, ldb, ops[m - 1].m2mc_lo, np, 4 * np);
  }
  if (threadIdx.x < TN) {
    const int grp = threadIdx.x >> 2;
    node[threadIdx.x] = (grp < ngrp) ? rg[rg_lo + q0 + grp] + int(threadIdx.x & 3) : -1;
    orow[threadIdx.x] = P + threadIdx.x * ldp;
  }
  pdl_wait();  // M2L results and the parents' locals come from the kernels before
  pdl_trigger();
  __syncthreads();
  for (int i = threadIdx.x; i < TN * np; i += NT) {
    const int t = i / np, k = i % np;
    P[t * ldp + k] = (node[t] >= 0) ? ple[(size_t)node[t] * np + k] : 0.0;
    T[t * ldp + k] = 0.0;
  }
  for (int i = threadIdx.x; i < 16 * ldl; i += NT) Lp[i] = 0.f;
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
  if (m >= 3) {
    const LevelOpsDev &opp = ops[m - 1];
    for (int i = threadIdx.x; i < 8 * np; i += NT) {
      const int grp = i / np, k = i % np;
      const int n0 = node[4 * grp];
      Lp[grp * ldl + k] = (n0 >= 0) ? loc32[(size_t)parent[n0] * np + k] : 0.f;
    }
    if (threadIdx.x < 8) {
      const int n0 = node[4 * threadIdx.x];
      psum[threadIdx.x] = (n0 >= 0) ? lsum[parent[n0]] : 0.0;
    }
    cp_async_wait_all();
    __syncthreads();
    // L2L: [8 parents][4np] = Lp . (M2MC - c) + c * sum(Lp)   (flexmm/flexmm2d/fmm.py:140-147)
    double acc[4][4] = {};
    if (kStageB)
      warp_gemm_x3<4, true>(Lp, ldl, Bh, Bl, ldb, np, 0, 8 * warp, 8, 4 * np, acc);
    else
      warp_gemm_x3<4, false>(Lp, ldl, opp.m2mc_hi, opp.m2mc_lo, 4 * np, np, 0, 8 * warp, 8, 4 * np,
                             acc);
    if (g < 8) {
#pragma unroll
      for (int cb = 0; cb < 4; ++cb) {
        const int col = 8 * warp + 64 * cb + 2 * q;
        if (col < 4 * np) {
          const int c = col / np, i = col % np;
          const double r1 = opp.c_m2m * psum[g];
          if (i < neq) P[(4 * g + c) * ldp + i] += acc[cb][0] + r1;
          if (i + 1 < neq) P[(4 * g + c) * ldp + i + 1] += acc[cb][1] + r1;
        }
      }
    }
  }
  cp_async_wait_all();
  __syncthreads();
  c2e_tile<true>(cv, np, P, T, orow);
  __syncthreads();
  store_mixed(P, ldp, np, neq, node, TN, loc32, lsum);
}

// ------------------------------------------------------------ evaluation ----
// Per work item, everything the evaluation reads before its first source:
// the leaf's centre, its colleagues' charge sum and source ranges.  Built by
// one thread per item, so the evaluation kernel starts an item with a single
// coalesced 128-byte read (prefetched during the previous item).
struct __align__(16) EvalDesc {
  double cx, cy, csrc;
  int g, lev, t0, cnt;
  int rb[9];   // first sorted source of each colleague
  int rs[10];  // exclusive prefix of the colleagues' source counts
  int multi;   // the leaf's targets fill several items (one thread per target)
  int pad[2];
};
static_assert(sizeof(EvalDesc) == 128, "EvalDesc is read as 32 words");

__global__ void k_eval_desc(const int4 *__restrict__ items, const int *__restrict__ n_items_ptr,
                            const int *__restrict__ coll, const int *__restrict__ bot,
                            const int *__restrict__ top, const double *__restrict__ xmid,
                            const double *__restrict__ ymid, const double *__restrict__ tsum,
                            EvalDesc *__restrict__ desc) {
  const int n_items = *n_items_ptr;
  for (int item = blockIdx.x * blockDim.x + threadIdx.x; item < n_items;
       item += gridDim.x * blockDim.x) {
    const int4 it = items[item];
    EvalDesc d;
    d.g = it.x;
    d.lev = it.y & EVAL_LEVEL_MASK;
    d.multi = (it.y & EVAL_MULTI) ? 1 : 0;
    d.t0 = it.z;
    d.cnt = it.w;
    d.cx = xmid[it.x];
    d.cy = ymid[it.x];
    double cs = 0.0;
    int acc = 0;
    d.rs[0] = 0;
#pragma unroll
    for (int c = 0; c < 9; ++c) {
      const int cg = coll[(size_t)it.x * 9 + c];
      const int b = cg >= 0 ? bot[cg] : 0, n = cg >= 0 ? top[cg] - b : 0;
      if (cg >= 0) cs += tsum[cg];
      d.rb[c] = b;
      acc += n;
      d.rs[c + 1] = acc;
    }
    d.csrc = cs;
    d.pad[0] = d.pad[1] = 0;
    desc[item] = d;
  }
}

// reciprocal on the special-function unit, denormals flushed
__device__ __forceinline__ float rcp_ftz(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// P2P pairs are summed in FP32 over at most 4 x 8 terms per thread, then in
// FP64 (cascaded summation: the FP32 rounding stays relative to short partial
// sums); the kernel offset terms are added in FP64.  NOUT = 1: potential;
// NOUT = 3: potential and its gradient in the target position (rows of out,
// stride ld_out); the gradient is summed on width-scaled coordinates and
// scaled by 1/w in FP64.
// PART: EVAL_FULL (L2T + P2P), EVAL_NEAR (P2P and its kernel-offset term
// only, into near[], caller's point order) or EVAL_FAR (L2T and its offset
// term only, plus near[]: out = far + near).
// resident blocks per SM the evaluation is built for (its register budget):
// the K0 polynomials need more registers than the log kernel's one log2
template <class KF32>
struct EvalOcc {
  static constexpr int blocks = EVAL_BLOCKS_PER_SM;
};
template <>
struct EvalOcc<ModHelmholtzF32> {
  static constexpr int blocks = 8;
};

template <class KF32, class KF64, int NOUT, int PART = EVAL_FULL>
__global__ void __launch_bounds__(TCH, NOUT == 1 ? EvalOcc<KF32>::blocks : 6)
    k_evaluate_mx(KernelParams kp, int neq, int np, const EvalDesc *__restrict__ desc,
                  const int *__restrict__ n_items_ptr, const double *__restrict__ sx,
                  const double *__restrict__ sy, const double *__restrict__ tau,
                  const LevelOpsDev *__restrict__ ops, const float *__restrict__ loc32,
                  const double *__restrict__ lsum, const double *__restrict__ txs,
                  const double *__restrict__ tys, const int *__restrict__ tperm, int check,
                  int self_eval, double *__restrict__ out, int64_t ld_out,
                  int *__restrict__ next_item, double *__restrict__ near = nullptr,
                  const int *hold = nullptr) {
  static_assert(PART == EVAL_FULL || NOUT == 1, "split evaluation: potential only");
  __shared__ EvalDesc D;
  __shared__ float4 src[SMAX];  // (x, y, charge, sorted index) in width units of the leaf
  // NOUT = 3: the low parts of the source coordinates (x = hi + lo): the
  // gradient is dominated by the closest pairs, whose FP32 differences would
  // otherwise lose the digits below 2^-24 of the leaf width
  __shared__ float2 src_lo[NOUT == 3 ? SMAX : 1];
  __shared__ double red[NOUT][TCH / 32];
  __shared__ int s_next, s_pair;
  const KF32 K(kp);
  const KF64 K64(kp);
  const int n_items = *n_items_ptr;
  const int *dw = reinterpret_cast<const int *>(desc);
  // items are handed out dynamically: the block works on `item`, holds the
  // descriptor of `nxt` in registers and fetches the index after that.
  // With `hold` (a near field that pauses and resumes in a second launch)
  // every item is claimed from the counter, and none while *hold is set.
  auto claim = [&]() -> int {
    if (*reinterpret_cast<const volatile int *>(hold)) return n_items;
    return atomicAdd(next_item, 1);
  };
  int item = blockIdx.x, nxt = blockIdx.x + gridDim.x;
  if (hold) {
    if (threadIdx.x == 0) {
      const int a = claim();
      s_next = a;
      s_pair = a < n_items ? claim() : n_items;
    }
    __syncthreads();
    item = s_next;
    nxt = s_pair;
    __syncthreads();
  }
  int nextw = 0;
  if (item < n_items && threadIdx.x < 32) nextw = __ldg(dw + (size_t)item * 32 + threadIdx.x);
  while (item < n_items) {
    if (threadIdx.x < 32) reinterpret_cast<int *>(&D)[threadIdx.x] = nextw;
    __syncthreads();
    if (nxt < n_items && threadIdx.x < 32) nextw = __ldg(dw + (size_t)nxt * 32 + threadIdx.x);
    int after = 0;
    if (threadIdx.x == 0)
      after = hold ? (nxt < n_items ? claim() : n_items) : atomicAdd(next_item, 1) + 2 * gridDim.x;
    const int g = D.g, lev = D.lev, t0 = D.t0, cnt = D.cnt;
    const int ns = PART == EVAL_FAR ? 0 : D.rs[9];
    int G = 1;
    if (!D.multi)
      while (2 * G * cnt <= TCH) G *= 2;
    const int t = threadIdx.x / G, sub = threadIdx.x % G;
    const bool valid = t < cnt;
    const double cx = D.cx, cy = D.cy;
    const double iw = ops[lev].inv_w, kofs = ops[lev].kofs;
    const double x = valid ? txs[t0 + t] : cx, y = valid ? tys[t0 + t] : cy;
    const double txd = (x - cx) * iw, tyd = (y - cy) * iw;
    const float tx = (float)txd, ty = (float)tyd;
    const float tx_lo = (float)(txd - (double)tx), ty_lo = (float)(tyd - (double)ty);
    double acc = 0.0, accx = 0.0, accy = 0.0;  // accx, accy: kScale * (dx, dy) / d2 sums
    if (lev >= 2 && valid && PART != EVAL_NEAR) {  // L2T (flexmm/flexmm2d/kifmm.py:106-120), operands through L1
      const float *Lg = loc32 + (size_t)g * np;
      const float *lx = ops[lev].lx32, *ly = ops[lev].ly32;
      if constexpr (NOUT == 1) {
        float p0 = 0.f, p1 = 0.f;
        int k = sub;
        for (; k + G < neq; k += 2 * G) {
          p0 = fmaf(K(tx - __ldg(lx + k), ty - __ldg(ly + k)), __ldg(Lg + k), p0);
          p1 = fmaf(K(tx - __ldg(lx + k + G), ty - __ldg(ly + k + G)), __ldg(Lg + k + G), p1);
        }
        if (k < neq) p0 = fmaf(K(tx - __ldg(lx + k), ty - __ldg(ly + k)), __ldg(Lg + k), p0);
        acc = (double)p0 + (double)p1;
      } else {
        float p0 = 0.f, px = 0.f, py = 0.f;
        for (int k = sub; k < neq; k += G) {
          const float dx = tx - __ldg(lx + k), dy = ty - __ldg(ly + k);
          const float d2 = fmaf(dy, dy, dx * dx);
          const float q = __ldg(Lg + k) * KF32::kScale;
          p0 = fmaf(K.radial(d2), q, p0);
          const float qr = rcp_ftz(d2) * q;
          px = fmaf(dx, qr, px);
          py = fmaf(dy, qr, py);
        }
        acc = (double)p0;
        accx = (double)px;
        accy = (double)py;
      }
    }
    // P2P (flexmm/flexmm2d/helpers.py:152-194): branch-free FP32 sweep with
    // the kernel's scale folded into the staged charges.  A pair closer than
    // FLT_MIN in squared width units (coincident in FP32) contributes 0 there
    // and is redone in FP64 on the exact coordinates: the one such pair a
    // thread meets (a source evaluated at itself) directly, more by a rescan.
    double exact = 0.0, exact_x = 0.0, exact_y = 0.0;
    // source evaluation (targets are the tree's sorted sources): the range
    // [own_lo, own_lo + own_n) of the item's concatenated sources that holds
    // its targets, and this target's own index there
    int own = -1, own_lo = 0, own_n = 0;
    if (self_eval) {
#pragma unroll
      for (int c = 0; c < 9; ++c) {
        const int n = D.rs[c + 1] - D.rs[c];
        if (t0 >= D.rb[c] && t0 < D.rb[c] + n) {
          own_lo = D.rs[c];
          own_n = n;
          if (valid && t0 + t < D.rb[c] + n) own = D.rs[c] + (t0 + t - D.rb[c]);
        }
      }
    }
    // untested sweeps first, except where most targets coincide with a
    // source that is not known by index (general-path source evaluation)
    const bool fast = self_eval || !check;
    for (int base = 0; base < ns; base += SMAX) {
      const int nb = min(SMAX, ns - base);
      if (base > 0) __syncthreads();  // previous chunk fully read
      for (int i = threadIdx.x; i < nb; i += TCH) {
        const int idx = base + i;
        int c = 0;
#pragma unroll
        for (int k = 1; k < 9; ++k) c += (idx >= D.rs[k]);
        const int j = D.rb[c] + (idx - D.rs[c]);
        const double qx = (sx[j] - cx) * iw, qy = (sy[j] - cy) * iw;
        src[i] = make_float4((float)qx, (float)qy, (float)tau[j] * KF32::kScale, __int_as_float(j));
        if constexpr (NOUT == 3)
          src_lo[i] = make_float2((float)(qx - (double)(float)qx), (float)(qy - (double)(float)qy));
      }
      __syncthreads();
      if (valid) {
        // a coincident pair: the source's kernel offset is already in csrc:
        // take it out and add the FP64 kernel unless the points coincide
        // exactly (check)
        auto fix = [&](int jj) {
          const int q = __float_as_int(src[jj].w);
          const double qx = sx[q], qy = sy[q];
          exact -= kofs * tau[q];
          if (!(check && x - qx == 0.0 && y - qy == 0.0)) {
            if constexpr (NOUT == 1)
              exact += K64(qx, qy, x, y) * tau[q];
            else
              K64.grad(qx, qy, x, y, tau[q], exact, exact_x, exact_y);
          }
        };
        // Fast sweep, no pair tests: a pair closer than FLT_MIN (squared,
        // width units) makes the flushed log2 (and reciprocal) infinite, so a
        // non-finite sum sends the chunk to the tested sweep below.  In source
        // evaluation the own leaf's range [sa, sb) is swept last, rotated so
        // that each thread starts after its own point and never meets it; the
        // other ranges have bounds common to all threads (no divergence).
        static_assert(KF32::kInfAtZero, "the fast sweep needs radial(d2 < FLT_MIN) = +-inf");
        const int sa = own_lo - base, sb = sa + own_n;
        const bool rot = own >= 0 && sa >= 0 && sb <= nb;
        const int o = own - base - sa;  // own point within [sa, sb)
        const double acc0 = acc, accx0 = accx, accy0 = accy;
        if (fast) {
          if constexpr (NOUT == 1) {
            float p0 = 0.f, p1 = 0.f, p2 = 0.f, p3 = 0.f;
            auto pair = [&](const float4 q, float &p) {
              const float dx = tx - q.x, dy = ty - q.y;
              p = fmaf(K.radial(fmaf(dy, dy, dx * dx)), q.z, p);
            };
            auto flush = [&] {
              acc += ((double)p0 + (double)p1) + ((double)p2 + (double)p3);
              p0 = p1 = p2 = p3 = 0.f;
            };
            auto sweep = [&](int lo, int hi) {
              int j = lo + sub, nsum = 0;
              for (; j + 3 * G < hi; j += 4 * G) {
                pair(src[j], p0);
                pair(src[j + G], p1);
                pair(src[j + 2 * G], p2);
                pair(src[j + 3 * G], p3);
                if (++nsum == 8) {
                  flush();
                  nsum = 0;
                }
              }
              for (; j < hi; j += G) pair(src[j], p0);
              flush();
            };
            if (rot) {
              sweep(0, sa);
              sweep(sb, nb);
              // own leaf: offsets 1 .. own_n-1 from the own point, cyclically
              int k = sub + 1;
              for (; k + G < own_n; k += 2 * G) {
                int j0 = o + k, j1 = o + k + G;
                j0 -= j0 >= own_n ? own_n : 0;
                j1 -= j1 >= own_n ? own_n : 0;
                pair(src[sa + j0], p0);
                pair(src[sa + j1], p1);
              }
              if (k < own_n) {
                int j0 = o + k;
                j0 -= j0 >= own_n ? own_n : 0;
                pair(src[sa + j0], p2);
              }
              flush();
            } else {
              sweep(0, nb);
            }
          } else {
            float p[2] = {0.f, 0.f}, px[2] = {0.f, 0.f}, py[2] = {0.f, 0.f};
            auto pair = [&](int jj, int a) {
              const float4 q = src[jj];
              const float2 ql = src_lo[jj];
              const float dx = (tx - q.x) + (tx_lo - ql.x), dy = (ty - q.y) + (ty_lo - ql.y);
              const float d2 = fmaf(dy, dy, dx * dx);
              p[a] = fmaf(K.radial(d2), q.z, p[a]);
              const float qr = rcp_ftz(d2) * q.z;
              px[a] = fmaf(dx, qr, px[a]);
              py[a] = fmaf(dy, qr, py[a]);
            };
            auto flush = [&] {
              acc += (double)p[0] + (double)p[1];
              accx += (double)px[0] + (double)px[1];
              accy += (double)py[0] + (double)py[1];
              p[0] = p[1] = px[0] = px[1] = py[0] = py[1] = 0.f;
            };
            auto sweep = [&](int lo, int hi) {
              int j = lo + sub, nsum = 0;
              for (; j + G < hi; j += 2 * G) {
                pair(j, 0);
                pair(j + G, 1);
                if (++nsum == 16) {
                  flush();
                  nsum = 0;
                }
              }
              if (j < hi) pair(j, 0);
              flush();
            };
            if (rot) {
              sweep(0, sa);
              sweep(sb, nb);
              for (int k = sub + 1; k < own_n; k += G) {
                int j0 = o + k;
                j0 -= j0 >= own_n ? own_n : 0;
                pair(sa + j0, (k / G) & 1);
              }
              flush();
            } else {
              sweep(0, nb);
            }
          }
        }
        bool finite = fast && isfinite(acc);
        if constexpr (NOUT == 3) finite = finite && isfinite(accx) && isfinite(accy);
        if (finite) {
          if (rot && sub == 0) fix(sa + o);  // all G threads of the target skipped it
        } else {
        acc = acc0;
        accx = accx0;
        accy = accy0;
        int nhit = 0, hj = 0;
        if constexpr (NOUT == 1) {
          float p0 = 0.f, p1 = 0.f, p2 = 0.f, p3 = 0.f;
          auto pair = [&](const float4 q, int jj, float &p) {
            const float dx = tx - q.x, dy = ty - q.y;
            const float d2 = fmaf(dy, dy, dx * dx);
            const bool z = d2 < 1.17549435e-38f;  // FLT_MIN
            nhit += z;
            hj = z ? jj : hj;
            const float v = K.radial(d2);
            p = fmaf(z ? 0.f : v, q.z, p);
          };
          int j = sub, nsum = 0;
          for (; j + 3 * G < nb; j += 4 * G) {
            pair(src[j], j, p0);
            pair(src[j + G], j + G, p1);
            pair(src[j + 2 * G], j + 2 * G, p2);
            pair(src[j + 3 * G], j + 3 * G, p3);
            if (++nsum == 8) {
              acc += ((double)p0 + (double)p1) + ((double)p2 + (double)p3);
              p0 = p1 = p2 = p3 = 0.f;
              nsum = 0;
            }
          }
          for (; j < nb; j += G) pair(src[j], j, p0);
          acc += ((double)p0 + (double)p1) + ((double)p2 + (double)p3);
        } else {
          float p[2] = {0.f, 0.f}, px[2] = {0.f, 0.f}, py[2] = {0.f, 0.f};
          auto pair = [&](const float4 q, int jj, int a) {
            // hi parts first: exact for close points (Sterbenz), then the low parts
            const float2 ql = src_lo[jj];
            const float dx = (tx - q.x) + (tx_lo - ql.x), dy = (ty - q.y) + (ty_lo - ql.y);
            const float d2 = fmaf(dy, dy, dx * dx);
            const bool z = d2 < 1.17549435e-38f;  // FLT_MIN
            nhit += z;
            hj = z ? jj : hj;
            p[a] = fmaf(z ? 0.f : K.radial(d2), q.z, p[a]);
            const float qr = z ? 0.f : rcp_ftz(d2) * q.z;
            px[a] = fmaf(dx, qr, px[a]);
            py[a] = fmaf(dy, qr, py[a]);
          };
          int j = sub, nsum = 0;
          for (; j + G < nb; j += 2 * G) {
            pair(src[j], j, 0);
            pair(src[j + G], j + G, 1);
            if (++nsum == 16) {
              acc += (double)p[0] + (double)p[1];
              accx += (double)px[0] + (double)px[1];
              accy += (double)py[0] + (double)py[1];
              p[0] = p[1] = px[0] = px[1] = py[0] = py[1] = 0.f;
              nsum = 0;
            }
          }
          if (j < nb) pair(src[j], j, 0);
          acc += (double)p[0] + (double)p[1];
          accx += (double)px[0] + (double)px[1];
          accy += (double)py[0] + (double)py[1];
        }
        if (nhit) {
          if (nhit == 1) {
            fix(hj);
          } else {
            for (int jj = sub; jj < nb; jj += G) {
              const float4 q4 = src[jj];
              float dx = tx - q4.x, dy = ty - q4.y;
              if constexpr (NOUT == 3) {
                dx += tx_lo - src_lo[jj].x;
                dy += ty_lo - src_lo[jj].y;
              }
              if (fmaf(dy, dy, dx * dx) < 1.17549435e-38f) fix(jj);
            }
          }
        }
        }  // tested sweep
      }
    }
    double r[NOUT];
    r[0] = acc + exact;
    if (sub == 0) {  // FP64 kernel-offset terms: colleagues' charges (P2P), locals' sum (L2T)
      const double cterm = PART == EVAL_FAR ? 0.0 : D.csrc;
      const double lterm = (PART == EVAL_NEAR || lev < 2) ? 0.0 : lsum[g];
      r[0] += kofs * (cterm + lterm);
    }
    if constexpr (NOUT == 3) {
      const double gs = KF32::kGradScale / (double)KF32::kScale * iw;
      r[1] = accx * gs + exact_x;
      r[2] = accy * gs + exact_y;
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
    if (threadIdx.x == 0) s_next = after;
    __syncthreads();  // D and src are rewritten by the next item
    item = nxt;
    nxt = s_next;
  }
}

// per node: FP64 sum of its charges, as a difference of prefix sums
__global__ void k_node_charge_sums(int total, const int *__restrict__ bot, const int *__restrict__ top,
                                   const double *__restrict__ pre, double *__restrict__ tsum) {
  for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < total; g += gridDim.x * blockDim.x)
    tsum[g] = pre[top[g]] - pre[bot[g]];
}

template <class KF32>
void upward_mx_impl(const PassArgs &a, const double *tau_s, const double *tsum, float *mult32,
                    double *msum, float *mult_tc, cudaStream_t s) {
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  const int np = a.np;
  if (th.L < 3) return;
  const size_t pbytes = sizeof(double) * ((size_t)TN * pad_ld(np) * 2 + c2e_stage_doubles(np));
  smem_limit(k_s2m_mx<KF32>, pbytes);
  PhaseTimer timer(PH_UPWARD, s);
  k_s2m_mx<KF32><<<work_grid((th.n_total() + TN - 1) / TN, 4), NT, pbytes, s>>>(a.kp, a.neq, np, th.L, td.dev_off.get(),
                                              td.uplist.get(), td.n_up.get(), td.bot.get(),
                                              td.top.get(), td.xmid.get(), td.ymid.get(),
                                              td.sx.get(), td.sy.get(), tau_s, tsum, a.ops_dev,
                                              mult32, msum, mult_tc);
  FMMB_CUDA(cudaGetLastError());
  // operators staged in shared memory when they fit (static smem ~1 KB aside)
  const bool stage_b = m2m_mx_smem(np, true) + 4096 <= smem_optin();
  const size_t mbytes = m2m_mx_smem(np, stage_b);
  auto kern = stage_b ? k_m2m_mx<true> : k_m2m_mx<false>;
  smem_limit(kern, mbytes);
  for (int m = th.L - 2; m >= 2; --m) {
    const int c_first = th.off[m + 1];
    const int n_groups = (th.off[m + 2] - th.off[m + 1]) / 4;
    if (n_groups == 0) continue;
    // level m's operators are staged while level m+1 finishes
    launch_pdl(kern, dim3((n_groups + TN - 1) / TN), dim3(NT), mbytes, s, m, a.neq, np, c_first,
               n_groups, td.parent.get(), a.ops_dev, mult32, msum, mult_tc);
  }
}

}  // namespace

void node_charge_sums(const PassArgs &a, const double *tau_s, double *tsum, cudaStream_t s) {
  const int total = a.th->n_total();
  const int64_t n = a.th->n_points;
  DevBuf<double> pre;
  pre.alloc(n + 1, s);
  FMMB_CUDA(cudaMemsetAsync(pre.get(), 0, sizeof(double), s));
  prefix_sum<double, true>(tau_s, pre.get() + 1, n, a.td->sort_fail.get(), false, s);
  k_node_charge_sums<<<grid_for(total, 256), 256, 0, s>>>(total, a.td->bot.get(), a.td->top.get(),
                                                          pre.get(), tsum);
  FMMB_CUDA(cudaGetLastError());
}

void run_upward_mixed(const PassArgs &a, const double *tau_s, const double *tsum, float *mult32,
                      double *msum, float *mult_tc, cudaStream_t s) {
  switch (a.kernel_id) {
    case KERNEL_LAPLACE: upward_mx_impl<LaplaceF32>(a, tau_s, tsum, mult32, msum, mult_tc, s); break;
    case KERNEL_MOD_HELMHOLTZ:
      upward_mx_impl<ModHelmholtzF32>(a, tau_s, tsum, mult32, msum, mult_tc, s);
      break;
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
}

void run_m2l_mixed(const PassArgs &a, const float *mult32, const float *mult_tc, const double *msum,
                   double *ple, int *err, cudaStream_t s) {
  const TreeHost &th = *a.th;
  if (th.L < 3) return;
  FMMB_CHECK(th.L <= FMM_MAX_LEVELS_DEV, ERR_INVALID_ARGUMENT, "too many levels");
  M2LTilesMx tl{};
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
  static const bool force_sync = [] {
    const char *e = getenv("FLEXMM_B200_M2L");
    return e && std::string(e) == "mma_sync";
  }();
  if (a.np <= TC_MAX_NP && !force_sync) {
    // tiles of 128 targets per (level, parity class)
    int ctiles = 0;
    M2LTilesMx tc{};
    tc.n_levels = th.L;
    for (int m = 0; m < th.L; ++m) {
      tc.rg_lo[m] = tl.rg_lo[m];
      tc.rg_cnt[m] = tl.rg_cnt[m];
      for (int c = 0; c < 4; ++c) {
        tc.tile_start[4 * m + c] = ctiles;
        if (m >= 2) ctiles += (tc.rg_cnt[m] + TCM - 1) / TCM;
      }
    }
    tc.tile_start[4 * th.L] = ctiles;
    // persistent: one CTA per SM (its shared memory admits no second one),
    // each walking tiles blockIdx.x, blockIdx.x + gridDim.x, ...
    const size_t sm = m2l_tc_smem_bytes(a.np);
    smem_limit(k_m2l_tc, sm);
    int dev = 0, sms = 0;
    FMMB_CUDA(cudaGetDevice(&dev));
    FMMB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    PhaseTimer timer(PH_M2L, s);
    k_m2l_tc<<<std::min(ctiles, sms), TC_THREADS, sm, s>>>(tc, ctiles, a.neq, a.np, a.td->rg.get(),
                                                           a.td->il.get(), a.ops_dev, mult_tc, msum,
                                                           ple, err, err + 1);
    FMMB_CUDA(cudaGetLastError());
    return;
  }
  const size_t sm = sizeof(float) * (size_t)TM * pad_f(a.np);
  PhaseTimer timer(PH_M2L, s);
  k_m2l_mx<<<tiles, 128, sm, s>>>(tl, a.neq, a.np, a.td->rg.get(), a.td->il.get(), a.ops_dev, mult32,
                                  msum, ple);
  FMMB_CUDA(cudaGetLastError());
}

void run_downward_mixed(const PassArgs &a, const double *ple, float *loc32, double *lsum,
                        cudaStream_t s) {
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  auto bytes = [&](bool stage_b) {
    return sizeof(double) * ((size_t)TN * pad_ld(a.np) * 2 + c2e_stage_doubles(a.np)) +
           sizeof(float) * ((size_t)16 * pad_f(a.np) + (stage_b ? (size_t)2 * a.np * ldb_f(4 * a.np) : 0));
  };
  const bool stage_b = bytes(true) + 4096 <= smem_optin();
  const size_t sm = bytes(stage_b);
  auto kern = stage_b ? k_downward_mx<true> : k_downward_mx<false>;
  smem_limit(kern, sm);
  for (int m = 2; m < th.L; ++m) {
    const int lo = th.rg_lo[m], cnt = th.rg_hi[m] - th.rg_lo[m];
    if (cnt <= 0) continue;
    PhaseTimer timer(PH_DOWNWARD, s);
    launch_pdl(kern, dim3((cnt + 7) / 8), dim3(NT), sm, s, m, a.neq, a.np, lo, cnt, td.rg.get(),
               td.parent.get(), a.ops_dev, ple, loc32, lsum);
  }
}

template <class KF32, class KF64>
void split_mixed_impl(const PassArgs &a, const double *tau_s, const double *tsum,
                      const float *loc32, const double *lsum, int check, double *out,
                      cudaStream_t s, const SplitEval &se) {
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  const int64_t m = th.n_points;
  const int total = th.n_total();
  FMMB_CUDA(cudaStreamWaitEvent(se.side, se.ready, 0));
  EvalItems it;
  eval_items(a, td.pkeys.get(), m, it, se.side);
  DevBuf<EvalDesc> desc;
  desc.alloc(total + m / TCH + 1, se.side);
  DevBuf<int> next_item;  // [0] near-field, [1] far-field hand-out counters
  next_item.alloc(2, se.side);
  next_item.zero(se.side);
  DevBuf<double> near;
  near.alloc(m, se.side);
  k_eval_desc<<<grid_for(total + m / TCH + 1, 256), 256, 0, se.side>>>(
      it.items.get(), it.n_items.get(), td.coll.get(), td.bot.get(), td.top.get(), td.xmid.get(),
      td.ymid.get(), tsum, desc.get());
  FMMB_CUDA(cudaGetLastError());
  {
    // the SMs keep their largest shared-memory carveout while near-field
    // blocks sit on them, so the level passes' CTAs still fit beside them
    static const bool carveout_set = [] {
      FMMB_CUDA(cudaFuncSetAttribute(k_evaluate_mx<KF32, KF64, 1, EVAL_NEAR>,
                                     cudaFuncAttributePreferredSharedMemoryCarveout,
                                     cudaSharedmemCarveoutMaxShared));
      return true;
    }();
    (void)carveout_set;
    PhaseTimer timer(PH_EVAL, se.side);
    // beside the upward pass until the M2L starts (hold), then beside the
    // downward pass, resuming from the same item counter
    for (int part = 0; part < (se.hold ? 2 : 1); ++part) {
      if (part == 1) {
        FMMB_CUDA(cudaStreamWaitEvent(se.side, se.m2l_done, 0));
        FMMB_CUDA(cudaMemsetAsync(se.hold, 0, sizeof(int), se.side));
      }
      k_evaluate_mx<KF32, KF64, 1, EVAL_NEAR>
          <<<work_grid(total + m / TCH + 1, part == 0 ? NEAR_BLOCKS_PER_SM_MIXED
                                                      : NEAR_BLOCKS_PER_SM_MIXED_RESUME),
             TCH, 0, se.side>>>(a.kp, a.neq, a.np, desc.get(), it.n_items.get(), td.sx.get(),
                                td.sy.get(), tau_s, a.ops_dev, loc32, lsum, td.sx.get(),
                                td.sy.get(), td.ordv.get(), check, 1, out, 0, next_item.get(),
                                near.get(), se.hold);
      FMMB_CUDA(cudaGetLastError());
    }
  }
  FMMB_CUDA(cudaEventRecord(se.near_done, se.side));
  FMMB_CUDA(cudaStreamWaitEvent(s, se.near_done, 0));
  {
    PhaseTimer timer(PH_EVAL, s);
    k_evaluate_mx<KF32, KF64, 1, EVAL_FAR>
        <<<work_grid(total + m / TCH + 1, EvalOcc<KF32>::blocks), TCH, 0, s>>>(
        a.kp, a.neq, a.np, desc.get(), it.n_items.get(), td.sx.get(), td.sy.get(), tau_s,
        a.ops_dev, loc32, lsum, td.sx.get(), td.sy.get(), td.ordv.get(), check, 1, out, 0,
        next_item.get() + 1, near.get());
    FMMB_CUDA(cudaGetLastError());
  }
  FMMB_CUDA(cudaEventRecord(se.far_done, s));
  FMMB_CUDA(cudaStreamWaitEvent(se.side, se.far_done, 0));
}

void run_evaluate_sources_split_mixed(const PassArgs &a, const double *tau_s,
                                      const double *tsum, const float *loc32, const double *lsum,
                                      int check, double *out, cudaStream_t s, const SplitEval &se) {
  if (a.th->n_points == 0) return;
  switch (a.kernel_id) {
    case KERNEL_LAPLACE:
      split_mixed_impl<LaplaceF32, LaplaceF64>(a, tau_s, tsum, loc32, lsum, check, out, s, se);
      break;
    case KERNEL_MOD_HELMHOLTZ:
      split_mixed_impl<ModHelmholtzF32, ModHelmholtzF64>(a, tau_s, tsum, loc32, lsum, check, out,
                                                         s, se);
      break;
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
}

void run_evaluate_mixed(const PassArgs &a, const double *tau_s, const double *tsum,
                        const float *loc32, const double *lsum, const double *txs,
                        const double *tys, const uint64_t *tkeys, const int *tperm, int64_t m,
                        int check, int nout, double *out, int64_t ld_out, cudaStream_t s,
                        const EvalItems *pre) {
  if (m == 0) return;
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  const int total = th.n_total();
  EvalItems own;
  if (!pre) eval_items(a, tkeys, m, own, s);
  const EvalItems &it = pre ? *pre : own;
  DevBuf<EvalDesc> desc;
  desc.alloc(total + m / TCH + 1, s);
  DevBuf<int> next_item;
  next_item.alloc(1, s);
  next_item.zero(s);
  k_eval_desc<<<grid_for(total + m / TCH + 1, 256), 256, 0, s>>>(
      it.items.get(), it.n_items.get(), td.coll.get(), td.bot.get(), td.top.get(), td.xmid.get(),
      td.ymid.get(), tsum, desc.get());
  FMMB_CUDA(cudaGetLastError());
  // targets that are the tree's own sorted sources: each target's own point
  // is left out of the pair sweep
  const int self_eval = txs == td.sx.get() && tys == td.sy.get();
  PhaseTimer timer(PH_EVAL, s);
  switch (a.kernel_id) {
    case KERNEL_LAPLACE: {
      auto kern = nout == 3 ? k_evaluate_mx<LaplaceF32, LaplaceF64, 3>
                            : k_evaluate_mx<LaplaceF32, LaplaceF64, 1>;
      const int per_sm = nout == 3 ? 6 : EVAL_BLOCKS_PER_SM;
      kern<<<work_grid(total + m / TCH + 1, per_sm), TCH, 0, s>>>(a.kp, a.neq, a.np, desc.get(),
                                                                it.n_items.get(),
                                        td.sx.get(), td.sy.get(), tau_s, a.ops_dev, loc32, lsum,
                                        txs, tys, tperm, check, self_eval, out, ld_out,
                                        next_item.get(), nullptr, nullptr);
      break;
    }
    case KERNEL_MOD_HELMHOLTZ: {  // potential only: the mixed gradient is the log kernel's
      FMMB_CHECK(nout == 1, ERR_UNSUPPORTED,
                 "the mixed form evaluates the modified Helmholtz potential only (gradients: FP64)");
      k_evaluate_mx<ModHelmholtzF32, ModHelmholtzF64, 1>
          <<<work_grid(total + m / TCH + 1, EvalOcc<ModHelmholtzF32>::blocks), TCH, 0, s>>>(
              a.kp, a.neq, a.np, desc.get(), it.n_items.get(), td.sx.get(), td.sy.get(), tau_s,
              a.ops_dev, loc32, lsum, txs, tys, tperm, check, self_eval, out, ld_out,
              next_item.get(), nullptr, nullptr);
      break;
    }
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
  FMMB_CUDA(cudaGetLastError());
}

}  // namespace fmmb
