// FMM passes (FP64): upward (S2M / M2M + check-to-equivalent), offset-grouped
// M2L, downward (L2L + check-to-equivalent) and evaluation (L2T + P2P).
//
// Reference path: flexmm/flexmm2d/fmm.py:67-176 (passes), kifmm.py:83-144
// (S2M, C2E, L2T), helpers.py:5-33 (M2L factors), helpers.py:152-194 (P2P).
// Differences of form, not of result:
//  * check-to-equivalent is applied as VH^T diag(1/S) U^T, the factored SVD
//    solve (flexmm/kifmm2d/scalar/helpers.py:240-248), never an explicit
//    inverse; it agrees with the reference's LU solve to ~1e-15;
//  * M2L is target-centric: a tile of target boxes gathers the source
//    multipoles of one offset and multiplies by that offset's dense or
//    SVD-factored operator, accumulating all 40 offsets in registers (the
//    reference multiplies every multipole by every offset, then gathers);
//  * L2L is parent-centric: one GEMM per tile of 8 parents produces the
//    partial locals of their 32 children.
#include <cub/cub.cuh>

#include "fmm.cuh"
#include "timing.cuh"

namespace fmmb {
namespace {

constexpr int TN = 32;    // nodes per tile
constexpr int NT = 256;   // threads per tile CTA
constexpr int TCH = 128;  // targets per evaluation work item

// acc[r][c] += sum_k A[(row0 + r) * lda + k] * B[k * ldb + col0 + c], r < R, c < 4
template <int R>
__device__ __forceinline__ void gemm_acc(const double *__restrict__ A, int lda,
                                         const double *__restrict__ B, int ldb, int K, int row0,
                                         int col0, double (&acc)[R][4]) {
#pragma unroll 4
  for (int k = 0; k < K; ++k) {
    const double2 b01 = *reinterpret_cast<const double2 *>(B + (size_t)k * ldb + col0);
    const double2 b23 = *reinterpret_cast<const double2 *>(B + (size_t)k * ldb + col0 + 2);
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const double a = A[(row0 + r) * lda + k];
      acc[r][0] = fma(a, b01.x, acc[r][0]);
      acc[r][1] = fma(a, b01.y, acc[r][1]);
      acc[r][2] = fma(a, b23.x, acc[r][2]);
      acc[r][3] = fma(a, b23.y, acc[r][3]);
    }
  }
}

template <int R>
__device__ __forceinline__ void zero_acc(double (&acc)[R][4]) {
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int c = 0; c < 4; ++c) acc[r][c] = 0.0;
}

// Check-to-equivalent on a tile held in smem P[TN][NP] -> T (scratch) -> out rows.
// out[t][i] = sum_k VH[k][i] * sinv[k] * sum_j U[j][k] * P[t][j]
__device__ void c2e_tile(const LevelOpsDev &op, int np, const double *P, double *T, int nloc,
                         double *out_base, const uint8_t *write_mask) {
  const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
  const int row0 = 2 * ty, col0 = 4 * tx;
  double acc[2][4];
  zero_acc(acc);
  if (col0 < np) gemm_acc<2>(P, np, op.u, np, np, row0, col0, acc);
  if (col0 < np) {
#pragma unroll
    for (int r = 0; r < 2; ++r)
#pragma unroll
      for (int c = 0; c < 4; ++c) T[(row0 + r) * np + col0 + c] = acc[r][c] * op.sinv[col0 + c];
  }
  __syncthreads();
  zero_acc(acc);
  if (col0 < np) gemm_acc<2>(T, np, op.vh, np, np, row0, col0, acc);
  if (col0 < np) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int t = row0 + r;
      if (t < nloc && (!write_mask || write_mask[t])) {
        double *o = out_base + (size_t)t * np + col0;
        reinterpret_cast<double2 *>(o)[0] = make_double2(acc[r][0], acc[r][1]);
        reinterpret_cast<double2 *>(o)[1] = make_double2(acc[r][2], acc[r][3]);
      }
    }
  }
}

// ---------------------------------------------------------------- upward ----
template <class KF>
__global__ void __launch_bounds__(NT) k_upward(int m, KernelParams kp, int neq, int np, int g_begin,
                                               int g_end, const uint8_t *__restrict__ flags,
                                               const int *__restrict__ bot,
                                               const int *__restrict__ top,
                                               const int *__restrict__ child,
                                               const double *__restrict__ xmid,
                                               const double *__restrict__ ymid,
                                               const double *__restrict__ sx,
                                               const double *__restrict__ sy,
                                               const double *__restrict__ tau,
                                               const LevelOpsDev *__restrict__ ops,
                                               double *__restrict__ mult) {
  extern __shared__ double smem[];
  double *P = smem;             // [TN][np]   check potentials
  double *A = P + TN * np;      // [TN][4np]  children multipoles; later C2E scratch
  const KF K(kp);
  const LevelOpsDev &op = ops[m];
  const int g0 = g_begin + blockIdx.x * TN;
  const int nloc = min(TN, g_end - g0);
  for (int i = threadIdx.x; i < TN * np; i += NT) P[i] = 0.0;
  for (int i = threadIdx.x; i < TN * 4 * np; i += NT) A[i] = 0.0;
  __syncthreads();
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  // S2M (flexmm/flexmm2d/kifmm.py:96-105) for leaves and fake leaves with
  // points; gather children multipoles for boxes with children (M2M)
  for (int t = warp; t < nloc; t += NT / 32) {
    const int g = g0 + t;
    const uint8_t f = flags[g];
    const int b = bot[g], e = top[g];
    const bool up = (((f & NF_LEAF) && !(f & NF_XLIST)) || (f & NF_FAKE)) && e > b;
    if (up) {
      const double cx = xmid[g], cy = ymid[g];
      for (int k = lane; k < neq; k += 32) {
        const double lxk = op.lx[k], lyk = op.ly[k];
        double acc = 0.0;
        for (int j = b; j < e; ++j) acc = fma(K(sx[j] - cx, sy[j] - cy, lxk, lyk), tau[j], acc);
        P[t * np + k] = acc;
      }
    } else if (f & NF_CHILDREN) {
      const int c0 = child[g];
      for (int q = lane; q < 4 * np; q += 32) A[t * 4 * np + q] = mult[(size_t)(c0 + q / np) * np + q % np];
    }
  }
  __syncthreads();
  // M2M: P[t] = M2MC . [children]  (flexmm/flexmm2d/fmm.py:93-96)
  {
    const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
    const int row0 = 2 * ty, col0 = 4 * tx;
    double acc[2][4];
    zero_acc(acc);
    if (col0 < np) gemm_acc<2>(A, 4 * np, op.m2mct, np, 4 * np, row0, col0, acc);
    __syncthreads();
    if (col0 < np) {
#pragma unroll
      for (int r = 0; r < 2; ++r) {
        const int t = row0 + r;
        if (t < nloc && (flags[g0 + t] & NF_CHILDREN))
#pragma unroll
          for (int c = 0; c < 4; ++c) P[t * np + col0 + c] = acc[r][c];
      }
    }
  }
  __syncthreads();
  c2e_tile(op, np, P, A, nloc, mult + (size_t)g0 * np, nullptr);
}

// ------------------------------------------------------------------- M2L ----
__global__ void __launch_bounds__(NT) k_m2l(const int *__restrict__ tile_start, int L,
                                            const int *__restrict__ off, int np,
                                            const int *__restrict__ il,
                                            const LevelOpsDev *__restrict__ ops,
                                            const double *__restrict__ mult,
                                            double *__restrict__ ple) {
  extern __shared__ double smem[];
  double *G = smem;           // [TN][np] gathered source multipoles
  double *W = G + TN * np;    // [TN][np] SVD intermediate
  int m = 2;
  while (m + 1 < L && tile_start[m + 1] <= (int)blockIdx.x) ++m;
  const int g0 = off[m] + TN * (blockIdx.x - tile_start[m]);
  const int nloc = min(TN, off[m + 1] - g0);
  const LevelOpsDev &op = ops[m];
  const int ty = threadIdx.x / 16, tx = threadIdx.x % 16;
  const int row0 = 2 * ty, col0 = 4 * tx;
  double acc[2][4];
  zero_acc(acc);
  for (int o = 0; o < N_OFFSETS; ++o) {
    const int kind = op.kind[o];
    if (kind == M2L_NULL) continue;
    const int has = (threadIdx.x < nloc) ? (il[(size_t)(g0 + threadIdx.x) * N_OFFSETS + o] >= 0) : 0;
    if (!__syncthreads_or(has)) continue;
    for (int i = threadIdx.x; i < TN * np; i += NT) {
      const int t = i / np, k = i % np;
      const int s = (t < nloc) ? il[(size_t)(g0 + t) * N_OFFSETS + o] : -1;
      G[i] = (s >= 0) ? mult[(size_t)s * np + k] : 0.0;
    }
    __syncthreads();
    if (kind == M2L_DENSE) {
      if (col0 < np) gemm_acc<2>(G, np, op.m2l[o], np, np, row0, col0, acc);
    } else {
      const int rp = op.rp[o];
      double w[2][4];
      zero_acc(w);
      if (col0 < rp) gemm_acc<2>(G, np, op.m2l[o], rp, np, row0, col0, w);
      if (col0 < rp) {
#pragma unroll
        for (int r = 0; r < 2; ++r)
#pragma unroll
          for (int c = 0; c < 4; ++c) W[(row0 + r) * rp + col0 + c] = w[r][c];
      }
      __syncthreads();
      if (col0 < np) gemm_acc<2>(W, rp, op.m2l[o] + (size_t)np * rp, np, rp, row0, col0, acc);
    }
    __syncthreads();
  }
  if (col0 < np) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const int t = row0 + r;
      if (t < nloc) {
        double *o = ple + (size_t)(g0 + t) * np + col0;
        reinterpret_cast<double2 *>(o)[0] = make_double2(acc[r][0], acc[r][1]);
        reinterpret_cast<double2 *>(o)[1] = make_double2(acc[r][2], acc[r][3]);
      }
    }
  }
}

// -------------------------------------------------------------- downward ----
__global__ void __launch_bounds__(NT) k_downward(int m, int np, int g_begin, int g_end,
                                                 const uint8_t *__restrict__ flags,
                                                 const int *__restrict__ parent,
                                                 const LevelOpsDev *__restrict__ ops,
                                                 const double *__restrict__ ple,
                                                 double *__restrict__ loc) {
  extern __shared__ double smem[];
  double *P = smem;            // [TN][np] = [8][4np] partial locals
  double *T = P + TN * np;     // [TN][np] scratch (parent locals, then C2E)
  __shared__ uint8_t real[TN];
  const LevelOpsDev &op = ops[m];
  const LevelOpsDev &opp = ops[m - 1];
  const int g0 = g_begin + blockIdx.x * TN;
  const int nloc = min(TN, g_end - g0);
  if (threadIdx.x < TN) real[threadIdx.x] = (threadIdx.x < nloc) && !(flags[g0 + threadIdx.x] & NF_FAKE);
  for (int i = threadIdx.x; i < TN * np; i += NT) {
    const int t = i / np;
    P[i] = (t < nloc) ? ple[(size_t)g0 * np + i] : 0.0;
    T[i] = 0.0;
  }
  __syncthreads();
  if (m >= 3) {
    // parent locals of the 8 sibling groups
    for (int i = threadIdx.x; i < 8 * np; i += NT) {
      const int q = i / np, k = i % np;
      const int t = 4 * q;
      T[i] = (t < nloc && real[t]) ? loc[(size_t)parent[g0 + t] * np + k] : 0.0;
    }
    __syncthreads();
    // L2L: [8 parents][4np] += Lp . M2MC  (flexmm/flexmm2d/fmm.py:140-147)
    const int ty = threadIdx.x / 64, tx = threadIdx.x % 64;
    const int row0 = 2 * ty, col0 = 4 * tx;
    double acc[2][4];
    zero_acc(acc);
    if (col0 < 4 * np) gemm_acc<2>(T, np, opp.m2mc, 4 * np, np, row0, col0, acc);
    __syncthreads();
    if (col0 < 4 * np) {
#pragma unroll
      for (int r = 0; r < 2; ++r)
#pragma unroll
        for (int c = 0; c < 4; ++c) P[(row0 + r) * 4 * np + col0 + c] += acc[r][c];
    }
    __syncthreads();
  }
  c2e_tile(op, np, P, T, nloc, loc + (size_t)g0 * np, real);
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
    if (flags[g] & NF_LEAF) {
      const int sh = 2 * (MAXD - lev);
      const uint64_t c = code[g];
      int64_t l0 = 0, h0 = m;
      const uint64_t vlo = c << sh, vhi = (c + 1) << sh;
      while (l0 < h0) {
        int64_t md = (l0 + h0) >> 1;
        if (tkeys[md] < vlo) l0 = md + 1; else h0 = md;
      }
      b = int(l0);
      h0 = m;
      while (l0 < h0) {
        int64_t md = (l0 + h0) >> 1;
        if (tkeys[md] < vhi) l0 = md + 1; else h0 = md;
      }
      e = int(l0);
    }
    tb[g] = b;
    te[g] = e;
    nchunk[g] = (e - b + TCH - 1) / TCH;
  }
}

template <class KF>
__global__ void __launch_bounds__(TCH) k_evaluate(KernelParams kp, int neq, int np, int total_nodes,
                                                  int L, const int *__restrict__ off,
                                                  const int *__restrict__ choff,
                                                  const int *__restrict__ nchunk,
                                                  const int *__restrict__ tb,
                                                  const int *__restrict__ te,
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
                                                  double *__restrict__ out) {
  __shared__ double Ls[64], lxs[64], lys[64];
  __shared__ double ssx[TCH], ssy[TCH], stau[TCH];
  const KF K(kp);
  const int n_items = choff[total_nodes - 1] + nchunk[total_nodes - 1];
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    int lo = 0, hi = total_nodes;  // last g with choff[g] <= item
    while (hi - lo > 1) {
      int mid = (lo + hi) >> 1;
      if (choff[mid] <= item) lo = mid; else hi = mid;
    }
    const int g = lo;
    int lev = 0;
    {
      int a = 0, b = L;
      while (b - a > 1) {
        int mid = (a + b) >> 1;
        if (off[mid] <= g) a = mid; else b = mid;
      }
      lev = a;
    }
    const int ch = item - choff[g];
    const int t0 = tb[g] + ch * TCH;
    const int cnt = min(TCH, te[g] - t0);
    const bool valid = threadIdx.x < cnt;
    const int ti = t0 + threadIdx.x;
    const double x = valid ? txs[ti] : 0.0, y = valid ? tys[ti] : 0.0;
    double u = 0.0;
    // L2T (flexmm/flexmm2d/kifmm.py:106-120); locals of levels 0-1 are zero
    if (lev >= 2) {
      for (int k = threadIdx.x; k < neq; k += TCH) {
        Ls[k] = loc[(size_t)g * np + k];
        lxs[k] = ops[lev].lx[k];
        lys[k] = ops[lev].ly[k];
      }
      __syncthreads();
      if (valid) {
        const double dx = x - xmid[g], dy = y - ymid[g];
        for (int k = 0; k < neq; ++k) u = fma(K(lxs[k], lys[k], dx, dy), Ls[k], u);
      }
    }
    // P2P over the colleagues' sorted source ranges (flexmm/flexmm2d/helpers.py:152-194)
    for (int c = 0; c < 9; ++c) {
      const int cg = coll[(size_t)g * 9 + c];
      if (cg < 0) break;
      const int b = bot[cg], e = top[cg];
      double part = 0.0;
      for (int j0 = b; j0 < e; j0 += TCH) {
        const int nj = min(TCH, e - j0);
        __syncthreads();
        if (threadIdx.x < nj) {
          ssx[threadIdx.x] = sx[j0 + threadIdx.x];
          ssy[threadIdx.x] = sy[j0 + threadIdx.x];
          stau[threadIdx.x] = tau[j0 + threadIdx.x];
        }
        __syncthreads();
        if (valid) {
          for (int j = 0; j < nj; ++j) {
            const double qx = ssx[j], qy = ssy[j];
            if (check && x - qx == 0.0 && y - qy == 0.0) continue;
            part = fma(K(qx, qy, x, y), stau[j], part);
          }
        }
      }
      u += part;
    }
    if (valid) out[tperm[ti]] = u;
    __syncthreads();
  }
}

// FP64 direct sum (kernel_apply / kernel_apply_single_check,
// flexmm/flexmm2d/helpers.py:91-116): all sources, one target per thread,
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
void upward_impl(const PassArgs &a, const double *tau_s, double *mult, cudaStream_t s) {
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  const int np = a.np;
  const size_t sm = sizeof(double) * (size_t)TN * np * 5;
  FMMB_CUDA(cudaFuncSetAttribute(k_upward<KF>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(sizeof(double) * TN * 64 * 5)));
  for (int m = th.L - 1; m >= 2; --m) {
    const int gb = th.off[m], ge = th.off[m + 1];
    const int tiles = (ge - gb + TN - 1) / TN;
    PhaseTimer timer(PH_UPWARD, s);
    k_upward<KF><<<tiles, NT, sm, s>>>(m, a.kp, a.neq, np, gb, ge, td.flags.get(), td.bot.get(),
                                       td.top.get(), td.child.get(), td.xmid.get(), td.ymid.get(),
                                       td.sx.get(), td.sy.get(), tau_s, a.ops_dev, mult);
    FMMB_CUDA(cudaGetLastError());
  }
}

template <class KF>
void evaluate_impl(const PassArgs &a, const double *tau_s, const double *loc, const double *txs,
                   const double *tys, const uint64_t *tkeys, const int *tperm, int64_t m, int check,
                   double *out, cudaStream_t s) {
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  const int total = th.n_total();
  DevBuf<int> tb, te, nch, choff;
  tb.alloc(total, s);
  te.alloc(total, s);
  nch.alloc(total, s);
  choff.alloc(total, s);
  k_leaf_targets<<<grid_for(total, 256), 256, 0, s>>>(total, th.L, td.dev_off.get(), td.code.get(),
                                                      td.flags.get(), tkeys, m, tb.get(), te.get(),
                                                      nch.get());
  FMMB_CUDA(cudaGetLastError());
  size_t bytes = 0;
  FMMB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, bytes, nch.get(), choff.get(), total, s));
  DevBuf<uint8_t> tmp;
  tmp.alloc(bytes, s);
  FMMB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.get(), bytes, nch.get(), choff.get(), total, s));
  PhaseTimer timer(PH_EVAL, s);
  k_evaluate<KF><<<148 * 8, TCH, 0, s>>>(a.kp, a.neq, a.np, total, th.L, td.dev_off.get(),
                                         choff.get(), nch.get(), tb.get(), te.get(), td.coll.get(),
                                         td.bot.get(), td.top.get(), td.xmid.get(), td.ymid.get(),
                                         td.sx.get(), td.sy.get(), tau_s, a.ops_dev, loc, txs, tys,
                                         tperm, check, out);
  FMMB_CUDA(cudaGetLastError());
}

}  // namespace

void run_upward(const PassArgs &a, const double *tau_s, double *mult, cudaStream_t s) {
  switch (a.kernel_id) {
    case KERNEL_LAPLACE: upward_impl<LaplaceF64>(a, tau_s, mult, s); break;
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
}

void run_m2l(const PassArgs &a, const double *mult, double *ple, cudaStream_t s) {
  const TreeHost &th = *a.th;
  if (th.L < 3) return;
  std::vector<int> ts(th.L + 1, 0);
  int tiles = 0;
  for (int m = 2; m < th.L; ++m) {
    ts[m] = tiles;
    tiles += (th.off[m + 1] - th.off[m] + TN - 1) / TN;
  }
  ts[th.L] = tiles;
  DevBuf<int> tsd;
  tsd.alloc(th.L + 1, s);
  FMMB_CUDA(cudaMemcpyAsync(tsd.get(), ts.data(), ts.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  const size_t sm = sizeof(double) * (size_t)TN * a.np * 2;
  PhaseTimer timer(PH_M2L, s);
  k_m2l<<<tiles, NT, sm, s>>>(tsd.get(), th.L, a.td->dev_off.get(), a.np, a.td->il.get(), a.ops_dev,
                              mult, ple);
  FMMB_CUDA(cudaGetLastError());
}

void run_downward(const PassArgs &a, const double *ple, double *loc, cudaStream_t s) {
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  const size_t sm = sizeof(double) * (size_t)TN * a.np * 2;
  for (int m = 2; m < th.L; ++m) {
    const int gb = th.off[m], ge = th.off[m + 1];
    const int tiles = (ge - gb + TN - 1) / TN;
    PhaseTimer timer(PH_DOWNWARD, s);
    k_downward<<<tiles, NT, sm, s>>>(m, a.np, gb, ge, td.flags.get(), td.parent.get(), a.ops_dev,
                                     ple, loc);
    FMMB_CUDA(cudaGetLastError());
  }
}

void run_evaluate(const PassArgs &a, const double *tau_s, const double *loc, const double *txs,
                  const double *tys, const uint64_t *tkeys, const int *tperm, int64_t m, int check,
                  double *out, cudaStream_t s) {
  if (m == 0) return;
  switch (a.kernel_id) {
    case KERNEL_LAPLACE:
      evaluate_impl<LaplaceF64>(a, tau_s, loc, txs, tys, tkeys, tperm, m, check, out, s);
      break;
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
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
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
  FMMB_CUDA(cudaGetLastError());
}

void gather_sorted(const double *v, const int *perm, int64_t n, double *o, cudaStream_t s) {
  if (n == 0) return;
  k_gather_sorted<<<grid_for(n, 256), 256, 0, s>>>(v, perm, n, o);
  FMMB_CUDA(cudaGetLastError());
}

}  // namespace fmmb
