// Black-box (Chebyshev) FMM passes in FP64 (flexmm/flexmm2d/bbfmm.py).
//
// The expansions of a box are p x p Chebyshev coefficients on the box scaled
// to [-1, 1]^2 (NQ = p^2, rows padded to np):
//  * S2M: Chebyshev moments of the box's sources,
//    M[a p + b] = sum_j T_a(x_j) T_b(y_j) tau_j (anterpolate2, bbfmm.py:11-24,
//    source2pMs, bbfmm.py:186-196); no check-to-equivalent step;
//  * M2M / L2L: the level-independent M2MC [NQ x 4NQ] and its transpose
//    (bbfmm.py:145-161) on the contiguous child rows of each parent group;
//  * M2L: per level and offset VI K VI^T (bbfmm.py:101-122), the 40 offsets
//    of a level applied in one row-GEMM launch (rowgemm.cuh) over the
//    stacked operators: each tile of 64 target boxes of one parity class
//    reads the source multipole of each offset it meets, and skips the
//    offsets absent for the whole tile;
//  * L2T: the local coefficients evaluated as a 2-D Chebyshev series
//    (chebeval2d1, bbfmm.py:25-31, L2targets, bbfmm.py:198-210);
//  * P2P: the same colleague sweep as the KIFMM evaluation.
// M2M, L2L and M2L are FP64 tensor-core row GEMMs (rowgemm.cuh) with their
// gathers and scatters fused into the loads and stores; moments and
// evaluation are the kernels below.

#include <algorithm>
#include <string>

#include "dense.cuh"
#include "rowgemm.cuh"
#include "fmm.cuh"
#include "timing.cuh"

namespace fmmb {
namespace {

constexpr int BB_MAX_P = 16;
constexpr int TCH_BB = 128;   // evaluation threads per work item
constexpr int SMAX_BB = 1024;  // sources staged per evaluation pass

// 2 / width per level: maps a box to [-1, 1]^2 (width_adj, bbfmm.py:122)
struct BBScale {
  double inv_hw[FMM_MAX_LEVELS_DEV];
};

// S2M moments, one warp per S2M node; lane owns outputs q = lane + 32 k
__global__ void __launch_bounds__(128) k_bb_s2m(int p, int np, int L, BBScale sc,
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
                                                double *__restrict__ mult) {
  __shared__ double Tx[4][32][BB_MAX_P], Ty[4][32][BB_MAX_P], tw[4][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_up = *n_up_ptr, nq = p * p;
  int qa[8], qb[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int q = lane + 32 * k;
    qa[k] = q < nq ? q / p : 0;
    qb[k] = q < nq ? q % p : 0;
  }
  for (int i = blockIdx.x * 4 + warp; i < n_up; i += gridDim.x * 4) {
    const int g = uplist[i];
    const double a = sc.inv_hw[node_level_of(off, L, g)];
    const double cx = xmid[g], cy = ymid[g];
    const int b = bot[g], e = top[g];
    double acc[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) acc[k] = 0.0;
    for (int j0 = b; j0 < e; j0 += 32) {
      const int nj = min(32, e - j0);
      if (lane < nj) {
        const double x = (sx[j0 + lane] - cx) * a, y = (sy[j0 + lane] - cy) * a;
        double t0 = 1.0, t1 = x, u0 = 1.0, u1 = y;
        Tx[warp][lane][0] = 1.0;
        Ty[warp][lane][0] = 1.0;
        for (int n = 1; n < p; ++n) {
          Tx[warp][lane][n] = t1;
          Ty[warp][lane][n] = u1;
          const double t2 = 2.0 * x * t1 - t0, u2 = 2.0 * y * u1 - u0;
          t0 = t1;
          t1 = t2;
          u0 = u1;
          u1 = u2;
        }
        tw[warp][lane] = tau[j0 + lane];
      }
      __syncwarp();
      for (int jj = 0; jj < nj; ++jj) {
        const double t = tw[warp][jj];
#pragma unroll
        for (int k = 0; k < 8; ++k)
          if (lane + 32 * k < nq) acc[k] = fma(Tx[warp][jj][qa[k]] * Ty[warp][jj][qb[k]], t, acc[k]);
      }
      __syncwarp();
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const int q = lane + 32 * k;
      if (q < np) mult[(size_t)g * np + q] = q < nq ? acc[k] : 0.0;
    }
  }
}

// Evaluation: L2T as a 2-D Chebyshev series of the leaf's local coefficients,
// P2P over the colleagues (as k_evaluate).  One work item = (leaf, up to 128
// of its targets); G threads share a target.  NOUT = 3 adds the gradient in
// the target position: the series' derivative (T_n' by its recurrence,
// chebeval2d_dx / _dy, bbfmm.py:32-45) and the kernel's gradient.
template <class KF, int NOUT>
__global__ void __launch_bounds__(TCH_BB) k_bb_evaluate(KernelParams kp, int p, int np, BBScale sc,
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
                                                        const double *__restrict__ loc,
                                                        const double *__restrict__ txs,
                                                        const double *__restrict__ tys,
                                                        const int *__restrict__ tperm, int check,
                                                        double *__restrict__ out, int64_t ld_out) {
  __shared__ double ssx[SMAX_BB], ssy[SMAX_BB], stau[SMAX_BB];
  __shared__ int rb[9], rs[10];
  __shared__ double red[NOUT][TCH_BB / 32];
  const KF K(kp);
  const int n_items = *n_items_ptr;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int4 it = items[item];
    const int g = it.x, lev = it.y, t0 = it.z, cnt = it.w;
    int G = 1;
    while (2 * G * cnt <= TCH_BB) G *= 2;
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
    double u = 0.0, gx = 0.0, gy = 0.0;
    if (lev >= 2 && valid) {
      // sum_a T_a(x) sum_b c[a p + b] T_b(y), rows a split over the G threads
      const double a = sc.inv_hw[lev];
      const double xh = (x - xmid[g]) * a, yh = (y - ymid[g]) * a;
      double ty[BB_MAX_P], dty[BB_MAX_P];
      ty[0] = 1.0;
      ty[1] = yh;
      dty[0] = 0.0;
      dty[1] = 1.0;
#pragma unroll
      for (int b = 2; b < BB_MAX_P; ++b) {
        ty[b] = 2.0 * yh * ty[b - 1] - ty[b - 2];
        if (NOUT == 3) dty[b] = 2.0 * ty[b - 1] + 2.0 * yh * dty[b - 1] - dty[b - 2];
      }
      const double *cr = loc + (size_t)g * np;
      double tp = 1.0, tc = xh;    // T_{ar-1}, T_ar as ar advances
      double dtp = 0.0, dtc = 1.0;  // their derivatives
      for (int ar = 0; ar < p; ++ar) {
        const double tx = ar == 0 ? 1.0 : tc, dtx = ar == 0 ? 0.0 : dtc;
        if (ar % G == sub) {
          double s = 0.0, sd = 0.0;
#pragma unroll
          for (int b = 0; b < BB_MAX_P; ++b)
            if (b < p) {
              const double c = __ldg(cr + ar * p + b);
              s = fma(c, ty[b], s);
              if (NOUT == 3) sd = fma(c, dty[b], sd);
            }
          u = fma(tx, s, u);
          if (NOUT == 3) {
            gx = fma(dtx, s, gx);
            gy = fma(tx, sd, gy);
          }
        }
        if (ar >= 1) {
          const double tn = 2.0 * xh * tc - tp;
          if (NOUT == 3) {
            const double dtn = 2.0 * tc + 2.0 * xh * dtc - dtp;
            dtp = dtc;
            dtc = dtn;
          }
          tp = tc;
          tc = tn;
        }
      }
      gx *= a;  // d/dx = (2 / w) d/dxh
      gy *= a;
    }
    __syncthreads();
    auto pair = [&](int j) -> double {
      const double qx = ssx[j], qy = ssy[j];
      const double v = K(qx, qy, x, y) * stau[j];
      return (check && x - qx == 0.0 && y - qy == 0.0) ? 0.0 : v;
    };
    const int ns = rs[9];
    double u1 = 0.0, u2 = 0.0, u3 = 0.0;
    for (int base = 0; base < ns; base += SMAX_BB) {
      const int nb = min(SMAX_BB, ns - base);
      for (int i = threadIdx.x; i < nb; i += TCH_BB) {
        const int idx = base + i;
        int c = 0;
        while (idx >= rs[c + 1]) ++c;
        const int j = rb[c] + (idx - rs[c]);
        ssx[i] = sx[j];
        ssy[i] = sy[j];
        stau[i] = tau[j];
      }
      __syncthreads();
      if (valid) {
        if constexpr (NOUT == 1) {
          int j = sub;
          for (; j + 3 * G < nb; j += 4 * G) {
            u += pair(j);
            u1 += pair(j + G);
            u2 += pair(j + 2 * G);
            u3 += pair(j + 3 * G);
          }
          for (; j < nb; j += G) u += pair(j);
        } else {
          for (int j = sub; j < nb; j += G) {
            const double qx = ssx[j], qy = ssy[j];
            if (!(check && x - qx == 0.0 && y - qy == 0.0)) K.grad(qx, qy, x, y, stau[j], u, gx, gy);
          }
        }
      }
      __syncthreads();
    }
    double r[3] = {(u + u1) + (u2 + u3), gx, gy};
#pragma unroll
    for (int o = 0; o < NOUT; ++o) {
      double w = r[o];
      for (int q = min(G, 32) >> 1; q >= 1; q >>= 1) w += __shfl_xor_sync(0xffffffffu, w, q);
      if (G > 32) {
        if ((threadIdx.x & 31) == 0) red[o][threadIdx.x >> 5] = w;
        __syncthreads();
        if (sub == 0) {
          w = 0.0;
          for (int q = 0; q < G / 32; ++q) w += red[o][(threadIdx.x >> 5) + q];
        }
      }
      if (valid && sub == 0) out[o * ld_out + tperm[t0 + t]] = w;
    }
    __syncthreads();
  }
}

BBScale bb_scale(const TreeHost &th) {
  BBScale sc{};
  for (int m = 0; m < th.L && m < FMM_MAX_LEVELS_DEV; ++m) sc.inv_hw[m] = 2.0 / th.width[m];
  return sc;
}

}  // namespace

void run_bb_upward(const BBArgs &b, const double *tau_s, double *mult, cudaStream_t s) {
  const TreeHost &th = *b.th;
  const TreeDev &td = *b.td;
  if (th.L < 3) return;
  FMMB_CHECK(th.L <= FMM_MAX_LEVELS_DEV, ERR_INVALID_ARGUMENT, "too many levels");
  const int np = b.np;
  const BBScale sc = bb_scale(th);
  PhaseTimer timer(PH_UPWARD, s);
  k_bb_s2m<<<work_grid(th.n_total(), 8), 128, 0, s>>>(b.p, np, th.L, sc, td.dev_off.get(), td.uplist.get(),
                                   td.n_up.get(), td.bot.get(), td.top.get(), td.xmid.get(),
                                   td.ymid.get(), td.sx.get(), td.sy.get(), tau_s, mult);
  FMMB_CUDA(cudaGetLastError());
  for (int m = th.L - 2; m >= 2; --m) {
    const int c_first = th.off[m + 1];
    const int n_groups = (th.off[m + 2] - th.off[m + 1]) / 4;
    if (n_groups == 0) continue;
    // parent rows = children rows (contiguous, 4np wide) . M2MC^T (fmm.py:93-96)
    rowgemm(RowsContig{mult + (size_t)c_first * np, 4 * (int64_t)np, n_groups, 4 * np},
            StoreParents{td.parent.get(), mult, c_first, np}, row_tiles(n_groups), b.m2mct, np, np,
            4 * np, s);
  }
}

void run_bb_downward(const BBArgs &b, const double *mult, double *ple, cudaStream_t s) {
  const TreeHost &th = *b.th;
  const TreeDev &td = *b.td;
  if (th.L < 3) return;
  const int np = b.np;
  for (int m = 2; m < th.L; ++m) {
    const int lo = th.rg_lo[m], n_groups = th.rg_hi[m] - th.rg_lo[m];
    if (n_groups == 0) continue;
    if (m >= 3) {  // L2L from level m-1: children += parent local . M2MC (bbfmm.py:161, fmm.py:140-147)
      PhaseTimer timer(PH_DOWNWARD, s);
      rowgemm(ParentRows{td.rg.get(), td.parent.get(), ple, lo, n_groups, np},
              AddChildRows{td.rg.get(), ple, lo, np}, row_tiles(n_groups), b.m2mc, 4 * np, 4 * np,
              np, s);
    }
    {  // M2L of level m: tiles of one parity class, absent offsets skipped (fmm.py:118-131)
      PhaseTimer timer(PH_M2L, s);
      const int tpc = row_tiles(n_groups);
      rowgemm(M2LRows{td.rg.get(), td.il.get(), mult, lo, n_groups, np, tpc},
              AddGroupRows{td.rg.get(), ple, lo, np}, 4 * tpc, b.m2l_cat[m], np, np, np, s);
    }
  }
}

void run_bb_evaluate(const BBArgs &b, const double *tau_s, const double *loc, const double *txs,
                     const double *tys, const uint64_t *tkeys, const int *tperm, int64_t m,
                     int check, int nout, double *out, int64_t ld_out, cudaStream_t s) {
  if (m == 0) return;
  const TreeDev &td = *b.td;
  PassArgs a{};
  a.th = b.th;
  a.td = b.td;
  EvalItems it;
  eval_items(a, tkeys, m, it, s);
  const BBScale sc = bb_scale(*b.th);
  PhaseTimer timer(PH_EVAL, s);
  auto launch = [&](auto kern) {
    kern<<<work_grid(b.th->n_total() + m / TCH_BB + 1, 8), TCH_BB, 0, s>>>(
        b.kp, b.p, b.np, sc, it.items.get(), it.n_items.get(),
                                    td.coll.get(), td.bot.get(), td.top.get(), td.xmid.get(),
                                    td.ymid.get(), td.sx.get(), td.sy.get(), tau_s, loc, txs, tys,
                                    tperm, check, out, ld_out);
  };
  switch (b.kernel_id) {
    case KERNEL_LAPLACE:
      nout == 3 ? launch(k_bb_evaluate<LaplaceF64, 3>) : launch(k_bb_evaluate<LaplaceF64, 1>);
      break;
    case KERNEL_MOD_HELMHOLTZ:
      nout == 3 ? launch(k_bb_evaluate<ModHelmholtzF64, 3>) : launch(k_bb_evaluate<ModHelmholtzF64, 1>);
      break;
    case KERNEL_RADIAL_TABLE:
      FMMB_CHECK(nout == 1, ERR_UNSUPPORTED, "tabulated kernels evaluate potentials only");
      launch(k_bb_evaluate<RadialTableF64, 1>);
      break;
    default: throw Error(ERR_UNSUPPORTED, "unknown kernel id");
  }
  FMMB_CUDA(cudaGetLastError());
}

}  // namespace fmmb
