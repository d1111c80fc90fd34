// Stokes FMM passes in FP64 (flexmm/kifmm2d/vector/stokes_fmm.py:550-858).
//
// A box carries 2 Neq + 1 values (row of np doubles): the equivalent forces
// (fx, fy) on Neq points of a circle plus one extra unknown of the corrected
// (pressure-augmented) forms; check values are the velocities (u, v) on Neq
// points plus the pressure at the circle's centre.  Per level:
//  * upward: partial = S2M (velocities on the check circle from the leaf's
//    sources; pressure row 0, as upwards_pass, stokes_fmm.py:259-291, ignores
//    kernel_add's pressure) + M2MC . children (extra unknowns excluded), then
//    the factored-SVD solve of the corrected equivalent-to-check form
//    (E2C_SVD, stokes_fmm.py:553-558);
//  * downward: partial locals += L2LC . parent local (real sibling groups) and
//    += M2L . source multipoles (the 40 offsets in one row-GEMM launch,
//    tiles of one parity class skipping absent offsets), then the C2E solve,
//    extra unknown dropped (stokes_fmm.py:712-733);
//  * evaluation: (u, v, p) from the leaf's local forces on the large circle
//    (local_expansion_evaluation, stokes_fmm.py:331-360) plus the colleagues'
//    sources (neighbor_evaluation, stokes_fmm.py:361-396).
// Solves and translations are FP64 tensor-core row GEMMs (rowgemm.cuh) on
// the plan's stream, gathers and scatters fused into their loads and stores.

#include <algorithm>

#include "dense.cuh"
#include "rowgemm.cuh"
#include "fmm.cuh"
#include "timing.cuh"

namespace fmmb {
namespace {

constexpr int TCH_ST = 128;
constexpr int SMAX_ST = 1024;

struct StokesCircles {
  const double *lx[FMM_MAX_LEVELS_DEV], *ly[FMM_MAX_LEVELS_DEV];  // large circle, per level
};

// one Stokeslet pair, unscaled: u, v times 1/(4 pi), p times 1/(2 pi) later
// (kernel_apply_single, stokes_fmm.py:166-187)
__device__ __forceinline__ void stokeslet(double dx, double dy, double fx, double fy, double &u,
                                          double &v, double &p) {
  const double id2 = 1.0 / (dx * dx + dy * dy);
  const double logid = 0.5 * log(id2);
  const double dxdy = dx * dy * id2;
  u += (logid + dx * dx * id2) * fx + dxdy * fy;
  v += dxdy * fx + (logid + dy * dy * id2) * fy;
  p += (fx * dx + fy * dy) * id2;
}

// one stresslet (double-layer) pair, unscaled like stokeslet: strength
// (sgx, sgy) along the normal (nx, ny), d = (dx, dy) target - source
// (kernel_apply_single_with_dipole, stokes_fmm.py:187-235):
//   u_a += 4 (d.n) d_a d_b / r^4 sigma_b,
//   p   += 2 (-n_b / r^2 + 2 d_b (d.n) / r^4) sigma_b
__device__ __forceinline__ void stresslet(double dx, double dy, double sgx, double sgy, double nx,
                                          double ny, double &u, double &v, double &p) {
  const double id2 = 1.0 / (dx * dx + dy * dy);
  const double dn = dx * nx + dy * ny;
  const double c = 4.0 * dn * id2 * id2;
  const double gxy = c * dx * dy;
  u += c * dx * dx * sgx + gxy * sgy;
  v += gxy * sgx + c * dy * dy * sgy;
  p += 2.0 * (-nx * id2 + 0.5 * dx * c) * sgx + 2.0 * (-ny * id2 + 0.5 * dy * c) * sgy;
}

// S2M: velocities at the large circle's points from the box's sources; one
// warp per S2M node, lane k owns check points k and k + 32.  DIP: the
// sources also carry stresslets (upwards_pass_dipole, stokes_fmm.py:294-322).
template <bool DIP>
__global__ void __launch_bounds__(128) k_stokes_s2m(int neq, int np, int L, StokesCircles cir,
                                                    const int *__restrict__ off,
                                                    const int *__restrict__ uplist,
                                                    const int *__restrict__ n_up_ptr,
                                                    const int *__restrict__ bot,
                                                    const int *__restrict__ top,
                                                    const double *__restrict__ xmid,
                                                    const double *__restrict__ ymid,
                                                    const double *__restrict__ sx,
                                                    const double *__restrict__ sy,
                                                    const double *__restrict__ fx,
                                                    const double *__restrict__ fy,
                                                    double *__restrict__ partial,
                                                    const double *__restrict__ sgx,
                                                    const double *__restrict__ sgy,
                                                    const double *__restrict__ dnx,
                                                    const double *__restrict__ dny) {
  __shared__ double qx[4][32], qy[4][32], qf[4][32], qg[4][32];
  __shared__ double qs[DIP ? 4 : 1][32], qt[DIP ? 4 : 1][32], qn[DIP ? 4 : 1][32],
      qm[DIP ? 4 : 1][32];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n_up = *n_up_ptr;
  for (int i = blockIdx.x * 4 + warp; i < n_up; i += gridDim.x * 4) {
    const int g = uplist[i];
    const int m = node_level_of(off, L, g);
    const double cx = xmid[g], cy = ymid[g];
    double ex[2], ey[2], u[2] = {0.0, 0.0}, v[2] = {0.0, 0.0}, p[2] = {0.0, 0.0};
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = lane + 32 * h;
      ex[h] = k < neq ? cir.lx[m][k] : 0.0;
      ey[h] = k < neq ? cir.ly[m][k] : 0.0;
    }
    const int b = bot[g], e = top[g];
    for (int j0 = b; j0 < e; j0 += 32) {
      const int nj = min(32, e - j0);
      if (lane < nj) {
        qx[warp][lane] = sx[j0 + lane] - cx;
        qy[warp][lane] = sy[j0 + lane] - cy;
        qf[warp][lane] = fx[j0 + lane];
        qg[warp][lane] = fy[j0 + lane];
        if constexpr (DIP) {
          qs[warp][lane] = sgx[j0 + lane];
          qt[warp][lane] = sgy[j0 + lane];
          qn[warp][lane] = dnx[j0 + lane];
          qm[warp][lane] = dny[j0 + lane];
        }
      }
      __syncwarp();
#pragma unroll
      for (int h = 0; h < 2; ++h)
        if (lane + 32 * h < neq)
          for (int j = 0; j < nj; ++j) {
            const double dx = ex[h] - qx[warp][j], dy = ey[h] - qy[warp][j];
            stokeslet(dx, dy, qf[warp][j], qg[warp][j], u[h], v[h], p[h]);
            if constexpr (DIP)
              stresslet(dx, dy, qs[warp][j], qt[warp][j], qn[warp][j], qm[warp][j], u[h], v[h],
                        p[h]);
          }
      __syncwarp();
    }
    const double us = 0.25 / M_PI;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int k = lane + 32 * h;
      if (k < neq) {
        partial[(size_t)g * np + k] = u[h] * us;
        partial[(size_t)g * np + neq + k] = v[h] * us;
      }
    }
  }
}

// Evaluation: (u, v, p) rows of out (stride ld_out).  One work item = (leaf,
// up to 128 of its targets); G threads share a target.  DIP: the near field
// adds the sources' stresslets (neighbor_evaluation_dipole,
// stokes_fmm.py:399-441); the far field is the same local expansion.
template <bool DIP>
__global__ void __launch_bounds__(TCH_ST) k_stokes_evaluate(
    int neq, int np, StokesCircles cir, const int4 *__restrict__ items,
    const int *__restrict__ n_items_ptr, const int *__restrict__ coll, const int *__restrict__ bot,
    const int *__restrict__ top, const double *__restrict__ xmid, const double *__restrict__ ymid,
    const double *__restrict__ sx, const double *__restrict__ sy, const double *__restrict__ fx,
    const double *__restrict__ fy, const double *__restrict__ loc, const double *__restrict__ txs,
    const double *__restrict__ tys, const int *__restrict__ tperm, int check,
    double *__restrict__ out, int64_t ld_out, const double *__restrict__ sgx,
    const double *__restrict__ sgy, const double *__restrict__ dnx,
    const double *__restrict__ dny) {
  constexpr int SM = DIP ? SMAX_ST / 2 : SMAX_ST;  // 48 KB of static shared memory at most
  __shared__ double ssx[SM], ssy[SM], sfx[SM], sfy[SM];
  __shared__ double ssg[DIP ? SM : 1], stg[DIP ? SM : 1], snx[DIP ? SM : 1], sny[DIP ? SM : 1];
  __shared__ int rb[9], rs[10];
  __shared__ double red[3][TCH_ST / 32];
  const int n_items = *n_items_ptr;
  for (int item = blockIdx.x; item < n_items; item += gridDim.x) {
    const int4 it = items[item];
    const int g = it.x, lev = it.y, t0 = it.z, cnt = it.w;
    int G = 1;
    while (2 * G * cnt <= TCH_ST) G *= 2;
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
    double u = 0.0, v = 0.0, p = 0.0;
    if (lev >= 2 && valid) {  // L2T: local forces on the large circle
      const double dx0 = x - xmid[g], dy0 = y - ymid[g];
      const double *lf = loc + (size_t)g * np;
      for (int k = sub; k < neq; k += G)
        stokeslet(dx0 - cir.lx[lev][k], dy0 - cir.ly[lev][k], lf[k], lf[neq + k], u, v, p);
    }
    __syncthreads();
    const int ns = rs[9];
    for (int base = 0; base < ns; base += SM) {
      const int nb = min(SM, ns - base);
      for (int i = threadIdx.x; i < nb; i += TCH_ST) {
        const int idx = base + i;
        int c = 0;
        while (idx >= rs[c + 1]) ++c;
        const int j = rb[c] + (idx - rs[c]);
        ssx[i] = sx[j];
        ssy[i] = sy[j];
        sfx[i] = fx[j];
        sfy[i] = fy[j];
        if constexpr (DIP) {
          ssg[i] = sgx[j];
          stg[i] = sgy[j];
          snx[i] = dnx[j];
          sny[i] = dny[j];
        }
      }
      __syncthreads();
      if (valid)
        for (int j = sub; j < nb; j += G) {
          const double dx = x - ssx[j], dy = y - ssy[j];
          if (check && dx == 0.0 && dy == 0.0) continue;
          stokeslet(dx, dy, sfx[j], sfy[j], u, v, p);
          if constexpr (DIP) stresslet(dx, dy, ssg[j], stg[j], snx[j], sny[j], u, v, p);
        }
      __syncthreads();
    }
    double r[3] = {u * (0.25 / M_PI), v * (0.25 / M_PI), p * (0.5 / M_PI)};
#pragma unroll
    for (int o = 0; o < 3; ++o) {
      double w = r[o];
      for (int s = min(G, 32) >> 1; s >= 1; s >>= 1) w += __shfl_xor_sync(0xffffffffu, w, s);
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

StokesCircles circles(const StokesArgs &a) {
  StokesCircles c{};
  for (int m = 0; m < a.th->L && m < FMM_MAX_LEVELS_DEV; ++m) {
    c.lx[m] = a.lev[m].lx;
    c.ly[m] = a.lev[m].ly;
  }
  return c;
}

// rows of x := ((b . U) . VHs), row-major np x np operators, n contiguous rows
void solve_rows(const StokesArgs &a, const double *u, const double *vhs, const double *b, double *x,
                double *tmp, int n, cudaStream_t s) {
  const int np = a.np;
  rowgemm(RowsContig{b, np, n, np}, StoreRows{tmp, np}, row_tiles(n), u, np, np, np, s);
  rowgemm(RowsContig{tmp, np, n, np}, StoreRows{x, np}, row_tiles(n), vhs, np, np, np, s);
}

}  // namespace

void run_stokes_upward(const StokesArgs &a, const double *fx, const double *fy, double *partial,
                       double *mult, cudaStream_t s) {
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  if (th.L < 3) return;
  FMMB_CHECK(th.L <= FMM_MAX_LEVELS_DEV, ERR_INVALID_ARGUMENT, "too many levels");
  const int np = a.np;
  PhaseTimer timer(PH_UPWARD, s);
  auto s2m = a.sgx ? k_stokes_s2m<true> : k_stokes_s2m<false>;
  s2m<<<work_grid(th.n_total(), 8), 128, 0, s>>>(a.neq, np, th.L, circles(a), td.dev_off.get(),
                                                 td.uplist.get(), td.n_up.get(), td.bot.get(),
                                                 td.top.get(), td.xmid.get(), td.ymid.get(),
                                                 td.sx.get(), td.sy.get(), fx, fy, partial, a.sgx,
                                                 a.sgy, a.dnx, a.dny);
  FMMB_CUDA(cudaGetLastError());
  int max_rows = 0;
  for (int m = 2; m < th.L; ++m) max_rows = std::max(max_rows, th.off[m + 1] - th.off[m]);
  DevBuf<double> tmp;
  tmp.alloc((size_t)max_rows * np, s);
  for (int m = th.L - 1; m >= 2; --m) {
    if (m <= th.L - 2) {  // partial of level m's parents = children . M2MC
      const int c_first = th.off[m + 1];
      const int n_groups = (th.off[m + 2] - th.off[m + 1]) / 4;
      if (n_groups > 0)
        rowgemm(RowsContig{mult + (size_t)c_first * np, 4 * (int64_t)np, n_groups, 4 * np},
                StoreParents{td.parent.get(), partial, c_first, np}, row_tiles(n_groups),
                a.lev[m].m2mc, np, np, 4 * np, s);
    }
    const int r0 = th.off[m], n = th.off[m + 1] - th.off[m];
    if (n > 0)
      solve_rows(a, a.lev[m].e2c_u, a.lev[m].e2c_vhs, partial + (size_t)r0 * np,
                 mult + (size_t)r0 * np, tmp.get(), n, s);
  }
}

void run_stokes_downward(const StokesArgs &a, const double *mult, double *ple, double *loc,
                         cudaStream_t s) {
  const TreeHost &th = *a.th;
  const TreeDev &td = *a.td;
  if (th.L < 3) return;
  const int np = a.np;
  int max_groups = 0, max_rows = 0;
  for (int m = 2; m < th.L; ++m) {
    max_groups = std::max(max_groups, th.rg_hi[m] - th.rg_lo[m]);
    max_rows = std::max(max_rows, th.off[m + 1] - th.off[m]);
  }
  DevBuf<double> tmp;
  tmp.alloc((size_t)std::max(max_rows, 1) * np, s);
  for (int m = 2; m < th.L; ++m) {
    const int lo = th.rg_lo[m], n_groups = th.rg_hi[m] - th.rg_lo[m];
    if (n_groups > 0) {
      if (m >= 3) {  // L2L from level m-1 (stokes_fmm.py:726-733)
        PhaseTimer timer(PH_DOWNWARD, s);
        rowgemm(ParentRows{td.rg.get(), td.parent.get(), loc, lo, n_groups, np},
                AddChildRows{td.rg.get(), ple, lo, np}, row_tiles(n_groups), a.lev[m - 1].l2lc,
                4 * np, 4 * np, np, s);
      }
      // M2L: tiles of one parity class, absent offsets skipped
      PhaseTimer timer(PH_M2L, s);
      const int tpc = row_tiles(n_groups);
      rowgemm(M2LRows{td.rg.get(), td.il.get(), mult, lo, n_groups, np, tpc},
              AddGroupRows{td.rg.get(), ple, lo, np}, 4 * tpc, a.lev[m].m2l_cat, np, np, np, s);
    }
    const int r0 = th.off[m], nr = th.off[m + 1] - th.off[m];
    if (nr > 0)
      solve_rows(a, a.lev[m].c2e_u, a.lev[m].c2e_vhs, ple + (size_t)r0 * np, loc + (size_t)r0 * np,
                 tmp.get(), nr, s);
  }
}

void run_stokes_evaluate(const StokesArgs &a, const double *fx, const double *fy, const double *loc,
                         const double *txs, const double *tys, const uint64_t *tkeys,
                         const int *tperm, int64_t m, int check, double *out, int64_t ld_out,
                         cudaStream_t s) {
  if (m == 0) return;
  const TreeDev &td = *a.td;
  PassArgs pa{};
  pa.th = a.th;
  pa.td = a.td;
  EvalItems it;
  eval_items(pa, tkeys, m, it, s);
  PhaseTimer timer(PH_EVAL, s);
  auto ev = a.sgx ? k_stokes_evaluate<true> : k_stokes_evaluate<false>;
  ev<<<work_grid(a.th->n_total() + m / TCH_ST + 1, 8), TCH_ST, 0, s>>>(
      a.neq, a.np, circles(a), it.items.get(), it.n_items.get(), td.coll.get(), td.bot.get(),
      td.top.get(), td.xmid.get(), td.ymid.get(), td.sx.get(), td.sy.get(), fx, fy, loc, txs, tys,
      tperm, check, out, ld_out, a.sgx, a.sgy, a.dnx, a.dny);
  FMMB_CUDA(cudaGetLastError());
}

}  // namespace fmmb
