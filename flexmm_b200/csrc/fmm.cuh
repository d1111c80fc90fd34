// FMM passes over a TreeDev.  Expansions are stored per node (level-major,
// padded to NP columns): multipoles (equivalent densities on the small
// circle), partial locals from M2L, and locals (equivalent densities on the
// large circle).
#pragma once

#include "kernels.cuh"
#include "tree.cuh"

namespace fmmb {

constexpr int M2L_NULL = 0, M2L_DENSE = 1, M2L_SVD = 2;
constexpr int FMM_MAX_LEVELS_DEV = 30;  // levels 0..29 (keys hold 29 digits)

// Device view of one width's operators (all arrays zero padded to NP).
struct LevelOpsDev {
  const double *lx, *ly;  // [Neq] check circle (upward) / equivalent circle (downward)
  const double *u;        // [NP x NP]  S2L = U diag(S) VH
  const double *sinv;     // [NP]       1/S (0 where S <= tol, and in padding)
  const double *vh;       // [NP x NP]
  const double *m2mct;    // [4NP x NP] m2mct[c*NP+k][i] = M2MC[i][c*Neq+k]
  const double *m2mc;     // [NP x 4NP] m2mc[k][c*NP+i] = M2MC[k][c*Neq+i]
  const double *m2l[N_OFFSETS];  // dense: D^T [NP x NP]; svd: M1^T [NP x RP] then M2^T [RP x NP]
  int kind[N_OFFSETS];
  int rp[N_OFFSETS];
  // mixed precision: operators minus their mean c (the mean enters exactly as
  // c * sum(input), in FP64), rounded to TF32 as hi + lo pairs, B layout [K][N]
  const float *lx32, *ly32;             // [NP]
  const float *m2mct_hi, *m2mct_lo;     // [4NP x NP]
  const float *m2mc_hi, *m2mc_lo;       // [NP x 4NP]
  const float *m2l_hi[N_OFFSETS], *m2l_lo[N_OFFSETS];  // [NP x NP] dense (D - c)^T
  const float *m2l_tc_hi[N_OFFSETS], *m2l_tc_lo[N_OFFSETS];  // [NT x NP] (D - c), NT = NP rounded to 16
  double c_m2m;
  double c_m2l[N_OFFSETS];
  // kernel scaling of the FP32 evaluations: coordinates are multiplied by
  // inv_w (1/width for scale-invariant kernels, else 1) and kofs (the
  // kernel's offset(width), else 0) times the charge sum is added in FP64;
  // lx32 / ly32 hold the check circle already scaled
  double inv_w, kofs;
};

constexpr int PREC_FP64 = 0, PREC_MIXED = 1;

struct PassArgs {
  int kernel_id;
  KernelParams kp;
  int neq, np;
  const TreeDev *td;
  const TreeHost *th;
  const LevelOpsDev *ops_dev;   // device array indexed by level
  // dipole sources (Laplace double layer): per sorted source the dipole
  // vector strength * normal; null when the sources carry charges only
  const double *dvx = nullptr, *dvy = nullptr;
};

// Black-box (Chebyshev) FMM (bbfmm.cu): p x p coefficients per box, NQ = p^2
// padded to np columns; M2MC [np x 4np] row-major (level independent);
// m2l_cat[m]: level m's 40 M2L operators stacked transposed, [40 np x np]
// row-major, rows o np .. o np + np - 1 holding (VI K VI^T)^T of offset o
// (zero for a null offset); m2mct = M2MC^T [4np x np].
struct BBArgs {
  int kernel_id;
  KernelParams kp;
  int p, np;
  const TreeDev *td;
  const TreeHost *th;
  const double *m2mc, *m2mct;
  const double *m2l_cat[FMM_MAX_LEVELS_DEV];
};
void run_bb_upward(const BBArgs &b, const double *tau_sorted, double *mult, cudaStream_t s);
// M2L and L2L, level by level; the locals are the partial locals (no solve)
void run_bb_downward(const BBArgs &b, const double *mult, double *ple, cudaStream_t s);
// nout = 1 potential, 3 potential and target gradient (rows, stride ld_out)
void run_bb_evaluate(const BBArgs &b, const double *tau_sorted, const double *loc,
                     const double *txs, const double *tys, const uint64_t *tkeys, const int *tperm,
                     int64_t m, int check, int nout, double *out, int64_t ld_out, cudaStream_t s);

// Stokes FMM (stokes.cu): rows of np = pad8(2 Neq + 1) doubles; per level
// the large circle and the row-major operators of the GEMMs:
//   e2c_u, e2c_vhs [np x np]: E2C solve x = (b . U) . (diag(1/S) VH);
//   c2e_u, c2e_vhs [np x np]: C2E solve, the extra unknown's column zeroed;
//   m2mc [4np x np]: parent check row = children rows . m2mc;
//   l2lc [np x 4np]: children partial-local rows = local row . l2lc;
//   m2l_cat [40np x np]: the 40 M2L operators stacked, each transposed.
struct StokesArgs {
  int neq, np;
  const TreeDev *td;
  const TreeHost *th;
  // double-layer (stresslet) sources: strengths (sigma) and normals, sorted;
  // null when the sources carry forces only (build_expansions_dipole,
  // stokes_fmm.py:738-826)
  const double *sgx = nullptr, *sgy = nullptr, *dnx = nullptr, *dny = nullptr;
  struct Level {
    const double *lx, *ly;
    const double *e2c_u, *e2c_vhs, *c2e_u, *c2e_vhs, *m2mc, *l2lc, *m2l_cat;
  } lev[FMM_MAX_LEVELS_DEV];
};
void run_stokes_upward(const StokesArgs &a, const double *fx, const double *fy, double *partial,
                       double *mult, cudaStream_t s);
void run_stokes_downward(const StokesArgs &a, const double *mult, double *ple, double *loc,
                         cudaStream_t s);
// out rows (u, v, p), stride ld_out
void run_stokes_evaluate(const StokesArgs &a, const double *fx, const double *fy, const double *loc,
                         const double *txs, const double *tys, const uint64_t *tkeys,
                         const int *tperm, int64_t m, int check, double *out, int64_t ld_out,
                         cudaStream_t s);

// n_rhs charge columns (stride n_src, sorted order) and their locals (stride
// col_stride): out row r (stride ld_out) for column r
void run_evaluate_multi(const PassArgs &a, const double *tau_sorted, int64_t n_src, int n_rhs,
                        const double *loc, int64_t col_stride, const double *txs, const double *tys,
                        const uint64_t *tkeys, const int *tperm, int64_t m, int check, double *out,
                        int64_t ld_out, cudaStream_t s);
// Split own-source evaluation: the near field (P2P) runs on `side` as soon
// as `ready` (recorded on the plan stream once the charges are sorted) has
// passed, beside the level passes still queued on the plan stream; the far
// field (L2T) runs on the plan stream after them and adds the near field.
// near_done / far_done are scratch events of the plan.  Scratch lives on the
// side stream and is released there after the plan stream has used it.
struct SplitEval {
  cudaStream_t side;
  cudaEvent_t ready, near_done, far_done;
  // mixed form: the near field pauses while the M2L runs.  hold (device int)
  // is set on the plan stream before the M2L and m2l_done recorded after
  // it; the near-field kernel takes no new items while hold is set, and a
  // second launch after m2l_done finishes the rest.  hold NULL: one launch.
  int *hold = nullptr;
  cudaEvent_t m2l_done = nullptr;
};
// near-field blocks per SM, leaving room for the level passes: FP64 (28 KB of
// shared memory each) beside the DMMA M2L tiles; mixed (17 KB each) beside
// the upward pass until the M2L (which it leaves to the persistent tcgen05
// CTAs), then beside the downward pass.  Mixed, measured at 1M (step ms,
// two runs each, one box): before / after the M2L 3/10 1.277-1.281, 2/10
// 1.282-1.286, 6/10 1.253-1.262, 8/10 1.245-1.247, 12/10 1.287, 6/8
// 1.247-1.249, 6/12 1.273-1.277.  FP64 (step ms, same way): 2 5.10, 3 3.86,
// 4 3.350-3.351, 6 3.194, 8 3.197-3.204.
constexpr int NEAR_BLOCKS_PER_SM = 6;
constexpr int NEAR_BLOCKS_PER_SM_MIXED = 8;
constexpr int NEAR_BLOCKS_PER_SM_MIXED_RESUME = 10;  // after the M2L, beside the downward pass
void run_evaluate_sources_split(const PassArgs &a, const double *tau_sorted, const double *loc,
                                int check, double *out, cudaStream_t s, const SplitEval &se);
void run_evaluate_sources_split_mixed(const PassArgs &a, const double *tau_sorted,
                                      const double *tsum, const float *loc32, const double *lsum,
                                      int check, double *out, cudaStream_t s, const SplitEval &se);
// The FP64 passes; n_rhs charge columns at once (multi-RHS: column r's
// charges at tau_sorted + r * tstride, its expansions at + r * cstride),
// one launch per level for all columns.
void run_upward(const PassArgs &a, const double *tau_sorted, double *mult, cudaStream_t s,
                int n_rhs = 1, int64_t tstride = 0, int64_t cstride = 0);
void run_m2l(const PassArgs &a, const double *mult, double *ple, cudaStream_t s, int n_rhs = 1,
             int64_t cstride = 0);
void run_downward(const PassArgs &a, const double *ple, double *loc, cudaStream_t s,
                  int n_rhs = 1, int64_t cstride = 0);
// targets: sorted coordinates, sorted keys, permutation sorted -> original
void run_direct(int kernel_id, const KernelParams &kp, const double *sx, const double *sy,
                const double *tau, int64_t ns, const double *tx, const double *ty, int64_t nt,
                int check, double *out, cudaStream_t s);
void gather_sorted(const double *v, const int *perm, int64_t n, double *o, cudaStream_t s);
void gather_sorted_i64(const int64_t *v, const int *perm, int64_t n, int64_t *o, cudaStream_t s);
// near field only (local evaluator): out[i] = sum over the target's
// colleagues' sources; scat (sorted) / tcat (caller's order) categories, or null
void run_local_evaluate(const PassArgs &a, const double *tau_sorted, const double *txs,
                        const double *tys, const uint64_t *tkeys, const int *tperm, int64_t m,
                        int check, const int64_t *scat, const int64_t *tcat, double *out,
                        cudaStream_t s);
// the FP64 passes' table-driven log2 and the library log2 at n device points
void run_diag_log2(const double *x, int64_t n, double *out_tab, double *out_lib, cudaStream_t s);
// nout = 1: potential into out[m]; nout = 3: potential and its gradient in the
// target position into out[0..2][m] (row stride ld_out)
struct EvalItems;
// (pre: work items already built for txs, tys; else built from tkeys)
void run_evaluate(const PassArgs &a, const double *tau_sorted, const double *loc,
                  const double *txs, const double *tys, const uint64_t *tkeys, const int *tperm,
                  int64_t m, int check, int nout, double *out, int64_t ld_out, cudaStream_t s,
                  const EvalItems *pre = nullptr);

// Evaluation work items: per leaf its range of sorted targets, split into
// chunks of 128 targets; choff = exclusive scan of the chunk counts.
struct EvalItems {
  DevBuf<int> tb, te, nch, choff;
  DevBuf<int4> items;   // (leaf, level | EVAL_MULTI, first sorted target, count)
  DevBuf<int> n_items;  // device count of items
};
// item .y: the leaf's level, plus EVAL_MULTI when the leaf's targets fill more
// than one item (targets placed in no particular order inside the leaf): then
// every item of the leaf gives one thread per target (G = 1), so that a
// target's arithmetic does not depend on which item holds it
constexpr int EVAL_LEVEL_MASK = 0xFF, EVAL_MULTI = 0x100;
constexpr int EVAL_CHUNK = 128;  // targets per evaluation work item
// parts of an evaluation: both, the near field (P2P) alone, the far field (L2T) alone
constexpr int EVAL_FULL = 0, EVAL_NEAR = 1, EVAL_FAR = 2;
void eval_items(const PassArgs &a, const uint64_t *tkeys, int64_t m, EvalItems &it, cudaStream_t s);
// Work items for targets (tx, ty) in the caller's order, binned into the
// leaves instead of sorted: writes txs, tys (leaf by leaf) and tperm.
void eval_items_binned(const PassArgs &a, const double *tx, const double *ty, int64_t m,
                       EvalItems &it, double *txs, double *tys, int *tperm, cudaStream_t s);

// Mixed precision (fmm_mixed.cu): FP32 multipoles / locals with FP64 sums.
void node_charge_sums(const PassArgs &a, const double *tau_sorted, double *tsum, cudaStream_t s);
// mult_tc: [node][TF32 hi np | lo np] copy of mult32, the tcgen05 M2L operand
void run_upward_mixed(const PassArgs &a, const double *tau_sorted, const double *tsum, float *mult32,
                      double *msum, float *mult_tc, cudaStream_t s);
void run_m2l_mixed(const PassArgs &a, const float *mult32, const float *mult_tc, const double *msum,
                   double *ple, int *err, cudaStream_t s);  // err: 2 zeroed ints (flag, tile counter)
void run_downward_mixed(const PassArgs &a, const double *ple, float *loc32, double *lsum,
                        cudaStream_t s);
void run_evaluate_mixed(const PassArgs &a, const double *tau_sorted, const double *tsum,
                        const float *loc32, const double *lsum, const double *txs,
                        const double *tys, const uint64_t *tkeys, const int *tperm, int64_t m,
                        int check, int nout, double *out, int64_t ld_out, cudaStream_t s,
                        const EvalItems *pre = nullptr);

// Evaluation with caller-provided scratch: tb, te, nch, choff hold one int
// per tree node, temp holds evaluate_scratch_bytes(nodes) bytes.
size_t evaluate_scratch_bytes(int total_nodes);
void run_evaluate_scratch(const PassArgs &a, const double *tau_sorted, const double *loc,
                          const double *txs, const double *tys, const uint64_t *tkeys,
                          const int *tperm, int64_t m, int check, double *out, int *tb, int *te,
                          int *nch, int *choff, int4 *items, int *n_items, void *temp,
                          size_t temp_bytes, cudaStream_t s);

}  // namespace fmmb
