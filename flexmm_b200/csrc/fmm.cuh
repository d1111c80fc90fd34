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
};

struct PassArgs {
  int kernel_id;
  KernelParams kp;
  int neq, np;
  const TreeDev *td;
  const TreeHost *th;
  const LevelOpsDev *ops_dev;   // device array indexed by level
  std::vector<LevelOpsDev> ops_host;
};

void run_upward(const PassArgs &a, const double *tau_sorted, double *mult, cudaStream_t s);
void run_m2l(const PassArgs &a, const double *mult, double *ple, cudaStream_t s);
void run_downward(const PassArgs &a, const double *ple, double *loc, cudaStream_t s);
// targets: sorted coordinates, sorted keys, permutation sorted -> original
void run_direct(int kernel_id, const KernelParams &kp, const double *sx, const double *sy,
                const double *tau, int64_t ns, const double *tx, const double *ty, int64_t nt,
                int check, double *out, cudaStream_t s);
void gather_sorted(const double *v, const int *perm, int64_t n, double *o, cudaStream_t s);
void run_evaluate(const PassArgs &a, const double *tau_sorted, const double *loc,
                  const double *txs, const double *tys, const uint64_t *tkeys, const int *tperm,
                  int64_t m, int check, double *out, cudaStream_t s);

// Evaluation with caller-provided scratch: tb, te, nch, choff hold one int
// per tree node, temp holds evaluate_scratch_bytes(nodes) bytes.
size_t evaluate_scratch_bytes(int total_nodes);
void run_evaluate_scratch(const PassArgs &a, const double *tau_sorted, const double *loc,
                          const double *txs, const double *tys, const uint64_t *tkeys,
                          const int *tperm, int64_t m, int check, double *out, int *tb, int *te,
                          int *nch, int *choff, void *temp, size_t temp_bytes, cudaStream_t s);

}  // namespace fmmb
