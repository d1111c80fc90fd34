/* flexmm_b200: C ABI of the B200 2D FMM evaluation path.
 *
 * The reference (dbstein/flexmm) is a Python + Numba package with no native
 * interface; these entry points replace the pieces of its Python object model
 * that do the work, and the Python package flexmm_b200 binds them with ctypes
 * behind the reference's own class names and signatures:
 *
 *   fmm_ops_*            the operator cache of a Helper: one entry per box
 *                        width (KI_Helper.prepare / KI_Precomputation,
 *                        flexmm/flexmm2d/kifmm.py:13-82; FloatDict keyed by
 *                        width, flexmm/flexmm2d/float_dict.py:23-24)
 *   fmm_plan_create      FMM.__init__ -> Tree(x, y, Ncutoff, bbox)
 *                        (flexmm/flexmm2d/fmm.py:33-58, flexmm/tree.py:451-518)
 *   fmm_plan_info /      the tree's level widths, to fill and bind the
 *   fmm_plan_bind        operator cache (KI_Helper.prepare, kifmm.py:67-82)
 *   fmm_plan_bind_levels the same for all levels at once
 *   fmm_build_expansions FMM.build_expansions(tau) (fmm.py:151-153)
 *   fmm_evaluate         FMM.source_evaluation / target_evaluation
 *                        (fmm.py:158-176); check=1 skips coincident pairs
 *                        (helpers.py:99-107)
 *   fmm_tree_export      the tree arrays (Tree.Levels[*], tree.py:275-360)
 *
 * Conventions: every function returns 0 (FMM_OK) or an FMM_ERR_* code and
 * never aborts; fmm_last_error() gives the message of the calling thread's
 * last failure.  Point, charge and output pointers are DEVICE pointers owned
 * by the caller; `stream` is a cudaStream_t (NULL = legacy default stream).
 * A plan must be used from one stream.  An operator set must outlive the
 * plans bound to it.  Plans are independent and may be used concurrently.
 */
#ifndef FLEXMM_B200_H
#define FLEXMM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FMM_OK 0
#define FMM_ERR_INVALID_ARGUMENT 1
#define FMM_ERR_CUDA 2
#define FMM_ERR_TREE_TOO_DEEP 3
#define FMM_ERR_NOT_READY 4
#define FMM_ERR_UNSUPPORTED 5
#define FMM_ERR_CAPACITY 6

/* kernels, registered under the reference's example names */
#define FMM_KERNEL_LAPLACE 0 /* Laplace_Eval, examples/kifmm_laplace.py:24-29 */

#define FMM_N_OFFSETS 40 /* far-field offsets (-3..3)^2 minus (-1..1)^2; id walks ox outer, oy inner */
#define FMM_MAX_LEVELS 30
#define FMM_MAX_NEQUIV 64

typedef struct fmm_ops fmm_ops;
typedef struct fmm_plan fmm_plan;

/* Operators of one box width (row-major, natural sizes, n = nequiv).
 * Replaces KI_Precomputation (flexmm/flexmm2d/kifmm.py:13-62) and
 * Precomputation.compress / M2L_Evaluator (flexmm/flexmm2d/helpers.py:5-33,
 * 196-218). */
typedef struct fmm_level_ops {
  double width;                    /* box width w of this level               */
  const double *large_x, *large_y; /* [n] check circle of radius w(4-sqrt2)/2 */
  const double *c2e_u;             /* [n*n] U of S2L = U diag(S) VH          */
  const double *c2e_sinv;          /* [n] 1/S (0 for discarded values)        */
  const double *c2e_vh;            /* [n*n] VH                                */
  const double *m2mc;              /* [n * 4n] child equivalent circles -> check circle */
  const int *m2l_rank;             /* [40] -1 dense, 0 null, r > 0 SVD rank   */
  const double *const *m2l_a;      /* [40] dense: M2L [n*n]; SVD: M2 [n*r]    */
  const double *const *m2l_b;      /* [40] SVD: M1 [r*n]; otherwise unused    */
} fmm_level_ops;

/* Stokes FMM operator set (kifmm2d/vector/stokes_fmm.py:550-858): Nequiv
 * points per circle, 2 Nequiv + 1 values per box.  Per box width the host
 * supplies (n1 = 2 Nequiv + 1, n2 = 2 Nequiv, row-major, FP64):
 *   large_x/y [Nequiv]  the check / local-equivalent circle (dd = 0.1);
 *   e2c_u, e2c_sinv, e2c_vh   SVD of the corrected small-to-large form
 *                             [n1 x n1], 1/S with 0 where S < 1e-15;
 *   c2e_u, c2e_sinv, c2e_vh   the same for the large-to-small form;
 *   m2mc [n1 x 4 n2]      children equivalent forces -> parent check values;
 *   l2lc [4 n1 x n2]      parent local forces -> children partial locals;
 *   m2l: per offset rank < 0 dense [n1 x n2], rank > 0 M2 [n1 x r], M1 [r x n2].
 * (Precomputation, stokes_fmm.py:541-591.)  Plans on such a set build with
 * fmm_build_expansions2 and evaluate with FMM_EVAL_STOKES. */
typedef struct fmm_stokes_level_ops {
  double width;
  const double *large_x, *large_y;
  const double *e2c_u, *e2c_sinv, *e2c_vh;
  const double *c2e_u, *c2e_sinv, *c2e_vh;
  const double *m2mc, *l2lc;
  const int *m2l_rank;
  const double *const *m2l_a;
  const double *const *m2l_b;
} fmm_stokes_level_ops;
int fmm_stokes_ops_create(int nequiv, fmm_ops **out);
int fmm_stokes_ops_add(fmm_ops *ops, const fmm_stokes_level_ops *lv, int *level_id);
/* FMM.build_expansions(taux, tauy) of the Stokes FMM (stokes_fmm.py:642-735):
 * device forces in the caller's source order. */
int fmm_build_expansions2(fmm_plan *plan, const double *fx, const double *fy, void *stream);
/* The Stokes FMM's build_expansions_dipole(taux, tauy, sigmax, sigmay, dipx,
 * dipy) (stokes_fmm.py:738-826): forces plus stresslets of strength
 * (sigma_x, sigma_y) along the normals (dip_nx, dip_ny), device arrays in the
 * caller's source order.  Its evaluations (FMM_EVAL_STOKES) add the
 * stresslets' near field (evaluate_to_points_dipole, stokes_fmm.py:844-858);
 * the expansions carry both. */
int fmm_build_expansions2_dipole(fmm_plan *plan, const double *fx, const double *fy,
                                 const double *sigma_x, const double *sigma_y,
                                 const double *dip_nx, const double *dip_ny, void *stream);

/* Kernel ids: 0 Laplace -log(r^2)/(4 pi) (examples/kifmm_laplace.py:24-29);
 * 1 modified Helmholtz K0(k r)/(2 pi), kparams[0] = k
 * (examples/kifmm_modified_helmholtz.py:25-39); 2 a tabulated radial kernel
 * f(r), kparams[0] = the id from fmm_kernel_table_create. */
#define FMM_KERNEL_MOD_HELMHOLTZ 1
#define FMM_KERNEL_RADIAL_TABLE 2
/* Register a radial kernel f(r) tabulated as Chebyshev series on the octaves
 * [2^j, 2^(j+1)), j = j0 .. j0 + n_octaves - 1: coef[n_octaves][n_cheb],
 * series in u = (2 r - 3 2^j) / 2^j.  Replaces the reference examples'
 * function_generator tables (examples/bbfmm_struve.py:34-46,
 * kifmm_modified_helmholtz.py:28).  Distances outside the range are clamped
 * to it.  Tables live until the process exits. */
int fmm_kernel_table_create(const double *coef, int j0, int n_octaves, int n_cheb, int *table_id);

/* Black-box (Chebyshev) FMM operator set, BB_FMM / BB_Helper
 * (flexmm/flexmm2d/bbfmm.py:133-231): Chebyshev order p (2..16, NQ = p^2
 * coefficients per box) and the level-independent M2MC [NQ x 4NQ] (child
 * blocks ordered (-,-), (-,+), (+,-), (+,+)), row-major host memory.  Plans
 * built on it run S2M moments, M2M, M2L, L2L, L2T as the reference's BB_FMM,
 * in FP64; fmm_plan_create / bind / build_expansions / evaluate take it like
 * a KIFMM set. */
#define FMM_BB_MAX_P 16
int fmm_bb_ops_create(int kernel_id, const double *kparams, int p, const double *m2mc,
                      fmm_ops **out);
/* One box width's 40 M2L operators VI K VI^T (bbfmm.py:101-122), in the
 * fmm_level_ops convention: rank < 0 dense [NQ x NQ] in m2l_a, rank > 0 the
 * factors M2 [NQ x r] (m2l_a) and M1 [r x NQ] (m2l_b), 0 none. */
typedef struct fmm_bb_level_ops {
  double width;
  const int *m2l_rank;
  const double *const *m2l_a;
  const double *const *m2l_b;
} fmm_bb_level_ops;
int fmm_bb_ops_add(fmm_ops *ops, const fmm_bb_level_ops *lv, int *level_id);

int fmm_ops_create(int kernel_id, const double *kernel_params /* [4] or NULL */, int nequiv,
                   fmm_ops **out);
int fmm_ops_add(fmm_ops *ops, const fmm_level_ops *level, int *level_id);
int fmm_ops_destroy(fmm_ops *ops);

/* Build the quadtree of n sources (device x, y) with at most ncutoff points
 * per leaf over the square bbox = {xmin, xmax, ymin, ymax} (host array).
 * Device memory comes from the device's default stream-ordered pool; the
 * first plan on a device sets that pool to keep freed memory and reserves up
 * to 1 GiB (at most 1/8 of the free memory) in it, so that later plans do
 * not map memory while earlier work is still queued. */
int fmm_plan_create(fmm_ops *ops, const double *x, const double *y, int64_t n, int ncutoff,
                    const double *bbox, void *stream, fmm_plan **out);
/* Near-field-only evaluation, the LocalEvaluator family
 * (flexmm/flexmm2d/local_evaluator.py, local_evaluator_category.py,
 * periodic_local_evaluator_category.py; LocalTree, flexmm/local_tree.py):
 * fmm_plan_create_local builds the tree of fmm_plan_create except that a box
 * splits only while it holds more than ncutoff points AND its width exceeds
 * 2 min_width (local_tree.py:191-222), on an operator set of the kernel
 * (fmm_ops_create; no levels need binding).  fmm_local_evaluate sums, at m
 * device points, the kernel over the sources of the target leaf's
 * colleagues only -- no far field -- with charges tau (caller's source
 * order); check != 0 skips coincident sources; src_cat / tgt_cat (device
 * int64, both or neither) leave out sources whose category equals the
 * target's (local_evaluator_category.py:33-38).  out[m] is overwritten. */
int fmm_plan_create_local(fmm_ops *ops, const double *x, const double *y, int64_t n, int ncutoff,
                          double min_width, const double *bbox, void *stream, fmm_plan **out);
int fmm_local_evaluate(fmm_plan *plan, const double *tau, const double *tx, const double *ty,
                       int64_t m, int check, const int64_t *src_cat, const int64_t *tgt_cat,
                       double *out, void *stream);

/* n_levels and, for each level, its box width and node count (host arrays of
 * FMM_MAX_LEVELS entries). */
int fmm_plan_info(fmm_plan *plan, int *n_levels, double *widths, int *n_nodes);
/* Arithmetic of the passes (the precision forms of the path):
 *   FMM_PRECISION_FP64   everything in FP64 (matches the reference to 1e-12);
 *   FMM_PRECISION_MIXED  FP32 kernel evaluations (P2P with compensated sums),
 *                        split-precision (3xTF32) tensor-core M2M / M2L / L2L
 *                        with FP32 accumulate on mean-deflated operators,
 *                        FP64 check-to-equivalent and final accumulation.
 *                        KIFMM plans of the Laplace kernel (potential and
 *                        gradient) and the modified Helmholtz kernel
 *                        (potential; FP32 K0 from the Abramowitz-Stegun
 *                        polynomials); other plans return FMM_ERR_UNSUPPORTED.
 * Set before fmm_build_expansions (it invalidates previous expansions). */
#define FMM_PRECISION_FP64 0
#define FMM_PRECISION_MIXED 1
int fmm_plan_set_precision(fmm_plan *plan, int precision);
/* Use operator entry level_id (from fmm_ops_add) for tree level `level`. */
int fmm_plan_bind(fmm_plan *plan, int level, int level_id);
/* fmm_plan_bind for levels 0 .. n_levels-1 in one call: level_ids[l] for
 * level l (-1 leaves a level unbound).  Same operator cache as
 * fmm_plan_bind (KI_Helper.prepare, kifmm.py:67-82). */
int fmm_plan_bind_levels(fmm_plan *plan, int n_levels, const int *level_ids);
/* tau: device charges [n] in the caller's (original) source order. */
int fmm_build_expansions(fmm_plan *plan, const double *tau, void *stream);
/* Potential at m device points into device out[m]; check != 0 skips sources
 * that coincide with the target (source evaluation). */
int fmm_evaluate(fmm_plan *plan, const double *tx, const double *ty, int64_t m, int check,
                 double *out, void *stream);
/* Potential at the plan's own source points (the coordinates given to
 * fmm_plan_create, as the tree build copied them) into device out[n], in the
 * caller's original source order; check != 0 skips coincident sources.
 * Equal to fmm_evaluate(plan, x, y, n, check, out, stream) on unchanged x, y,
 * without re-reading, re-locating and re-sorting the points: the tree already
 * holds them sorted by leaf.  Replaces FMM.source_evaluation(x, y) called on
 * the FMM's own sources (flexmm/flexmm2d/fmm.py:158-159, 162-176). */
int fmm_evaluate_sources(fmm_plan *plan, int check, double *out, void *stream);

/* Charges and dipoles: the Laplace single plus double layer of the
 * reference's kifmm2d FMM with the example's upwardor Laplace_Both_Eval
 * (build_expansions(tau, 'slp+dlp', extras), flexmm/kifmm2d/scalar/fmm.py:73-124,
 * 168-176; examples/pure_kifmm_laplace_dipoles.py:31-40, 94-98): source j
 * carries the charge tau[j] (NULL: none) and the dipole of strength
 * dip_str[j] along the normal (dip_nx[j], dip_ny[j]), all device arrays in the
 * caller's source order.  The field at t of a source at s is
 *   -log|t - s|^2 / (4 pi) tau + (n . (t - s)) / |t - s|^2 / (2 pi) str.
 * FP64 KIFMM plans of the Laplace kernel.  Evaluations after it (potential
 * only) include both layers in the near field; the expansions carry both. */
int fmm_build_expansions_dipole(fmm_plan *plan, const double *tau, const double *dip_str,
                                const double *dip_nx, const double *dip_ny, void *stream);

/* Several charge columns on one tree (multi-RHS; the reference's kifmm2d
 * FMM takes tau [k, N], flexmm/kifmm2d/scalar/fmm.py:71-87): column r is
 * tau[r * ld_tau .. + n), caller's source order.  FP64 KIFMM plans.  The
 * evaluation computes each kernel value once for up to 8 columns; result
 * row r is out[r * ld_out .. + m).  fmm_evaluate after a multi build uses
 * column 0. */
int fmm_build_expansions_multi(fmm_plan *plan, const double *tau, int n_rhs, int64_t ld_tau,
                               void *stream);
int fmm_evaluate_multi(fmm_plan *plan, const double *tx, const double *ty, int64_t m, int check,
                       double *out, int64_t ld_out, void *stream);
int fmm_evaluate_sources_multi(fmm_plan *plan, int check, double *out, int64_t ld_out, void *stream);

/* Several outputs per point, as the reference's named evaluators
 * (kifmm2d FMM.register_evaluator + evaluate_to_points,
 * flexmm/kifmm2d/scalar/fmm.py:172-199, helpers.py:176-238):
 *   FMM_EVAL_POTENTIAL  1 row:  u
 *   FMM_EVAL_GRADIENT   3 rows: u, du/dx, du/dy (derivatives in the target
 *                       position; examples/pure_kifmm_laplace_gradient.py:32-55)
 * Row r of the result is out[r * ld_out .. r * ld_out + m), ld_out >= m. */
#define FMM_EVAL_POTENTIAL 0
#define FMM_EVAL_GRADIENT 1
#define FMM_EVAL_STOKES 2 /* Stokes plans: 3 rows u, v, p (stokes_fmm.py:820-835) */
int fmm_evaluate_outputs(fmm_plan *plan, int evaluator, const double *tx, const double *ty,
                         int64_t m, int check, double *out, int64_t ld_out, void *stream);
/* The same at the plan's own source points (see fmm_evaluate_sources). */
int fmm_evaluate_sources_outputs(fmm_plan *plan, int evaluator, int check, double *out,
                                 int64_t ld_out, void *stream);
/* Release the plan's expansions (and its sorted charges), keeping the tree:
 * a later fmm_build_expansions forms them again.  The differentiation form
 * (torch.autograd) uses it to recompute expansions in its backward pass
 * instead of holding them between forward and backward.  No counterpart in
 * the reference, whose FMM objects hold their expansions. */
int fmm_plan_drop_expansions(fmm_plan *plan);
/* Move the plan's sources to new coordinates (device x, y in the caller's
 * original order) without rebuilding the tree: every source keeps the leaf
 * the tree gave it ("frozen tree"; points may leave their box slightly).
 * Expansions must be built again afterwards.  For finite-difference checks
 * and optimisation loops over slowly moving points; no counterpart in the
 * reference, whose Tree copies the points once (flexmm/tree.py:459-460). */
int fmm_plan_move_sources(fmm_plan *plan, const double *x, const double *y, void *stream);
/* Releases the plan without waiting for the GPU: its device memory returns to
 * the pool in stream order on the plan's stream (one stream per plan), so a
 * loop that builds a plan per step keeps the host ahead of the GPU. */
int fmm_plan_destroy(fmm_plan *plan);
/* Wait for the plan's work and report failures of it: FMM_ERR_CUDA when a
 * kernel stopped one of its bounded waits (the results are then invalid). */
int fmm_plan_status(fmm_plan *plan);

/* Copy the tree to host arrays sized by fmm_plan_info (nodes = sum n_nodes):
 * xmin, ymin [nodes]; bot, top, parent, child [nodes]; flags [nodes]
 * (1 leaf, 2 fake leaf, 4 X-list, 8 has children); coll [nodes*9];
 * il [nodes*40] (source node per offset, -1 none); ordv [n] (sorted ->
 * original source index).  Any pointer may be NULL. */
int fmm_tree_export(fmm_plan *plan, double *xmin, double *ymin, int *bot, int *top, int *parent,
                    int *child, uint8_t *flags, int *coll, int *il, int *ordv);

/* FP64 direct sum over all ns sources at nt targets (device pointers);
 * check != 0 skips coincident pairs.  Replaces kernel_apply /
 * kernel_apply_single_check (flexmm/flexmm2d/helpers.py:91-116); used as the
 * accuracy reference. */
int fmm_direct(int kernel_id, const double *kernel_params, const double *sx, const double *sy,
               const double *tau, int64_t ns, const double *tx, const double *ty, int64_t nt,
               int check, double *out, void *stream);

/* Per-kernel CUDA-event timing, the per-phase timers of the reference's
 * verbose mode (flexmm/flexmm2d/fmm.py:24-30, 55-58, 106-107, 148-149).
 * fmm_timing_read returns, per phase, the summed milliseconds and the number
 * of timed launches since the last read, then clears them.  Phases:
 * 0 tree build (span), 1 targets into leaves (binning for KIFMM plans, a
 * sort for black-box and Stokes plans, and the work items), 2 upward, 3 M2L, 4 downward,
 * 5 evaluation (L2T + P2P), 6 direct sum, 7-9 the tree build's three
 * stages (keys/sort/initial splits, 2:1 closure and X-list, node arrays),
 * 10 expansion set-up (charge gather, buffers, charge sums). */
#define FMM_N_PHASES 12
int fmm_timing_enable(int on);
int fmm_timing_read(double *ms /* [FMM_N_PHASES] */, int64_t *launches /* [FMM_N_PHASES] */);

/* Whether evaluation at a plan's own sources runs split: the near field
 * (P2P) on a side stream, started once the charges are sorted, beside the
 * upward/M2L/downward passes, and the far field (L2T) after them.  mode 1 on,
 * 0 off (one evaluation kernel after the passes), -1 the default (on for
 * both forms; the environment variable FLEXMM_B200_SPLIT_EVAL=0/1 overrides
 * the default).  Process-wide; results
 * agree to rounding either way.  No reference counterpart (the reference
 * evaluates after its passes, flexmm/flexmm2d/fmm.py:150-157). */
int fmm_set_split_evaluation(int mode);

/* Allocation-free fmm_evaluate, for callers that cannot allocate device
 * memory at evaluation time: e.g. an application that has reserved the whole
 * GPU for its own pool, or a loop that must not touch the allocator.  It has
 * no counterpart in the reference.  It serves FP64 KIFMM plans (Laplace,
 * modified Helmholtz and tabulated radial kernels; the potential, one value
 * per target) and refuses mixed-precision, black-box and Stokes plans with
 * FMM_ERR_UNSUPPORTED before queueing any work.  For the plans it serves it
 * computes what fmm_evaluate computes, with the plan built and expanded
 * beforehand; its scratch is a
 * 24 MiB array inside the library (held on every GPU that loads it until
 * exit), shared by all calls and keeping the last call's contents.  Calls
 * that overlap on the GPU race on it: serialise them.  The first call on a
 * device looks up the array's device address once (cudaGetSymbolAddress);
 * make that first call before any stream capture.  Limits: m <=
 * FMM_NOALLOC_MAX_TARGETS targets and a tree of at most FMM_NOALLOC_MAX_NODES
 * nodes; larger requests fail with FMM_ERR_CAPACITY. */
#define FMM_NOALLOC_MAX_TARGETS 262144
#define FMM_NOALLOC_MAX_NODES 262144
int fmm_evaluate_noalloc(fmm_plan *plan, const double *tx, const double *ty, int64_t m, int check,
                         double *out, void *stream);

/* Diagnostic: the table-driven log2 that the FP64 passes use for the
 * Laplace kernel (exponent split, a 257-entry table of 1/F and log2 F,
 * degree-5 series; Tang, ACM TOMS 16, 1990) and CUDA's log2, at n device
 * points x, into out_table and out_library.  For tests of its accuracy. */
int fmm_diag_log2(const double *x, int64_t n, double *out_table, double *out_library,
                  void *stream);

const char *fmm_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
