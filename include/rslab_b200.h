/*
 * rslab_b200 — C ABI of the B200-native supernodal LDL^T factor + solve.
 *
 * The drop-in boundary for RSLAB's symmetric direct-solver path.  Every entry
 * point takes plain pointers and sizes, returns an int status (0 = ok) and
 * never throws; rslab_last_error() gives the message of the calling thread's
 * last failure.  Status codes mirror RslabError (src/error.rs:15-55).
 *
 * Reference interfaces replaced (paths in the RSLAB source tree):
 *   rslab_analyze        LdltSymbolic::analyze / analyze_with
 *                        (src/numeric/sparse_solver.rs:493,506) ->
 *                        multifrontal_ldlt::analyze_with (src/numeric/multifrontal_ldlt.rs:1667)
 *   rslab_analyze_tuned  LdltSolver::tuned + nd_bakeoff (src/numeric/sparse_solver.rs:108-131,231-266)
 *   rslab_symbolic_estimate LdltSymbolic::estimate_memory / symbolic_factor_nnz
 *                        (src/numeric/sparse_solver.rs:550-660)
 *   rslab_factor         LdltSymbolic::factor (src/numeric/sparse_solver.rs:677) ->
 *                        factor_numeric (src/numeric/multifrontal_ldlt.rs:1851)
 *   rslab_refactor       LdltSymbolic::factor on a new value set of the same
 *                        pattern (frequency sweeps, src/numeric/sparse_solver.rs:457-478)
 *   rslab_solve          LdltSolver::solve / solve_many (src/numeric/sparse_solver.rs:274,302)
 *   rslab_mixed_factor   MixedLdltSolver::factor / factor_with (src/numeric/mixed.rs:234,245)
 *   rslab_mixed_solve    MixedLdltSolver::solve / solve_to (src/numeric/mixed.rs:258,267)
 *   rslab_tier_factor    MixedLdltSolver::factor with the precision chosen per
 *                        matrix (src/numeric/mixed.rs:234); rslab_tier_mlp_*
 *                        (the network that chooses it) have no counterpart
 *   rslab_factor_info    LdltSolver::inertia / n_perturbed / diagnostics
 *                        (src/numeric/sparse_solver.rs:81,72,57)
 *   rslab_export_factors LdltFactors (src/dense/ldlt_generic.rs:31-66), the
 *                        factor_numeric return value
 *   rslab_compress_factors / rslab_cfac_*  CompressedLdltFactors (src/dense/ldlt_generic.rs:434-536)
 *   rslab_amd_order      rslab_amd::amd_order (crates/rslab-amd/src/lib.rs:66)
 *   rslab_metis_order    rslab_metis::metis_order_full (crates/rslab-metis/src/lib.rs:204)
 */
#ifndef RSLAB_B200_H
#define RSLAB_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RSLAB_ABI_VERSION 1

/* Status codes (RslabError). */
#define RSLAB_OK 0
#define RSLAB_NUMERICALLY_RANK_DEFICIENT 1
#define RSLAB_INVALID_INPUT 2
#define RSLAB_DIMENSION_MISMATCH 3
#define RSLAB_CUDA_ERROR 4

/* Scalar fields: the reference's f64 / Complex<f64> / f32 / Complex<f32>.
 * Complex values are interleaved (re, im) pairs; complex matrices are
 * complex-SYMMETRIC (A = A^T), never Hermitian. */
#define RSLAB_F64 0
#define RSLAB_C64 1
#define RSLAB_F32 2
#define RSLAB_C32 3

/* Orderings (OrderingMethod, src/symbolic/mod.rs:28). */
#define RSLAB_ORDER_AMD 0      /* rslab_amd::amd_order (crates/rslab-amd/src/lib.rs:66) */
#define RSLAB_ORDER_METIS_ND 1 /* rslab_metis::metis_order (crates/rslab-metis/src/lib.rs:184) */
#define RSLAB_ORDER_NATURAL 2
#define RSLAB_ORDER_GIVEN 3

/* Zero-pivot policy (ZeroPivotAction, src/numeric/multifrontal_ldlt.rs:165). */
#define RSLAB_PIVOT_FAIL 0
#define RSLAB_PIVOT_PERTURB 1
/* ZeroPivotAction::ForceAccept: static pivoting with the floor
 * max(max|A_scaled|, 1) * eps computed on the device at factor time
 * (factor_left_looking, src/numeric/multifrontal_ldlt.rs:3355-3358). */
#define RSLAB_PIVOT_FORCE_ACCEPT 2

/* Equilibration (ScalingStrategy): one-pass inf-norm (default) or identity. */
#define RSLAB_SCALING_ONEPASS 0
#define RSLAB_SCALING_IDENTITY 1

typedef struct rslab_sym_handle rslab_sym_handle;
typedef struct rslab_fac_handle rslab_fac_handle;

/* Analyze-time half of SolverSettings (defaults :583-614). */
typedef struct {
  int32_t ordering;            /* RSLAB_ORDER_* (default AMD) */
  int64_t nemin;               /* 16 */
  int32_t relax;               /* relaxed amalgamation on (1) */
  int64_t relax_max_width;     /* 256 */
  int64_t relax_max_extra_rows;/* 64 */
  int32_t hybrid_liu;          /* child reordering (scheduling only) */
  int64_t panel_nb;            /* BK panel width, 64 (128 when ncol >= 512); clamped to [8, 128] */
  const int64_t* given_perm;   /* RSLAB_ORDER_GIVEN: new-to-old permutation */
} rslab_analyze_settings;

/* Numeric half of SolverSettings. */
typedef struct {
  int32_t on_zero_pivot;       /* RSLAB_PIVOT_FAIL | RSLAB_PIVOT_PERTURB */
  double abs_floor;            /* PerturbToEps floor */
  int32_t scaling;             /* RSLAB_SCALING_* */
  int32_t use_graph;           /* capture factor / solve as CUDA graphs (1) */
  void* stream;                /* cudaStream_t to run on, or NULL for a private one */
  int32_t schur_engine;        /* RSLAB_SCHUR_*: how descendant updates run (AUTO) */
  double drop_tol;             /* > 0: incomplete factor, drop |L_ip| < drop_tol * max_i |L_ip| per
                                * column (SolverSettings::drop_tol, multifrontal_ldlt.rs:2359-2367) */
  int32_t overlap;             /* schedule: run the Schur update beyond the next block and the next
                                * level's early descendant updates on side streams (1, default) or
                                * everything in order on one stream (0); the factor is the same */
  int32_t method;              /* RSLAB_METHOD_*: SolverSettings::method (FactorMethod,
                                * multifrontal_ldlt.rs:283) */
} rslab_factor_settings;

/* Numeric schedule.  RSLAB_METHOD_LEFT_LOOKING (default): every supernode
 * gathers its descendants' updates (cmod, per the schur_engine).
 * RSLAB_METHOD_MULTIFRONTAL: every supernode's front is its panel plus a
 * contribution block; the children's contribution blocks are extend-added
 * into it (in child order, deterministic), the panel is factored with the same
 * Bunch-Kaufman kernels, and the contribution block becomes CB - L21 D L21^T
 * for the parent (factor_front + extend-add, multifrontal_ldlt.rs:901,
 * 1494-1510).  Same pivoting; the sums run in another order, so the factors
 * agree with the left-looking ones to rounding.  schur_engine picks the panel
 * kernels as for the left-looking method and, for f64 / c64, the engine of the
 * contribution-block products (FP64 tensor-core tiles or the CUDA-core FMA
 * tiles; the f32 / c32 ones run on the CUDA cores).  It holds every
 * contribution block (sum of (nrow - ncol)^2 scalars) for the factor's
 * lifetime and allocates none of the left-looking update buffers. */
#define RSLAB_METHOD_LEFT_LOOKING 0
#define RSLAB_METHOD_MULTIFRONTAL 1

/* Descendant (cmod) updates.  RSLAB_SCHUR_TENSOR: per (updater, target) pair
 * a dense product over the updater's contiguous rows, in GEMM tiles on the
 * tensor cores (f32 / c32: tcgen05 3xTF32 split products with fp32
 * accumulation, operands staged by TMA, complex products in the 3M form of
 * three real products; f64 / c64: FP64 DMMA), written to a
 * level workspace and assembled into the targets in update order
 * (deterministic; parity with the oracle by tolerance).  RSLAB_SCHUR_FMA: FMA
 * on the CUDA cores in the oracle's operation order (bit-exact).
 * RSLAB_SCHUR_AUTO (default): TENSOR when the analysis' model flops reach
 * RSLAB_SCHUR_AUTO_MIN_FLOPS, else FMA — below that size the workspace and
 * assembly launches cost more than the tiles save, and the factor keeps the
 * oracle's bits (and so its pivot decisions on near-singular KKT systems).
 * rslab_factor_info reports the engine a factor ran with. */
#define RSLAB_SCHUR_TENSOR 0
#define RSLAB_SCHUR_FMA 1
#define RSLAB_SCHUR_AUTO 2
#define RSLAB_SCHUR_AUTO_MIN_FLOPS 2.0e8

typedef struct {
  int64_t n, nnz, nsuper, nlevels;
  int64_t factor_nnz_sym;      /* sum of symbolic column counts */
  int64_t panel_elems;         /* device panel pool size in scalars */
  double flops_model;          /* sum_s sum_{m=r-c+1}^{r} (m^2 - 1) */
  double flops_proxy;          /* sum_s r^2 c (factor_flops of the reference) */
  int32_t renumbered;
  int64_t amd_ncmpa, amd_ndense;
  double amd_ndiv, amd_nms_ldl, amd_nms_lu;
  int64_t n_factor_launches, n_solve_launches;
  /* tensor-core cmod plan: 128 x 64 tiles, (updater, tile) pairs, and K
   * chunks staged (16 complex / 32 real updater columns per chunk) */
  int64_t tc_tiles, tc_pairs, tc_chunks_complex, tc_chunks_real;
} rslab_symbolic_info_t;

typedef struct {
  int32_t status;              /* last factor status */
  int64_t failing_supernode;
  int64_t inertia_pos, inertia_neg, inertia_zero;
  int64_t n_perturbed;
  double factor_ms, solve_ms;  /* device time of the last factor / solve */
  int32_t dtype, dtype_hi;
  int32_t multiprocessors;     /* SMs of the handle's device (the reference's Diagnostics::threads
                                * counts CPU workers) */
  int32_t schur_engine;        /* RSLAB_SCHUR_TENSOR or RSLAB_SCHUR_FMA: the engine AUTO resolved to */
  int32_t method;              /* RSLAB_METHOD_* */
} rslab_factor_info_t;

typedef struct {
  int64_t ir_iters;
  int64_t gmres_iters;
  double backward_error;       /* max over right-hand sides */
  int32_t certified;           /* backward_error <= target for every rhs */
} rslab_mixed_info;

int rslab_version(void);
const char* rslab_last_error(void);
int rslab_device_count(int* count);

void rslab_default_analyze_settings(rslab_analyze_settings* s);
void rslab_default_factor_settings(rslab_factor_settings* s);

/* Phase 1: analyze a lower-triangle CSC pattern (n, col_ptr[n+1], row_idx). */
int rslab_analyze(int64_t n, const int64_t* col_ptr, const int64_t* row_idx,
                  const rslab_analyze_settings* settings, rslab_sym_handle** out);
/* CscMatrix::validate (src/sparse/csc.rs:157) for a lower-triangular CSC: col_ptr
 * starts at 0, ends at nnz and never decreases; row indices in [0, n), on or
 * below the diagonal and strictly increasing in each column.  Returns
 * RSLAB_INVALID_INPUT with a message naming the first offending column. */
int rslab_validate_lower_csc(int64_t n, const int64_t* col_ptr, const int64_t* row_idx, int64_t nnz);
int rslab_symbolic_info(const rslab_sym_handle* sym, rslab_symbolic_info_t* info);

/* A-priori memory and work estimate of an analysis for a scalar of
 * value_bytes bytes: LdltSymbolic::estimate_memory
 * (src/numeric/sparse_solver.rs:561-660; estimate_left_looking,
 * src/diagnostics.rs:116-175) and LdltSymbolic::symbolic_factor_nnz (:550).
 * panel_live_peak_bytes is the live-panel peak of the left-looking refcount
 * free schedule; factor_flops = sum_s nrow^2 ncol. */
typedef struct {
  int64_t value_bytes, factor_nnz, factor_bytes, panels_all_bytes;
  int64_t panel_live_peak_bytes, transient_peak_bytes;
  uint64_t factor_flops, critical_path_flops;
  int64_t max_tree_width;
  int64_t symbolic_factor_nnz; /* exact column-count fill x 1.2 (src/symbolic/mod.rs:1189,1202) */
  /* MemoryEstimate::mf_transient_peak_bytes (src/diagnostics.rs:30-40): the
   * figure for RSLAB_METHOD_MULTIFRONTAL, which here keeps every contribution
   * block resident: transient_peak_bytes + sum (nrow - ncol)^2 value_bytes */
  int64_t mf_transient_peak_bytes;
} rslab_memory_estimate_t;
int rslab_symbolic_estimate(const rslab_sym_handle* sym, int64_t value_bytes, rslab_memory_estimate_t* est);

/* The default settings pick behind LdltSolver::factor: LdltSolver::tuned
 * (src/numeric/sparse_solver.rs:108-131) with the nested-dissection bakeoff
 * nd_bakeoff (:231-266).  Analyses with the default settings (AMD); when
 * n >= 10,000 and that analysis predicts factor_flops >= 5e9 for a scalar
 * of value_bytes bytes, analyses again with MetisND and adopts it only if its
 * factor_flops is below 0.75x, its symbolic_factor_nnz is not larger and its
 * live-panel peak is not larger (constants :31-36).  *ordering_used gets the
 * RSLAB_ORDER_* of the returned analysis. */
#define RSLAB_ND_BAKEOFF_MIN_FLOPS 5000000000LL
#define RSLAB_ND_BAKEOFF_MIN_N 10000
#define RSLAB_ND_BAKEOFF_ADOPT_RATIO 0.75
int rslab_analyze_tuned(int64_t n, const int64_t* col_ptr, const int64_t* row_idx, int64_t value_bytes,
                        rslab_sym_handle** out, int32_t* ordering_used);
int rslab_symbolic_export(const rslab_sym_handle* sym, int64_t* perm, int64_t* sn_first, int64_t* sn_ncol,
                          int64_t* sn_nrow, int64_t* sn_level, int64_t* child_ptr, int64_t* child_idx,
                          int64_t* col_counts, int64_t* parent);
void rslab_free_symbolic(rslab_sym_handle* sym);

/* Independent systems as one analysis (no reference counterpart: the
 * reference factors them one call at a time; `rslab_factor_batch` of the
 * design sketch is this entry plus rslab_factor on the concatenated values).
 * System i keeps its own LdltSymbolic::analyze result (orderings, supernodes
 * and update lists identical to a lone analysis); the systems are laid out
 * block-diagonally (columns and stored entries concatenated in input order)
 * so one launch per assembly-tree level covers that level of every system.
 * Values / right-hand sides of the batch are the systems' arrays
 * concatenated; rslab_mixed_solve on a batch handle certifies every
 * (system, column) unit separately. */
int rslab_analyze_batch(int64_t count, const int64_t* n, const int64_t* const* col_ptr,
                        const int64_t* const* row_idx, const rslab_analyze_settings* settings,
                        rslab_sym_handle** out);
/* count systems; seg_begin[count+1] column offsets; nnz_begin[count+1] value offsets. */
int rslab_batch_layout(const rslab_sym_handle* sym, int64_t* count, int64_t* seg_begin, int64_t* nnz_begin);
/* Per (system, column) backward errors of the handle's last rslab_mixed_solve,
 * index system * nrhs + column; *count = systems * nrhs (at most cap written). */
int rslab_mixed_batch_result(const rslab_fac_handle* fac, int64_t cap, double* backward_error, int64_t* count);

/* Phases 2-3: equilibrate + numeric factor on the GPU.  `values` follow the
 * analysed pattern's row_idx order; host memory unless values_on_device.  On a
 * singular pivot returns RSLAB_NUMERICALLY_RANK_DEFICIENT and still hands
 * back the handle (for rslab_factor_info); it must be freed. */
int rslab_factor(rslab_sym_handle* sym, int dtype, const void* values, int values_on_device,
                 const rslab_factor_settings* settings, rslab_fac_handle** out);
int rslab_refactor(rslab_fac_handle* fac, const void* values, int values_on_device);
/* Static pivot reuse across a value sweep of one pattern (the LDL^T
 * counterpart of the reference's static-pivot sweep,
 * src/numeric/multifrontal_lu.rs:3551: factor once with the pivot search,
 * then refactor new values without it).  Every factor that searches records
 * its Bunch-Kaufman steps (1x1 / 2x2 and the interchange of each step); with
 * on = 1 the following refactors replay that record instead of searching, a
 * zero or (with static pivoting) tiny pivot being perturbed as usual; on = 0
 * restores the search.  Pair it with refinement (rslab_mixed_solve) and fall
 * back to a searching refactor when a solve does not certify. */
int rslab_set_pivot_reuse(rslab_fac_handle* fac, int on);
/* x = A^-1 b, b and x row-major n x nrhs. */
int rslab_solve(rslab_fac_handle* fac, const void* b, int64_t nrhs, void* x, int on_device);
/* LdltSolver::solve_refined (src/numeric/sparse_solver.rs:335-375): solve, then
 * up to max_iter corrections x += A^-1 (b - A x) against the factored values,
 * in the factor's field, keeping per column the iterate of smallest ||r||_inf. */
int rslab_solve_refined(rslab_fac_handle* fac, const void* b, int64_t nrhs, int64_t max_iter, void* x,
                        int on_device);
int rslab_factor_info(const rslab_fac_handle* fac, rslab_factor_info_t* info);
void* rslab_factor_stream(const rslab_fac_handle* fac);
/* Eager refactor with per-launch CUDA events: device ms, launches and
 * algorithmic flops per kernel class ([0] equilibration + assembly, [1] cmod,
 * [2] BK panel getf2, [3] deep-row replay, [4] in-panel Schur, [5] total).
 * A measurement aid with no reference counterpart. */
int rslab_factor_profile(rslab_fac_handle* fac, double* kind_ms, int64_t* kind_launches, double* kind_flops);
/* Eager solve with per-launch CUDA events ([0] permute in/out, [1] forward
 * diagonal, [2] forward push, [3] D solve, [4] backward off-diagonal dots,
 * [5] backward diagonal, [6] total).  A measurement aid with no reference
 * counterpart. */
int rslab_solve_profile(rslab_fac_handle* fac, int64_t nrhs, double* kind_ms, int64_t* kind_launches);
/* Per-launch rows of the handle's last factor/solve profile: launch kind
 * (0 cmod, 1 getf2, 2 deep replay, 3 panel Schur, 4 forward diagonal,
 * 5 forward push, 6 backward dots, 7 backward diagonal, 8-11 see below, 13
 * multifrontal extend-add, 14 G = L21 D, 15 diagonal-block inverses, 17
 * tensor-core panel Schur (tcgen05 or DMMA tiles), 18/19 forward/backward
 * block-chain solve, 21 deep rows as a product with the block transform, 22
 * block transform, 23 forward push partial-sum reduction, 24 multifrontal
 * contribution block, -1 other; 12, 16 and 20 are not launched any more: the
 * chain items gather their own right-hand sides and sum split dots), grid
 * size and device ms.  *count = rows available; at most cap are written.
 * A measurement aid with no reference counterpart.  Kinds 8-11 are the
 * tensor-core cmod's GEMM tiles, its assembly and the real / complex operand
 * split. */
int rslab_profile_trace(const rslab_fac_handle* fac, int64_t cap, int32_t* kind, int32_t* grid, float* ms,
                        int64_t* count);
/* Reference LdltFactors layout; pass NULL arrays to query *nnz_out first. */
int rslab_export_factors(const rslab_fac_handle* fac, int64_t* l_col_ptr, int64_t* l_row_idx, void* l_values,
                         void* d_diag, void* d_subdiag, uint8_t* two_by_two, int64_t* perm, double* scale,
                         int64_t* nnz_out);
void rslab_free_factor(rslab_fac_handle* fac);

/* CompressedLdltFactors (src/dense/ldlt_generic.rs:434-536): the factor in
 * the LdltFactors layout with uint32 index arrays and pivot permutation, on
 * the host, and its single-right-hand-side solve with the reference's
 * solve_ldlt expressions (bit-identical to it on the same factors; like the
 * reference container it solves with the factors of the equilibrated matrix,
 * A_hat = S A S, S the rslab_export_factors scale).  rslab_compress_factors
 * returns RSLAB_INVALID_INPUT when n or nnz(L) does not fit 32 bits (the
 * reference's from_factors returns None).  index_bytes = 4 (n + 1 + nnz + n). */
typedef struct rslab_cfac_handle rslab_cfac_handle;
int rslab_compress_factors(const rslab_fac_handle* fac, rslab_cfac_handle** out);
int rslab_cfac_info(const rslab_cfac_handle* c, int64_t* n, int64_t* nnz, int64_t* index_bytes, int32_t* dtype);
int rslab_cfac_export(const rslab_cfac_handle* c, uint32_t* l_col_ptr, uint32_t* l_row_idx, void* l_values,
                      void* d_diag, void* d_subdiag, uint8_t* two_by_two, uint32_t* perm);
int rslab_cfac_solve(const rslab_cfac_handle* c, const void* rhs, void* x);
void rslab_free_cfac(rslab_cfac_handle* c);

/* Mixed precision: factor cast(A) in f32/c32, refine against the f64/c64 A. */
int rslab_mixed_factor(rslab_sym_handle* sym, int dtype_hi, const void* values_hi, int values_on_device,
                       const rslab_factor_settings* settings, rslab_fac_handle** out);
int rslab_mixed_solve(rslab_fac_handle* fac, const void* b, int64_t nrhs, double target, void* x, int on_device,
                      rslab_mixed_info* info);

/* Right-preconditioned restarted block GMRES (gmres_block,
 * src/numeric/iterative.rs:1881) on the handle's FP64 matrix (the original
 * matrix of a refined handle, the input of an f64 / c64 factor) with the
 * handle's factor as the preconditioner (Preconditioner for LdltSolver,
 * iterative.rs:178-190).  b, x0 (optional: NULL = zero start) and x are
 * row-major n x s, the layout of rslab_solve (the reference's block API is
 * column-major).  Columns run in groups of 16 in lockstep, one block
 * preconditioner apply and one block product per step; block classical
 * Gram-Schmidt with a per-column second pass, in-cycle deflation of
 * converged columns.  iters = block steps of the longest group, final_res[s]
 * = ||b_c - A x_c||_2 / ||b_c||_2, *converged = every column reached tol. */
int rslab_gmres_block(rslab_fac_handle* fac, const void* b, int64_t s, double tol, int64_t max_iter, int64_t restart,
                      const void* x0, void* x, int on_device, int64_t* iters, double* final_res, int* converged);

/* Precision tiers of a refined factor.  The tier fixes the precision the
 * factor is computed and stored in; refinement always runs against the
 * original FP64 matrix and certifies the normwise backward error. */
#define RSLAB_TIER_FP64 0   /* factor in the matrix's own field (f64 / c64) */
#define RSLAB_TIER_FP32 1   /* f32 / c32 factor, CUDA-core descendant updates */
#define RSLAB_TIER_TF32X3 2 /* f32 / c32 factor, 3xTF32 tensor-core descendant updates */

/* Refined factor in a chosen precision tier: rslab_mixed_factor generalised
 * (src/numeric/mixed.rs:234-256 factors in f32 / c32 only).  The handle is
 * solved with rslab_mixed_solve whatever the tier; RSLAB_TIER_FP64 makes the
 * plain FP64 factor the preconditioner of the same refinement ladder (the
 * fallback when a low tier does not certify). */
int rslab_tier_factor(rslab_sym_handle* sym, int dtype_hi, int tier, const void* values_hi, int values_on_device,
                      const rslab_factor_settings* settings, rslab_fac_handle** out);

/* Tier network: 8 features -> 64 -> 64 -> 3 tier probabilities (ReLU hidden
 * layers, softmax output), FP32.  No counterpart in the reference: it picks
 * the precision tier above per matrix, trained on labels the solver makes by
 * running every tier and keeping the cheapest one that certifies.  Parameters
 * (RSLAB_TIER_MLP_PARAMS floats): W1[64][8], b1[64], W2[64][64], b2[64],
 * W3[3][64], b3[3], rows = output units.  x is m x 8 row-major (already
 * standardised), y holds labels 0..2, w optional per-sample weights (NULL =
 * 1).  on_device = 1: every array is device memory. */
#define RSLAB_TIER_FEATURES 8
#define RSLAB_TIER_HIDDEN 64
#define RSLAB_TIER_COUNT 3
#define RSLAB_TIER_MLP_PARAMS 4931
/* probs: m x 3 softmax outputs. */
int rslab_tier_mlp_forward(const float* params, const float* x, int64_t m, float* probs, int on_device);
/* Gradient of the weighted mean cross-entropy sum_s w_s CE_s / sum_s w_s
 * with respect to the parameters (grad: RSLAB_TIER_MLP_PARAMS floats), and
 * that loss. */
int rslab_tier_mlp_grad(const float* params, const float* x, const int32_t* y, const float* w, int64_t m,
                        float* grad, float* loss, int on_device);
/* `epochs` full-batch Adam steps (beta 0.9 / 0.999, eps 1e-8, rate lr) on the
 * same loss, params updated in place; loss_curve[e] (optional) = the loss
 * before step e. */
int rslab_tier_mlp_train(float* params, const float* x, const int32_t* y, const float* w, int64_t m, int64_t epochs,
                         float lr, float* loss_curve, int on_device);

/* Synthetic-workload generator: m unit draws of the xorshift64* state
 * `state`; returns the advanced state. */
uint64_t rslab_rng_units(uint64_t state, int64_t m, double* out);

/* AMD on a full symmetric pattern; stats7 = ncmpa, ndense, ndiv, nms_ldl,
 * nms_lu, mass eliminations, supervariable merges. */
int rslab_amd_order(int64_t n, const int64_t* col_ptr, const int64_t* row_idx, int64_t* perm, double* stats7);

/* MetisND on a full symmetric pattern: rslab_metis::metis_order_full
 * (crates/rslab-metis/src/lib.rs:204) with the given seed, the opt-in
 * quasi-dense column quotient (dense_quotient != 0; columns of off-diagonal
 * degree above dense_threshold, or max(40, ceil(10 sqrt(n))) when it is < 0,
 * are ordered last, densest first) and otherwise default options; seed 1
 * without the quotient = metis_order (:184).  perm = new-to-old. */
int rslab_metis_order(int64_t n, const int64_t* col_ptr, const int64_t* row_idx, uint64_t seed, int dense_quotient,
                      int64_t dense_threshold, int64_t* perm);

/* Allocation-free dense panel factor.  No counterpart in the reference: an
 * addition for callers that cannot allocate device memory at factor time
 * (code embedded in another library's memory pool, capped or frozen
 * allocators, real-time loops that must not risk cudaMalloc latency or an
 * out-of-memory failure).  Factors one caller-owned dense panel
 * (nrow x ncol column-major device memory: the fully-summed block on top of
 * the off-diagonal rows, lower part) in place with the same panel-bounded
 * Bunch-Kaufman kernels as rslab_factor, writing d, dsub, kind (0 = 1x1,
 * 1/2 = first/second column of a 2x2 block), lperm (pivot position ->
 * pre-pivot column, ncol each) and status[4] (code, failing block, perturbed
 * count, unused), all caller-owned device memory.  All scratch lives in one
 * 1 MiB static device array that every GPU loading the library keeps until
 * exit: nrow <= 4096, ncol <= 1024 and panel_nb in [8, 64]; larger panels
 * are rejected with RSLAB_INVALID_INPUT.  Calls no allocator.  The first call
 * on a device looks up that array's device address, so make it before any
 * stream capture.  Every call shares the array: calls whose work overlaps
 * on the GPU (different streams, no ordering between them) race. */
int rslab_panel_factor_noalloc(int dtype, void* panel, int64_t nrow, int64_t ncol, int64_t panel_nb, void* d,
                               void* dsub, uint8_t* kind, int32_t* lperm, int32_t* status, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* RSLAB_B200_H */
