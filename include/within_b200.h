/*
 * within_b200.h -- C ABI of the B200-native solve phase of `within`.
 *
 * The entry points replace the reference's Rust API (paths relative to the
 * reference's crates/ directory):
 *
 *   within_solver_new          Solver::new               within/src/solver.rs:415-430
 *   within_solver_solve        Solver::solve             within/src/solver.rs:157-239
 *   within_solver_solve_batch  Solver::solve_batch       within/src/solver.rs:241-277
 *   within_solver_n_dofs/_obs  Solver::{n_dofs,n_obs}    within/src/solver.rs:284-292
 *   within_solve / _batch      orchestrate::{solve,solve_batch}  within/src/orchestrate.rs:151-184
 *   within_solver_free         Drop for Solver
 *   within_last_error          Display of WithinError    within/src/error.rs:61-90
 *
 * Configuration mirrors SolverParams / Preconditioner / LocalSolverConfig
 * (within/src/config.rs:43-236).  Every computation runs on the current CUDA
 * device through hand-written sm_100a kernels; there is no CPU fallback: when
 * no device is usable the calls fail with WITHIN_ERR_CUDA.
 *
 * Layouts: categories element (i, q) is codes[i*row_stride + q*col_stride]
 * (F-order: row_stride 1, col_stride n_obs).  Batch inputs and outputs are
 * RHS-major (column j of an F-order (n, k) array starts at j*n), matching
 * BatchSolveResult (within/src/orchestrate.rs:58-135).
 *
 * Thread safety: a solver may be used from several host threads; calls on one
 * solver are serialised internally.
 */
#ifndef WITHIN_B200_H
#define WITHIN_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes: one per WithinError variant (within/src/error.rs:25-59). */
enum {
    WITHIN_OK = 0,
    WITHIN_ERR_EMPTY_OBSERVATIONS = 1,
    WITHIN_ERR_OBSERVATION_COUNT_MISMATCH = 2,
    WITHIN_ERR_WEIGHT_COUNT_MISMATCH = 3,
    WITHIN_ERR_OVERFLOW = 4,
    WITHIN_ERR_SINGULAR_DIAGONAL = 5,
    WITHIN_ERR_LOCAL_SOLVER_BUILD = 6,
    WITHIN_ERR_PRECONDITIONER_BUILD = 7,
    WITHIN_ERR_ITERATIVE_SOLVE = 8,
    WITHIN_ERR_INVALID_ARGUMENT = 9, /* configuration rejected (PyValueError in within-py) */
    WITHIN_ERR_CUDA = 10             /* device unavailable or a CUDA call failed */
};

enum { WITHIN_KRYLOV_CG = 0, WITHIN_KRYLOV_GMRES = 1, WITHIN_KRYLOV_LSMR = 2 };
enum { WITHIN_OPERATOR_IMPLICIT = 0, WITHIN_OPERATOR_EXPLICIT = 1 };
enum { WITHIN_PRECOND_OFF = 0, WITHIN_PRECOND_ADDITIVE = 1, WITHIN_PRECOND_MULTIPLICATIVE = 2 };
/* Arithmetic of the inner Krylov solve.  FP64 is the plain drop-in; MIXED runs the
 * operator and Schwarz applies in FP32 inside an FP64 iterative-refinement loop. */
enum { WITHIN_PRECISION_FP64 = 0, WITHIN_PRECISION_MIXED = 1 };

/* SolverParams (within/src/config.rs:205-236). */
typedef struct {
    int32_t krylov;          /* WITHIN_KRYLOV_* */
    int32_t gmres_restart;   /* KrylovMethod::Gmres { restart } */
    int32_t operator_repr;   /* WITHIN_OPERATOR_* */
    double tol;
    int32_t maxiter;
    int32_t max_refinements;
    int32_t precision;       /* WITHIN_PRECISION_* (LSMR always runs in FP64) */
    int32_t lsmr_local_size; /* KrylovMethod::Lsmr { local_size }: windowed reorthogonalization
                                against this many past v vectors; 0 = None (lsmr.rs:106-121) */
} within_params;

/* Preconditioner + LocalSolverConfig (within/src/config.rs:76-117, 174-183). */
typedef struct {
    int32_t kind;                  /* WITHIN_PRECOND_* */
    uint64_t approx_chol_seed;
    uint32_t approx_chol_split;    /* split_merge; 0 or 1 = None */
    int32_t approx_schur_enabled;  /* 0 = exact Schur complement */
    uint64_t approx_schur_seed;
    uint32_t approx_schur_split;
    int32_t dense_threshold;
    int32_t reduction_strategy;    /* ReductionStrategy: 0 Auto, 1 AtomicScatter, 2 ParallelReduction
                                      (reported by the diagnostics; the device path has one reduction) */
} within_preconditioner;

typedef struct {
    int32_t converged;
    int32_t iterations;      /* Krylov iterations including refinement */
    double final_residual;   /* ||D'W(y - D x)|| / ||D'W y|| */
    double time_total;       /* seconds */
    double time_setup;
    double time_solve;
} within_solve_stats;

typedef struct within_solver within_solver;

/* Fill the reference defaults: CG, implicit, tol 1e-8, maxiter 1000, 2 refinements
 * (config.rs:227-236); additive Schwarz with LocalSolverConfig::solver_default()
 * (config.rs:108-117, within-py/src/lib.rs:546-552). */
void within_default_params(within_params *params);
void within_default_preconditioner(within_preconditioner *precond);

/* Solver::new.  weights may be NULL (unit weights).  precond may be NULL (no
 * preconditioner, Preconditioner.Off).  On success *out owns the device copy of
 * the design and the preconditioner factors. */
int within_solver_new(const uint32_t *codes, size_t n_obs, size_t n_factors,
                      int64_t row_stride, int64_t col_stride, const double *weights,
                      const within_params *params, const within_preconditioner *precond,
                      within_solver **out);
void within_solver_free(within_solver *solver);

size_t within_solver_n_dofs(const within_solver *solver);
size_t within_solver_n_obs(const within_solver *solver);
size_t within_solver_n_factors(const within_solver *solver);

/* Solver::solve: y (n_obs), x (n_dofs), demeaned (n_obs) are host buffers. */
int within_solver_solve(within_solver *solver, const double *y, double *x, double *demeaned,
                        within_solve_stats *stats);

/* Solver::solve_batch: ys (n_obs*k, RHS-major), x (n_dofs*k), demeaned (n_obs*k) host
 * buffers; stats has k entries; time_total of entry 0 is the batch total.  Calls on one
 * solver from several host threads are safe: each call has its own device buffers and
 * copy stream, the solves take turns, and a call's upload and download overlap the other
 * calls' solves (pinned host buffers make the copies asynchronous). */
int within_solver_solve_batch(within_solver *solver, const double *ys, size_t k, double *x,
                              double *demeaned, within_solve_stats *stats);

/* Same as solve_batch with device buffers, on the given CUDA stream (NULL = the
 * solver's own stream).  Inputs stay resident in HBM; no host copies of vectors. */
int within_solver_solve_batch_device(within_solver *solver, const double *d_ys, size_t k,
                                     double *d_x, double *d_demeaned, within_solve_stats *stats,
                                     void *cuda_stream);

/* One-shot orchestrate::solve / solve_batch (build, solve, free). */
int within_solve(const uint32_t *codes, size_t n_obs, size_t n_factors, int64_t row_stride,
                 int64_t col_stride, const double *y, const double *weights,
                 const within_params *params, const within_preconditioner *precond, double *x,
                 double *demeaned, within_solve_stats *stats);
int within_solve_batch(const uint32_t *codes, size_t n_obs, size_t n_factors, int64_t row_stride,
                       int64_t col_stride, const double *ys, size_t k, const double *weights,
                       const within_params *params, const within_preconditioner *precond,
                       double *x, double *demeaned, within_solve_stats *stats);

/* One problem of within_solve_many: a design, its weights (NULL = unit) and k RHS
 * (n_obs*k, RHS-major), with caller-provided outputs x (n_dofs*k, where n_dofs is the
 * sum over factors of max code + 1), demeaned (n_obs*k) and stats (k entries).
 * status receives the problem's result code. */
typedef struct {
    const uint32_t *codes;
    size_t n_obs, n_factors;
    int64_t row_stride, col_stride;
    const double *weights;
    const double *ys;
    size_t k;
    double *x;
    double *demeaned;
    within_solve_stats *stats;
    int32_t status;
} within_problem;

/* Many independent problems of uneven size (orchestrate::solve_batch applied to each),
 * solved concurrently: up to `concurrency` problems (<= 0: one per host core) are in flight at once,
 * each with its own solver and CUDA stream, so the kernels of small problems share the
 * GPU.  Every problem is attempted; the return value is WITHIN_OK or the code of the
 * first failed problem (its message in within_last_error), and each status says which.
 * The reference has no single call for this: its callers loop over problems. */
int within_solve_many(within_problem *problems, size_t n_problems, const within_params *params,
                      const within_preconditioner *precond, int32_t concurrency);

/* Operator applies on host vectors, for parity tests against the CPU oracle
 * (Operator::apply of GramianOperator, within/src/operator/gramian.rs:84-89, and of
 * FePreconditioner, within/src/operator/preconditioner.rs:108-154).
 * x, y: n_dofs*k RHS-major.  Precision follows the solver's params. */
int within_solver_apply_gramian(within_solver *solver, const double *x, size_t k, double *y);
int within_solver_apply_preconditioner(within_solver *solver, const double *r, size_t k, double *z);
/* D x (matvec_d, domain.rs:390-395): x n_dofs*k -> y n_obs*k; D'W r (rmatvec_wdt, :409-417). */
int within_solver_matvec_d(within_solver *solver, const double *x, size_t k, double *y);
int within_solver_rmatvec_wdt(within_solver *solver, const double *r, size_t k, double *x);

/* Setup introspection, for bit-exact checks of the integer setup against the oracle.
 * factor_meta: n_levels[q], offsets[q] (WeightedDesign::from_store, domain.rs:133-155). */
void within_solver_factor_meta(const within_solver *solver, int64_t *n_levels, int64_t *offsets);
int32_t within_solver_n_subdomains(const within_solver *solver);
/* info[8] = q, r, n_local, n_q, n_r, eliminate_q, reduced_kind (0 dense, 1 ac), n_reduced */
void within_solver_subdomain_info(const within_solver *solver, int32_t i, int64_t *info);
void within_solver_subdomain_indices(const within_solver *solver, int32_t i, uint32_t *gidx,
                                     double *pou);
/* Preconditioner persistence (FePreconditioner pickling and FePreconditioner(bytes),
 * within-py/src/lib.rs:890-913; Solver::with_preconditioner, within/src/solver.rs:433-446).
 * The bytes are this library's own format (magic "WB200PC", version, checksum); they
 * hold the configuration, every subdomain with its local factor and, for multiplicative
 * Schwarz, the explicit Gramian of its residual updates.  Reading rejects corrupted or
 * inconsistent bytes with WITHIN_ERR_INVALID_ARGUMENT before anything reaches the GPU.
 *
 * preconditioner_bytes: with buf NULL, *len receives the size; otherwise buf (of *len
 * bytes) receives the bytes.  WITHIN_ERR_INVALID_ARGUMENT when the solver has none.
 * new_with_preconditioner: a solver on a design that reuses the preconditioner instead of
 * building one (its dof count must equal the design's).
 * preconditioner_from_bytes: a handle holding only the preconditioner; it supports
 * apply_preconditioner, n_dofs, the subdomain queries and the diagnostics, and rejects
 * solves and the operator applies.  Free it with within_solver_free.
 * preconditioner_kind: 0 none, 1 additive, 2 multiplicative. */
int within_solver_preconditioner_bytes(within_solver *solver, uint8_t *buf, size_t *len);
int within_solver_new_with_preconditioner(const uint32_t *codes, size_t n_obs, size_t n_factors,
                                          int64_t row_stride, int64_t col_stride, const double *weights,
                                          const within_params *params, const uint8_t *data, size_t len,
                                          within_solver **out);
int within_preconditioner_from_bytes(const uint8_t *data, size_t len, within_solver **out);
int32_t within_solver_preconditioner_kind(const within_solver *solver);

/* FePreconditioner::subdomain_inner_parallel_work (within/src/operator/preconditioner.rs:64-79):
 * per subdomain, the work estimate of local_solver.rs:348-356 (2 nnz(C) + n_local when
 * the larger side has more than 10,000 rows, else 0).  work has n_subdomains entries. */
void within_solver_subdomain_inner_work(const within_solver *solver, int64_t *work);

/* AdditiveSchwarzDiagnostics (schwarz-precond/src/schwarz/additive/planning.rs:141-210;
 * within-py/src/lib.rs:200-260).  Strategies: 0 Auto, 1 AtomicScatter, 2
 * ParallelReduction.  `resolved_reduction_strategy` is the reference CPU scheduler's
 * choice for `threads` worker threads (planning.rs:71-135; <= 0: one per host core); the
 * device executor always adds subdomain results with atomics. */
typedef struct {
    int32_t reduction_strategy;
    int32_t resolved_reduction_strategy;
    int64_t n_subdomains;
    int64_t n_dofs;
    int64_t total_inner_parallel_work;
    int64_t max_inner_parallel_work;
    int64_t total_scatter_dofs;
    double outer_parallel_capacity;
    double scatter_overlap;
} within_additive_diagnostics;
/* WITHIN_ERR_INVALID_ARGUMENT unless the solver was built with additive Schwarz
 * (the reference returns None then: preconditioner.rs:98-106). */
int within_solver_additive_diagnostics(const within_solver *solver, int32_t threads,
                                       within_additive_diagnostics *out);
/* AC factor of subdomain i: sizes[5] = n, n_levels, nnz, n_columns, n_core (zeros for
 * dense subdomains).  Arrays: level_ptr (n_levels+1), col_vertex/col_diag (n_columns),
 * col_ptr (n_columns+1), col_idx/col_coef (nnz), core_vertex (n_core),
 * core_z (n_core*n_core row-major anchored inverse of the dense core). */
void within_solver_ac_sizes(const within_solver *solver, int32_t i, int64_t *sizes);
void within_solver_ac_arrays(const within_solver *solver, int32_t i, int32_t *level_ptr,
                             int32_t *col_vertex, double *col_diag, int32_t *col_ptr,
                             int32_t *col_idx, double *col_coef, int32_t *core_vertex,
                             double *core_z);

/* Test hook for the failure path of a local solve (no counterpart in the reference, whose
 * tests use a failing LocalSolver stub: schwarz-precond/tests/schwarz.rs:947-1001).  With
 * `on`, the approximate-Cholesky sweeps' grid barriers wait for one block more than the
 * grid has, with a short limit (about a millisecond per wait): the waits run out, the
 * device error flag is set and the launches end; no GPU fault is involved.  Such a local
 * solve did not complete, and, as in the reference, within_solver_apply_preconditioner
 * returns z filled with NaN (Preconditioner::apply, additive/preconditioner.rs:197-201)
 * while a solve returns WITHIN_ERR_ITERATIVE_SOLVE (CG's try_apply, cg.rs:69, 104).
 * WITHIN_ERR_INVALID_ARGUMENT when the preconditioner has no such sweeps. */
int within_solver_inject_sweep_timeout(within_solver *solver, int32_t on);

/* Tuning knob (no counterpart in the reference, whose approximate-Cholesky solve,
 * approx_chol::Factor::solve_in_place, is sequential).  The longest run of consecutive
 * levels of an approximate-Cholesky sweep direction with at most `max_chunks` row pieces
 * each (default 512; at least two levels) runs in one thread-block cluster, separated by
 * the cluster's hardware barrier; the other levels run in cooperative grid launches with
 * grid barriers.  0 puts every level on the grid.  Same arithmetic in the same order
 * either way.  WITHIN_ERR_INVALID_ARGUMENT for a negative value. */
int within_solver_set_sweep_cluster(within_solver *solver, int64_t max_chunks);

/* Coarse space for CG (no counterpart in the reference; it augments the additive Schwarz
 * apply, schwarz-precond/src/schwarz/additive/executor.rs:59-147, inside CG,
 * schwarz-precond/src/solve/cg.rs:45-133).  With a coarse basis Z (n_dofs x 32), CG's
 * preconditioner becomes M^-1 r + Z E^+ Z' r with E = Z' G Z (FP64; E^+ drops the
 * null-space directions of G), which is symmetric positive semi-definite, so CG stays
 * valid and every solve still runs to the same tolerance.  GMRES, LSMR and
 * apply_preconditioner do not use it.
 *
 * The learned basis comes from a message-passing network over the level graph (one node
 * per level; edges weighted by the off-diagonal of G = D'WD): 16 input features per level
 * (factor, log weighted count, log count, 10 hashed probe signs from `seed`), three
 * layers H' = tanh([Ahat H, H] W + b) of 64 units with Ahat = D^-1/2 (G - diag G) D^-1/2,
 * and Z = D^-1/2 H W_o.  Weights are used in BF16 (tensor cores, FP32 accumulation); the
 * parameter vector is FP32 (W_0 32x64, b_0, W_1 128x64, b_1, W_2 128x64, b_2, W_o 64x32,
 * row-major): within_coarse_net_params() values.
 *
 * set_coarse_net: evaluate the network on the solver's design and install its basis.
 * set_coarse_basis: install a given basis (Z: n_dofs x k, RHS-major, k <= 32).
 * clear_coarse: back to plain Schwarz.  coarse_basis: the installed basis (n_dofs x 32).
 * set_coarse_targets / coarse_net_grad: training on this design: targets V (n_dofs x t,
 * t <= 32, orthonormal columns in the D^1/2-scaled space), loss
 * L = 1 - tr(B' A^-1 B)/t with A = Zt'Zt, B = Zt'V (Zt = D^1/2 Z: the fraction of the
 * targets outside span(Z)), its gradient for every parameter (FP32, same layout), and
 * optionally Zt (n_dofs x 32 RHS-major).  release_coarse_training frees the buffers. */
int32_t within_coarse_net_params(void);
int within_solver_set_coarse_net(within_solver *solver, const float *params, size_t n_params, uint64_t seed);
int within_solver_set_coarse_basis(within_solver *solver, const double *z, size_t k);
int within_solver_clear_coarse(within_solver *solver);
int within_solver_coarse_basis(within_solver *solver, double *z);
int within_solver_set_coarse_targets(within_solver *solver, const double *v, size_t t);
int within_coarse_net_grad(within_solver *solver, const float *params, uint64_t seed, float *grad, double *loss,
                           float *zt);
int within_solver_release_coarse_training(within_solver *solver);

/* Block shape of the observation pass for k RHS in elem_bytes (4 FP32, 8 FP64)
 * precision: observations per work chunk (16, 32 or 64) and resident blocks per SM (1
 * or 2).  The solver's autotuner picks them the first time it needs the pass (each
 * candidate timed on the solver's own design; cached per shape class for the process).
 * Returns 0 when tuned, 1 when not tuned yet (the defaults, 32 and 2, are reported).
 * A measurement hook with no counterpart in the reference. */
int within_solver_obs_config(const within_solver *solver, int32_t k, int32_t elem_bytes, int32_t *obs_per_chunk,
                             int32_t *blocks_per_sm);

/* Where the observation pass for k RHS in elem_bytes precision adds the run sums of a
 * factor's most frequent levels: 0 in a table in each block's shared memory, 1 in a
 * per-block copy in global memory (16-byte vector reductions in L2), -1 not tuned yet.
 * The autotuner tries both for designs that have such levels.  No counterpart in the
 * reference. */
int32_t within_solver_obs_hot_global(const within_solver *solver, int32_t k, int32_t elem_bytes);

/* Right-hand sides per lane of the observation pass for k RHS in elem_bytes precision:
 * 4, or 8 for wide lanes (FP32 operator apply with k > 4: the per-observation control is
 * shared by 8 RHS, with half the threads per block); -1 not tuned yet.  The autotuner
 * tries both where wide lanes apply.  No counterpart in the reference. */
int32_t within_solver_obs_rhs_per_lane(const within_solver *solver, int32_t k, int32_t elem_bytes);

/* Hybrid operator apply (no counterpart in the reference; it computes the same
 * GramianOperator::apply, operator/gramian.rs:84-89).  The blocks of G = D'WD between the
 * factor with the most levels (primary) and the small factors held in the observation
 * pass's lane-group tables stay implicit: one pass over the observations, with no code of
 * any other factor read.  Every other block is a factor-pair cross-tabulation of the
 * additive Schwarz setup, applied as CSR rows.  The autotuner times it against the
 * observation pass once per shape class and keeps the faster.  Its primary-major part
 * has two forms: lane-group tables of the small factors (prim_rows_kernel), and, for 16
 * RHS and at most 48 small-factor levels (each factor padded to 8), products of per-warp
 * weight tiles on the FP64 tensor cores (prim_mma_kernel).  within_solver_set_hybrid
 * fixes the choice for k RHS in elem_bytes precision: 0 off, 1 tables, 2 tensor cores (1
 * and 2 build the arrays here; outside any stream capture); WITHIN_ERR_INVALID_ARGUMENT
 * when the solver has no additive Schwarz preconditioner, uses the assembled Gramian, or
 * has no (or more than two) small factors, or for 2 where the tile does not apply.
 * within_solver_hybrid returns the form in use (0, 1 or 2) or -1 (not decided yet), with
 * the autotuner's time per apply of the faster form in *ms (0 when not timed; ms may be
 * null). */
int within_solver_set_hybrid(within_solver *solver, int32_t k, int32_t elem_bytes, int32_t on);
int32_t within_solver_hybrid(const within_solver *solver, int32_t k, int32_t elem_bytes, float *ms);
/* Algorithmic bytes of one hybrid apply for k RHS of elem_bytes per element (0 when the
 * solver holds no hybrid arrays): the small factors' codes and the weights once per
 * observation, the CSR entries (column 4 bytes, value elem_bytes) of the primary levels'
 * C_PO rows and of the other rows, their row pointers, and x read and y written once
 * (2 elem_bytes n_dofs kp). */
int64_t within_solver_hybrid_bytes(const within_solver *solver, int32_t k, int32_t elem_bytes);

/* The autotuner's measured time (milliseconds per operator apply, the best of two
 * sweeps over the candidates) of each candidate shape for k RHS in elem_bytes precision:
 * ms[c] for c < n and c < 24, where c = wide * 12 + hot_global * 6 +
 * 2 * log2(obs_per_chunk / 16) + blocks_per_sm - 1 (wide: 8 RHS per lane); 0 for
 * candidates not timed (a shape class tuned earlier in the process, no hot levels, or
 * no wide lanes for this precision and k).  A measurement hook with no counterpart in the reference. */
int within_solver_obs_tune_times(const within_solver *solver, int32_t k, int32_t elem_bytes, float *ms, int32_t n);

/* Fixes the observation pass's shape for k RHS in elem_bytes precision instead of
 * autotuning it: obs_per_chunk 16, 32 or 64, blocks_per_sm 1 or 2, and `variant` the sum
 * of 1 for the hot tables in per-block global copies (see within_solver_obs_hot_global;
 * the copies are allocated here) and 2 for wide lanes (see
 * within_solver_obs_rhs_per_lane; FP32, k > 4 and the exact kernels only: at most 3
 * factors, or 4 with at most one small factor in lane-group tables; otherwise
 * WITHIN_ERR_INVALID_ARGUMENT).  For reproducible timing and for testing each variant.
 * No counterpart in the reference. */
int within_solver_set_obs_config(within_solver *solver, int32_t k, int32_t elem_bytes, int32_t obs_per_chunk,
                                 int32_t blocks_per_sm, int32_t variant);

/* Algorithmic bytes of one Schwarz apply over k RHS with elem_bytes (4 or 8) per vector
 * element, counted from the built subdomains: per subdomain 2 (4+s) nnz(C_i) for the
 * cross block read twice (reduced right-hand side and back substitution), 12 n_i for the
 * slots' indices and weights, 2 s n_i k for the local vector, plus s (n_keep-1)^2 for a
 * dense anchored factor or 2 (4+s) nnz(L_AC) + s n_core^2 for an approximate-Cholesky
 * factor.  0 for a solver without subdomains.  A measurement hook with no counterpart in
 * the reference (the per-subdomain sizes follow local_solver.rs:360-449). */
int64_t within_solver_schwarz_bytes(const within_solver *solver, int32_t k, int32_t elem_bytes);

/* Number of kernels this solver has launched so far, and its setup wall time (s).
 * Measurement hooks with no counterpart in the reference. */
int64_t within_solver_gpu_launches(const within_solver *solver);
double within_solver_setup_time(const within_solver *solver);
/* Event timing of selected launches on the solver's stream (off by default; turning it
 * on resets the totals).  which: 0 operator apply D'WD in FP64, 1 the same in FP32,
 * 2 Schwarz apply in FP64, 3 the same in FP32. */
void within_solver_set_profiling(within_solver *solver, int32_t on);
void within_solver_kernel_time(const within_solver *solver, int32_t which, int64_t *launches,
                               double *total_ms);

/* G x = D'W(D x) like within_solver_apply_gramian, but on device buffers and without
 * allocating: d_x and d_y are n_dofs*k RHS-major device arrays, k <= 32, and the work
 * is queued on `cuda_stream` (NULL = the solver's stream) without waiting for it.
 * This entry point has no counterpart in the reference.  It exists for callers that
 * cannot allocate device memory while they run -- code under a fixed memory budget or
 * a custom allocator, or loops that cannot take an allocation's synchronisation.  Its
 * working space is a static 16 MiB device array (resident on every GPU that loads the
 * library until exit), so 2 x n_dofs x k (k rounded up to 4, 8, 16 or 32) must not
 * exceed 2^21 doubles; larger sizes are rejected with WITHIN_ERR_INVALID_ARGUMENT.
 * The first call on a device looks the array's address up (cudaGetSymbolAddress);
 * make that first call before any stream capture.  Every call shares the one array:
 * calls whose work overlaps on the GPU (different streams, or several solvers) race.
 * Arithmetic is FP64 whatever the solver's precision. */
int within_solver_apply_gramian_noalloc(within_solver *solver, const double *d_x, size_t k,
                                        double *d_y, void *cuda_stream);

/* Message of the last failed call on this host thread ("" when none). */
const char *within_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* WITHIN_B200_H */
