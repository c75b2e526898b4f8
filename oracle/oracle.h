/*
 * oracle.h -- CPU FP64 restatement of the `within` solve phase.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path in
 * `within_b200`: only the tests, `__graft_entry__.smoke()` and the CPU-baseline
 * leg of `bench.py` load it.  The product library never links or calls it.
 *
 * Parity status
 *   - Design ops (D x, D'r, D'W r, diag), CSR transpose, bipartite components,
 *     exact and anchored-dense Schur complements and CG are pinned against the
 *     literal vectors of the reference's own unit tests (tests/golden/).
 *   - The approximate-Cholesky factor and the clique-tree sampler belong to the
 *     external crate approx-chol 0.1.0, which is not vendored.  They are
 *     restated here from Gao, Kyng & Spielman (arXiv:2303.00709); their values
 *     are "parity unpinned" and are checked only at the solution level
 *     (demeaned residuals and x modulo the null space).
 */
#ifndef WITHIN_ORACLE_H
#define WITHIN_ORACLE_H

#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct oracle_solver oracle_solver;

/* krylov: 0 = CG, 1 = GMRES, 2 = LSMR.  precond_kind: 0 = off, 1 = additive, 2 = multiplicative.
 * approx_schur_enabled: 0 = exact Schur complement, 1 = sampled (clique tree). */
typedef struct {
    int32_t krylov;
    int32_t gmres_restart;
    double tol;
    int32_t maxiter;
    int32_t max_refinements;
    int32_t precond_kind;
    uint64_t approx_chol_seed;
    uint32_t approx_chol_split;   /* 1 = no split (reference split_merge None) */
    int32_t approx_schur_enabled;
    uint64_t approx_schur_seed;
    uint32_t approx_schur_split;
    int32_t dense_threshold;
    int32_t lsmr_local_size;      /* krylov 2 (LSMR): windowed reorthogonalization, 0 = off */
} oracle_params;

/* codes: element (i, q) at codes[i*row_stride + q*col_stride].  weights may be NULL. */
int oracle_solver_new(const uint32_t *codes, int64_t n_obs, int32_t n_factors,
                      int64_t row_stride, int64_t col_stride, const double *weights,
                      const oracle_params *params, oracle_solver **out,
                      char *err, int errlen);
void oracle_solver_free(oracle_solver *s);

int64_t oracle_n_dofs(const oracle_solver *s);
int64_t oracle_n_obs(const oracle_solver *s);
void oracle_factor_meta(const oracle_solver *s, int64_t *n_levels, int64_t *offsets);

/* y: n_obs.  x: n_dofs.  demeaned: n_obs. */
int oracle_solve(oracle_solver *s, const double *y, double *x, double *demeaned,
                 int32_t *converged, int32_t *iterations, double *final_residual,
                 char *err, int errlen);
/* ys, demeaned: RHS-major (k blocks of n_obs); x: k blocks of n_dofs.  Threads over RHS. */
int oracle_solve_batch(oracle_solver *s, const double *ys, int32_t k, double *x,
                       double *demeaned, int32_t *converged, int32_t *iterations,
                       double *final_residual, int32_t n_threads, char *err, int errlen);

/* Operator pieces, for kernel-level parity tests. */
void oracle_matvec_d(const oracle_solver *s, const double *x, double *y);
void oracle_rmatvec_wdt(const oracle_solver *s, const double *r, double *x);
void oracle_rmatvec_dt(const oracle_solver *s, const double *r, double *x);
void oracle_gramian_diagonal(const oracle_solver *s, double *diag);
void oracle_apply_gramian(const oracle_solver *s, const double *x, double *y);
int oracle_apply_precond(oracle_solver *s, const double *r, double *z);

/* LSMR on a dense row-major operator a (rows x cols) with an optional dense M^-1
 * (cols x cols), for known-answer tests of the recurrences (lsmr/tests.rs).
 * stop_reason: 0 zero rhs, 1 A'b = 0, 2 residual tolerance, 3 normal-equation
 * tolerance, 4 breakdown, 5 max iterations. */
int oracle_lsmr_dense(const double *a, int64_t rows, int64_t cols, const double *minv, const double *b, double tol,
                      int32_t maxiter, int32_t local_size, double *x, int32_t *converged, int32_t *iterations,
                      int32_t *stop_reason);

/* Setup structure, for bit-exact checks of the integer setup. */
int32_t oracle_n_subdomains(const oracle_solver *s);
/* info[0..7] = q, r, n_local, n_q, n_r, eliminate_q, reduced_kind (0 dense, 1 ac), n_reduced */
void oracle_subdomain_info(const oracle_solver *s, int32_t i, int64_t *info);
void oracle_subdomain_indices(const oracle_solver *s, int32_t i, uint32_t *gidx, double *pou);
/* Sizes of the AC factor of subdomain i: [n, n_levels, nnz, n_columns, n_core]; zeros when dense. */
void oracle_ac_sizes(const oracle_solver *s, int32_t i, int64_t *sizes);
void oracle_ac_arrays(const oracle_solver *s, int32_t i, int32_t *level_ptr, int32_t *col_vertex,
                      double *col_diag, int32_t *col_ptr, int32_t *col_idx, double *col_coef,
                      int32_t *core_vertex, double *core_z);
/* CSR of the subdomain's C block (n_q x n_r): sizes [nnz] then arrays. */
int64_t oracle_crosstab_nnz(const oracle_solver *s, int32_t i);
void oracle_crosstab(const oracle_solver *s, int32_t i, uint32_t *indptr, uint32_t *indices,
                     double *data, double *diag_q, double *diag_r);

/* Standalone pieces pinned by the reference's unit tests. */
void oracle_csr_transpose(int32_t nrows, int32_t ncols, const uint32_t *indptr,
                          const uint32_t *indices, const double *data, uint32_t *t_indptr,
                          uint32_t *t_indices, double *t_data);
/* Dense SPD / general operator CG, reference semantics; a may be NULL for identity. */
int oracle_dense_cg(int32_t n, const double *a, const double *m_inv_diag, const double *b,
                    double tol, int32_t maxiter, double *x, int32_t *converged,
                    int32_t *iterations, double *residual_norm);
int oracle_dense_gmres(int32_t n, const double *a, const double *m_inv_diag, const double *b,
                       double tol, int32_t maxiter, int32_t restart, double *x,
                       int32_t *converged, int32_t *iterations, double *residual_norm);

#ifdef __cplusplus
}
#endif
#endif
