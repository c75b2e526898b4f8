/*
 * oracle.c -- CPU FP64 restatement of the `within` solve phase.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path (see oracle.h).
 * Every function cites the reference file:line it restates; paths are relative
 * to the reference's `crates/` directory.  Plain sequential C (the batch entry
 * point runs right-hand sides on OpenMP threads, as the reference runs them on
 * Rayon tasks, within/src/solver.rs:242-277).
 */
#include "oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------- */
/* utilities                                                                 */
/* ------------------------------------------------------------------------- */

static void *xcalloc(size_t n, size_t sz) {
    void *p = calloc(n ? n : 1, sz ? sz : 1);
    if (!p) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return p;
}
static void *xrealloc(void *p, size_t sz) {
    void *q = realloc(p, sz ? sz : 1);
    if (!q) { fprintf(stderr, "oracle: out of memory\n"); abort(); }
    return q;
}
static void set_err(char *err, int errlen, const char *fmt, ...) {
    if (!err || errlen <= 0) return;
    va_list ap; va_start(ap, fmt); vsnprintf(err, (size_t)errlen, fmt, ap); va_end(ap);
}

/* splitmix64 (Steele, Lea & Flood 2014): the sampler's random stream. */
static uint64_t sm64_next(uint64_t *s) {
    uint64_t z = (*s += 0x9E3779B97F4A7C15ULL);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
static double sm64_u01(uint64_t *s) { return (double)(sm64_next(s) >> 11) * 0x1.0p-53; }
static uint64_t mix64(uint64_t x) { uint64_t s = x; return sm64_next(&s); }

static double vnorm(const double *v, int64_t n) {
    double s = 0.0;                       /* schwarz-precond/src/solve.rs:32-38 */
    for (int64_t i = 0; i < n; i++) s += v[i] * v[i];
    return sqrt(s);
}
static double vdot(const double *a, const double *b, int64_t n) {
    double s = 0.0;                       /* schwarz-precond/src/solve.rs:26-29 */
    for (int64_t i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

/* ------------------------------------------------------------------------- */
/* design: within/src/domain.rs:133-431                                      */
/* ------------------------------------------------------------------------- */

typedef struct {
    int64_t n;
    int32_t Q;
    uint32_t *codes;   /* owned, factor-major: codes[q*n + i] */
    double *w;         /* NULL = unit weights */
    int64_t *nlev, *off;
    int64_t ndofs;
} design_t;

/* WeightedDesign::from_store, domain.rs:133-155: n_levels = max+1, offsets = prefix sum. */
static void design_init(design_t *d) {
    d->nlev = xcalloc((size_t)d->Q, sizeof(int64_t));
    d->off = xcalloc((size_t)d->Q, sizeof(int64_t));
    int64_t off = 0;
    for (int q = 0; q < d->Q; q++) {
        uint32_t mx = 0;
        const uint32_t *c = d->codes + (size_t)q * d->n;
        for (int64_t i = 0; i < d->n; i++) if (c[i] > mx) mx = c[i];
        d->nlev[q] = (int64_t)mx + 1;
        d->off[q] = off;
        off += d->nlev[q];
    }
    d->ndofs = off;
}
static inline uint32_t lev(const design_t *d, int64_t i, int q) { return d->codes[(size_t)q * d->n + i]; }
static inline double wt(const design_t *d, int64_t i) { return d->w ? d->w[i] : 1.0; }

/* matvec_d, domain.rs:390-395 (gather_add :312-345, factor-major order). */
static void design_matvec_d(const design_t *d, const double *x, double *y) {
    for (int64_t i = 0; i < d->n; i++) y[i] = 0.0;
    for (int q = 0; q < d->Q; q++) {
        const uint32_t *c = d->codes + (size_t)q * d->n;
        const double *xq = x + d->off[q];
        for (int64_t i = 0; i < d->n; i++) y[i] += xq[c[i]];
    }
}
/* rmatvec_dt / rmatvec_wdt, domain.rs:398-417 (scatter_add :359-387). */
static void design_rmatvec(const design_t *d, const double *r, double *x, int weighted) {
    for (int64_t j = 0; j < d->ndofs; j++) x[j] = 0.0;
    for (int q = 0; q < d->Q; q++) {
        const uint32_t *c = d->codes + (size_t)q * d->n;
        double *xq = x + d->off[q];
        if (weighted && d->w) {
            for (int64_t i = 0; i < d->n; i++) xq[c[i]] += d->w[i] * r[i];
        } else {
            for (int64_t i = 0; i < d->n; i++) xq[c[i]] += r[i];
        }
    }
}
/* gramian_diagonal, domain.rs:422-431. */
static void design_diag(const design_t *d, double *diag) {
    for (int64_t j = 0; j < d->ndofs; j++) diag[j] = 0.0;
    for (int q = 0; q < d->Q; q++)
        for (int64_t i = 0; i < d->n; i++) diag[d->off[q] + lev(d, i, q)] += wt(d, i);
}

/* ------------------------------------------------------------------------- */
/* CSR block: within/src/operator/csr_block.rs                               */
/* ------------------------------------------------------------------------- */

typedef struct {
    int32_t nrows, ncols;
    uint32_t *indptr, *indices;
    double *data;
} csr_t;

static void csr_free(csr_t *a) { free(a->indptr); free(a->indices); free(a->data); memset(a, 0, sizeof *a); }
static int64_t csr_nnz(const csr_t *a) { return a->indptr ? (int64_t)a->indptr[a->nrows] : 0; }

/* CsrBlock::transpose, csr_block.rs:31-62 (stable counting scatter). */
static csr_t csr_transpose(const csr_t *a) {
    csr_t t; t.nrows = a->ncols; t.ncols = a->nrows;
    int64_t nnz = csr_nnz(a);
    t.indptr = xcalloc((size_t)t.nrows + 1, sizeof(uint32_t));
    t.indices = xcalloc((size_t)nnz, sizeof(uint32_t));
    t.data = xcalloc((size_t)nnz, sizeof(double));
    for (int64_t e = 0; e < nnz; e++) t.indptr[a->indices[e] + 1]++;
    for (int32_t i = 0; i < t.nrows; i++) t.indptr[i + 1] += t.indptr[i];
    uint32_t *cur = xcalloc((size_t)t.nrows + 1, sizeof(uint32_t));
    memcpy(cur, t.indptr, sizeof(uint32_t) * (size_t)t.nrows);
    for (int32_t r = 0; r < a->nrows; r++)
        for (uint32_t e = a->indptr[r]; e < a->indptr[r + 1]; e++) {
            uint32_t dst = a->indices[e], pos = cur[dst]++;
            t.indices[pos] = (uint32_t)r;
            t.data[pos] = a->data[e];
        }
    free(cur);
    return t;
}

void oracle_csr_transpose(int32_t nrows, int32_t ncols, const uint32_t *indptr,
                          const uint32_t *indices, const double *data, uint32_t *t_indptr,
                          uint32_t *t_indices, double *t_data) {
    csr_t a = { nrows, ncols, (uint32_t *)indptr, (uint32_t *)indices, (double *)data };
    csr_t t = csr_transpose(&a);
    int64_t nnz = csr_nnz(&t);
    memcpy(t_indptr, t.indptr, sizeof(uint32_t) * ((size_t)ncols + 1));
    memcpy(t_indices, t.indices, sizeof(uint32_t) * (size_t)nnz);
    memcpy(t_data, t.data, sizeof(double) * (size_t)nnz);
    csr_free(&t);
}

/* ------------------------------------------------------------------------- */
/* Cross-tab: within/src/operator/gramian/cross_tab.rs                       */
/* ------------------------------------------------------------------------- */

typedef struct {
    csr_t c, ct;        /* C: n_q x n_r, CT: n_r x n_q */
    double *dq, *dr;
} crosstab_t;

static void crosstab_free(crosstab_t *x) { csr_free(&x->c); csr_free(&x->ct); free(x->dq); free(x->dr); }

/* build_for_pair_with_active, cross_tab.rs:246-265 with build_compact_mapping :95-145 and the
 * bucket accumulation :568-664 (the dense-table path :532-562 sums in the same observation
 * order, so both give identical values; one routine serves both). Returns 0 for an empty pair. */
static int crosstab_build(const design_t *d, int q, int r, uint8_t **active, crosstab_t *out,
                          uint32_t **l2g_out, int32_t *nq_out) {
    int64_t Lq = d->nlev[q], Lr = d->nlev[r];
    uint32_t *qmap = xcalloc((size_t)Lq, sizeof(uint32_t));
    uint32_t *rmap = xcalloc((size_t)Lr, sizeof(uint32_t));
    int32_t nq = 0, nr = 0;
    for (int64_t j = 0; j < Lq; j++) qmap[j] = active[q][j] ? (uint32_t)nq++ : UINT32_MAX;
    for (int64_t k = 0; k < Lr; k++) rmap[k] = active[r][k] ? (uint32_t)nr++ : UINT32_MAX;
    if (nq == 0 || nr == 0) { free(qmap); free(rmap); return 0; }
    uint32_t *l2g = xcalloc((size_t)nq + (size_t)nr, sizeof(uint32_t));
    int32_t p = 0;
    for (int64_t j = 0; j < Lq; j++) if (active[q][j]) l2g[p++] = (uint32_t)(d->off[q] + j);
    for (int64_t k = 0; k < Lr; k++) if (active[r][k]) l2g[p++] = (uint32_t)(d->off[r] + k);

    double *dq = xcalloc((size_t)nq, sizeof(double)), *dr = xcalloc((size_t)nr, sizeof(double));
    uint32_t *bptr = xcalloc((size_t)nq + 1, sizeof(uint32_t));
    for (int64_t i = 0; i < d->n; i++) {
        uint32_t cj = qmap[lev(d, i, q)], ck = rmap[lev(d, i, r)];
        double w = wt(d, i);
        dq[cj] += w; dr[ck] += w; bptr[cj + 1]++;
    }
    for (int32_t j = 0; j < nq; j++) bptr[j + 1] += bptr[j];
    uint32_t total = bptr[nq];
    uint32_t *bcol = xcalloc(total, sizeof(uint32_t));
    double *bval = xcalloc(total, sizeof(double));
    uint32_t *cur = xcalloc((size_t)nq + 1, sizeof(uint32_t));
    memcpy(cur, bptr, sizeof(uint32_t) * (size_t)nq);
    for (int64_t i = 0; i < d->n; i++) {
        uint32_t cj = qmap[lev(d, i, q)], ck = rmap[lev(d, i, r)];
        uint32_t pos = cur[cj]++;
        bcol[pos] = ck; bval[pos] = wt(d, i);
    }
    /* per-row dedup with a dense workspace; columns emitted ascending, zeros dropped */
    double *work = xcalloc((size_t)nr, sizeof(double));
    uint8_t *seen = xcalloc((size_t)nr, 1);
    uint32_t *touched = xcalloc((size_t)nr + 1, sizeof(uint32_t));
    csr_t c; c.nrows = nq; c.ncols = nr;
    c.indptr = xcalloc((size_t)nq + 1, sizeof(uint32_t));
    size_t cap = total ? total : 1;
    c.indices = xcalloc(cap, sizeof(uint32_t)); c.data = xcalloc(cap, sizeof(double));
    uint32_t nnz = 0;
    for (int32_t row = 0; row < nq; row++) {
        int32_t nt = 0;
        for (uint32_t e = bptr[row]; e < bptr[row + 1]; e++) {
            uint32_t col = bcol[e];
            if (!seen[col]) { seen[col] = 1; touched[nt++] = col; }
            work[col] += bval[e];
        }
        /* insertion-free ascending order: counting via sort of touched */
        for (int32_t a = 1; a < nt; a++) {          /* small rows: insertion sort */
            uint32_t key = touched[a]; int32_t b = a - 1;
            while (b >= 0 && touched[b] > key) { touched[b + 1] = touched[b]; b--; }
            touched[b + 1] = key;
        }
        for (int32_t a = 0; a < nt; a++) {
            uint32_t col = touched[a];
            if (work[col] != 0.0) { c.indices[nnz] = col; c.data[nnz] = work[col]; nnz++; }
            work[col] = 0.0; seen[col] = 0;
        }
        c.indptr[row + 1] = nnz;
    }
    free(work); free(seen); free(touched); free(bcol); free(bval); free(bptr); free(cur);
    free(qmap); free(rmap);
    out->c = c; out->ct = csr_transpose(&c); out->dq = dq; out->dr = dr;
    *l2g_out = l2g; *nq_out = nq;
    return 1;
}

typedef struct { int32_t nq, nr; int32_t *qi, *ri; } comp_t;
static int cmp_i32(const void *a, const void *b) { int32_t x = *(const int32_t *)a, y = *(const int32_t *)b; return (x > y) - (x < y); }

/* bipartite_connected_components, cross_tab.rs:381-444: DFS from compact nodes 0..n_q+n_r
 * (q-nodes first), explicit stack, indices sorted per component. */
static int32_t crosstab_components(const crosstab_t *x, comp_t **out) {
    int32_t nq = x->c.nrows, nr = x->c.ncols, n = nq + nr;
    uint8_t *vis = xcalloc((size_t)n, 1);
    int32_t *stack = xcalloc((size_t)n + 1, sizeof(int32_t));
    int32_t *buf = xcalloc((size_t)n + 1, sizeof(int32_t));
    int32_t ncomp = 0, cap = 4;
    comp_t *comps = xcalloc((size_t)cap, sizeof(comp_t));
    for (int32_t s = 0; s < n; s++) {
        if (vis[s]) continue;
        vis[s] = 1;
        int32_t sp = 0, nb = 0;
        stack[sp++] = s;
        while (sp) {
            int32_t node = stack[--sp];
            buf[nb++] = node;
            if (node < nq) {
                for (uint32_t e = x->c.indptr[node]; e < x->c.indptr[node + 1]; e++) {
                    int32_t g = nq + (int32_t)x->c.indices[e];
                    if (!vis[g]) { vis[g] = 1; stack[sp++] = g; }
                }
            } else {
                int32_t ri = node - nq;
                for (uint32_t e = x->ct.indptr[ri]; e < x->ct.indptr[ri + 1]; e++) {
                    int32_t g = (int32_t)x->ct.indices[e];
                    if (!vis[g]) { vis[g] = 1; stack[sp++] = g; }
                }
            }
        }
        comp_t cp; cp.nq = 0; cp.nr = 0;
        for (int32_t a = 0; a < nb; a++) { if (buf[a] < nq) cp.nq++; else cp.nr++; }
        cp.qi = xcalloc((size_t)cp.nq + 1, sizeof(int32_t));
        cp.ri = xcalloc((size_t)cp.nr + 1, sizeof(int32_t));
        /* sorted member lists (sort_unstable in the reference) */
        int32_t a1 = 0, a2 = 0;
        for (int32_t a = 0; a < nb; a++) { if (buf[a] < nq) cp.qi[a1++] = buf[a]; else cp.ri[a2++] = buf[a] - nq; }
        qsort(cp.qi, (size_t)cp.nq, sizeof(int32_t), cmp_i32);
        qsort(cp.ri, (size_t)cp.nr, sizeof(int32_t), cmp_i32);
        if (ncomp == cap) { cap *= 2; comps = xrealloc(comps, sizeof(comp_t) * (size_t)cap); }
        comps[ncomp++] = cp;
    }
    free(vis); free(stack); free(buf);
    *out = comps;
    return ncomp;
}

/* extract_component, cross_tab.rs:450-501. */
static crosstab_t crosstab_extract(const crosstab_t *x, const comp_t *cp) {
    int32_t nq = cp->nq, nr = cp->nr;
    uint32_t *qre = xcalloc((size_t)x->c.nrows, sizeof(uint32_t));
    uint32_t *rre = xcalloc((size_t)x->c.ncols, sizeof(uint32_t));
    for (int32_t i = 0; i < x->c.nrows; i++) qre[i] = UINT32_MAX;
    for (int32_t i = 0; i < x->c.ncols; i++) rre[i] = UINT32_MAX;
    for (int32_t a = 0; a < nq; a++) qre[cp->qi[a]] = (uint32_t)a;
    for (int32_t a = 0; a < nr; a++) rre[cp->ri[a]] = (uint32_t)a;
    crosstab_t o;
    o.dq = xcalloc((size_t)nq, sizeof(double)); o.dr = xcalloc((size_t)nr, sizeof(double));
    for (int32_t a = 0; a < nq; a++) o.dq[a] = x->dq[cp->qi[a]];
    for (int32_t a = 0; a < nr; a++) o.dr[a] = x->dr[cp->ri[a]];
    int64_t cap = 0;
    for (int32_t a = 0; a < nq; a++) cap += x->c.indptr[cp->qi[a] + 1] - x->c.indptr[cp->qi[a]];
    csr_t c; c.nrows = nq; c.ncols = nr;
    c.indptr = xcalloc((size_t)nq + 1, sizeof(uint32_t));
    c.indices = xcalloc((size_t)cap + 1, sizeof(uint32_t)); c.data = xcalloc((size_t)cap + 1, sizeof(double));
    uint32_t nnz = 0;
    for (int32_t a = 0; a < nq; a++) {
        int32_t old = cp->qi[a];
        for (uint32_t e = x->c.indptr[old]; e < x->c.indptr[old + 1]; e++) {
            uint32_t nc = rre[x->c.indices[e]];
            if (nc != UINT32_MAX) { c.indices[nnz] = nc; c.data[nnz] = x->c.data[e]; nnz++; }
        }
        c.indptr[a + 1] = nnz;
    }
    free(qre); free(rre);
    o.c = c; o.ct = csr_transpose(&c);
    return o;
}

/* ------------------------------------------------------------------------- */
/* Square CSR (Schur complement): schwarz-precond/src/sparse_matrix.rs       */
/* ------------------------------------------------------------------------- */

typedef struct { int32_t n; uint32_t *indptr, *indices; double *data; } smat_t;
static void smat_free(smat_t *m) { free(m->indptr); free(m->indices); free(m->data); memset(m, 0, sizeof *m); }

/* ------------------------------------------------------------------------- */
/* Elimination + Schur: within/src/operator/schur_complement.rs              */
/* ------------------------------------------------------------------------- */

typedef struct {
    int elim_q;               /* eliminate_q = n_q >= n_r, schur_complement.rs:174 */
    int32_t n_keep, n_elim;
    double *inv_diag;         /* 1/D_elim, :178-191 (zero diagonal -> SingularDiagonal) */
    const double *diag_elim, *diag_keep;
    const csr_t *k2e, *e2k;   /* keep->elim and elim->keep blocks, :199-203 */
} elim_t;

static int elim_init(const crosstab_t *x, elim_t *e, char *err, int errlen) {
    int32_t nq = x->c.nrows, nr = x->c.ncols;
    e->elim_q = nq >= nr;
    e->n_keep = e->elim_q ? nr : nq;
    e->n_elim = e->elim_q ? nq : nr;
    e->diag_elim = e->elim_q ? x->dq : x->dr;
    e->diag_keep = e->elim_q ? x->dr : x->dq;
    e->k2e = e->elim_q ? &x->ct : &x->c;
    e->e2k = e->elim_q ? &x->c : &x->ct;
    e->inv_diag = xcalloc((size_t)e->n_elim, sizeof(double));
    for (int32_t i = 0; i < e->n_elim; i++) {
        double dd = e->diag_elim[i];
        if (dd > 0.0) e->inv_diag[i] = 1.0 / dd;
        else {
            set_err(err, errlen, "zero diagonal in %s block at index %d",
                    e->elim_q ? "q (elim)" : "r (elim)", (int)i);
            free(e->inv_diag); e->inv_diag = NULL;
            return -1;
        }
    }
    return 0;
}

/* SchurLaplacian::from_elimination, schur_complement.rs:331-378, 394-412 (exact, row workspace). */
static smat_t schur_exact(const elim_t *e) {
    int32_t n = e->n_keep;
    double *work = xcalloc((size_t)n, sizeof(double));
    int32_t *touched = xcalloc((size_t)n + 1, sizeof(int32_t));
    uint8_t *in = xcalloc((size_t)n, 1);
    smat_t s; s.n = n; s.indptr = xcalloc((size_t)n + 1, sizeof(uint32_t));
    size_t cap = (size_t)n * 4 + 16, nnz = 0;
    s.indices = xcalloc(cap, sizeof(uint32_t)); s.data = xcalloc(cap, sizeof(double));
    for (int32_t i = 0; i < n; i++) {
        int32_t nt = 0;
        work[i] = e->diag_keep[i]; touched[nt++] = i; in[i] = 1;
        for (uint32_t f = e->k2e->indptr[i]; f < e->k2e->indptr[i + 1]; f++) {
            uint32_t k = e->k2e->indices[f];
            double scale = e->k2e->data[f] * e->inv_diag[k];
            for (uint32_t b = e->e2k->indptr[k]; b < e->e2k->indptr[k + 1]; b++) {
                uint32_t j = e->e2k->indices[b];
                if (!in[j]) { in[j] = 1; touched[nt++] = (int32_t)j; }
                work[j] -= scale * e->e2k->data[b];
            }
        }
        for (int32_t a = 1; a < nt; a++) {
            int32_t key = touched[a], b = a - 1;
            while (b >= 0 && touched[b] > key) { touched[b + 1] = touched[b]; b--; }
            touched[b + 1] = key;
        }
        if (nnz + (size_t)nt > cap) {
            while (nnz + (size_t)nt > cap) cap *= 2;
            s.indices = xrealloc(s.indices, cap * sizeof(uint32_t));
            s.data = xrealloc(s.data, cap * sizeof(double));
        }
        for (int32_t a = 0; a < nt; a++) {
            int32_t j = touched[a];
            double v = work[j];
            if (v != 0.0 || j == i) { s.indices[nnz] = (uint32_t)j; s.data[nnz] = v; nnz++; }
            work[j] = 0.0; in[j] = 0;
        }
        s.indptr[i + 1] = (uint32_t)nnz;
    }
    free(work); free(touched); free(in);
    return s;
}

/* anchored_minor_from_elimination, schur_complement.rs:490-527: the top-left (n-1)^2 minor. */
static double *schur_anchored_minor(const elim_t *e) {
    int32_t n = e->n_keep;
    if (n <= 1) return NULL;
    int32_t m = n - 1;
    double *a = xcalloc((size_t)m * (size_t)m, sizeof(double));
    for (int32_t i = 0; i < m; i++) a[(size_t)i * m + i] = e->diag_keep[i];
    for (int32_t i = 0; i < m; i++)
        for (uint32_t f = e->k2e->indptr[i]; f < e->k2e->indptr[i + 1]; f++) {
            uint32_t k = e->k2e->indices[f];
            double scale = e->k2e->data[f] * e->inv_diag[k];
            for (uint32_t b = e->e2k->indptr[k]; b < e->e2k->indptr[k + 1]; b++) {
                uint32_t j = e->e2k->indices[b];
                if ((int32_t)j < m) a[(size_t)i * m + j] -= scale * e->e2k->data[b];
            }
        }
    return a;
}

typedef struct { uint32_t lo, hi; double w; } edge_t;
typedef struct { edge_t *e; size_t n, cap; } edges_t;
static void edges_push(edges_t *v, uint32_t a, uint32_t b, double w) {
    if (v->n == v->cap) { v->cap = v->cap ? v->cap * 2 : 64; v->e = xrealloc(v->e, v->cap * sizeof(edge_t)); }
    edge_t x; x.lo = a < b ? a : b; x.hi = a < b ? b : a; x.w = w;
    v->e[v->n++] = x;
}

typedef struct { uint32_t col; double w; } nbr_t;

/* Order neighbours by (weight, column) ascending: the clique-tree order. */
static int cmp_nbr_w(const void *pa, const void *pb) {
    const nbr_t *a = pa, *b = pb;
    if (a->w < b->w) return -1;
    if (a->w > b->w) return 1;
    return (a->col > b->col) - (a->col < b->col);
}

/*
 * Clique-tree sampling (Gao, Kyng & Spielman, arXiv:2303.00709, the sampled
 * replacement of an eliminated vertex's clique; called by the reference at
 * schur_complement.rs:128-139 through approx-chol, not vendored).
 * Neighbours (each split into `split` copies of weight w/split) are sorted by
 * weight; copy i (all but the last) links to one later copy j drawn with
 * probability w_j / S_i, S_i = sum of weights after i, with edge weight
 * w_i * S_i / d.  E[edge(a,b)] = w_a w_b / d, the clique's weight.  Links
 * between copies of one neighbour are self-loops and are dropped.  One uniform
 * draw per copy i from splitmix64(seed).
 */
static void clique_tree_sample(nbr_t *nb, int32_t deg, uint32_t split, double d, uint64_t seed,
                               edges_t *out, nbr_t *scratch, double *cum, double *suf) {
    if (split < 1) split = 1;
    int32_t m = deg * (int32_t)split;
    nbr_t *v = scratch;
    for (int32_t a = 0, p = 0; a < deg; a++)
        for (uint32_t s = 0; s < split; s++, p++) { v[p].col = nb[a].col; v[p].w = nb[a].w / (double)split; }
    qsort(v, (size_t)m, sizeof(nbr_t), cmp_nbr_w);
    double acc = 0.0;
    for (int32_t a = 0; a < m; a++) { acc += v[a].w; cum[a] = acc; }
    acc = 0.0;
    for (int32_t a = m - 1; a >= 0; a--) { suf[a] = acc; acc += v[a].w; }
    uint64_t st = seed;
    for (int32_t i = 0; i + 1 < m; i++) {
        double u = sm64_u01(&st);
        if (!(suf[i] > 0.0)) continue;
        double target = cum[i] + u * suf[i];
        int32_t lo = i + 1, hi = m - 1;          /* smallest j > i with cum[j] > target */
        while (lo < hi) { int32_t mid = (lo + hi) >> 1; if (cum[mid] > target) hi = mid; else lo = mid + 1; }
        int32_t j = lo;
        if (v[j].col == v[i].col) continue;
        edges_push(out, v[i].col, v[j].col, v[i].w * suf[i] / d);
    }
}

static int cmp_edge(const void *pa, const void *pb) {
    const edge_t *a = pa, *b = pb;
    if (a->lo != b->lo) return a->lo < b->lo ? -1 : 1;
    if (a->hi != b->hi) return a->hi < b->hi ? -1 : 1;
    return 0;
}
/* Stable sort by (lo, hi) then sum duplicates in emission order (sort_and_dedup, :259-277). */
static void edges_sort_merge(edges_t *v) {
    if (v->n <= 1) return;
    /* stable: sort (key, emission index) */
    typedef struct { edge_t e; size_t idx; } ie_t;
    ie_t *t = xcalloc(v->n, sizeof(ie_t));
    for (size_t a = 0; a < v->n; a++) { t[a].e = v->e[a]; t[a].idx = a; }
    /* merge sort for stability */
    ie_t *tmp = xcalloc(v->n, sizeof(ie_t));
    for (size_t width = 1; width < v->n; width *= 2) {
        for (size_t lo = 0; lo < v->n; lo += 2 * width) {
            size_t mid = lo + width < v->n ? lo + width : v->n;
            size_t hi = lo + 2 * width < v->n ? lo + 2 * width : v->n;
            size_t a = lo, b = mid, o = lo;
            while (a < mid && b < hi) {
                if (cmp_edge(&t[b].e, &t[a].e) < 0) tmp[o++] = t[b++]; else tmp[o++] = t[a++];
            }
            while (a < mid) tmp[o++] = t[a++];
            while (b < hi) tmp[o++] = t[b++];
        }
        ie_t *sw = t; t = tmp; tmp = sw;
    }
    size_t w = 0;
    v->e[0] = t[0].e;
    for (size_t a = 1; a < v->n; a++) {
        if (t[a].e.lo == v->e[w].lo && t[a].e.hi == v->e[w].hi) v->e[w].w += t[a].e.w;
        else v->e[++w] = t[a].e;
    }
    v->n = w + 1;
    free(t); free(tmp);
}

/* build_laplacian_csr, schur_complement.rs:534-586: rows [lower | diag | upper], -w off-diagonal. */
static smat_t laplacian_from_edges(const edges_t *v, int32_t n) {
    uint32_t *lc = xcalloc((size_t)n, sizeof(uint32_t)), *uc = xcalloc((size_t)n, sizeof(uint32_t));
    double *dg = xcalloc((size_t)n, sizeof(double));
    for (size_t a = 0; a < v->n; a++) {
        uc[v->e[a].lo]++; lc[v->e[a].hi]++;
        dg[v->e[a].lo] += v->e[a].w; dg[v->e[a].hi] += v->e[a].w;
    }
    smat_t s; s.n = n; s.indptr = xcalloc((size_t)n + 1, sizeof(uint32_t));
    for (int32_t i = 0; i < n; i++) s.indptr[i + 1] = s.indptr[i] + lc[i] + 1 + uc[i];
    size_t nnz = s.indptr[n];
    s.indices = xcalloc(nnz, sizeof(uint32_t)); s.data = xcalloc(nnz, sizeof(double));
    uint32_t *lcur = xcalloc((size_t)n, sizeof(uint32_t)), *ucur = xcalloc((size_t)n, sizeof(uint32_t));
    for (int32_t i = 0; i < n; i++) {
        lcur[i] = s.indptr[i]; ucur[i] = s.indptr[i] + lc[i] + 1;
        uint32_t p = s.indptr[i] + lc[i];
        s.indices[p] = (uint32_t)i; s.data[p] = dg[i];
    }
    for (size_t a = 0; a < v->n; a++) {
        uint32_t lo = v->e[a].lo, hi = v->e[a].hi;
        uint32_t p = ucur[lo]++; s.indices[p] = hi; s.data[p] = -v->e[a].w;
        p = lcur[hi]++; s.indices[p] = lo; s.data[p] = -v->e[a].w;
    }
    free(lc); free(uc); free(dg); free(lcur); free(ucur);
    return s;
}

/* ApproxSchurComplement::compute, schur_complement.rs:697-711 with par_emit :234-252:
 * stars of degree > 1 emit sampled clique trees with seed = seed + k. */
static smat_t schur_approx(const elim_t *e, uint64_t seed, uint32_t split) {
    edges_t ed = {0};
    int32_t maxdeg = 1;
    for (int32_t k = 0; k < e->n_elim; k++) {
        int32_t dg = (int32_t)(e->e2k->indptr[k + 1] - e->e2k->indptr[k]);
        if (dg > maxdeg) maxdeg = dg;
    }
    size_t sc = (size_t)maxdeg * (split ? split : 1) + 1;
    nbr_t *nb = xcalloc((size_t)maxdeg + 1, sizeof(nbr_t)), *scr = xcalloc(sc, sizeof(nbr_t));
    double *cum = xcalloc(sc, sizeof(double)), *suf = xcalloc(sc, sizeof(double));
    for (int32_t k = 0; k < e->n_elim; k++) {
        uint32_t b = e->e2k->indptr[k], en = e->e2k->indptr[k + 1];
        int32_t dg = (int32_t)(en - b);
        if (dg <= 1) continue;
        for (int32_t a = 0; a < dg; a++) { nb[a].col = e->e2k->indices[b + a]; nb[a].w = e->e2k->data[b + a]; }
        clique_tree_sample(nb, dg, split, e->diag_elim[k], seed + (uint64_t)k, &ed, scr, cum, suf);
    }
    free(nb); free(scr); free(cum); free(suf);
    edges_sort_merge(&ed);
    smat_t s = laplacian_from_edges(&ed, e->n_keep);
    free(ed.e);
    return s;
}

/* ------------------------------------------------------------------------- */
/* Approximate Cholesky (restated from GKS 2025; approx-chol is not vendored) */
/* ------------------------------------------------------------------------- */

/*
 * Factor of a Laplacian S as a product of eliminations L D L^T.  Vertices are
 * eliminated in rounds; each round is a maximal independent set of the current
 * graph chosen greedily by (degree, hash) -- so the eliminations of one round
 * commute and a triangular sweep needs one step per round.  Eliminating v with
 * merged neighbour weights w_u and d = sum w_u records the column
 * (u, w_u/d) and pivot d, and replaces v's clique by a sampled clique tree
 * (splitting each neighbour into `split` copies; split = 1 is plain AC).
 * A vertex with no live neighbours gets d = 0 and anchors its component.
 * Off-diagonal entries alone define the Laplacian (the diagonal is implied).
 * Once at most AC_CORE_MAX vertices remain, elimination stops: the remaining
 * Laplacian (the core, exact from there on) is kept dense and replaced by its
 * anchored inverse Z -- in each connected component of the core the largest
 * vertex is pinned to 0 and the rest solve against the SPD minor -- so the
 * core's solve is one dense product instead of a chain of tiny rounds.
 */
typedef struct {
    int32_t n, nlev, ncol;
    int32_t *level_ptr;   /* nlev+1, into column order */
    int32_t *col_vertex;  /* ncol */
    double *col_diag;     /* ncol */
    int32_t *col_ptr;     /* ncol+1 */
    int32_t *col_idx;     /* nnz */
    double *col_coef;     /* nnz */
    int32_t ncore;        /* vertices left when the rounds stop (n - ncol) */
    int32_t *core_vertex; /* ncore, ascending */
    double *core_z;       /* ncore x ncore row-major anchored inverse of the core Laplacian */
} acf_t;

static void acf_free(acf_t *f) {
    free(f->level_ptr); free(f->col_vertex); free(f->col_diag); free(f->col_ptr);
    free(f->col_idx); free(f->col_coef); free(f->core_vertex); free(f->core_z); memset(f, 0, sizeof *f);
}

/* Rounds stop once at most this many vertices remain; those form the dense core. */
#define AC_CORE_MAX 1024
/* Rounds also stop once one would eliminate fewer than max(AC_STALL_MIN, remaining /
   AC_STALL_DIV) vertices (the remaining graph has turned dense); if more than
   AC_CORE_MAX vertices remain then, they become one last level of pivots: the diagonal
   of the remaining Laplacian, without off-diagonal entries. */
#define AC_STALL_MIN 32
#define AC_STALL_DIV 128

typedef struct { nbr_t *a; int32_t n, cap; } adj_t;
static void adj_push(adj_t *l, uint32_t c, double w) {
    if (l->n == l->cap) { l->cap = l->cap ? l->cap * 2 : 8; l->a = xrealloc(l->a, sizeof(nbr_t) * (size_t)l->cap); }
    l->a[l->n].col = c; l->a[l->n].w = w; l->n++;
}
/* stable bottom-up merge sort of neighbour records by column */
static void nbr_stable_sort(nbr_t *a, int32_t m, nbr_t *tmp) {
    nbr_t *src = a, *dst = tmp;
    for (int32_t width = 1; width < m; width *= 2) {
        for (int32_t lo = 0; lo < m; lo += 2 * width) {
            int32_t mid = lo + width < m ? lo + width : m, hi = lo + 2 * width < m ? lo + 2 * width : m;
            int32_t x = lo, y = mid, o = lo;
            while (x < mid && y < hi) { if (src[y].col < src[x].col) dst[o++] = src[y++]; else dst[o++] = src[x++]; }
            while (x < mid) dst[o++] = src[x++];
            while (y < hi) dst[o++] = src[y++];
        }
        nbr_t *sw = src; src = dst; dst = sw;
    }
    if (src != a) memcpy(a, src, sizeof(nbr_t) * (size_t)m);
}
/* compact an adjacency list: drop dead neighbours, sort by column (stable), sum duplicates
 * in list order.  tmp must hold l->n records. */
static void adj_compact(adj_t *l, const uint8_t *dead, nbr_t *tmp) {
    int32_t m = 0;
    for (int32_t a = 0; a < l->n; a++) if (!dead[l->a[a].col]) l->a[m++] = l->a[a];
    nbr_stable_sort(l->a, m, tmp);
    int32_t w = 0;
    for (int32_t a = 0; a < m; a++) {
        if (w > 0 && l->a[w - 1].col == l->a[a].col) l->a[w - 1].w += l->a[a].w;
        else l->a[w++] = l->a[a];
    }
    l->n = w;
}

typedef struct { int32_t deg; uint64_t h; int32_t v; } rk_t;
static int cmp_rk(const void *pa, const void *pb) {
    const rk_t *a = pa, *b = pb;
    if (a->deg != b->deg) return a->deg < b->deg ? -1 : 1;
    if (a->h != b->h) return a->h < b->h ? -1 : 1;
    return (a->v > b->v) - (a->v < b->v);
}

static int dense_llt(double *a, int32_t m);

/* In-place inverse of an SPD row-major matrix through its Cholesky factor:
 * A = L L^T, then A^-1 = L^-T L^-1.  Returns -1 when a pivot is not positive. */
static int spd_inverse(double *a, int32_t m) {
    if (dense_llt(a, m)) return -1;
    /* invert L in place (lower triangle) */
    for (int32_t j = 0; j < m; j++) {
        a[(size_t)j * m + j] = 1.0 / a[(size_t)j * m + j];
        for (int32_t i = j + 1; i < m; i++) {
            double s = 0.0;
            for (int32_t k = j; k < i; k++) s += a[(size_t)i * m + k] * a[(size_t)k * m + j];
            a[(size_t)i * m + j] = -s / a[(size_t)i * m + i];
        }
    }
    /* Z = Linv^T Linv, symmetric; lower triangle computed then mirrored */
    double *z = xcalloc((size_t)m * (size_t)m, sizeof(double));
    for (int32_t i = 0; i < m; i++)
        for (int32_t j = 0; j <= i; j++) {
            double s = 0.0;
            for (int32_t k = i; k < m; k++) s += a[(size_t)k * m + i] * a[(size_t)k * m + j];
            z[(size_t)i * m + j] = s;
            z[(size_t)j * m + i] = s;
        }
    memcpy(a, z, sizeof(double) * (size_t)m * (size_t)m);
    free(z);
    return 0;
}

/* Dense core of an AC factor: live vertices ascending, their exact Laplacian from the
 * current adjacency, anchored inverse per connected component (anchor = largest vertex). */
static void ac_build_core(acf_t *f, adj_t *g, const uint8_t *dead, nbr_t *tmp, int32_t *maxlen) {
    int32_t n = f->n, r = 0;
    int32_t *loc = xcalloc((size_t)n + 1, sizeof(int32_t));
    for (int32_t v = 0; v < n; v++) loc[v] = dead[v] ? -1 : r++;
    f->ncore = r;
    f->core_vertex = xcalloc((size_t)r + 1, sizeof(int32_t));
    f->core_z = xcalloc((size_t)r * (size_t)r + 1, sizeof(double));
    if (r == 0) { free(loc); return; }
    for (int32_t v = 0; v < n; v++) if (!dead[v]) f->core_vertex[loc[v]] = v;
    double *S = xcalloc((size_t)r * (size_t)r, sizeof(double));
    int32_t *parent = xcalloc((size_t)r, sizeof(int32_t));
    for (int32_t a = 0; a < r; a++) parent[a] = a;
    for (int32_t a = 0; a < r; a++) {
        adj_t *L = &g[f->core_vertex[a]];
        if (L->n > *maxlen) { *maxlen = L->n * 2; }
        nbr_t *t2 = xcalloc((size_t)L->n + 1, sizeof(nbr_t));
        (void)tmp;
        adj_compact(L, dead, t2);
        free(t2);
        for (int32_t b = 0; b < L->n; b++) {
            int32_t c = loc[L->a[b].col];
            S[(size_t)a * r + c] -= L->a[b].w;
            S[(size_t)a * r + a] += L->a[b].w;
            int32_t x = a, y = c;
            while (parent[x] != x) x = parent[x];
            while (parent[y] != y) y = parent[y];
            if (x != y) { if (x < y) parent[y] = x; else parent[x] = y; }
        }
    }
    int32_t *root = xcalloc((size_t)r, sizeof(int32_t));
    for (int32_t a = 0; a < r; a++) { int32_t x = a; while (parent[x] != x) x = parent[x]; root[a] = x; }
    int32_t *mem = xcalloc((size_t)r, sizeof(int32_t));
    uint8_t *done = xcalloc((size_t)r, 1);
    for (int32_t a = 0; a < r; a++) {
        if (done[root[a]]) continue;
        done[root[a]] = 1;
        int32_t p = 0;
        for (int32_t b = a; b < r; b++) if (root[b] == root[a]) mem[p++] = b;
        int32_t m = p - 1;                       /* last member is the anchor */
        if (m <= 0) continue;
        double *A = xcalloc((size_t)m * (size_t)m, sizeof(double));
        for (int32_t i = 0; i < m; i++)
            for (int32_t j = 0; j < m; j++) A[(size_t)i * m + j] = S[(size_t)mem[i] * r + mem[j]];
        if (spd_inverse(A, m) == 0) {
            for (int32_t i = 0; i < m; i++)
                for (int32_t j = 0; j < m; j++) f->core_z[(size_t)mem[i] * r + mem[j]] = A[(size_t)i * m + j];
        }
        free(A);
    }
    free(S); free(parent); free(root); free(mem); free(done); free(loc);
}

static acf_t ac_build(const smat_t *s, uint64_t seed, uint32_t split) {
    int32_t n = s->n;
    acf_t f; memset(&f, 0, sizeof f);
    f.n = n;
    adj_t *g = xcalloc((size_t)n + 1, sizeof(adj_t));
    for (int32_t i = 0; i < n; i++)
        for (uint32_t e = s->indptr[i]; e < s->indptr[i + 1]; e++) {
            uint32_t j = s->indices[e];
            if ((int32_t)j != i && s->data[e] < 0.0) adj_push(&g[i], j, -s->data[e]);
        }
    uint8_t *dead = xcalloc((size_t)n + 1, 1), *blocked = xcalloc((size_t)n + 1, 1);
    rk_t *rk = xcalloc((size_t)n + 1, sizeof(rk_t));
    int32_t *picked = xcalloc((size_t)n + 1, sizeof(int32_t));
    f.level_ptr = xcalloc((size_t)n + 2, sizeof(int32_t));
    f.col_vertex = xcalloc((size_t)n + 1, sizeof(int32_t));
    f.col_diag = xcalloc((size_t)n + 1, sizeof(double));
    f.col_ptr = xcalloc((size_t)n + 2, sizeof(int32_t));
    size_t ccap = 64, cnnz = 0;
    f.col_idx = xcalloc(ccap, sizeof(int32_t)); f.col_coef = xcalloc(ccap, sizeof(double));
    int32_t maxlen = 8;
    nbr_t *tmp = xcalloc((size_t)maxlen, sizeof(nbr_t));
    int32_t ncol = 0, remaining = n;
    size_t scap = 16;
    nbr_t *scr = xcalloc(scap, sizeof(nbr_t));
    double *cum = xcalloc(scap, sizeof(double)), *suf = xcalloc(scap, sizeof(double));
    edges_t fill = {0};
    while (remaining > AC_CORE_MAX) {
        int32_t nr = 0;
        for (int32_t v = 0; v < n; v++) {
            if (dead[v]) continue;
            if (g[v].n > maxlen) { maxlen = g[v].n * 2; tmp = xrealloc(tmp, sizeof(nbr_t) * (size_t)maxlen); }
            adj_compact(&g[v], dead, tmp);
            rk[nr].deg = g[v].n; rk[nr].h = mix64(seed ^ ((uint64_t)v * 0xD1B54A32D192ED03ULL)); rk[nr].v = v;
            nr++;
        }
        qsort(rk, (size_t)nr, sizeof(rk_t), cmp_rk);
        int32_t np = 0;
        for (int32_t a = 0; a < nr; a++) {
            int32_t v = rk[a].v;
            if (blocked[v]) continue;
            picked[np++] = v;
            blocked[v] = 1;
            for (int32_t b = 0; b < g[v].n; b++) blocked[g[v].a[b].col] = 1;
        }
        {
            int64_t lim = (int64_t)remaining / AC_STALL_DIV;
            if (lim < AC_STALL_MIN) lim = AC_STALL_MIN;
            if ((int64_t)np < lim) {  /* the remaining graph has turned dense: stop */
                for (int32_t a = 0; a < nr; a++) blocked[rk[a].v] = 0;
                break;
            }
        }
        f.level_ptr[f.nlev] = ncol;
        for (int32_t a = 0; a < np; a++) {
            int32_t v = picked[a];
            adj_t *L = &g[v];
            double d = 0.0;
            for (int32_t b = 0; b < L->n; b++) d += L->a[b].w;
            f.col_vertex[ncol] = v;
            f.col_diag[ncol] = L->n > 0 ? d : 0.0;
            f.col_ptr[ncol] = (int32_t)cnnz;
            if (cnnz + (size_t)L->n > ccap) {
                while (cnnz + (size_t)L->n > ccap) ccap *= 2;
                f.col_idx = xrealloc(f.col_idx, ccap * sizeof(int32_t));
                f.col_coef = xrealloc(f.col_coef, ccap * sizeof(double));
            }
            for (int32_t b = 0; b < L->n; b++) {
                f.col_idx[cnnz] = (int32_t)L->a[b].col;
                f.col_coef[cnnz] = L->a[b].w / d;
                cnnz++;
            }
            ncol++;
            if (L->n > 1) {
                size_t need = (size_t)L->n * (split ? split : 1) + 1;
                if (need > scap) {
                    scap = need * 2;
                    scr = xrealloc(scr, scap * sizeof(nbr_t));
                    cum = xrealloc(cum, scap * sizeof(double)); suf = xrealloc(suf, scap * sizeof(double));
                }
                fill.n = 0;
                clique_tree_sample(L->a, L->n, split, d, seed + (uint64_t)v, &fill, scr, cum, suf);
                for (size_t e = 0; e < fill.n; e++) {
                    adj_push(&g[fill.e[e].lo], fill.e[e].hi, fill.e[e].w);
                    adj_push(&g[fill.e[e].hi], fill.e[e].lo, fill.e[e].w);
                }
            }
        }
        for (int32_t a = 0; a < np; a++) { dead[picked[a]] = 1; }
        for (int32_t a = 0; a < nr; a++) blocked[rk[a].v] = 0;
        remaining -= np;
        f.nlev++;
    }
    if (remaining > AC_CORE_MAX) {
        /* stalled, larger than a core: one last level of pivots (weighted degree in the
           remaining graph) without off-diagonal entries */
        f.level_ptr[f.nlev] = ncol;
        for (int32_t v = 0; v < n; v++) {
            if (dead[v]) continue;
            if (g[v].n > maxlen) { maxlen = g[v].n * 2; tmp = xrealloc(tmp, sizeof(nbr_t) * (size_t)maxlen); }
            adj_compact(&g[v], dead, tmp);
            double d = 0.0;
            for (int32_t b = 0; b < g[v].n; b++) d += g[v].a[b].w;
            f.col_vertex[ncol] = v;
            f.col_diag[ncol] = g[v].n > 0 ? d : 0.0;
            f.col_ptr[ncol] = (int32_t)cnnz;
            ncol++;
        }
        for (int32_t v = 0; v < n; v++) dead[v] = 1;
        f.nlev++;
    }
    f.level_ptr[f.nlev] = ncol;
    f.col_ptr[ncol] = (int32_t)cnnz;
    f.ncol = ncol;
    ac_build_core(&f, g, dead, tmp, &maxlen);
    for (int32_t v = 0; v < n; v++) free(g[v].a);
    free(g); free(dead); free(blocked); free(rk); free(picked); free(tmp);
    free(scr); free(cum); free(suf); free(fill.e);
    return f;
}

/* Solve L D L^T y = b in place: forward y_u += c*y_v, pivots, backward y_v += sum c*y_u. */
static void ac_solve(const acf_t *f, double *y) {
    for (int32_t c = 0; c < f->ncol; c++) {
        double yv = y[f->col_vertex[c]];
        for (int32_t e = f->col_ptr[c]; e < f->col_ptr[c + 1]; e++) y[f->col_idx[e]] += f->col_coef[e] * yv;
    }
    for (int32_t c = 0; c < f->ncol; c++) {
        int32_t v = f->col_vertex[c];
        y[v] = f->col_diag[c] > 0.0 ? y[v] / f->col_diag[c] : 0.0;
    }
    if (f->ncore > 0) {
        int32_t r = f->ncore;
        double *yc = xcalloc((size_t)r, sizeof(double));
        for (int32_t a = 0; a < r; a++) yc[a] = y[f->core_vertex[a]];
        for (int32_t a = 0; a < r; a++) {
            double s = 0.0;
            for (int32_t b = 0; b < r; b++) s += f->core_z[(size_t)a * r + b] * yc[b];
            y[f->core_vertex[a]] = s;
        }
        free(yc);
    }
    for (int32_t c = f->ncol - 1; c >= 0; c--) {
        int32_t v = f->col_vertex[c];
        double s = y[v];
        for (int32_t e = f->col_ptr[c]; e < f->col_ptr[c + 1]; e++) s += f->col_coef[e] * y[f->col_idx[e]];
        y[v] = s;
    }
}

/* ------------------------------------------------------------------------- */
/* Local solver: within/src/operator/local_solver.rs                         */
/* ------------------------------------------------------------------------- */

typedef struct {
    int q, r;
    int32_t nidx;
    uint32_t *gidx;
    double *pou;            /* NULL = uniform (PartitionWeights::Uniform) */
    crosstab_t ct;
    int elim_q;
    double *inv_diag;
    int kind;               /* 0 dense anchored Cholesky, 1 approximate Cholesky */
    int32_t n_red;
    double *L;              /* dense: (n_red-1)^2 row-major lower factor */
    acf_t ac;
} subdomain_t;

/* Plain lower Cholesky of an SPD row-major matrix (faer LLT in the reference,
 * local_solver.rs:229-243).  Returns -1 when a pivot is not positive. */
static int dense_llt(double *a, int32_t m) {
    for (int32_t j = 0; j < m; j++) {
        double s = a[(size_t)j * m + j];
        for (int32_t k = 0; k < j; k++) s -= a[(size_t)j * m + k] * a[(size_t)j * m + k];
        if (!(s > 0.0)) return -1;
        double ljj = sqrt(s);
        a[(size_t)j * m + j] = ljj;
        for (int32_t i = j + 1; i < m; i++) {
            double t = a[(size_t)i * m + j];
            for (int32_t k = 0; k < j; k++) t -= a[(size_t)i * m + k] * a[(size_t)j * m + k];
            a[(size_t)i * m + j] = t / ljj;
        }
        for (int32_t i = 0; i < j; i++) a[(size_t)i * m + j] = 0.0;
    }
    return 0;
}
/* AnchoredDenseCholesky::solve_in_place, local_solver.rs:252-299. */
static void dense_anchored_solve(const double *l, int32_t n, double *x) {
    if (n == 0) return;
    if (n == 1) { x[0] = 0.0; return; }
    int32_t m = n - 1;
    for (int32_t i = 0; i < m; i++) {
        double s = x[i];
        for (int32_t j = 0; j < i; j++) s -= l[(size_t)i * m + j] * x[j];
        x[i] = s / l[(size_t)i * m + i];
    }
    for (int32_t i = m - 1; i >= 0; i--) {
        double s = x[i];
        for (int32_t j = i + 1; j < m; j++) s -= l[(size_t)j * m + i] * x[j];
        x[i] = s / l[(size_t)i * m + i];
    }
    x[m] = 0.0;
}

static void negate_from(double *v, int32_t from, int32_t n) { for (int32_t i = from; i < n; i++) v[i] = -v[i]; }
static void subtract_mean(double *v, int32_t n) {      /* local_solver.rs:91-99 */
    if (n == 0) return;
    double s = 0.0;
    for (int32_t i = 0; i < n; i++) s += v[i];
    double mean = s / (double)n;
    for (int32_t i = 0; i < n; i++) v[i] -= mean;
}

/* build_reduced_schur_factor, operator/schwarz.rs:274-303 (dense fast path when
 * 0 < threshold and n_keep <= threshold, else exact or sampled Schur + AC). */
static int subdomain_build(subdomain_t *sd, const oracle_params *p, char *err, int errlen) {
    elim_t e;
    if (elim_init(&sd->ct, &e, err, errlen)) return -1;
    sd->elim_q = e.elim_q;
    sd->inv_diag = e.inv_diag;
    int32_t n_keep = e.n_keep;
    if (p->dense_threshold > 0 && n_keep <= p->dense_threshold) {
        double *minor = schur_anchored_minor(&e);
        int ok = 1;
        if (n_keep > 1) ok = dense_llt(minor, n_keep - 1) == 0;
        if (ok) { sd->kind = 0; sd->n_red = n_keep; sd->L = minor; return 0; }
        free(minor);
    }
    smat_t s = p->approx_schur_enabled ? schur_approx(&e, p->approx_schur_seed, p->approx_schur_split)
                                       : schur_exact(&e);
    sd->kind = 1;
    sd->n_red = n_keep;
    sd->ac = ac_build(&s, p->approx_chol_seed, p->approx_chol_split);
    smat_free(&s);
    return 0;
}

/* BlockElimSolver::solve_local_with_parallelism, local_solver.rs:360-449.
 * rhs has n + n_red entries (scratch tail), sol has n entries. */
static void local_solve(const subdomain_t *sd, double *rhs, double *sol) {
    const crosstab_t *ct = &sd->ct;
    int32_t nq = ct->c.nrows, nr = ct->c.ncols, n = nq + nr;
    negate_from(rhs, nq, n);
    subtract_mean(rhs, n);
    double *red = rhs + n;
    if (sd->elim_q) {
        for (int32_t i = 0; i < nq; i++) rhs[i] *= sd->inv_diag[i];
        for (int32_t i = 0; i < nr; i++) {         /* red = rhs_r + C^T rhs_q */
            double acc = rhs[nq + i];
            for (uint32_t e = ct->ct.indptr[i]; e < ct->ct.indptr[i + 1]; e++)
                acc += ct->ct.data[e] * rhs[ct->ct.indices[e]];
            red[i] = acc;
        }
        subtract_mean(red, sd->n_red);
        double *sk = sol + nq;
        memcpy(sk, red, sizeof(double) * (size_t)sd->n_red);
        if (sd->kind == 0) dense_anchored_solve(sd->L, sd->n_red, sk); else ac_solve(&sd->ac, sk);
        for (int32_t i = 0; i < nq; i++) {         /* backsub :111-151 */
            double s = 0.0;
            for (uint32_t e = ct->c.indptr[i]; e < ct->c.indptr[i + 1]; e++) s += ct->c.data[e] * sk[ct->c.indices[e]];
            sol[i] = rhs[i] + sd->inv_diag[i] * s;
        }
    } else {
        for (int32_t i = 0; i < nr; i++) rhs[nq + i] *= sd->inv_diag[i];
        for (int32_t i = 0; i < nq; i++) {         /* red = rhs_q + C rhs_r */
            double acc = rhs[i];
            for (uint32_t e = ct->c.indptr[i]; e < ct->c.indptr[i + 1]; e++)
                acc += ct->c.data[e] * rhs[nq + ct->c.indices[e]];
            red[i] = acc;
        }
        subtract_mean(red, sd->n_red);
        memcpy(sol, red, sizeof(double) * (size_t)sd->n_red);
        if (sd->kind == 0) dense_anchored_solve(sd->L, sd->n_red, sol); else ac_solve(&sd->ac, sol);
        for (int32_t i = 0; i < nr; i++) {
            double s = 0.0;
            for (uint32_t e = ct->ct.indptr[i]; e < ct->ct.indptr[i + 1]; e++) s += ct->ct.data[e] * sol[ct->ct.indices[e]];
            sol[nq + i] = rhs[nq + i] + sd->inv_diag[i] * s;
        }
    }
    subtract_mean(sol, n);
    negate_from(sol, nq, n);
}

/* ------------------------------------------------------------------------- */
/* Solver state                                                              */
/* ------------------------------------------------------------------------- */

struct oracle_solver {
    design_t d;
    oracle_params p;
    int32_t nsub;
    subdomain_t *sub;
    int32_t max_local;
    /* explicit Gramian (multiplicative Schwarz only): symmetric CSR, cols ascending */
    int64_t *g_ptr;
    uint32_t *g_idx;
    double *g_val;
};

/* build_local_domains, domain/factor_pairs.rs:63-80, pairs (q<r) in order :252-260, one
 * subdomain per component with indices q-levels then r-levels :244-250, PoU weights
 * 1/sqrt(count) unless every index is unique :272-304. */
static int build_domains(oracle_solver *s, char *err, int errlen) {
    design_t *d = &s->d;
    uint8_t **active = xcalloc((size_t)d->Q, sizeof(uint8_t *));
    for (int q = 0; q < d->Q; q++) {                       /* find_all_active_levels :75-89 */
        active[q] = xcalloc((size_t)d->nlev[q], 1);
        for (int64_t i = 0; i < d->n; i++) active[q][lev(d, i, q)] = 1;
    }
    int32_t cap = 8; s->nsub = 0;
    s->sub = xcalloc((size_t)cap, sizeof(subdomain_t));
    for (int q = 0; q < d->Q; q++)
        for (int r = q + 1; r < d->Q; r++) {
            crosstab_t full; uint32_t *l2g; int32_t nqf;
            if (!crosstab_build(d, q, r, active, &full, &l2g, &nqf)) continue;
            comp_t *comps; int32_t nc = crosstab_components(&full, &comps);
            for (int32_t c = 0; c < nc; c++) {
                if (s->nsub == cap) { cap *= 2; s->sub = xrealloc(s->sub, sizeof(subdomain_t) * (size_t)cap); }
                subdomain_t *sd = &s->sub[s->nsub++];
                memset(sd, 0, sizeof *sd);
                sd->q = q; sd->r = r;
                sd->ct = nc == 1 ? full : crosstab_extract(&full, &comps[c]);
                sd->nidx = comps[c].nq + comps[c].nr;
                sd->gidx = xcalloc((size_t)sd->nidx, sizeof(uint32_t));
                for (int32_t a = 0; a < comps[c].nq; a++) sd->gidx[a] = l2g[comps[c].qi[a]];
                for (int32_t a = 0; a < comps[c].nr; a++) sd->gidx[comps[c].nq + a] = l2g[nqf + comps[c].ri[a]];
            }
            if (nc != 1) crosstab_free(&full);
            for (int32_t c = 0; c < nc; c++) { free(comps[c].qi); free(comps[c].ri); }
            free(comps); free(l2g);
        }
    for (int q = 0; q < d->Q; q++) free(active[q]);
    free(active);
    uint32_t *cnt = xcalloc((size_t)d->ndofs + 1, sizeof(uint32_t));
    for (int32_t i = 0; i < s->nsub; i++)
        for (int32_t a = 0; a < s->sub[i].nidx; a++) cnt[s->sub[i].gidx[a]]++;
    s->max_local = 0;
    for (int32_t i = 0; i < s->nsub; i++) {
        subdomain_t *sd = &s->sub[i];
        int uniq = 1;
        for (int32_t a = 0; a < sd->nidx; a++) if (cnt[sd->gidx[a]] > 1) { uniq = 0; break; }
        if (!uniq) {
            sd->pou = xcalloc((size_t)sd->nidx, sizeof(double));
            for (int32_t a = 0; a < sd->nidx; a++) sd->pou[a] = 1.0 / sqrt((double)cnt[sd->gidx[a]]);
        }
        if (sd->nidx > s->max_local) s->max_local = sd->nidx;
    }
    free(cnt);
    for (int32_t i = 0; i < s->nsub; i++)
        if (subdomain_build(&s->sub[i], &s->p, err, errlen)) return -1;
    return 0;
}

/* Explicit symmetric CSR of G (Gramian::build, gramian/explicit.rs:207): per global row,
 * the diagonal plus every cross-tab row of the factor pairs it belongs to, cols ascending. */
typedef struct { uint32_t col; double w; } gent_t;
static int cmp_gent(const void *pa, const void *pb) {
    const gent_t *a = pa, *b = pb;
    return (a->col > b->col) - (a->col < b->col);
}
static void build_explicit_gramian(oracle_solver *s) {
    design_t *d = &s->d;
    int64_t m = d->ndofs;
    double *diag = xcalloc((size_t)m, sizeof(double));
    design_diag(d, diag);
    /* count pair entries per row from the full (uncompacted) pair cross products */
    int64_t *cnt = xcalloc((size_t)m + 1, sizeof(int64_t));
    int64_t npairs = (int64_t)d->Q * (d->Q - 1) / 2;
    /* per pair: sort (gq, gr) keys of all observations, merge -> entries */
    gent_t **rows = xcalloc((size_t)m, sizeof(gent_t *));
    int64_t *rn = xcalloc((size_t)m, sizeof(int64_t)), *rc = xcalloc((size_t)m, sizeof(int64_t));
    (void)npairs;
    for (int q = 0; q < d->Q; q++)
        for (int r = q + 1; r < d->Q; r++) {
            int64_t Lq = d->nlev[q];
            /* bucket observations by q-level, dedup r-levels per row */
            int64_t *bp = xcalloc((size_t)Lq + 1, sizeof(int64_t));
            for (int64_t i = 0; i < d->n; i++) bp[lev(d, i, q) + 1]++;
            for (int64_t j = 0; j < Lq; j++) bp[j + 1] += bp[j];
            int64_t *cur = xcalloc((size_t)Lq + 1, sizeof(int64_t));
            memcpy(cur, bp, sizeof(int64_t) * (size_t)Lq);
            gent_t *b = xcalloc((size_t)d->n + 1, sizeof(gent_t));
            for (int64_t i = 0; i < d->n; i++) {
                int64_t pos = cur[lev(d, i, q)]++;
                b[pos].col = (uint32_t)(d->off[r] + lev(d, i, r)); b[pos].w = wt(d, i);
            }
            for (int64_t j = 0; j < Lq; j++) {
                int64_t lo = bp[j], hi = bp[j + 1];
                if (hi - lo > 1) {
                    /* stable merge sort by col */
                    int64_t len = hi - lo;
                    gent_t *t = xcalloc((size_t)len, sizeof(gent_t));
                    gent_t *src = b + lo, *dst = t;
                    for (int64_t width = 1; width < len; width *= 2) {
                        for (int64_t a0 = 0; a0 < len; a0 += 2 * width) {
                            int64_t mid = a0 + width < len ? a0 + width : len, e0 = a0 + 2 * width < len ? a0 + 2 * width : len;
                            int64_t x = a0, y = mid, o = a0;
                            while (x < mid && y < e0) { if (src[y].col < src[x].col) dst[o++] = src[y++]; else dst[o++] = src[x++]; }
                            while (x < mid) dst[o++] = src[x++];
                            while (y < e0) dst[o++] = src[y++];
                        }
                        gent_t *sw = src; src = dst; dst = sw;
                    }
                    if (src != b + lo) memcpy(b + lo, src, sizeof(gent_t) * (size_t)len);
                    free(t);
                }
                uint32_t gq = (uint32_t)(d->off[q] + j);
                for (int64_t e = lo; e < hi;) {
                    uint32_t col = b[e].col; double w = 0.0;
                    while (e < hi && b[e].col == col) { w += b[e].w; e++; }
                    if (w == 0.0) continue;
                    /* row gq gets (col, w); row col gets (gq, w) */
                    uint32_t rr[2] = { gq, col }, cc[2] = { col, gq };
                    for (int t2 = 0; t2 < 2; t2++) {
                        uint32_t row = rr[t2];
                        if (rn[row] == rc[row]) { rc[row] = rc[row] ? rc[row] * 2 : 4; rows[row] = xrealloc(rows[row], sizeof(gent_t) * (size_t)rc[row]); }
                        rows[row][rn[row]].col = cc[t2]; rows[row][rn[row]].w = w; rn[row]++;
                    }
                }
            }
            free(bp); free(cur); free(b);
        }
    s->g_ptr = xcalloc((size_t)m + 1, sizeof(int64_t));
    for (int64_t i = 0; i < m; i++) s->g_ptr[i + 1] = s->g_ptr[i] + rn[i] + 1;
    s->g_idx = xcalloc((size_t)s->g_ptr[m] + 1, sizeof(uint32_t));
    s->g_val = xcalloc((size_t)s->g_ptr[m] + 1, sizeof(double));
    for (int64_t i = 0; i < m; i++) {
        if (rows[i] == NULL) { rows[i] = xcalloc(1, sizeof(gent_t)); }
        rows[i] = xrealloc(rows[i], sizeof(gent_t) * (size_t)(rn[i] + 1));
        rows[i][rn[i]].col = (uint32_t)i; rows[i][rn[i]].w = diag[i];
        qsort(rows[i], (size_t)rn[i] + 1, sizeof(gent_t), cmp_gent);
        for (int64_t a = 0; a <= rn[i]; a++) {
            s->g_idx[s->g_ptr[i] + a] = rows[i][a].col;
            s->g_val[s->g_ptr[i] + a] = rows[i][a].w;
        }
        free(rows[i]);
    }
    free(rows); free(rn); free(rc); free(cnt); free(diag);
}

/* ------------------------------------------------------------------------- */
/* Operators                                                                 */
/* ------------------------------------------------------------------------- */

typedef struct { const oracle_solver *s; double *tmp; double *rl; double *zl; double *rw; double *wl; } work_t;

static void work_init(work_t *w, const oracle_solver *s) {
    w->s = s;
    w->tmp = xcalloc((size_t)s->d.n + 1, sizeof(double));
    w->rl = xcalloc((size_t)2 * s->max_local + 2, sizeof(double));
    w->zl = xcalloc((size_t)2 * s->max_local + 2, sizeof(double));
    w->rw = xcalloc((size_t)s->d.ndofs + 1, sizeof(double));
    w->wl = xcalloc((size_t)s->max_local + 1, sizeof(double));
}
static void work_free(work_t *w) { free(w->tmp); free(w->rl); free(w->zl); free(w->rw); free(w->wl); }

/* GramianOperator::apply, operator/gramian.rs:84-89. */
static void op_gramian(work_t *w, const double *x, double *y) {
    design_matvec_d(&w->s->d, x, w->tmp);
    design_rmatvec(&w->s->d, w->tmp, y, 1);
}

/* Additive Schwarz apply: out = sum_i R_i^T D_i A_i^+ D_i R_i r
 * (additive/executor.rs:59-147, local_solve.rs:182-248, domain.rs:190-243). */
static void op_additive(work_t *w, const double *r, double *z) {
    const oracle_solver *s = w->s;
    for (int64_t j = 0; j < s->d.ndofs; j++) z[j] = 0.0;
    for (int32_t i = 0; i < s->nsub; i++) {
        const subdomain_t *sd = &s->sub[i];
        for (int32_t a = 0; a < sd->nidx; a++) w->rl[a] = sd->pou ? r[sd->gidx[a]] * sd->pou[a] : r[sd->gidx[a]];
        local_solve(sd, w->rl, w->zl);
        for (int32_t a = 0; a < sd->nidx; a++) z[sd->gidx[a]] += sd->pou ? w->zl[a] * sd->pou[a] : w->zl[a];
    }
}

/* Multiplicative Schwarz apply (multiplicative.rs:128-168, 214-245) with the explicit
 * Gramian residual updater (residual_update.rs:36-53); forward sweep only. */
static void op_multiplicative(work_t *w, const double *r, double *z) {
    const oracle_solver *s = w->s;
    int64_t m = s->d.ndofs;
    for (int64_t j = 0; j < m; j++) { z[j] = 0.0; w->rw[j] = r[j]; }
    for (int32_t i = 0; i < s->nsub; i++) {
        const subdomain_t *sd = &s->sub[i];
        for (int32_t a = 0; a < sd->nidx; a++) w->rl[a] = sd->pou ? w->rw[sd->gidx[a]] * sd->pou[a] : w->rw[sd->gidx[a]];
        local_solve(sd, w->rl, w->zl);
        for (int32_t a = 0; a < sd->nidx; a++) z[sd->gidx[a]] += sd->pou ? w->zl[a] * sd->pou[a] : w->zl[a];
        for (int32_t a = 0; a < sd->nidx; a++) {
            double c = sd->pou ? sd->pou[a] * w->zl[a] : w->zl[a];
            if (c == 0.0) continue;
            uint32_t row = sd->gidx[a];
            for (int64_t e = s->g_ptr[row]; e < s->g_ptr[row + 1]; e++) w->rw[s->g_idx[e]] -= c * s->g_val[e];
        }
    }
}

static void op_precond(work_t *w, const double *r, double *z) {
    if (w->s->p.precond_kind == 1) op_additive(w, r, z);
    else if (w->s->p.precond_kind == 2) op_multiplicative(w, r, z);
    else for (int64_t j = 0; j < w->s->d.ndofs; j++) z[j] = r[j];
}

/* ------------------------------------------------------------------------- */
/* Krylov: schwarz-precond/src/solve/{cg,gmres}.rs                           */
/* ------------------------------------------------------------------------- */

typedef void (*apply_fn)(void *ctx, const double *x, double *y);
typedef struct { double *x; int converged; int iterations; double res; } kres_t;

/* cg_solve_preconditioned, cg.rs:45-133 (pAp <= 0 exit, EPS^2 stagnation guard). */
static kres_t krylov_cg(int64_t n, apply_fn A, apply_fn M, void *ctx, const double *b, double tol, int maxiter) {
    kres_t out; out.x = xcalloc((size_t)n + 1, sizeof(double));
    double bn = vnorm(b, n);
    if (bn < DBL_EPSILON) { out.converged = 1; out.iterations = 0; out.res = 0.0; return out; }
    double *x = out.x, *r = xcalloc((size_t)n + 1, sizeof(double)), *z = xcalloc((size_t)n + 1, sizeof(double));
    double *p = xcalloc((size_t)n + 1, sizeof(double)), *ap = xcalloc((size_t)n + 1, sizeof(double));
    memcpy(r, b, sizeof(double) * (size_t)n);
    M(ctx, r, z);
    memcpy(p, z, sizeof(double) * (size_t)n);
    double rz = vdot(r, z, n), rz0 = rz, rn = bn;
    out.converged = 0; out.iterations = maxiter;
    for (int it = 1; it <= maxiter; it++) {
        A(ctx, p, ap);
        double pap = vdot(p, ap, n);
        if (pap <= 0.0) { out.iterations = it; goto done; }
        double alpha = rz / pap, rr = 0.0;
        for (int64_t i = 0; i < n; i++) { x[i] += alpha * p[i]; r[i] -= alpha * ap[i]; rr += r[i] * r[i]; }
        rn = sqrt(rr);
        if (rn / bn <= tol) { out.converged = 1; out.iterations = it; goto done; }
        M(ctx, r, z);
        double rzn = vdot(r, z, n);
        double thr = DBL_EPSILON * DBL_EPSILON * fmax(fabs(rz0), DBL_MIN);
        if (fabs(rzn) < thr) { out.converged = rn / bn <= tol; out.iterations = it; goto done; }
        double beta = rzn / rz;
        for (int64_t i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        rz = rzn;
    }
done:
    out.res = rn;
    free(r); free(z); free(p); free(ap);
    return out;
}

/* gmres_solve, gmres.rs:348-452 with arnoldi_cycle :238-317, MGS :201-220, Givens :486-494,
 * back substitution :499-519, update :523-530. */
static kres_t krylov_gmres(int64_t n, apply_fn A, apply_fn M, void *ctx, const double *b, double tol,
                           int maxiter, int restart) {
    kres_t out; out.x = xcalloc((size_t)n + 1, sizeof(double));
    double bn = vnorm(b, n);
    if (bn < DBL_EPSILON) { out.converged = 1; out.iterations = 0; out.res = 0.0; return out; }
    int m = restart > 0 ? restart : 1;
    double abs_tol = tol * bn;
    double *x = out.x, *r = xcalloc((size_t)n + 1, sizeof(double)), *w = xcalloc((size_t)n + 1, sizeof(double));
    double *V = xcalloc((size_t)(m + 1) * (size_t)n + 1, sizeof(double));
    double *Z = xcalloc((size_t)m * (size_t)n + 1, sizeof(double));
    int stride = m + 1;
    double *H = xcalloc((size_t)m * (size_t)stride + 1, sizeof(double));
    double *cs = xcalloc((size_t)m + 1, sizeof(double)), *sn = xcalloc((size_t)m + 1, sizeof(double));
    double *g = xcalloc((size_t)m + 2, sizeof(double)), *y = xcalloc((size_t)m + 1, sizeof(double));
    int total = 0;
#define HG(i, j) H[(size_t)(j) * stride + (i)]
    for (;;) {
        A(ctx, x, r);
        for (int64_t i = 0; i < n; i++) r[i] = b[i] - r[i];
        double beta = vnorm(r, n);
        if (beta <= abs_tol) { out.converged = 1; out.iterations = total; out.res = beta; break; }
        if (total >= maxiter) { out.converged = 0; out.iterations = total; out.res = beta; break; }
        memset(H, 0, sizeof(double) * (size_t)m * stride);
        memset(cs, 0, sizeof(double) * (size_t)m); memset(sn, 0, sizeof(double) * (size_t)m);
        memset(g, 0, sizeof(double) * (size_t)(m + 1));
        g[0] = beta;
        for (int64_t i = 0; i < n; i++) V[i] = r[i] * (1.0 / beta);
        int cyc = (maxiter - total) < m ? (maxiter - total) : m;
        int j = 0, outcome = 3; /* 0 conv, 1 maxiter, 2 breakdown, 3 restart */
        double hmax = 0.0, resid = 0.0;
        while (j < cyc) {
            M(ctx, V + (size_t)j * n, Z + (size_t)j * n);
            A(ctx, Z + (size_t)j * n, w);
            double lmax = 0.0;
            for (int i = 0; i <= j; i++) {
                double hij = vdot(w, V + (size_t)i * n, n);
                HG(i, j) = hij;
                if (fabs(hij) > lmax) lmax = fabs(hij);
                for (int64_t k = 0; k < n; k++) w[k] -= hij * V[(size_t)i * n + k];
            }
            double hj1 = vnorm(w, n);
            HG(j + 1, j) = hj1;
            hmax = fmax(fmax(hmax, lmax), hj1);
            for (int i = 0; i < j; i++) {
                double a = HG(i, j), bb = HG(i + 1, j);
                double t = cs[i] * a + sn[i] * bb;
                HG(i + 1, j) = -sn[i] * a + cs[i] * bb;
                HG(i, j) = t;
            }
            double a = HG(j, j), bb = HG(j + 1, j), rr = hypot(a, bb), c, sgv;
            if (rr == 0.0) { c = 1.0; sgv = 0.0; } else { c = a / rr; sgv = bb / rr; }
            cs[j] = c; sn[j] = sgv;
            HG(j, j) = c * a + sgv * bb;
            HG(j + 1, j) = 0.0;
            double t = c * g[j] + sgv * g[j + 1];
            g[j + 1] = -sgv * g[j] + c * g[j + 1];
            g[j] = t;
            j++; total++;
            resid = fabs(g[j]);
            if (resid <= abs_tol) { outcome = 0; break; }
            if (total >= maxiter) { outcome = 1; break; }
            if (hj1 > 1e-14 * hmax) {
                for (int64_t k = 0; k < n; k++) V[(size_t)j * n + k] = w[k] * (1.0 / hj1);
            } else { outcome = 2; break; }
        }
        for (int i = j - 1; i >= 0; i--) {
            double s = g[i];
            for (int k = i + 1; k < j; k++) s -= HG(i, k) * y[k];
            double dg = HG(i, i);
            y[i] = fabs(dg) < 1e-14 * (1.0 + fabs(s)) ? 0.0 : s / dg;
        }
        for (int k = 0; k < j; k++)
            for (int64_t i = 0; i < n; i++) x[i] += y[k] * Z[(size_t)k * n + i];
        if (outcome == 0) { out.converged = 1; out.iterations = total; out.res = resid; break; }
        if (outcome == 1) { out.converged = 0; out.iterations = total; out.res = resid; break; }
        if (outcome == 2) {
            A(ctx, x, r);
            for (int64_t i = 0; i < n; i++) r[i] = b[i] - r[i];
            double res = vnorm(r, n);
            out.converged = res <= abs_tol; out.iterations = total; out.res = res; break;
        }
    }
#undef HG
    free(r); free(w); free(V); free(Z); free(H); free(cs); free(sn); free(g); free(y);
    return out;
}

/* ------------------------------------------------------------------------- */
/* LSMR: schwarz-precond/src/solve/lsmr.rs, lsmr/bidiag.rs, lsmr/recurrence.rs */
/* (Fong & Saunders 2011, Algorithm 2.8; Modified Golub-Kahan with M ~ A'A)   */
/* ------------------------------------------------------------------------- */

/* WeightedDesignOperator, within/src/operator.rs:111-190: A = W^(1/2) D. */
typedef struct { work_t *w; const double *sw; double *tmp; } rect_t;
static void rect_apply(rect_t *R, const double *x, double *y) {
    const design_t *d = &R->w->s->d;
    design_matvec_d(d, x, y);
    if (R->sw) for (int64_t i = 0; i < d->n; i++) y[i] *= R->sw[i];
}
static void rect_adjoint(rect_t *R, const double *u, double *x) {
    const design_t *d = &R->w->s->d;
    if (R->sw) {
        for (int64_t i = 0; i < d->n; i++) R->tmp[i] = R->sw[i] * u[i];
        design_rmatvec(d, R->tmp, x, 0);
    } else {
        design_rmatvec(d, u, x, 0);
    }
}

/* Givens::new (recurrence.rs:24-31). */
typedef struct { double c, s, r; } givens_t;
static givens_t givens(double a, double b) {
    givens_t g; g.r = hypot(a, b);
    if (g.r > 0.0) { g.c = a / g.r; g.s = b / g.r; } else { g.c = 1.0; g.s = 0.0; }
    return g;
}
typedef struct { double rho, rho_bar, theta_new, theta_bar, zeta; } rot_t;

/* Ring of past v (and p~ = M v) vectors for windowed MGS (bidiag.rs:86-260): capacity
 * min(local_size, rows, cols), swept oldest first. */
typedef struct { double *v, *p; int64_t n; int cap, next, count; } ring_t;
static void ring_sweep(const ring_t *g, double *v, double *p) {
    int start = g->count < g->cap ? 0 : g->next;
    for (int i = 0; i < g->count; i++) {
        int idx = (start + i) % g->cap;
        const double *vj = g->v + (size_t)idx * g->n;
        if (p) {  /* M-weighted: c = <v, p_j>, v -= c v_j, p -= c p_j */
            const double *pj = g->p + (size_t)idx * g->n;
            double c = vdot(v, pj, g->n);
            for (int64_t a = 0; a < g->n; a++) { v[a] += -c * vj[a]; p[a] += -c * pj[a]; }
        } else {
            double c = vdot(v, vj, g->n);
            for (int64_t a = 0; a < g->n; a++) v[a] += -c * vj[a];
        }
    }
}
static void ring_push(ring_t *g, const double *v, const double *p, double pscale) {
    memcpy(g->v + (size_t)g->next * g->n, v, sizeof(double) * (size_t)g->n);
    if (p) for (int64_t a = 0; a < g->n; a++) g->p[(size_t)g->next * g->n + a] = p[a] * pscale;
    g->next = (g->next + 1) % g->cap;
    if (g->count < g->cap) g->count++;
}

/* A rectangular operator (rows x cols) and an optional preconditioner M^-1 (cols). */
typedef struct {
    void *ctx; int64_t rows, cols;
    void (*apply)(void *, const double *, double *);
    void (*adjoint)(void *, const double *, double *);
    void (*minv)(void *, const double *, double *);   /* NULL: no preconditioner */
} lsmr_op_t;
static void cb_rect_apply(void *c, const double *x, double *y) { rect_apply((rect_t *)c, x, y); }
static void cb_rect_adjoint(void *c, const double *u, double *x) { rect_adjoint((rect_t *)c, u, x); }
static void cb_rect_minv(void *c, const double *r, double *z) { op_precond(((rect_t *)c)->w, r, z); }

/* mlsmr (lsmr.rs:122-262): min ||b - A x||; with a preconditioner M ~ A'A, the Modified
 * Golub-Kahan process (one M^-1 per iteration).  Returns x, converged, iterations;
 * *stop_out (if given): 0 zero rhs, 1 A'b = 0, 2 residual tolerance, 3 normal-equation
 * tolerance, 4 breakdown, 5 max iterations (LsmrStopReason, lsmr.rs:86-100). */
static kres_t krylov_lsmr_op(const lsmr_op_t *A, const double *b, double tol, int maxiter, int local_size,
                             int *stop_out) {
    const int64_t no = A->rows, nd = A->cols;
    const int precond = A->minv != NULL;
    int stop_reason = 0;
    kres_t out; out.x = xcalloc((size_t)nd + 1, sizeof(double));
    out.converged = 1; out.iterations = 0; out.res = 0.0;
    double bnorm = vnorm(b, no);
    if (bnorm == 0.0) { if (stop_out) *stop_out = 0; return out; }   /* zero_rhs_result */
    double *u = xcalloc((size_t)no + 1, sizeof(double)), *av = xcalloc((size_t)no + 1, sizeof(double));
    double *v = xcalloc((size_t)nd + 1, sizeof(double)), *atu = xcalloc((size_t)nd + 1, sizeof(double));
    double *pt = xcalloc((size_t)nd + 1, sizeof(double)), *h = xcalloc((size_t)nd + 1, sizeof(double));
    double *hb = xcalloc((size_t)nd + 1, sizeof(double)), *x = out.x;
    ring_t ring; ring.n = nd; ring.next = 0; ring.count = 0;
    ring.cap = local_size; if (ring.cap > no) ring.cap = (int)no; if (ring.cap > nd) ring.cap = (int)nd;
    if (ring.cap < 0) ring.cap = 0;
    ring.v = ring.cap ? xcalloc((size_t)ring.cap * (size_t)nd, sizeof(double)) : NULL;
    ring.p = (ring.cap && precond) ? xcalloc((size_t)ring.cap * (size_t)nd, sizeof(double)) : NULL;
    /* init (bidiag.rs: GolubKahan::init, ModifiedGolubKahan::init) */
    double beta = sqrt(vdot(b, b, no)), alpha, beta_prev_inv = 1.0;
    if (beta > 0.0) for (int64_t i = 0; i < no; i++) u[i] = b[i] * (1.0 / beta);
    if (!precond) {
        A->adjoint(A->ctx, u, v);
        alpha = sqrt(vdot(v, v, nd));
        if (alpha > 0.0) for (int64_t j = 0; j < nd; j++) v[j] *= 1.0 / alpha;
        if (ring.cap) ring_push(&ring, v, NULL, 0.0);
    } else {
        A->adjoint(A->ctx, u, pt);
        A->minv(A->ctx, pt, v);
        double vp = vdot(v, pt, nd);
        alpha = vp > 0.0 ? sqrt(vp) : 0.0;
        if (alpha > 0.0) for (int64_t j = 0; j < nd; j++) v[j] *= 1.0 / alpha;
        if (ring.cap) ring_push(&ring, v, pt, alpha > 0.0 ? 1.0 / alpha : 0.0);
    }
    if (alpha == 0.0) { out.res = bnorm; stop_reason = 1; goto done; }   /* A'b = 0 */
    /* lsmr_from_bidiag (lsmr.rs:204-262) */
    double alpha_bar = alpha, phi_bar = beta, c_bar = 1.0, s_bar = 0.0, zeta_bar = alpha * beta;
    double abs_tol = tol * bnorm, a2 = alpha * alpha;
    rot_t prev = {1.0, 1.0, 0.0, 0.0, 0.0};
    memcpy(h, v, sizeof(double) * (size_t)nd);
    out.converged = 0; out.iterations = maxiter; stop_reason = 5;
    for (int itn = 1; itn <= maxiter; itn++) {
        /* one bidiagonalization step: (alpha, beta) and the normalized v */
        double sa, sb;
        if (!precond) {
            A->apply(A->ctx, v, av);
            double bsq = 0.0;
            for (int64_t i = 0; i < no; i++) { u[i] = av[i] + (-alpha) * u[i]; bsq += u[i] * u[i]; }
            sb = sqrt(bsq);
            if (sb == 0.0) {
                memset(v, 0, sizeof(double) * (size_t)nd); alpha = 0.0; sa = 0.0;
            } else {
                for (int64_t i = 0; i < no; i++) u[i] *= 1.0 / sb;
                A->adjoint(A->ctx, u, atu);
                double asq = 0.0;
                for (int64_t j = 0; j < nd; j++) { v[j] = atu[j] + (-sb) * v[j]; asq += v[j] * v[j]; }
                if (ring.cap) { ring_sweep(&ring, v, NULL); asq = vdot(v, v, nd); }
                sa = sqrt(asq);
                if (sa > 0.0) for (int64_t j = 0; j < nd; j++) v[j] *= 1.0 / sa;
                if (ring.cap) ring_push(&ring, v, NULL, 0.0);
                alpha = sa;
            }
        } else {
            double scale = -(alpha * beta_prev_inv);
            A->apply(A->ctx, v, av);
            double bsq = 0.0;
            for (int64_t i = 0; i < no; i++) { u[i] = av[i] + scale * u[i]; bsq += u[i] * u[i]; }
            sb = sqrt(bsq);
            if (sb == 0.0) {
                memset(v, 0, sizeof(double) * (size_t)nd); memset(pt, 0, sizeof(double) * (size_t)nd);
                alpha = 0.0; beta_prev_inv = 0.0; sa = 0.0;
            } else {
                double binv = 1.0 / sb, pc = sb / alpha;
                A->adjoint(A->ctx, u, atu);
                for (int64_t j = 0; j < nd; j++) pt[j] = binv * atu[j] + (-pc) * pt[j];
                A->minv(A->ctx, pt, v);
                if (ring.cap) ring_sweep(&ring, v, pt);
                double vp = vdot(v, pt, nd);
                sa = vp > 0.0 ? sqrt(vp) : 0.0;
                if (sa > 0.0) for (int64_t j = 0; j < nd; j++) v[j] *= 1.0 / sa;
                if (ring.cap) ring_push(&ring, v, pt, sa > 0.0 ? 1.0 / sa : 0.0);
                alpha = sa; beta_prev_inv = binv;
            }
        }
        a2 += sa * sa + sb * sb;                                     /* ConvergenceState::observe */
        /* LsmrRecurrenceState::step (recurrence.rs:92-140) */
        givens_t ph = givens(alpha_bar, sb);
        double theta_new = ph.s * sa, alpha_bar_new = -ph.c * sa, phi_bar_new = ph.s * phi_bar;
        double theta_bar = s_bar * ph.r;
        givens_t pb = givens(c_bar * ph.r, theta_new);
        double zeta = pb.c * zeta_bar, zeta_bar_new = -pb.s * zeta_bar;
        alpha_bar = alpha_bar_new; phi_bar = phi_bar_new; c_bar = pb.c; s_bar = pb.s; zeta_bar = zeta_bar_new;
        rot_t cur = {ph.r, pb.r, theta_new, theta_bar, zeta};
        /* SolutionState::update (recurrence.rs:186-240) */
        double dx = cur.rho * cur.rho_bar, dh = prev.rho * prev.rho_bar;
        double t_x = fabs(dx) > DBL_EPSILON ? cur.zeta / dx : 0.0;
        double t_hbar = fabs(dh) > DBL_EPSILON ? cur.theta_bar * cur.rho / dh : 0.0;
        double t_h = fabs(cur.rho) > DBL_EPSILON ? cur.theta_new / cur.rho : 0.0;
        for (int64_t j = 0; j < nd; j++) {
            double h_old = h[j], hbj = h_old - t_hbar * hb[j];
            hb[j] = hbj; x[j] += t_x * hbj; h[j] = v[j] - t_h * h_old;
        }
        /* ConvergenceState::check (recurrence.rs:272-284) */
        double residual = fabs(phi_bar);
        int stop = residual <= abs_tol;
        if (!stop) {
            double an = fmax(sqrt(a2), DBL_MIN), normar = fabs(zeta_bar);
            stop = normar / (an * fmax(residual, DBL_MIN)) <= tol;
        }
        out.res = residual;
        if (stop || sa == 0.0) {
            out.converged = 1; out.iterations = itn;
            stop_reason = stop ? (residual <= abs_tol ? 2 : 3) : 4;
            break;
        }
        prev = cur;
    }
done:
    if (stop_out) *stop_out = stop_reason;
    free(u); free(av); free(v); free(atu); free(pt); free(h); free(hb); free(ring.v); free(ring.p);
    return out;
}

/* The design operator A = W^(1/2) D with the solver's preconditioner. */
static kres_t krylov_lsmr(rect_t *R, int precond, const double *b, double tol, int maxiter, int local_size) {
    lsmr_op_t A = {R, R->w->s->d.n, R->w->s->d.ndofs, cb_rect_apply, cb_rect_adjoint, precond ? cb_rect_minv : NULL};
    return krylov_lsmr_op(&A, b, tol, maxiter, local_size, NULL);
}

/* Dense operators for the known-answer tests of the LSMR recurrences: A row-major
 * rows x cols, minv (optional) row-major cols x cols. */
typedef struct { const double *a, *minv; int64_t rows, cols; } dense_op_t;
static void dense_apply(void *c, const double *x, double *y) {
    const dense_op_t *d = (const dense_op_t *)c;
    for (int64_t i = 0; i < d->rows; i++) {
        double t = 0.0;
        for (int64_t j = 0; j < d->cols; j++) t += d->a[i * d->cols + j] * x[j];
        y[i] = t;
    }
}
static void dense_adjoint(void *c, const double *u, double *x) {
    const dense_op_t *d = (const dense_op_t *)c;
    for (int64_t j = 0; j < d->cols; j++) {
        double t = 0.0;
        for (int64_t i = 0; i < d->rows; i++) t += d->a[i * d->cols + j] * u[i];
        x[j] = t;
    }
}
static void dense_minv(void *c, const double *r, double *z) {
    const dense_op_t *d = (const dense_op_t *)c;
    for (int64_t i = 0; i < d->cols; i++) {
        double t = 0.0;
        for (int64_t j = 0; j < d->cols; j++) t += d->minv[i * d->cols + j] * r[j];
        z[i] = t;
    }
}
int oracle_lsmr_dense(const double *a, int64_t rows, int64_t cols, const double *minv, const double *b, double tol,
                      int32_t maxiter, int32_t local_size, double *x, int32_t *converged, int32_t *iterations,
                      int32_t *stop_reason) {
    dense_op_t d = {a, minv, rows, cols};
    lsmr_op_t A = {&d, rows, cols, dense_apply, dense_adjoint, minv ? dense_minv : NULL};
    int stop = 0;
    kres_t r = krylov_lsmr_op(&A, b, tol, maxiter, local_size, &stop);
    memcpy(x, r.x, sizeof(double) * (size_t)cols);
    *converged = r.converged; *iterations = r.iterations; *stop_reason = stop;
    free(r.x);
    return 0;
}

static void cb_gramian(void *ctx, const double *x, double *y) { op_gramian((work_t *)ctx, x, y); }
static void cb_precond(void *ctx, const double *x, double *y) { op_precond((work_t *)ctx, x, y); }

static kres_t krylov_solve(work_t *w, const double *rhs, double tol) {
    const oracle_solver *s = w->s;
    if (s->p.krylov == 1)
        return krylov_gmres(s->d.ndofs, cb_gramian, cb_precond, w, rhs, tol, s->p.maxiter, s->p.gmres_restart);
    return krylov_cg(s->d.ndofs, cb_gramian, cb_precond, w, rhs, tol, s->p.maxiter);
}

/* Solver::solve + iterative_refinement, within/src/solver.rs:209-238, 296-347. */
static void solve_one(work_t *w, const double *y, double *x_out, double *dem, int32_t *conv,
                      int32_t *iters, double *fres) {
    const oracle_solver *s = w->s;
    int64_t m = s->d.ndofs, n = s->d.n;
    double *rhs = xcalloc((size_t)m + 1, sizeof(double));
    design_rmatvec(&s->d, y, rhs, 1);
    double rn = vnorm(rhs, m); if (rn < 1e-15) rn = 1e-15;
    if (s->p.krylov == 2) {
        /* Solver::solve, LSMR branch (solver.rs:162-203): b = W^(1/2) y, mlsmr, then the
         * demeaning and the normal-equation residual; no refinement */
        rect_t R; R.w = w; R.sw = NULL; R.tmp = NULL;
        double *sw = NULL, *b = xcalloc((size_t)n + 1, sizeof(double));
        if (s->d.w) {
            sw = xcalloc((size_t)n + 1, sizeof(double));
            for (int64_t i = 0; i < n; i++) sw[i] = sqrt(s->d.w[i]);
            R.sw = sw; R.tmp = xcalloc((size_t)n + 1, sizeof(double));
        }
        for (int64_t i = 0; i < n; i++) b[i] = sw ? sw[i] * y[i] : y[i];
        kres_t r = krylov_lsmr(&R, s->p.precond_kind != 0, b, s->p.tol, s->p.maxiter, s->p.lsmr_local_size);
        design_matvec_d(&s->d, r.x, dem);
        for (int64_t i = 0; i < n; i++) dem[i] = y[i] - dem[i];
        double *corr = xcalloc((size_t)m + 1, sizeof(double));
        design_rmatvec(&s->d, dem, corr, 1);
        *fres = vnorm(corr, m) / rn;
        *conv = r.converged; *iters = r.iterations;
        memcpy(x_out, r.x, sizeof(double) * (size_t)m);
        free(r.x); free(corr); free(b); free(sw); free(R.tmp); free(rhs);
        return;
    }
    double abs_tol = s->p.tol * rn;
    kres_t k0 = krylov_solve(w, rhs, s->p.tol);
    double *x = k0.x;
    int iterations = k0.iterations, converged = k0.converged;
    double *corr = xcalloc((size_t)m + 1, sizeof(double));
    for (int it = 0; it < s->p.max_refinements; it++) {
        design_matvec_d(&s->d, x, dem);
        for (int64_t i = 0; i < n; i++) dem[i] = y[i] - dem[i];
        design_rmatvec(&s->d, dem, corr, 1);
        double cn = vnorm(corr, m);
        if (cn <= abs_tol) break;
        double ct = abs_tol / cn; if (ct > 1.0) ct = 1.0;
        kres_t kc = krylov_solve(w, corr, ct);
        for (int64_t j = 0; j < m; j++) x[j] += kc.x[j];
        iterations += kc.iterations; converged = kc.converged;
        free(kc.x);
    }
    design_matvec_d(&s->d, x, dem);
    for (int64_t i = 0; i < n; i++) dem[i] = y[i] - dem[i];
    design_rmatvec(&s->d, dem, corr, 1);
    *fres = vnorm(corr, m) / rn;
    *conv = converged; *iters = iterations;
    memcpy(x_out, x, sizeof(double) * (size_t)m);
    free(x); free(corr); free(rhs);
}

/* ------------------------------------------------------------------------- */
/* Public entry points                                                       */
/* ------------------------------------------------------------------------- */

int oracle_solver_new(const uint32_t *codes, int64_t n_obs, int32_t n_factors, int64_t row_stride,
                      int64_t col_stride, const double *weights, const oracle_params *params,
                      oracle_solver **out, char *err, int errlen) {
    *out = NULL;
    if (n_obs <= 0) { set_err(err, errlen, "no observations provided"); return 1; }
    if (n_factors <= 0) { set_err(err, errlen, "no factors provided"); return 1; }
    oracle_solver *s = xcalloc(1, sizeof(oracle_solver));
    s->p = *params;
    s->d.n = n_obs; s->d.Q = n_factors;
    s->d.codes = xcalloc((size_t)n_obs * (size_t)n_factors, sizeof(uint32_t));
    for (int q = 0; q < n_factors; q++)
        for (int64_t i = 0; i < n_obs; i++) s->d.codes[(size_t)q * n_obs + i] = codes[i * row_stride + q * col_stride];
    if (weights) {
        s->d.w = xcalloc((size_t)n_obs, sizeof(double));
        memcpy(s->d.w, weights, sizeof(double) * (size_t)n_obs);
    }
    design_init(&s->d);
    if (s->p.precond_kind != 0) {
        if (build_domains(s, err, errlen)) { oracle_solver_free(s); return 5; }
    }
    if (s->p.precond_kind == 2) build_explicit_gramian(s);
    *out = s;
    return 0;
}

void oracle_solver_free(oracle_solver *s) {
    if (!s) return;
    for (int32_t i = 0; i < s->nsub; i++) {
        subdomain_t *sd = &s->sub[i];
        free(sd->gidx); free(sd->pou); crosstab_free(&sd->ct); free(sd->inv_diag); free(sd->L); acf_free(&sd->ac);
    }
    free(s->sub); free(s->d.codes); free(s->d.w); free(s->d.nlev); free(s->d.off);
    free(s->g_ptr); free(s->g_idx); free(s->g_val);
    free(s);
}

int64_t oracle_n_dofs(const oracle_solver *s) { return s->d.ndofs; }
int64_t oracle_n_obs(const oracle_solver *s) { return s->d.n; }
void oracle_factor_meta(const oracle_solver *s, int64_t *n_levels, int64_t *offsets) {
    for (int q = 0; q < s->d.Q; q++) { n_levels[q] = s->d.nlev[q]; offsets[q] = s->d.off[q]; }
}

int oracle_solve(oracle_solver *s, const double *y, double *x, double *demeaned, int32_t *converged,
                 int32_t *iterations, double *final_residual, char *err, int errlen) {
    (void)err; (void)errlen;
    work_t w; work_init(&w, s);
    solve_one(&w, y, x, demeaned, converged, iterations, final_residual);
    work_free(&w);
    return 0;
}

int oracle_solve_batch(oracle_solver *s, const double *ys, int32_t k, double *x, double *demeaned,
                       int32_t *converged, int32_t *iterations, double *final_residual,
                       int32_t n_threads, char *err, int errlen) {
    (void)err; (void)errlen;
    int64_t n = s->d.n, m = s->d.ndofs;
#ifdef _OPENMP
    if (n_threads < 1) n_threads = 1;
#pragma omp parallel for schedule(dynamic, 1) num_threads(n_threads)
#endif
    for (int32_t c = 0; c < k; c++) {
        work_t w; work_init(&w, s);
        solve_one(&w, ys + (size_t)c * n, x + (size_t)c * m, demeaned + (size_t)c * n,
                  converged + c, iterations + c, final_residual + c);
        work_free(&w);
    }
    (void)n_threads;
    return 0;
}

void oracle_matvec_d(const oracle_solver *s, const double *x, double *y) { design_matvec_d(&s->d, x, y); }
void oracle_rmatvec_wdt(const oracle_solver *s, const double *r, double *x) { design_rmatvec(&s->d, r, x, 1); }
void oracle_rmatvec_dt(const oracle_solver *s, const double *r, double *x) { design_rmatvec(&s->d, r, x, 0); }
void oracle_gramian_diagonal(const oracle_solver *s, double *diag) { design_diag(&s->d, diag); }
void oracle_apply_gramian(const oracle_solver *s, const double *x, double *y) {
    work_t w; work_init(&w, s); op_gramian(&w, x, y); work_free(&w);
}
int oracle_apply_precond(oracle_solver *s, const double *r, double *z) {
    work_t w; work_init(&w, s); op_precond(&w, r, z); work_free(&w); return 0;
}

int32_t oracle_n_subdomains(const oracle_solver *s) { return s->nsub; }
void oracle_subdomain_info(const oracle_solver *s, int32_t i, int64_t *info) {
    const subdomain_t *sd = &s->sub[i];
    info[0] = sd->q; info[1] = sd->r; info[2] = sd->nidx; info[3] = sd->ct.c.nrows; info[4] = sd->ct.c.ncols;
    info[5] = sd->elim_q; info[6] = sd->kind; info[7] = sd->n_red;
}
void oracle_subdomain_indices(const oracle_solver *s, int32_t i, uint32_t *gidx, double *pou) {
    const subdomain_t *sd = &s->sub[i];
    memcpy(gidx, sd->gidx, sizeof(uint32_t) * (size_t)sd->nidx);
    for (int32_t a = 0; a < sd->nidx; a++) pou[a] = sd->pou ? sd->pou[a] : 1.0;
}
void oracle_ac_sizes(const oracle_solver *s, int32_t i, int64_t *sizes) {
    const subdomain_t *sd = &s->sub[i];
    for (int a = 0; a < 5; a++) sizes[a] = 0;
    if (sd->kind != 1) return;
    sizes[0] = sd->ac.n; sizes[1] = sd->ac.nlev; sizes[2] = sd->ac.col_ptr[sd->ac.ncol];
    sizes[3] = sd->ac.ncol; sizes[4] = sd->ac.ncore;
}
void oracle_ac_arrays(const oracle_solver *s, int32_t i, int32_t *level_ptr, int32_t *col_vertex,
                      double *col_diag, int32_t *col_ptr, int32_t *col_idx, double *col_coef,
                      int32_t *core_vertex, double *core_z) {
    const acf_t *f = &s->sub[i].ac;
    memcpy(level_ptr, f->level_ptr, sizeof(int32_t) * (size_t)(f->nlev + 1));
    memcpy(col_vertex, f->col_vertex, sizeof(int32_t) * (size_t)f->ncol);
    memcpy(col_diag, f->col_diag, sizeof(double) * (size_t)f->ncol);
    memcpy(col_ptr, f->col_ptr, sizeof(int32_t) * (size_t)(f->ncol + 1));
    memcpy(col_idx, f->col_idx, sizeof(int32_t) * (size_t)f->col_ptr[f->ncol]);
    memcpy(col_coef, f->col_coef, sizeof(double) * (size_t)f->col_ptr[f->ncol]);
    memcpy(core_vertex, f->core_vertex, sizeof(int32_t) * (size_t)f->ncore);
    memcpy(core_z, f->core_z, sizeof(double) * (size_t)f->ncore * (size_t)f->ncore);
}
int64_t oracle_crosstab_nnz(const oracle_solver *s, int32_t i) { return csr_nnz(&s->sub[i].ct.c); }
void oracle_crosstab(const oracle_solver *s, int32_t i, uint32_t *indptr, uint32_t *indices, double *data,
                     double *diag_q, double *diag_r) {
    const crosstab_t *x = &s->sub[i].ct;
    int64_t nnz = csr_nnz(&x->c);
    memcpy(indptr, x->c.indptr, sizeof(uint32_t) * ((size_t)x->c.nrows + 1));
    memcpy(indices, x->c.indices, sizeof(uint32_t) * (size_t)nnz);
    memcpy(data, x->c.data, sizeof(double) * (size_t)nnz);
    memcpy(diag_q, x->dq, sizeof(double) * (size_t)x->c.nrows);
    memcpy(diag_r, x->dr, sizeof(double) * (size_t)x->c.ncols);
}

/* dense helpers for the CG/GMRES known-answer tests (schwarz-precond/src/solve/cg.rs:150-330) */
typedef struct { int32_t n; const double *a; const double *m; } dense_ctx;
static void cb_dense_a(void *ctx, const double *x, double *y) {
    dense_ctx *c = ctx;
    for (int32_t i = 0; i < c->n; i++) { double s = 0.0; for (int32_t j = 0; j < c->n; j++) s += c->a[(size_t)i * c->n + j] * x[j]; y[i] = s; }
}
static void cb_dense_m(void *ctx, const double *x, double *y) {
    dense_ctx *c = ctx;
    for (int32_t i = 0; i < c->n; i++) y[i] = c->m ? c->m[i] * x[i] : x[i];
}
int oracle_dense_cg(int32_t n, const double *a, const double *m_inv_diag, const double *b, double tol,
                    int32_t maxiter, double *x, int32_t *converged, int32_t *iterations, double *residual_norm) {
    dense_ctx c = { n, a, m_inv_diag };
    kres_t r = krylov_cg(n, cb_dense_a, cb_dense_m, &c, b, tol, maxiter);
    memcpy(x, r.x, sizeof(double) * (size_t)n);
    *converged = r.converged; *iterations = r.iterations; *residual_norm = r.res;
    free(r.x);
    return 0;
}
int oracle_dense_gmres(int32_t n, const double *a, const double *m_inv_diag, const double *b, double tol,
                       int32_t maxiter, int32_t restart, double *x, int32_t *converged, int32_t *iterations,
                       double *residual_norm) {
    dense_ctx c = { n, a, m_inv_diag };
    kres_t r = krylov_gmres(n, cb_dense_a, cb_dense_m, &c, b, tol, maxiter, restart);
    memcpy(x, r.x, sizeof(double) * (size_t)n);
    *converged = r.converged; *iterations = r.iterations; *residual_norm = r.res;
    free(r.x);
    return 0;
}
