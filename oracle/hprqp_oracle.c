/*
 * hprqp_oracle.c -- serial CPU restatement of the HPR-QP algorithm.
 *
 * TEST INFRASTRUCTURE ONLY (see hprqp_oracle.h).  Every routine names the
 * reference file:line it restates.  Paths are relative to the reference
 * project (PolyU-IOR/HPR-QP-C).  Where the reference's CPU backend and CUDA
 * backend disagree, the difference is selected by `mode` and commented with
 * [GPU]/[CPU] tags.
 */
#define _POSIX_C_SOURCE 200809L
#include "hprqp_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* ------------------------------------------------------------------------ */
/* small dense helpers (src/shared/vector.c:24-55)                           */
/* ------------------------------------------------------------------------ */

static double o_dot(const double *a, const double *b, size_t n)
{
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

static double o_norm2(const double *a, size_t n) { return sqrt(o_dot(a, a, n)); }

static double o_norm_inf(const double *a, size_t n)
{
    double m = 0.0;
    for (size_t i = 0; i < n; ++i) {
        double v = fabs(a[i]);
        if (v > m) m = v;
    }
    return m;
}

static double o_clamp(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

static double *o_zeros(size_t n) { return (double *)calloc(n ? n : 1, sizeof(double)); }

static double o_now(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ------------------------------------------------------------------------ */
/* CSR                                                                        */
/* ------------------------------------------------------------------------ */

typedef struct OCsr {
    size_t nrow, ncol, nnz;
    size_t *rp;
    size_t *ci;
    double *v;
} OCsr;

static void csr_free(OCsr *a)
{
    free(a->rp);
    free(a->ci);
    free(a->v);
    memset(a, 0, sizeof(*a));
}

static int csr_alloc(OCsr *a, size_t nrow, size_t ncol, size_t nnz)
{
    a->nrow = nrow;
    a->ncol = ncol;
    a->nnz = nnz;
    a->rp = (size_t *)calloc(nrow + 1, sizeof(size_t));
    a->ci = (size_t *)calloc(nnz ? nnz : 1, sizeof(size_t));
    a->v = (double *)calloc(nnz ? nnz : 1, sizeof(double));
    return (a->rp && a->ci && a->v) ? ORACLE_OK : ORACLE_ALLOC;
}

static int csr_copy(OCsr *d, const OCsr *s)
{
    if (csr_alloc(d, s->nrow, s->ncol, s->nnz) != ORACLE_OK) return ORACLE_ALLOC;
    memcpy(d->rp, s->rp, (s->nrow + 1) * sizeof(size_t));
    memcpy(d->ci, s->ci, s->nnz * sizeof(size_t));
    memcpy(d->v, s->v, s->nnz * sizeof(double));
    return ORACLE_OK;
}

/* Counting-sort transpose, stable in source row order.
 * Restates matrix_csr_transpose, src/shared/sparse.c:81-125. */
static int csr_transpose(OCsr *t, const OCsr *a)
{
    if (csr_alloc(t, a->ncol, a->nrow, a->nnz) != ORACLE_OK) return ORACLE_ALLOC;
    for (size_t k = 0; k < a->nnz; ++k) t->rp[a->ci[k] + 1] += 1;
    for (size_t r = 0; r < t->nrow; ++r) t->rp[r + 1] += t->rp[r];
    size_t *next = (size_t *)malloc((t->nrow ? t->nrow : 1) * sizeof(size_t));
    if (!next) return ORACLE_ALLOC;
    memcpy(next, t->rp, t->nrow * sizeof(size_t));
    for (size_t r = 0; r < a->nrow; ++r)
        for (size_t k = a->rp[r]; k < a->rp[r + 1]; ++k) {
            size_t pos = next[a->ci[k]]++;
            t->ci[pos] = r;
            t->v[pos] = a->v[k];
        }
    free(next);
    return ORACLE_OK;
}

/* Row-order serial SpMV: src/shared/sparse.c:127-145. */
void oracle_csr_matvec(size_t nrow, const size_t *rp, const size_t *ci, const double *v,
                       const double *x, double *y)
{
    for (size_t r = 0; r < nrow; ++r) {
        double s = 0.0;
        for (size_t k = rp[r]; k < rp[r + 1]; ++k) s += v[k] * x[ci[k]];
        y[r] = s;
    }
}

static void o_spmv(const OCsr *a, const double *x, double *y)
{
    oracle_csr_matvec(a->nrow, a->rp, a->ci, a->v, x, y);
}

/* ------------------------------------------------------------------------ */
/* model build + preprocess (src/shared/build.c:137-400, 504-621)            */
/* ------------------------------------------------------------------------ */

struct OracleModel {
    size_t n, m;
    OCsr Q, A, AT;
    double *c, *AL, *AU, *l, *u;
    double obj_constant;
};

typedef struct OEntry {
    size_t row, col, seq;
    double val;
} OEntry;

static int entry_cmp(const void *pa, const void *pb)
{
    const OEntry *a = (const OEntry *)pa, *b = (const OEntry *)pb;
    if (a->row != b->row) return a->row < b->row ? -1 : 1;
    if (a->col != b->col) return a->col < b->col ? -1 : 1;
    if (a->seq != b->seq) return a->seq < b->seq ? -1 : 1; /* deterministic ties */
    return 0;
}

/* Q <- factor*(Q + Q'), dropping |entry| <= tol before and after merging.
 * Restates symmetrize_q_matrix / build_csr_from_entries,
 * src/shared/build.c:163-252. */
static int symmetrize_q(OCsr *dst, const OCsr *src, double factor, double tol)
{
    size_t ne = 2 * src->nnz;
    OEntry *e = (OEntry *)malloc((ne ? ne : 1) * sizeof(OEntry));
    if (!e) return ORACLE_ALLOC;
    size_t k = 0;
    for (size_t r = 0; r < src->nrow; ++r)
        for (size_t p = src->rp[r]; p < src->rp[r + 1]; ++p) {
            double v = factor * src->v[p];
            e[k] = (OEntry){r, src->ci[p], k, v};
            ++k;
            e[k] = (OEntry){src->ci[p], r, k, v};
            ++k;
        }
    qsort(e, ne, sizeof(OEntry), entry_cmp);
    size_t u = 0;
    for (size_t i = 0; i < ne; ++i) {
        if (fabs(e[i].val) <= tol) continue;
        if (u > 0 && e[i].row == e[u - 1].row && e[i].col == e[u - 1].col)
            e[u - 1].val += e[i].val;
        else
            e[u++] = e[i];
    }
    size_t kept = 0;
    for (size_t i = 0; i < u; ++i) {
        if (fabs(e[i].val) <= tol) e[i].val = 0.0;
        if (e[i].val != 0.0) e[kept++] = e[i];
    }
    if (csr_alloc(dst, src->nrow, src->ncol, kept) != ORACLE_OK) {
        free(e);
        return ORACLE_ALLOC;
    }
    for (size_t i = 0; i < kept; ++i) dst->rp[e[i].row + 1] += 1;
    for (size_t r = 0; r < src->nrow; ++r) dst->rp[r + 1] += dst->rp[r];
    for (size_t i = 0; i < kept; ++i) {
        dst->ci[i] = e[i].col;
        dst->v[i] = e[i].val;
    }
    free(e);
    return ORACLE_OK;
}

void oracle_model_free(OracleModel *m)
{
    if (!m) return;
    csr_free(&m->Q);
    csr_free(&m->A);
    csr_free(&m->AT);
    free(m->c);
    free(m->AL);
    free(m->AU);
    free(m->l);
    free(m->u);
    free(m);
}

static double *dup_vec(const double *s, size_t n)
{
    double *d = (double *)malloc((n ? n : 1) * sizeof(double));
    if (d && n) memcpy(d, s, n * sizeof(double));
    return d;
}

static int csr_view_valid(size_t nrow, size_t ncol, size_t nnz, const size_t *rp, const size_t *ci)
{
    if (nrow > 0 && rp == NULL) return 0;
    if (nnz > 0 && ci == NULL) return 0;
    if (rp && (rp[0] != 0 || rp[nrow] != nnz)) return 0;
    for (size_t r = 0; rp && r < nrow; ++r)
        if (rp[r + 1] < rp[r]) return 0;
    for (size_t k = 0; k < nnz; ++k)
        if (ci[k] >= ncol) return 0;
    return 1;
}

int oracle_build(size_t n, size_t q_nnz, const size_t *q_rp, const size_t *q_ci, const double *q_v,
                 size_t m, size_t a_nnz, const size_t *a_rp, const size_t *a_ci, const double *a_v,
                 const double *c, const double *AL, const double *AU, const double *l,
                 const double *u, double obj_constant, OracleModel **out)
{
    /* validation: build.c:513-531 and preprocess_model build.c:339-379 */
    if (!out || !c || !l || !u) return ORACLE_INVALID;
    *out = NULL;
    if (!csr_view_valid(n, n, q_nnz, q_rp, q_ci) || !csr_view_valid(m, n, a_nnz, a_rp, a_ci))
        return ORACLE_INVALID;
    if (m > 0 && (!AL || !AU)) return ORACLE_INVALID;
    for (size_t k = 0; k < q_nnz; ++k)
        if (!isfinite(q_v[k])) return ORACLE_INVALID;
    for (size_t k = 0; k < a_nnz; ++k)
        if (!isfinite(a_v[k])) return ORACLE_INVALID;
    for (size_t i = 0; i < n; ++i) {
        if (!isfinite(c[i]) || isnan(l[i]) || isnan(u[i]) || l[i] > u[i]) return ORACLE_INVALID;
    }
    for (size_t i = 0; i < m; ++i)
        if (isnan(AL[i]) || isnan(AU[i]) || AL[i] > AU[i]) return ORACLE_INVALID;

    OracleModel *mo = (OracleModel *)calloc(1, sizeof(OracleModel));
    if (!mo) return ORACLE_ALLOC;
    OCsr qin = {n, n, q_nnz, (size_t *)q_rp, (size_t *)q_ci, (double *)q_v};
    size_t zero_rp = 0;
    if (n == 0) qin.rp = &zero_rp;
    if (symmetrize_q(&mo->Q, &qin, 0.5, 1e-15) != ORACLE_OK) goto fail;

    /* delete empty and free rows: build.c:254-337 */
    size_t kept = 0, kept_nnz = 0;
    for (size_t r = 0; r < m; ++r) {
        size_t len = a_rp[r + 1] - a_rp[r];
        int free_row = isinf(AL[r]) && AL[r] < 0 && isinf(AU[r]) && AU[r] > 0;
        if (len > 0 && !free_row) {
            kept++;
            kept_nnz += len;
        }
    }
    if (csr_alloc(&mo->A, kept, n, kept_nnz) != ORACLE_OK) goto fail;
    mo->AL = o_zeros(kept);
    mo->AU = o_zeros(kept);
    if (!mo->AL || !mo->AU) goto fail;
    size_t row = 0, pos = 0;
    for (size_t r = 0; r < m; ++r) {
        size_t len = a_rp[r + 1] - a_rp[r];
        int free_row = isinf(AL[r]) && AL[r] < 0 && isinf(AU[r]) && AU[r] > 0;
        if (len == 0 || free_row) continue;
        mo->AL[row] = AL[r];
        mo->AU[row] = AU[r];
        for (size_t k = a_rp[r]; k < a_rp[r + 1]; ++k) {
            mo->A.ci[pos] = a_ci[k];
            mo->A.v[pos] = a_v[k];
            ++pos;
        }
        mo->A.rp[++row] = pos;
    }
    if (csr_transpose(&mo->AT, &mo->A) != ORACLE_OK) goto fail;
    mo->n = n;
    mo->m = kept;
    mo->c = dup_vec(c, n);
    mo->l = dup_vec(l, n);
    mo->u = dup_vec(u, n);
    mo->obj_constant = obj_constant;
    if (!mo->c || !mo->l || !mo->u) goto fail;
    *out = mo;
    return ORACLE_OK;
fail:
    oracle_model_free(mo);
    return ORACLE_ALLOC;
}

size_t oracle_model_n(const OracleModel *m) { return m->n; }
size_t oracle_model_m(const OracleModel *m) { return m->m; }
size_t oracle_model_q_nnz(const OracleModel *m) { return m->Q.nnz; }
size_t oracle_model_a_nnz(const OracleModel *m) { return m->A.nnz; }

void oracle_model_export(const OracleModel *mo, size_t *q_rp, size_t *q_ci, double *q_v,
                         size_t *a_rp, size_t *a_ci, double *a_v, double *c, double *AL,
                         double *AU, double *l, double *u)
{
    memcpy(q_rp, mo->Q.rp, (mo->n + 1) * sizeof(size_t));
    memcpy(q_ci, mo->Q.ci, mo->Q.nnz * sizeof(size_t));
    memcpy(q_v, mo->Q.v, mo->Q.nnz * sizeof(double));
    memcpy(a_rp, mo->A.rp, (mo->m + 1) * sizeof(size_t));
    memcpy(a_ci, mo->A.ci, mo->A.nnz * sizeof(size_t));
    memcpy(a_v, mo->A.v, mo->A.nnz * sizeof(double));
    memcpy(c, mo->c, mo->n * sizeof(double));
    memcpy(l, mo->l, mo->n * sizeof(double));
    memcpy(u, mo->u, mo->n * sizeof(double));
    memcpy(AL, mo->AL, mo->m * sizeof(double));
    memcpy(AU, mo->AU, mo->m * sizeof(double));
}

/* ------------------------------------------------------------------------ */
/* scaled working problem                                                    */
/* ------------------------------------------------------------------------ */

typedef struct OProb {
    size_t n, m;
    OCsr Q, A, AT;
    double *c, *AL, *AU, *l, *u;
    double obj_constant;
    /* scaling (HPRQPScaling, include/shared/types.h:68-79) */
    double *row_norm, *col_norm;
    double b_scale, c_scale, norm_b, norm_c, norm_b_org, norm_c_org;
} OProb;

static void prob_free(OProb *p)
{
    csr_free(&p->Q);
    csr_free(&p->A);
    csr_free(&p->AT);
    free(p->c);
    free(p->AL);
    free(p->AU);
    free(p->l);
    free(p->u);
    free(p->row_norm);
    free(p->col_norm);
    memset(p, 0, sizeof(*p));
}

static double bound_measure(double al, double au)
{
    double a = isinf(al) ? 0.0 : fabs(al);
    double b = isinf(au) ? 0.0 : fabs(au);
    return a > b ? a : b;
}

/* Column factor sqrt(max|.|) or sqrt(sum|.|) over A's column j and Q's
 * row/column j.  [CPU] scans columns of A and Q (src/cpu/scale.c:62-147);
 * [GPU] scans rows of AT and Q (src/gpu/scale.cu:15-111). */
static void col_factors(const OProb *p, int use_sum, int mode, double *out)
{
    size_t n = p->n;
    if (mode == ORACLE_MODE_CPU_REF) {
        for (size_t j = 0; j < n; ++j) out[j] = 0.0;
        for (size_t r = 0; r < p->A.nrow; ++r)
            for (size_t k = p->A.rp[r]; k < p->A.rp[r + 1]; ++k) {
                double v = fabs(p->A.v[k]);
                if (use_sum) out[p->A.ci[k]] += v;
                else if (v > out[p->A.ci[k]]) out[p->A.ci[k]] = v;
            }
        for (size_t r = 0; r < p->Q.nrow; ++r)
            for (size_t k = p->Q.rp[r]; k < p->Q.rp[r + 1]; ++k) {
                double v = fabs(p->Q.v[k]);
                if (use_sum) out[p->Q.ci[k]] += v;
                else if (v > out[p->Q.ci[k]]) out[p->Q.ci[k]] = v;
            }
        for (size_t j = 0; j < n; ++j) {
            out[j] = sqrt(out[j]);
            if (out[j] == 0.0) out[j] = 1.0;
        }
    } else {
        for (size_t j = 0; j < n; ++j) {
            double acc = 0.0;
            for (size_t k = p->AT.rp[j]; k < p->AT.rp[j + 1]; ++k) {
                double v = fabs(p->AT.v[k]);
                if (use_sum) acc += v;
                else if (v > acc) acc = v;
            }
            for (size_t k = p->Q.rp[j]; k < p->Q.rp[j + 1]; ++k) {
                double v = fabs(p->Q.v[k]);
                if (use_sum) acc += v;
                else if (v > acc) acc = v;
            }
            out[j] = acc > 0.0 ? sqrt(acc) : 1.0;
        }
    }
}

/* Row factor over A's rows: src/cpu/scale.c:100-163, src/gpu/scale.cu:45-130. */
static void row_factors(const OProb *p, int use_sum, double *out)
{
    for (size_t r = 0; r < p->m; ++r) {
        double acc = 0.0;
        for (size_t k = p->A.rp[r]; k < p->A.rp[r + 1]; ++k) {
            double v = fabs(p->A.v[k]);
            if (use_sum) acc += v;
            else if (v > acc) acc = v;
        }
        out[r] = acc > 0.0 ? sqrt(acc) : 1.0;
    }
}

/* Apply one pass of row factors rf (m) and column factors cf (n).
 * [CPU] Q /= cf[i], /= cf[j]; A /= rf[r], /= cf[j] (src/cpu/scale.c:165-207);
 * AT rebuilt at the end.  [GPU] rows multiply by the reciprocal, columns
 * divide, and AT is scaled in place with the roles swapped
 * (src/gpu/scale.cu:113-150, 392-474). */
static void apply_factors(OProb *p, const double *rf, const double *cf, int mode)
{
    for (size_t i = 0; i < p->n; ++i) {
        if (mode == ORACLE_MODE_CPU_REF) {
            for (size_t k = p->Q.rp[i]; k < p->Q.rp[i + 1]; ++k) {
                p->Q.v[k] /= cf[i];
                p->Q.v[k] /= cf[p->Q.ci[k]];
            }
        } else {
            double rs = 1.0 / cf[i];
            for (size_t k = p->Q.rp[i]; k < p->Q.rp[i + 1]; ++k) p->Q.v[k] *= rs;
            for (size_t k = p->Q.rp[i]; k < p->Q.rp[i + 1]; ++k) p->Q.v[k] /= cf[p->Q.ci[k]];
        }
        p->c[i] /= cf[i];
        p->l[i] *= cf[i];
        p->u[i] *= cf[i];
    }
    for (size_t r = 0; r < p->m; ++r) {
        if (mode == ORACLE_MODE_CPU_REF) {
            for (size_t k = p->A.rp[r]; k < p->A.rp[r + 1]; ++k) {
                p->A.v[k] /= rf[r];
                p->A.v[k] /= cf[p->A.ci[k]];
            }
            if (!isinf(p->AL[r])) p->AL[r] /= rf[r];
            if (!isinf(p->AU[r])) p->AU[r] /= rf[r];
        } else {
            double rs = 1.0 / rf[r];
            for (size_t k = p->A.rp[r]; k < p->A.rp[r + 1]; ++k) p->A.v[k] *= rs;
            for (size_t k = p->A.rp[r]; k < p->A.rp[r + 1]; ++k) p->A.v[k] /= cf[p->A.ci[k]];
            p->AL[r] /= rf[r];
            p->AU[r] /= rf[r];
        }
    }
    if (mode != ORACLE_MODE_CPU_REF && p->m > 0) {
        for (size_t j = 0; j < p->n; ++j) {
            double rs = 1.0 / cf[j];
            for (size_t k = p->AT.rp[j]; k < p->AT.rp[j + 1]; ++k) p->AT.v[k] *= rs;
            for (size_t k = p->AT.rp[j]; k < p->AT.rp[j + 1]; ++k) p->AT.v[k] /= rf[p->AT.ci[k]];
        }
    }
}

/* Ruiz x10 (sqrt max-abs) then one Pock-Chambolle (sqrt sum-abs) pass.
 * Restates scale_problem, src/cpu/scale.c:231-319, and gpu_problem_scale,
 * src/gpu/scale.cu:332-560. */
static int prob_from_model(const OracleModel *mo, int use_scaling, int mode, OProb *p)
{
    memset(p, 0, sizeof(*p));
    p->n = mo->n;
    p->m = mo->m;
    if (csr_copy(&p->Q, &mo->Q) || csr_copy(&p->A, &mo->A) || csr_copy(&p->AT, &mo->AT))
        return ORACLE_ALLOC;
    p->c = dup_vec(mo->c, p->n);
    p->l = dup_vec(mo->l, p->n);
    p->u = dup_vec(mo->u, p->n);
    p->AL = dup_vec(mo->AL, p->m);
    p->AU = dup_vec(mo->AU, p->m);
    p->row_norm = o_zeros(p->m);
    p->col_norm = o_zeros(p->n);
    double *rf = o_zeros(p->m), *cf = o_zeros(p->n);
    if (!p->c || !p->l || !p->u || !p->AL || !p->AU || !p->row_norm || !p->col_norm || !rf || !cf)
        return ORACLE_ALLOC;
    p->obj_constant = mo->obj_constant;
    for (size_t r = 0; r < p->m; ++r) p->row_norm[r] = 1.0;
    for (size_t j = 0; j < p->n; ++j) p->col_norm[j] = 1.0;
    p->norm_b_org = 0.0;
    for (size_t r = 0; r < p->m; ++r) {
        double v = bound_measure(p->AL[r], p->AU[r]);
        if (v > p->norm_b_org) p->norm_b_org = v;
    }
    p->norm_c_org = o_norm_inf(p->c, p->n);
    if (use_scaling) {
        for (int pass = 0; pass < 11; ++pass) {
            int use_sum = pass == 10; /* pass 10 is the Pock-Chambolle pass */
            col_factors(p, use_sum, mode, cf);
            row_factors(p, use_sum, rf);
            for (size_t r = 0; r < p->m; ++r) p->row_norm[r] *= rf[r];
            for (size_t j = 0; j < p->n; ++j) p->col_norm[j] *= cf[j];
            apply_factors(p, rf, cf, mode);
        }
    }
    if (mode == ORACLE_MODE_CPU_REF) { /* src/cpu/scale.c:307-312 */
        csr_free(&p->AT);
        if (csr_transpose(&p->AT, &p->A) != ORACLE_OK) return ORACLE_ALLOC;
    }
    double nb = 0.0;
    for (size_t r = 0; r < p->m; ++r) {
        double v = bound_measure(p->AL[r], p->AU[r]);
        nb += v * v;
    }
    p->norm_b = sqrt(nb);
    p->norm_c = o_norm2(p->c, p->n);
    p->b_scale = 1.0;
    p->c_scale = 1.0;
    free(rf);
    free(cf);
    return ORACLE_OK;
}

int oracle_scale(const OracleModel *mo, int use_scaling, int mode, double *row_norm,
                 double *col_norm, double *q_val, double *a_val, double *c, double *l, double *u,
                 double *AL, double *AU, double *s4)
{
    OProb p;
    int st = prob_from_model(mo, use_scaling, mode, &p);
    if (st == ORACLE_OK) {
        memcpy(row_norm, p.row_norm, p.m * sizeof(double));
        memcpy(col_norm, p.col_norm, p.n * sizeof(double));
        memcpy(q_val, p.Q.v, p.Q.nnz * sizeof(double));
        memcpy(a_val, p.A.v, p.A.nnz * sizeof(double));
        memcpy(c, p.c, p.n * sizeof(double));
        memcpy(l, p.l, p.n * sizeof(double));
        memcpy(u, p.u, p.n * sizeof(double));
        memcpy(AL, p.AL, p.m * sizeof(double));
        memcpy(AU, p.AU, p.m * sizeof(double));
        s4[0] = p.norm_b_org;
        s4[1] = p.norm_c_org;
        s4[2] = p.norm_b;
        s4[3] = p.norm_c;
    }
    prob_free(&p);
    return st;
}

/* ------------------------------------------------------------------------ */
/* workspace (HPRQPWorkspace, include/shared/types.h:112-165)                 */
/* ------------------------------------------------------------------------ */

typedef struct OWs {
    size_t n, m;
    int mode;
    double sigma, lambda_A, lambda_Q;
    int Q_is_diag, noC, to_check;
    double *x, *x_bar, *x_hat, *w, *w_bar, *y, *y_bar, *Ax, *ATy, *ATy_bar, *ATdy, *Qw, *Qw_bar,
        *Qx, *dQw, *QATdy, *dx, *dy, *dw, *Rp, *Rd, *s, *z_bar, *tempv, *diag_Q, *fact1, *fact2,
        *fact, *fact_M, *last_x, *last_y, *last_Qw, *last_w, *last_ATy;
} OWs;

#define OWS_N_VECS 28
#define OWS_M_VECS 7

static double **ws_nvec(OWs *w, int i)
{
    double **t[OWS_N_VECS] = {&w->x,      &w->x_bar, &w->x_hat,  &w->w,      &w->w_bar,
                              &w->ATy,    &w->ATy_bar, &w->ATdy, &w->Qw,     &w->Qw_bar,
                              &w->Qx,     &w->dQw,   &w->QATdy,  &w->dx,     &w->dw,
                              &w->Rd,     &w->z_bar, &w->tempv,  &w->diag_Q, &w->fact1,
                              &w->fact2,  &w->fact,  &w->fact_M, &w->last_x, &w->last_Qw,
                              &w->last_w, &w->last_ATy, NULL};
    return t[i];
}

static double **ws_mvec(OWs *w, int i)
{
    double **t[OWS_M_VECS] = {&w->y, &w->y_bar, &w->Ax, &w->dy, &w->Rp, &w->s, &w->last_y};
    return t[i];
}

static void ws_free(OWs *w)
{
    for (int i = 0; i < OWS_N_VECS; ++i) {
        double **p = ws_nvec(w, i);
        if (p) free(*p);
    }
    for (int i = 0; i < OWS_M_VECS; ++i) free(*ws_mvec(w, i));
    memset(w, 0, sizeof(*w));
}

static int ws_alloc(OWs *w, size_t n, size_t m)
{
    memset(w, 0, sizeof(*w));
    w->n = n;
    w->m = m;
    for (int i = 0; i < OWS_N_VECS; ++i) {
        double **p = ws_nvec(w, i);
        if (!p) continue;
        *p = o_zeros(n);
        if (!*p) return ORACLE_ALLOC;
    }
    for (int i = 0; i < OWS_M_VECS; ++i) {
        double **p = ws_mvec(w, i);
        *p = o_zeros(m);
        if (!*p) return ORACLE_ALLOC;
    }
    return ORACLE_OK;
}

static void update_diag_factors(OWs *w)
{
    /* src/cpu/control.c:116-127, src/gpu/control.cu:73-92 */
    for (size_t i = 0; i < w->n; ++i) {
        double inv = 1.0 / (1.0 + w->sigma * w->diag_Q[i]);
        w->fact2[i] = inv;
        w->fact[i] = w->sigma * inv;
        w->fact1[i] = w->sigma * w->diag_Q[i] * inv;
        w->fact_M[i] = w->sigma * w->sigma * inv;
    }
}

/* Power iteration for lambda_max(M) with M = A*A' (is_a) or Q.
 * Restates src/cpu/eigs.c:19-153 and src/gpu/eigs.cu:185-383: probe
 * 1+(i+1)/(len+1), <=5000 iterations, stop when
 * ||Mq - lambda q|| / (||Mq|| + |lambda| + 1e-16) < 1e-4.
 * [GPU] normalises with a multiplication by 1/||z||, [CPU] by division. */
static double power_iteration(const OProb *p, int is_a, int mode)
{
    size_t len = is_a ? p->m : p->n;
    if (len == 0) return 0.0;
    if (!is_a && mode != ORACLE_MODE_CPU_REF && p->Q.nnz == 0) return 0.0;
    double *z = o_zeros(len), *q = o_zeros(len), *tmp = o_zeros(p->n);
    double lambda = 1.0;
    for (size_t i = 0; i < len; ++i) z[i] = 1.0 + ((double)i + 1.0) / ((double)len + 1.0);
    for (int it = 0; it < 5000; ++it) {
        double qn = o_norm2(z, len);
        if (qn <= 1e-16) {
            lambda = 0.0;
            break;
        }
        if (mode == ORACLE_MODE_CPU_REF) {
            for (size_t i = 0; i < len; ++i) q[i] = z[i] / qn;
        } else {
            double inv = 1.0 / qn;
            for (size_t i = 0; i < len; ++i) q[i] = z[i] * inv;
        }
        if (is_a) {
            o_spmv(&p->AT, q, tmp);
            o_spmv(&p->A, tmp, z);
        } else {
            o_spmv(&p->Q, q, z);
        }
        lambda = o_dot(q, z, len);
        double zn = o_norm2(z, len);
        for (size_t i = 0; i < len; ++i) q[i] = z[i] - lambda * q[i];
        double err = o_norm2(q, len) / (zn + fabs(lambda) + 1e-16);
        if (err < 1e-4) break;
    }
    free(z);
    free(q);
    free(tmp);
    return lambda < 0.0 ? 0.0 : lambda;
}

/* Setup after scaling: sigma0, noC, Q diagonal test, eigenvalues, diagonal
 * factors.  Restates workspace_allocate, src/cpu/workspace.c:191-247, and
 * gpu_workspace_setup, src/gpu/control.cu:156-241 (+ eigs.cu:385-423). */
static int ws_setup(OWs *w, const OProb *p, int mode)
{
    if (ws_alloc(w, p->n, p->m) != ORACLE_OK) return ORACLE_ALLOC;
    w->mode = mode;
    w->to_check = 1;
    size_t free_count = 0;
    for (size_t i = 0; i < p->n; ++i)
        if (isinf(p->l[i]) && isinf(p->u[i])) free_count++;
    w->noC = p->n > 0 && 5 * free_count > 4 * p->n;
    w->sigma = 1.0;
    if (p->norm_b > 1e-16 && p->norm_c > 1e-16 && p->norm_b < 1e16 && p->norm_c < 1e16)
        w->sigma = p->norm_b / p->norm_c;
    if (w->sigma <= 0.0) return ORACLE_INVALID;
    int is_diag = 1;
    double max_abs_diag = 0.0, max_diag = 0.0;
    for (size_t i = 0; i < p->n; ++i) {
        double d = 0.0;
        for (size_t k = p->Q.rp[i]; k < p->Q.rp[i + 1]; ++k) {
            if (p->Q.ci[k] == i) d += p->Q.v[k];
            else if (fabs(p->Q.v[k]) > 1e-15) is_diag = 0;
        }
        w->diag_Q[i] = d;
        if (fabs(d) > max_abs_diag) max_abs_diag = fabs(d);
        if (d > max_diag) max_diag = d;
    }
    w->Q_is_diag = is_diag;
    w->lambda_A = p->m > 0 ? power_iteration(p, 1, mode) * 1.05 : 0.0;
    if (is_diag) {
        /* [GPU] max |diag| via Idamax (eigs.cu:166-172); [CPU] max(0, diag) */
        w->lambda_Q = mode == ORACLE_MODE_CPU_REF ? max_diag : max_abs_diag;
    } else {
        w->lambda_Q = power_iteration(p, 0, mode) * 1.05;
    }
    if (is_diag) update_diag_factors(w);
    return ORACLE_OK;
}

int oracle_setup(const OracleModel *mo, int use_scaling, int mode, double *out5)
{
    OProb p;
    OWs w;
    memset(&w, 0, sizeof(w));
    int st = prob_from_model(mo, use_scaling, mode, &p);
    if (st == ORACLE_OK) st = ws_setup(&w, &p, mode);
    if (st == ORACLE_OK) {
        out5[0] = w.sigma;
        out5[1] = w.lambda_A;
        out5[2] = w.lambda_Q;
        out5[3] = w.Q_is_diag;
        out5[4] = w.noC;
    }
    ws_free(&w);
    prob_free(&p);
    return st;
}

/* ------------------------------------------------------------------------ */
/* one HPR step (src/cpu/iteration.c:250-294, src/gpu/iteration.cu:1386-1442) */
/* ------------------------------------------------------------------------ */

static void step_zxw1(OWs *w, const OProb *p, double h1, double h2)
{
    /* non-noC: src/cpu/iteration.c:85-123, gpu kernels iteration.cu:110-188 */
    double f2s = 1.0 / (1.0 + w->sigma * w->lambda_Q);
    double f1s = 1.0 - f2s;
    o_spmv(&p->Q, w->w, w->Qw);
    for (size_t i = 0; i < w->n; ++i) {
        double tmp = -w->Qw[i] + w->ATy[i] - p->c[i];
        double z_raw = w->x[i] + w->sigma * tmp;
        double xb = o_clamp(z_raw, p->l[i], p->u[i]);
        double xh = 2.0 * xb - w->x[i];
        double wb = w->Q_is_diag ? w->fact1[i] * w->w[i] + w->fact2[i] * xh
                                 : f1s * w->w[i] + f2s * xh;
        if (w->to_check) {
            w->dx[i] = xb - w->x[i];
            w->z_bar[i] = (xb - z_raw) / w->sigma;
        }
        /* [GPU] the partial kernel (to_check == 0) leaves x_bar untouched
         * (iteration.cu:153-188); [CPU] always stores it. */
        if (w->to_check || w->mode == ORACLE_MODE_CPU_REF) w->x_bar[i] = xb;
        w->x_hat[i] = xh;
        w->x[i] = h2 * xh + h1 * w->last_x[i];
        w->w_bar[i] = wb;
    }
    /* Q w_bar and tempv: iteration.c:136-143 / iteration.cu:372-403 */
    o_spmv(&p->Q, w->w_bar, w->Qw_bar);
    for (size_t i = 0; i < w->n; ++i)
        w->tempv[i] = w->x_hat[i] + w->sigma * (w->Qw[i] - w->Qw_bar[i]);
}

static void step_zxw1_noC(OWs *w, const OProb *p, double h1, double h2)
{
    /* src/cpu/iteration.c:19-83, gpu iteration.cu:190-280, 405-447, 831-920 */
    double f2s = 1.0 / (1.0 + w->sigma * w->lambda_Q);
    double f1s = 1.0 - f2s;
    if (w->m > 0) o_spmv(&p->AT, w->y, w->ATy);
    else
        for (size_t i = 0; i < w->n; ++i) w->ATy[i] = 0.0;
    for (size_t i = 0; i < w->n; ++i) {
        double tmp = -w->Qw[i] + w->ATy[i] - p->c[i];
        double z_raw = w->x[i] + w->sigma * tmp;
        double xb = o_clamp(z_raw, p->l[i], p->u[i]);
        double xh = 2.0 * xb - w->x[i];
        double wb = w->Q_is_diag ? w->fact1[i] * w->w[i] + w->fact2[i] * xh
                                 : f1s * w->w[i] + f2s * xh;
        double wh = 2.0 * wb - w->w[i];
        if (w->to_check) {
            w->dx[i] = xb - w->x[i];
            w->dw[i] = wb - w->w[i];
            w->z_bar[i] = (xb - z_raw) / w->sigma;
        }
        if (w->to_check || w->mode == ORACLE_MODE_CPU_REF) w->x_bar[i] = xb;
        w->x_hat[i] = xh;
        w->x[i] = h2 * xh + h1 * w->last_x[i];
        w->w_bar[i] = wb;
        w->w[i] = h2 * wh + h1 * w->last_w[i];
    }
    o_spmv(&p->Q, w->w_bar, w->Qw_bar);
    for (size_t i = 0; i < w->n; ++i) {
        double qw = w->Qw[i], qwb = w->Qw_bar[i];
        w->Qw[i] = h2 * (2.0 * qwb - qw) + h1 * w->last_Qw[i];
        w->tempv[i] = w->x_hat[i] + w->sigma * (qw - qwb);
    }
}

static void step_y(OWs *w, const OProb *p, double h1, double h2)
{
    /* src/cpu/iteration.c:107-156, gpu iteration.cu:449-571, 922-1008 */
    if (w->m == 0) return;
    o_spmv(&p->A, w->tempv, w->Ax);
    double f1 = w->lambda_A * w->sigma;
    double f2 = 1.0 / f1;
    for (size_t i = 0; i < w->m; ++i) {
        double s_raw = w->Ax[i] - f1 * w->y[i];
        double s_proj = o_clamp(s_raw, p->AL[i], p->AU[i]);
        double yb = f2 * (s_proj - s_raw);
        double yh = 2.0 * yb - w->y[i];
        if (w->to_check) {
            w->s[i] = s_proj;
            w->dy[i] = yb - w->y[i];
        }
        w->y_bar[i] = yb;
        w->y[i] = h2 * yh + h1 * w->last_y[i];
    }
}

static void step_w2(OWs *w, const OProb *p, double h1, double h2)
{
    /* src/cpu/iteration.c:200-230, gpu iteration.cu:573-697, 1010-1127 */
    double fs = w->sigma / (1.0 + w->sigma * w->lambda_Q);
    if (w->m > 0) o_spmv(&p->AT, w->y_bar, w->ATy_bar);
    for (size_t i = 0; i < w->n; ++i) {
        double f = w->Q_is_diag ? w->fact[i] : fs;
        double wbn = w->w_bar[i] + f * (w->ATy_bar[i] - w->ATy[i]);
        double wn = h1 * w->last_w[i] + h2 * (2.0 * wbn - w->w[i]);
        double an = h1 * w->last_ATy[i] + h2 * (2.0 * w->ATy_bar[i] - w->ATy[i]);
        if (w->to_check) {
            w->dw[i] = wbn - w->w[i];
            w->ATdy[i] = w->ATy_bar[i] - w->ATy[i];
        }
        /* [GPU] the partial w2 kernel does not store the corrected w_bar
         * (iteration.cu:605-630, 669-697) */
        if (w->to_check || w->mode == ORACLE_MODE_CPU_REF) w->w_bar[i] = wbn;
        w->w[i] = wn;
        w->ATy[i] = an;
    }
}

static void iteration_step(OWs *w, const OProb *p, size_t inner)
{
    double h1 = 1.0 / ((double)inner + 2.0);
    double h2 = 1.0 - h1;
    if (w->noC) {
        step_zxw1_noC(w, p, h1, h2);
        step_y(w, p, h1, h2);
        return;
    }
    step_zxw1(w, p, h1, h2);
    step_y(w, p, h1, h2);
    step_w2(w, p, h1, h2);
}

/* ------------------------------------------------------------------------ */
/* residuals (src/cpu/residuals.c:88-189, src/gpu/residuals.cu:81-183)       */
/* ------------------------------------------------------------------------ */

typedef struct ORes {
    int is_updated;
    double rp, rd, kkt, pobj, gap, dobj;
} ORes;

static void residuals(OWs *w, const OProb *p, ORes *r, size_t iter)
{
    memset(r, 0, sizeof(*r));
    o_spmv(&p->Q, w->x_bar, w->Qx);
    if (w->m > 0) {
        o_spmv(&p->A, w->x_bar, w->Ax);
        o_spmv(&p->AT, w->y_bar, w->ATdy);
    } else {
        for (size_t i = 0; i < w->n; ++i) w->ATdy[i] = 0.0;
    }
    double bc = p->b_scale * p->c_scale;
    double xqx = o_dot(w->x_bar, w->Qx, w->n);
    r->pobj = bc * (o_dot(p->c, w->x_bar, w->n) + 0.5 * xqx) + p->obj_constant;
    double mq = 0.0, ma = 0.0, max_ax = 0.0;
    for (size_t i = 0; i < w->n; ++i) {
        double sf = p->col_norm[i] * p->c_scale;
        double sq = fabs(w->Qx[i] * sf), sa = fabs(w->ATdy[i] * sf);
        w->Rd[i] = (w->Qx[i] + p->c[i] - w->ATdy[i] - w->z_bar[i]) * sf;
        if (sq > mq) mq = sq;
        if (sa > ma) ma = sa;
    }
    double ys = 0.0;
    if (w->m > 0) {
        for (size_t i = 0; i < w->m; ++i) {
            double proj = o_clamp(w->Ax[i], p->AL[i], p->AU[i]);
            double sf = p->row_norm[i] * p->b_scale;
            /* [GPU] s is overwritten with proj(A x_bar) (residuals.cu:28-50);
             * [CPU] s keeps the value from the last checked y-step. */
            if (w->mode != ORACLE_MODE_CPU_REF) w->s[i] = proj;
            w->Rp[i] = (proj - w->Ax[i]) * sf;
            double v = fabs(w->Ax[i] * sf);
            if (v > max_ax) max_ax = v;
        }
        ys = o_dot(w->y_bar, w->s, w->m);
    }
    r->dobj = bc * (-0.5 * xqx + o_dot(w->z_bar, w->x_bar, w->n) + ys) + p->obj_constant;
    r->gap = fabs(r->pobj - r->dobj) / (1.0 + fmax(fabs(r->pobj), fabs(r->dobj)));
    double nc = p->norm_c_org;
    r->rd = o_norm_inf(w->Rd, w->n) / (1.0 + fmax(nc, fmax(ma, mq)));
    if (w->m > 0) r->rp = o_norm_inf(w->Rp, w->m) / (1.0 + fmax(p->norm_b_org, max_ax));
    if (iter == 0) {
        double bv = 0.0;
        for (size_t i = 0; i < w->n; ++i) {
            double lo = p->l[i] - w->x_bar[i], hi = w->x_bar[i] - p->u[i], v = 0.0;
            if (lo > 0.0) v += lo;
            if (hi > 0.0) v += hi;
            v = fabs(v * (p->b_scale / p->col_norm[i]));
            if (v > bv) bv = v;
        }
        if (bv > r->rp) r->rp = bv;
    }
    r->kkt = fmax(r->rp, fmax(r->rd, r->gap));
    r->is_updated = 1;
}

/* ------------------------------------------------------------------------ */
/* restart / sigma / M-norm (src/cpu/control.c, src/gpu/control.cu)          */
/* ------------------------------------------------------------------------ */

typedef struct ORst {
    int flag, first;
    double last_gap, current_gap, save_gap;
    size_t inner, sufficient, necessary, long_restart, times;
    double weighted_norm, best_gap, best_sigma;
} ORst;

static void restart_init(ORst *r)
{
    /* src/cpu/control.c:129-142 */
    memset(r, 0, sizeof(*r));
    r->first = 1;
    r->save_gap = r->current_gap = r->last_gap = r->best_gap = INFINITY;
    r->best_sigma = 1.0;
    r->weighted_norm = INFINITY;
}

static double m_norm(OWs *w, const OProb *p)
{
    /* src/cpu/control.c:155-229, src/gpu/control.cu:243-332 */
    double m1 = 0.0, m3 = 0.0;
    double dx_sq = o_dot(w->dx, w->dx, w->n);
    double m2 = (1.0 / w->sigma) * dx_sq;
    o_spmv(&p->Q, w->dw, w->dQw);
    m2 -= 2.0 * o_dot(w->dQw, w->dx, w->n);
    if (w->m > 0) {
        double dy_sq = o_dot(w->dy, w->dy, w->m);
        m1 = w->sigma * w->lambda_A * dy_sq;
        o_spmv(&p->AT, w->dy, w->ATdy);
        o_spmv(&p->Q, w->ATdy, w->QATdy);
        m1 -= 2.0 * w->sigma * o_dot(w->dQw, w->ATdy, w->n);
        m2 += 2.0 * o_dot(w->ATdy, w->dx, w->n);
        if (w->Q_is_diag) {
            for (size_t i = 0; i < w->n; ++i) w->tempv[i] = w->ATdy[i] * w->fact_M[i];
            m3 = o_dot(w->tempv, w->QATdy, w->n);
            m1 += w->sigma * o_dot(w->dQw, w->dQw, w->n);
        } else {
            m3 = (w->sigma * w->sigma) / (1.0 + w->sigma * w->lambda_Q) *
                 o_dot(w->ATdy, w->QATdy, w->n);
            m1 += w->sigma * w->lambda_Q * o_dot(w->dw, w->dQw, w->n);
        }
    } else if (!w->Q_is_diag) {
        m1 = w->sigma * w->lambda_Q * o_dot(w->dw, w->dQw, w->n);
    }
    m2 += m1 > 0.0 ? m1 : 0.0;
    return sqrt((m2 > 0.0 ? m2 : 0.0) + (m3 > 0.0 ? m3 : 0.0));
}

static void restart_check(ORst *r, size_t iter, size_t check_iter, double sigma)
{
    /* src/cpu/control.c:231-282 */
    if (check_iter == 0) return;
    r->flag = 0;
    if (r->first) {
        if (iter == check_iter) {
            r->first = 0;
            r->flag = 1;
            r->weighted_norm = r->current_gap;
            r->best_gap = r->current_gap;
            r->best_sigma = sigma;
        }
        return;
    }
    if (iter % check_iter != 0) return;
    if (r->current_gap < 0.0) r->current_gap = 1e-6;
    if (r->current_gap <= 0.2 * r->last_gap) {
        r->sufficient++;
        r->flag = 1;
    }
    if (r->current_gap <= 0.8 * r->last_gap && r->current_gap > r->save_gap) {
        r->necessary++;
        r->flag = 2;
    }
    double f = (r->weighted_norm > 0.0 && r->current_gap / r->weighted_norm > 1e-1) ? 0.5 : 0.2;
    if ((double)r->inner >= f * (double)iter) {
        r->long_restart++;
        r->flag = 3;
    }
    if (r->best_gap > r->current_gap) {
        r->best_gap = r->current_gap;
        r->best_sigma = sigma;
    }
    r->save_gap = r->current_gap;
}

static void restart_post(ORst *r, size_t iter, size_t check_iter, double gap)
{
    /* src/cpu/control.c:284-305 */
    int at_check = check_iter > 0 && (iter + 1) % check_iter == 0;
    if (r->flag > 0 || at_check) {
        if (r->flag > 0) r->last_gap = gap;
        if (at_check) r->current_gap = gap;
    }
}

static double golden_scalar(double a, double b, double c, double d)
{
    /* src/cpu/control.c:45-77, src/gpu/cuda_common.h:115-147 */
    double left = 1e-12, right = 1e12;
    double ip = (sqrt(5.0) - 1.0) / 2.0, ip2 = (3.0 - sqrt(5.0)) / 2.0;
    double x1 = left + ip2 * (right - left), x2 = left + ip * (right - left);
#define OBJ(x) (a * (x) + b / (x) + c * (x) * (x) / (1.0 + d * (x)))
    double f1 = OBJ(x1), f2 = OBJ(x2);
    for (int it = 0; it < 256; ++it) {
        if (fabs(right - left) <= 1e-13 * fmax(1.0, fmax(fabs(left), fabs(right)))) break;
        if (f1 > f2) {
            left = x1;
            x1 = x2;
            f1 = f2;
            x2 = left + ip * (right - left);
            f2 = OBJ(x2);
        } else {
            right = x2;
            x2 = x1;
            f2 = f1;
            x1 = left + ip2 * (right - left);
            f1 = OBJ(x1);
        }
    }
#undef OBJ
    return 0.5 * (left + right);
}

static double diag_obj(OWs *w, double x, double a, double b)
{
    /* src/cpu/control.c:25-43, src/gpu/control.cu:60-71 + 444-446 */
    double dot = 0.0;
    for (size_t i = 0; i < w->n; ++i) {
        w->tempv[i] = w->QATdy[i] / (1.0 + x * w->diag_Q[i]);
        dot += w->ATdy[i] * w->tempv[i];
    }
    return a * x + b / x + x * x * dot;
}

static double golden_diag(OWs *w, double a, double b)
{
    /* src/cpu/control.c:79-114, src/gpu/control.cu:429-489 */
    double left = 1e-12, right = 1e12, phi = (sqrt(5.0) - 1.0) / 2.0;
    double x1 = right - phi * (right - left), x2 = left + phi * (right - left);
    double f1 = diag_obj(w, x1, a, b), f2 = diag_obj(w, x2, a, b);
    for (int it = 0; it < 200; ++it) {
        if (fabs(right - left) <= 1e-12 * fmax(1.0, fabs(left))) break;
        if (f1 > f2) {
            left = x1;
            x1 = x2;
            f1 = f2;
            x2 = left + phi * (right - left);
            f2 = diag_obj(w, x2, a, b);
        } else {
            right = x2;
            x2 = x1;
            f2 = f1;
            x1 = right - phi * (right - left);
            f1 = diag_obj(w, x1, a, b);
        }
    }
    return f1 < f2 ? x1 : x2;
}

static void sigma_update(OWs *w, const OProb *p, ORst *r, const ORes *res)
{
    /* src/cpu/control.c:307-411, src/gpu/control.cu:334-529 */
    if (r->flag < 1) return;
    double sigma_old = w->sigma, a = 0.0, c_term = 0.0, d_term = 0.0;
    for (size_t i = 0; i < w->n; ++i) {
        w->dx[i] = w->x_bar[i] - w->last_x[i];
        w->dw[i] = w->w_bar[i] - w->last_w[i];
    }
    double b = o_dot(w->dx, w->dx, w->n);
    o_spmv(&p->Q, w->dw, w->dQw);
    if (w->m > 0) {
        for (size_t i = 0; i < w->m; ++i) w->dy[i] = w->y_bar[i] - w->last_y[i];
        for (size_t i = 0; i < w->n; ++i) w->ATdy[i] = w->ATy_bar[i] - w->last_ATy[i];
        a = w->lambda_A * o_dot(w->dy, w->dy, w->m);
        a -= 2.0 * o_dot(w->dQw, w->ATdy, w->n);
        o_spmv(&p->Q, w->ATdy, w->QATdy);
    }
    if (w->Q_is_diag) {
        a += o_dot(w->dQw, w->dQw, w->n);
    } else {
        a += w->lambda_Q * o_dot(w->dw, w->dQw, w->n);
        if (w->m > 0) {
            c_term = o_dot(w->ATdy, w->QATdy, w->n);
            d_term = w->lambda_Q;
        }
    }
    a = a > 1e-12 ? a : 1e-12;
    b = b > 1e-12 ? b : 1e-12;
    double est;
    if (w->Q_is_diag && w->m > 0) est = golden_diag(w, a, b);
    else if (!w->Q_is_diag && w->m > 0)
        est = golden_scalar(a, b, c_term > 0.0 ? c_term : 0.0, d_term > 0.0 ? d_term : 0.0);
    else
        est = sqrt(b / a);
    est = o_clamp(est, 1e-12, 1e12);
    double fact = (r->best_gap > 0.0 && isfinite(r->best_gap))
                      ? exp(-0.05 * (r->current_gap / r->best_gap))
                      : 1.0;
    double cand = exp(fact * log(est) + (1.0 - fact) * log(r->best_sigma > 0.0 ? r->best_sigma : sigma_old));
    double kappa = 1.0;
    double t1 = fmax(fmin(res->rd, res->rp), fmin(res->gap, r->current_gap));
    if (t1 <= 9e-10 && res->rp > 0.0) {
        double ratio = res->rd / res->rp;
        kappa = t1 > 5e-10 ? o_clamp(sqrt(ratio), 1e-2, 100.0) : o_clamp(ratio, 1e-2, 100.0);
    }
    w->sigma = o_clamp(kappa * cand, 1e-12, 1e12);
    if (w->Q_is_diag && fabs(w->sigma - sigma_old) > 1e-15) update_diag_factors(w);
}

static void restart_apply(OWs *w, const OProb *p, ORst *r)
{
    /* src/cpu/control.c:413-458, src/gpu/control.cu:531-591 + solver.cu:74-92 */
    if (r->flag <= 0) return;
    for (size_t i = 0; i < w->n; ++i) {
        w->x[i] = w->last_x[i] = w->x_bar[i];
        w->w[i] = w->last_w[i] = w->w_bar[i];
    }
    if (w->m > 0) {
        for (size_t i = 0; i < w->m; ++i) w->y[i] = w->last_y[i] = w->y_bar[i];
        o_spmv(&p->AT, w->y_bar, w->ATy_bar);
        for (size_t i = 0; i < w->n; ++i) w->ATy[i] = w->last_ATy[i] = w->ATy_bar[i];
    }
    if (w->noC)
        for (size_t i = 0; i < w->n; ++i) w->Qw[i] = w->last_Qw[i] = w->Qw_bar[i];
    r->last_gap = r->current_gap;
    r->save_gap = INFINITY;
    r->times++;
    r->inner = 0;
}

/* ------------------------------------------------------------------------ */
/* outer loop (src/shared/solver_backend.c:119-208, 338-569)                  */
/* ------------------------------------------------------------------------ */

static size_t adaptive_step(size_t iter)
{
    size_t step = 10;
    if (iter == 0) return step;
    while (iter / step >= 100 && step <= SIZE_MAX / 10) step *= 10;
    return step;
}

static int should_print(const OracleParams *pr, size_t iter, double elapsed)
{
    if (pr->print_frequency == -1 &&
        (iter % adaptive_step(iter) == 0 || iter == pr->max_iter || elapsed > pr->time_limit))
        return 1;
    if (pr->print_frequency > 0 && (iter % (size_t)pr->print_frequency == 0 ||
                                    iter == pr->max_iter || elapsed > pr->time_limit))
        return 1;
    return 0;
}

static int should_check_next(const OracleParams *pr, const ORst *r, size_t next)
{
    int t = 0;
    if (pr->check_iter > 0 && next % pr->check_iter == 0) t = 1;
    if (r->flag > 0) t = 1;
    if (pr->print_frequency == -1 && next % adaptive_step(next) == 0) t = 1;
    if (pr->print_frequency > 0 && next % (size_t)pr->print_frequency == 0) t = 1;
    return t;
}

void oracle_params_default(OracleParams *p)
{
    p->stoptol = 1e-8;
    p->max_iter = 2147483647u;
    p->time_limit = 3600.0;
    p->check_iter = 100;
    p->print_frequency = -1;
    p->use_scaling = 1;
    p->mode = ORACLE_MODE_GPU_REF;
}

int oracle_solve(const OracleModel *mo, const OracleParams *pr, OracleResult *out, double *x,
                 double *y, double *z, double *wv)
{
    return oracle_solve_from(mo, pr, NULL, NULL, NULL, 0.0, out, x, y, z, wv);
}

/* Warm start: this project's addition (the reference always starts at
 * zero, its vectors zero-filled at allocation, src/gpu/context.cu:75-96),
 * restated from the batch solver's rules so that its iterates can be
 * checked: the iterates and the Halpern anchors start at the point scaled
 * like the data (x0 * col_norm / b_scale, w0 likewise, y0 * row_norm /
 * c_scale, the inverse of the output map), A'y (and Q w on the noC path)
 * are computed once, sigma0 > 0 replaces the data-based sigma0 (clamped to
 * [1e-12, 1e12]), and the point is not accepted as optimal at iteration 0. */
int oracle_solve_from(const OracleModel *mo, const OracleParams *pr, const double *x0, const double *y0,
                      const double *w0, double sigma0, OracleResult *out, double *x, double *y, double *z,
                      double *wv)
{
    if (!mo || !pr || !out) return ORACLE_INVALID;
    memset(out, 0, sizeof(*out));
    double t0 = o_now();
    OProb p;
    OWs w;
    memset(&w, 0, sizeof(w));
    int st = prob_from_model(mo, pr->use_scaling, pr->mode, &p);
    if (st == ORACLE_OK) st = ws_setup(&w, &p, pr->mode);
    if (st != ORACLE_OK) {
        ws_free(&w);
        prob_free(&p);
        return st;
    }
    const int warm = x0 != NULL;
    if (warm) {
        if (sigma0 > 0.0) {
            w.sigma = o_clamp(sigma0, 1e-12, 1e12);
            if (w.Q_is_diag) update_diag_factors(&w);
        }
        for (size_t i = 0; i < w.n; ++i) {
            const double cn = p.col_norm[i];
            const double xs = x0[i] * cn / p.b_scale, ws = (w0 ? w0[i] : x0[i]) * cn / p.b_scale;
            w.x[i] = w.x_bar[i] = w.x_hat[i] = w.last_x[i] = xs;
            w.w[i] = w.w_bar[i] = w.last_w[i] = ws;
        }
        for (size_t i = 0; i < w.m; ++i)
            w.y[i] = w.y_bar[i] = w.last_y[i] = y0 ? y0[i] * p.row_norm[i] / p.c_scale : 0.0;
        if (w.m > 0) {
            o_spmv(&p.AT, w.y, w.ATy);
            for (size_t i = 0; i < w.n; ++i) w.ATy_bar[i] = w.last_ATy[i] = w.ATy[i];
        }
        if (w.noC) {
            o_spmv(&p.Q, w.w, w.Qw);
            for (size_t i = 0; i < w.n; ++i) w.Qw_bar[i] = w.last_Qw[i] = w.Qw[i];
        }
    }
    ORes res;
    ORst rs;
    restart_init(&rs);
    size_t iter_4 = 0, iter_6 = 0;
    int first_4 = 1, first_6 = 1;
    residuals(&w, &p, &res, 0);
    if (first_4 && res.kkt < 1e-4) { iter_4 = 0; first_4 = 0; }
    if (first_6 && res.kkt < 1e-6) { iter_6 = 0; first_6 = 0; }
    int final_status = ORACLE_MAX_ITER;
    rs.best_sigma = w.sigma;
    size_t iter;
    for (iter = 0;; ++iter) {
        double el = o_now() - t0;
        if (iter > 0) {
            int print_yes = should_print(pr, iter, el);
            if ((pr->check_iter > 0 && iter % pr->check_iter == 0) || print_yes) {
                residuals(&w, &p, &res, iter);
                if (first_4 && res.kkt < 1e-4) { iter_4 = iter; first_4 = 0; }
                if (first_6 && res.kkt < 1e-6) { iter_6 = iter; first_6 = 0; }
            } else {
                res.is_updated = 0;
            }
        }
        if (res.kkt < pr->stoptol && !(warm && iter == 0)) final_status = ORACLE_OPTIMAL;
        else if (iter == pr->max_iter) final_status = ORACLE_MAX_ITER;
        else if (el > pr->time_limit) final_status = ORACLE_TIME_LIMIT;
        else final_status = ORACLE_CONTINUE;
        restart_check(&rs, iter, pr->check_iter, w.sigma);
        sigma_update(&w, &p, &rs, &res);
        restart_apply(&w, &p, &rs);
        if (final_status != ORACLE_CONTINUE) break;
        w.to_check = should_check_next(pr, &rs, iter + 1);
        iteration_step(&w, &p, rs.inner);
        if (rs.flag > 0 || (pr->check_iter > 0 && (iter + 1) % pr->check_iter == 0)) {
            double g = m_norm(&w, &p);
            if (!isfinite(g)) {
                ws_free(&w);
                prob_free(&p);
                return ORACLE_INVALID;
            }
            restart_post(&rs, iter, pr->check_iter, g);
        }
        rs.inner += 1;
    }
    out->status = final_status;
    out->iter = iter;
    out->iter_4 = iter_4 == 0 ? iter : iter_4;
    out->iter_6 = iter_6 == 0 ? iter : iter_6;
    out->primal_obj = res.pobj;
    out->residuals = res.kkt;
    out->gap = res.gap;
    out->err_rp = res.rp;
    out->err_rd = res.rd;
    out->dual_obj = res.dobj;
    out->sigma = w.sigma;
    out->lambda_max_A = w.lambda_A;
    out->lambda_max_Q = w.lambda_Q;
    out->Q_is_diag = w.Q_is_diag;
    out->noC = w.noC;
    out->restarts = rs.times;
    out->time = o_now() - t0;
    /* unscaled output: src/gpu/workspace.cu:427-511, src/shared/solver.c:67-106 */
    for (size_t i = 0; i < w.n; ++i) {
        double cn = p.col_norm[i];
        if (x) x[i] = p.b_scale * (w.x_bar[i] / cn);
        if (wv) wv[i] = p.b_scale * (w.w_bar[i] / cn);
        if (z) z[i] = p.c_scale * (w.z_bar[i] * cn);
    }
    for (size_t i = 0; i < w.m; ++i)
        if (y) y[i] = p.c_scale * (w.y_bar[i] / p.row_norm[i]);
    ws_free(&w);
    prob_free(&p);
    return final_status;
}

/* ------------------------------------------------------------------------ */
/* host FP64 KKT recomputation in the original space                         */
/* (formulas of src/cpu/residuals.c:123-189 with unit scaling, s = proj(Ax)) */
/* ------------------------------------------------------------------------ */

void oracle_kkt(const OracleModel *mo, const double *x, const double *y, const double *z,
                double *out)
{
    size_t n = mo->n, m = mo->m;
    double *qx = o_zeros(n), *aty = o_zeros(n), *ax = o_zeros(m);
    o_spmv(&mo->Q, x, qx);
    if (m) {
        o_spmv(&mo->A, x, ax);
        o_spmv(&mo->AT, y, aty);
    }
    double xqx = o_dot(x, qx, n);
    double pobj = o_dot(mo->c, x, n) + 0.5 * xqx + mo->obj_constant;
    double rd = 0.0, mq = 0.0, ma = 0.0;
    for (size_t i = 0; i < n; ++i) {
        double v = fabs(qx[i] + mo->c[i] - aty[i] - z[i]);
        if (v > rd) rd = v;
        if (fabs(qx[i]) > mq) mq = fabs(qx[i]);
        if (fabs(aty[i]) > ma) ma = fabs(aty[i]);
    }
    double nc = o_norm_inf(mo->c, n), nb = 0.0, rp = 0.0, max_ax = 0.0, ys = 0.0;
    for (size_t r = 0; r < m; ++r) {
        double bm = bound_measure(mo->AL[r], mo->AU[r]);
        if (bm > nb) nb = bm;
        double proj = o_clamp(ax[r], mo->AL[r], mo->AU[r]);
        if (fabs(proj - ax[r]) > rp) rp = fabs(proj - ax[r]);
        if (fabs(ax[r]) > max_ax) max_ax = fabs(ax[r]);
        ys += y[r] * proj;
    }
    double dobj = -0.5 * xqx + o_dot(z, x, n) + ys + mo->obj_constant;
    double err_rd = rd / (1.0 + fmax(nc, fmax(ma, mq)));
    double err_rp = m ? rp / (1.0 + fmax(nb, max_ax)) : 0.0;
    double gap = fabs(pobj - dobj) / (1.0 + fmax(fabs(pobj), fabs(dobj)));
    out[0] = err_rp;
    out[1] = err_rd;
    out[2] = gap;
    out[3] = pobj;
    out[4] = dobj;
    out[5] = fmax(err_rp, fmax(err_rd, gap));
    free(qx);
    free(aty);
    free(ax);
}
