/*
 * hprqp_oracle.h -- CPU oracle for the HPR-QP iteration loop.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain serial C restatement of the
 * reference algorithm (PolyU-IOR/HPR-QP-C), used as the checker by tests/,
 * by __graft_entry__.smoke() and by bench.py's cpu_baseline / reference
 * legs.  It is never linked into, called by or shipped with the product
 * library.
 *
 * Two semantic modes are provided because the reference's two backends
 * differ in a few places (documented at each use in hprqp_oracle.c):
 *   ORACLE_MODE_GPU_REF  the reference's CUDA backend (src/gpu, CUDA files): the
 *                        default, and what the B200 engine must match;
 *   ORACLE_MODE_CPU_REF  the reference's serial CPU backend (src/cpu, C files):
 *                        used to pin this restatement against the reference
 *                        CPU library compiled from its own sources.
 *
 * All index arrays are 0-based size_t CSR, like the reference host ABI.
 */
#ifndef HPRQP_ORACLE_H
#define HPRQP_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORACLE_MODE_GPU_REF 0
#define ORACLE_MODE_CPU_REF 1

/* status codes mirror HPRQPStatus */
#define ORACLE_OK 0
#define ORACLE_INVALID 1
#define ORACLE_ALLOC 2
#define ORACLE_MAX_ITER 4
#define ORACLE_TIME_LIMIT 5
#define ORACLE_OPTIMAL 6
#define ORACLE_CONTINUE 7

typedef struct OracleModel OracleModel;

typedef struct OracleParams {
    double stoptol;
    size_t max_iter;
    double time_limit;
    size_t check_iter;
    int print_frequency;
    int use_scaling;
    int mode;
} OracleParams;

typedef struct OracleResult {
    int status;
    size_t iter;
    size_t iter_4;
    size_t iter_6;
    double primal_obj;
    double residuals;
    double gap;
    double err_rp;
    double err_rd;
    double dual_obj;
    double sigma;
    double lambda_max_A;
    double lambda_max_Q;
    int Q_is_diag;
    int noC;
    size_t restarts;
    double time;
} OracleResult;

void oracle_params_default(OracleParams *p);

/* Build + preprocess (symmetrise Q, drop empty / free rows, validate). */
int oracle_build(size_t n, size_t q_nnz, const size_t *q_row_ptr, const size_t *q_col,
                 const double *q_val, size_t m, size_t a_nnz, const size_t *a_row_ptr,
                 const size_t *a_col, const double *a_val, const double *c, const double *AL,
                 const double *AU, const double *l, const double *u, double obj_constant,
                 OracleModel **out);
void oracle_model_free(OracleModel *model);
size_t oracle_model_n(const OracleModel *model);
size_t oracle_model_m(const OracleModel *model);
size_t oracle_model_q_nnz(const OracleModel *model);
size_t oracle_model_a_nnz(const OracleModel *model);
/* Export the preprocessed model (arrays sized by the getters above). */
void oracle_model_export(const OracleModel *model, size_t *q_row_ptr, size_t *q_col, double *q_val,
                         size_t *a_row_ptr, size_t *a_col, double *a_val, double *c, double *AL,
                         double *AU, double *l, double *u);

/* Full solve; x, w, z (n) and y (m) are caller-allocated, may be NULL. */
int oracle_solve(const OracleModel *model, const OracleParams *params, OracleResult *result,
                 double *x, double *y, double *z, double *w);

/* The same solve from a warm start (x0, w0: n; y0: m rows of the
 * preprocessed model; w0 and y0 may be NULL: x0 and zero; x0 == NULL is a
 * cold start) and an optional sigma0 (> 0), following the batch solver's
 * warm-start rules (an addition of this project, not in the reference). */
int oracle_solve_from(const OracleModel *model, const OracleParams *params, const double *x0,
                      const double *y0, const double *w0, double sigma0, OracleResult *result, double *x,
                      double *y, double *z, double *w);

/* Scaling only: fills row_norm (m), col_norm (n) and the scaled Q/A values
 * (arrays sized like the preprocessed model), plus scalars
 * [norm_b_org, norm_c_org, norm_b, norm_c]. */
int oracle_scale(const OracleModel *model, int use_scaling, int mode, double *row_norm,
                 double *col_norm, double *q_val, double *a_val, double *c, double *l, double *u,
                 double *AL, double *AU, double *scalars4);

/* Setup only: sigma0, lambda_max_A, lambda_max_Q, Q_is_diag, noC after scaling. */
int oracle_setup(const OracleModel *model, int use_scaling, int mode, double *out5);

/* y = M x for a size_t CSR matrix (serial, row order, reference summation). */
void oracle_csr_matvec(size_t nrow, const size_t *row_ptr, const size_t *col, const double *val,
                       const double *x, double *y);

/* KKT recomputation in the ORIGINAL space from (x, y, z), FP64 on the host:
 * out6 = [err_rp, err_rd, gap, primal_obj, dual_obj, kkt]. */
void oracle_kkt(const OracleModel *model, const double *x, const double *y, const double *z,
                double *out6);

#ifdef __cplusplus
}
#endif

#endif
