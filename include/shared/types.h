/*
 * Public ABI types of the HPR-QP engine.
 *
 * Every enum value and struct layout in this file is binary-identical to the
 * one a caller of PolyU-IOR/HPR-QP-C compiles against (include/shared/types.h
 * of that project), so an application, the Python ctypes wrapper or the Julia
 * ccall wrapper built for it links against this library unchanged.  Field
 * order, field types and enum numbering are therefore fixed; the comments are
 * this project's own.
 *
 * Fields that belong to subsystems this engine does not implement (the
 * equality Gram metric, CPU polishing) keep their slots so the layout stays
 * the same; the engine ignores them.  Second-order cones are supported by
 * solve_gpu (build_from_QAbc_soc, and QCQP rows lifted to cones); the batch
 * API and the adjoints reject models with cones.
 */
#ifndef HPRQP_TYPES_H
#define HPRQP_TYPES_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes.  Reference: include/shared/types.h:10-19. */
typedef enum HPRQPStatus {
    HPRQP_STATUS_OK = 0,
    HPRQP_STATUS_INVALID_ARGUMENT = 1,
    HPRQP_STATUS_ALLOCATION_FAILED = 2,
    HPRQP_STATUS_NOT_IMPLEMENTED = 3, /* also: any CUDA failure, int32 overflow */
    HPRQP_STATUS_MAX_ITER = 4,
    HPRQP_STATUS_TIME_LIMIT = 5,
    HPRQP_STATUS_OPTIMAL = 6,
    HPRQP_STATUS_CONTINUE = 7
} HPRQPStatus;

/* SpMV implementation choice.  This engine has one SpMV family (its own
 * row-block kernels); the field is accepted for ABI compatibility and
 * AUTO/CUSPARSE/CUSTOMIZED all select it.  Reference: types.h:21-25. */
typedef enum HPRQPSpmvMode {
    HPRQP_SPMV_MODE_AUTO = 0,
    HPRQP_SPMV_MODE_CUSPARSE = 1,
    HPRQP_SPMV_MODE_CUSTOMIZED = 2
} HPRQPSpmvMode;

/* Host CSR matrix: 0-based size_t indices, row_ptr[nrow] == nnz.
 * Reference: types.h:27-35. */
typedef struct HPRQPMatrixCSR {
    size_t nrow;
    size_t ncol;
    size_t nnz;
    size_t *row_ptr;
    size_t *col_ind;
    double *values;
    int owns_data;
} HPRQPMatrixCSR;

/* Second-order-cone description: the last variables and the last rows of a
 * model may form Lorentz cones (offsets of each cone's first entry).
 * Reference: types.h:37-48. */
typedef struct HPRQPSOCSpec {
    size_t num_var_cones;
    const size_t *var_offsets;
    size_t num_row_cones;
    const size_t *row_offsets;
    const double *rhs;
} HPRQPSOCSpec;

/* A preprocessed QP:  min 1/2 x'Qx + c'x + obj_constant
 *                     s.t. AL <= Ax <= AU,  l <= x <= u.
 * Q is stored symmetrised; AT is the explicit transpose of A.
 * Reference: types.h:50-66. */
typedef struct HPRQPModel {
    HPRQPMatrixCSR Q;
    HPRQPMatrixCSR A;
    HPRQPMatrixCSR AT;
    double *c;
    double *AL;
    double *AU;
    double *l;
    double *u;
    double obj_constant;
    int owns_data;
    size_t num_var_cones;
    size_t *var_cone_offsets;
    size_t num_row_cones;
    size_t *row_cone_offsets;
    double *soc_rhs;
} HPRQPModel;

/* Diagonal equilibration produced by Ruiz + Pock-Chambolle scaling.
 * Reference: types.h:68-79. */
typedef struct HPRQPScaling {
    double *row_norm;
    double *col_norm;
    double *l_org;
    double *u_org;
    double b_scale;
    double c_scale;
    double norm_b;
    double norm_c;
    double norm_b_org;
    double norm_c_org;
} HPRQPScaling;

/* Equality-Gram row metric policy (kept for ABI; this engine always runs
 * with the metric off).  Reference: types.h:81-86. */
typedef enum HPRQPGramMode {
    HPRQP_GRAM_OFF = 0,
    HPRQP_GRAM_AUTO = 1,
    HPRQP_GRAM_REQUEST = 2
} HPRQPGramMode;

/* Solver options.  Reference: types.h:88-110; defaults set by
 * params_set_defaults() follow src/shared/solver.c:133-157. */
typedef struct HPRQPParams {
    double stoptol;
    size_t max_iter;
    int use_gpu;
    int device_number;
    double time_limit;
    size_t check_iter;
    int print_frequency;
    int use_scaling;
    int verbose;
    HPRQPSpmvMode spmv_mode_q;
    HPRQPSpmvMode spmv_mode_a;
    HPRQPGramMode gram_mode;
    int polishing;               /* ignored: no CPU polishing in this engine */
    const char *polish_python;   /* ignored */
    const char *polish_worker;   /* ignored */
    const char *polish_directory;/* ignored */
    int polish_keep_files;       /* ignored */
    size_t polish_max_attempts;  /* ignored */
    double polish_episode_seconds; /* ignored */
    double polish_total_seconds; /* ignored */
    size_t polish_memory_bytes;  /* ignored */
} HPRQPParams;

/* Host-side view of the iterate state (the reference's CPU workspace; the
 * GPU engine keeps its state in device memory and only mirrors the scalar
 * fields here).  Reference: types.h:112-165. */
typedef struct HPRQPWorkspace {
    size_t m;
    size_t n;
    double sigma;
    double lambda_max_A;
    double lambda_max_Q;
    int Q_is_diag;
    int noC;
    int to_check;
    const HPRQPMatrixCSR *Q;
    const HPRQPMatrixCSR *A;
    const HPRQPMatrixCSR *AT;
    const double *c;
    const double *AL;
    const double *AU;
    const double *l;
    const double *u;
    double *x;
    double *x_bar;
    double *x_hat;
    double *w;
    double *w_bar;
    double *w_hat;
    double *y;
    double *y_bar;
    double *y_hat;
    double *Ax;
    double *ATy;
    double *ATy_bar;
    double *ATdy;
    double *Qw;
    double *Qw_bar;
    double *Qx;
    double *dQw;
    double *QATdy;
    double *dx;
    double *dy;
    double *dw;
    double *Rp;
    double *Rd;
    double *s;
    double *z_bar;
    double *tempv;
    double *diag_Q;
    double *fact1;
    double *fact2;
    double *fact;
    double *fact_M;
    double *last_x;
    double *last_y;
    double *last_Qw;
    double *last_w;
    double *last_ATy;
} HPRQPWorkspace;

/* Residuals in the original (unscaled) space.  Reference: types.h:167-175. */
typedef struct HPRQPResiduals {
    int is_updated;
    double err_Rp_org_bar;
    double err_Rd_org_bar;
    double KKTx_and_gap_org_bar;
    double primal_obj_bar;
    double rel_gap_bar;
    double dual_obj_bar;
} HPRQPResiduals;

/* Restart bookkeeping.  Reference: types.h:177-193. */
typedef struct HPRQPRestart {
    int restart_flag;
    int first_restart;
    double last_gap;
    double current_gap;
    double save_gap;
    size_t inner;
    size_t step;
    size_t sufficient;
    size_t necessary;
    size_t long_restart;
    size_t ratio;
    size_t times;
    double weighted_norm;
    double best_gap;
    double best_sigma;
} HPRQPRestart;

/* Solve output; x, y, z, w are malloc'd by the library and released by
 * results_free().  Reference: types.h:195-214. */
typedef struct HPRQPResults {
    size_t iter;
    size_t iter_4;
    size_t iter_6;
    double time;
    double time_4;
    double time_6;
    double primal_obj;
    double residuals;
    double gap;
    int status;
    double *x;
    double *y;
    double *z;
    double *w;
    size_t polish_attempts;
    int polish_accepted;
    int gram_active;
    double total_time;
} HPRQPResults;

#ifdef __cplusplus
}
#endif

#endif
