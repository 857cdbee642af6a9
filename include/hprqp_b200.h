/*
 * hprqp_b200.h -- engine diagnostics used by the parity tests and the
 * benchmark.  These have no counterpart in the reference's public API; the
 * reference exposes the same quantities only through internal headers
 * (include/gpu/*.h) to its own C tests.
 */
#ifndef HPRQP_B200_H
#define HPRQP_B200_H

#include <stddef.h>
#include <stdint.h>

#include "shared/types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* y = M x with the engine's row-block SpMV kernel (the product inside every
 * HPR step; the reference runs cuSPARSE CSR ALG2 or a thread-per-row dot,
 * src/gpu/spmv.cu:25-39, 511-659).  Host arrays in, host array out; the
 * kernel is replayed `reps` times (>= 1) and, when ms_per_spmv is non-NULL,
 * the mean device time of one product (CUDA events) is returned there.
 * A matrix whose stream is smaller than 256 MiB is evicted from L2 (a
 * 256 MiB buffer write) before every timed product, so each product reads it
 * from HBM; larger matrices do not fit in L2 and are timed back to back. */
HPRQPStatus hprqp_b200_spmv(size_t nrow, size_t ncol, size_t nnz, const size_t *row_ptr,
                            const size_t *col_ind, const double *values, const double *x, double *y,
                            int reps, double *ms_per_spmv);

/* Setup of a model exactly as solve_gpu performs it (upload, Ruiz x10 +
 * Pock-Chambolle scaling, Q-diagonal test, power iterations, sigma0).
 * out[0..4] = sigma0, lambda_max_A, lambda_max_Q, Q_is_diag, noC;
 * out[5..8] = norm_b_org, norm_c_org, norm_b, norm_c.
 * Each non-NULL array receives the scaled data (sizes of the preprocessed
 * model: row_norm m, col_norm n, q_val nnz(Q), a_val nnz(A), at_val nnz(A),
 * c/l/u n, AL/AU m).  Reference: gpu_problem_scale (src/gpu/scale.cu:332-560),
 * gpu_workspace_setup (src/gpu/control.cu:156-241). */
HPRQPStatus hprqp_b200_setup(const HPRQPModel *model, const HPRQPParams *params, double *out9,
                             double *row_norm, double *col_norm, double *q_val, double *a_val,
                             double *at_val, double *c, double *l, double *u, double *AL, double *AU);

/* Number of engine kernel launches issued by this process so far
 * (graph replays count each captured kernel). */
uint64_t hprqp_b200_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif
