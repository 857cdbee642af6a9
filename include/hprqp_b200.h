/*
 * hprqp_b200.h -- engine diagnostics used by the parity tests and the
 * benchmark.  These have no counterpart in the reference's public API; the
 * reference exposes the same quantities only through the internal headers
 * of its include/gpu directory to its own C tests.
 */
#ifndef HPRQP_B200_H
#define HPRQP_B200_H

#include <stddef.h>
#include <stdint.h>

#include "shared/types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* y = M x with the engine's tiled SpMV kernel (the product inside every
 * HPR step; the reference runs cuSPARSE CSR ALG2 or a thread-per-row dot,
 * src/gpu/spmv.cu:25-39, 511-659).  Host arrays in, host array out; after
 * one untimed launch the kernel is replayed `reps` times (>= 1) and, when
 * ms_per_spmv is non-NULL, the mean device time of one product (CUDA
 * events) is returned there.
 * A matrix whose stream is smaller than 256 MiB is evicted from L2 (a
 * 256 MiB buffer write) before every timed product, so each product reads it
 * from HBM; larger matrices do not fit in L2 and are timed back to back. */
HPRQPStatus hprqp_b200_spmv(size_t nrow, size_t ncol, size_t nnz, const size_t *row_ptr,
                            const size_t *col_ind, const double *values, const double *x, double *y,
                            int reps, double *ms_per_spmv);

/* The floor of any CSR product with this matrix's sparsity pattern (an
 * addition, a yardstick for hprqp_b200_spmv): one kernel streams every
 * column index and value once and gathers every x[col], with no row
 * structure (each warp takes 2048 consecutive entries).  Timed like
 * hprqp_b200_spmv (one untimed pass, then `reps` timed passes, the same L2
 * eviction rule); *ms_per_pass = mean device time of one pass, *checksum =
 * the sum of all products v[k] * x[col[k]] (the sum of the entries of M x,
 * up to rounding). */
HPRQPStatus hprqp_b200_gather_bound(size_t nrow, size_t ncol, size_t nnz, const size_t *row_ptr,
                                    const size_t *col_ind, const double *values, const double *x, int reps,
                                    double *ms_per_pass, double *checksum);

/* The solver's residual kernels at a caller-given point (x, y, z) in the
 * original space of the preprocessed model (x, z: n entries, y: m): setup as
 * solve_gpu performs it, then the fused residual SpMVs and reductions
 * (reference gpu_compute_residuals_value, src/gpu/residuals.cu:81-183);
 * iter == 0 adds the bound-violation term to errRp as at the first check. */
HPRQPStatus hprqp_b200_residuals(const HPRQPModel *model, const HPRQPParams *params, const double *x,
                                 const double *y, const double *z, size_t iter, HPRQPResiduals *out);

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

/* lambda_max(A A') * 1.05 -- the dual step-size bound that solve_gpu computes
 * at setup -- by the same power iteration, for callers that cannot allocate
 * device memory (their GPU memory belongs to another allocator or arena, or
 * device allocation is not allowed while they run).  No counterpart in the
 * reference, which only computes this inside its own setup.
 *
 * Inputs are device arrays owned by the caller: A (m x n) and its transpose
 * A' (n x m) in 0-based int32 CSR (row pointers, column indices, values),
 * which must be valid CSR of those shapes.  The result and the iteration
 * count are written to host memory.  `stream` is a cudaStream_t (NULL for the
 * legacy default stream); the call returns after the stream has executed it.
 * All work vectors live in one fixed 8 MiB device array inside this library:
 * 2*m + n must not exceed 1,046,526 (larger calls return
 * HPRQP_STATUS_INVALID_ARGUMENT).  The array is shared by all calls and
 * keeps the previous call's contents, so calls on the same device must not
 * overlap in time.  The first call on a device looks up the array's device
 * address (again after a cudaDeviceReset or a new primary context); make it
 * before any stream capture on that device.  `device` must be a visible
 * device (else HPRQP_STATUS_INVALID_ARGUMENT); the caller's current device is
 * restored before the call returns.  Nothing is allocated: no cudaMalloc, no
 * cudaFree, no allocating library call (the 8 MiB array is reserved when the
 * library's device code is loaded on the device, not by a call). */
HPRQPStatus hprqp_b200_power_lambda_noalloc(int device, size_t m, size_t n, const int *a_row_ptr,
                                            const int *a_col, const double *a_val, const int *at_row_ptr,
                                            const int *at_col, const double *at_val, void *stream,
                                            double *lambda_out, int *iterations_out);

/* Routing of solve_gpu (an addition: the reference runs every model through
 * its host-driven loop, src/shared/solver_backend.c:432-513).  A model
 * without cones whose products per iteration touch at most max_work
 * nonzeros (2 nnz(Q) + 2 nnz(A)) is solved in one CTA of the batch kernel
 * -- same method, same results up to rounding, one launch instead of host
 * round trips per iteration -- unless it is solved for the adjoint
 * (hprqp_solve_for_backward).  max_work = 0 sends every model through the
 * host-driven loop.  Process-wide; returns the previous value. */
size_t hprqp_b200_set_single_cta_max_work(size_t max_work);

/* Number of engine kernel launches issued by this process so far
 * (graph replays count each captured kernel). */
uint64_t hprqp_b200_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif
