/*
 * hprqp_batch.h -- batched solves and the implicit-differentiation adjoint.
 *
 * These entry points are additions: the reference (PolyU-IOR/HPR-QP-C) has
 * no batch API and no adjoint.  Each instance of a batch is solved with the
 * reference algorithm (same preprocessing, scaling, step, restart and sigma
 * rules as solve_gpu, reference src/gpu/solver.cu:127-232), to its own
 * tolerance, with its own sigma and restart state.
 *
 * A batch is given as one block-diagonal QP: instance k owns variables
 * [var_offsets[k], var_offsets[k+1]) and constraint rows
 * [row_offsets[k], row_offsets[k+1]); Q and A are the block-diagonal
 * matrices in host CSR form (entries outside an instance's block are
 * rejected with HPRQP_STATUS_INVALID_ARGUMENT).  All arrays are host memory.
 */
#ifndef HPRQP_BATCH_H
#define HPRQP_BATCH_H

#include <stddef.h>

#include "shared/types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct HPRQPBatch HPRQPBatch;

typedef struct HPRQPBatchParams {
    double stoptol;      /* per-instance relative KKT tolerance (default 1e-6) */
    size_t max_iter;     /* per instance (default INT_MAX) */
    double time_limit;   /* seconds for the whole batch (default 3600) */
    size_t check_iter;   /* residual / restart cadence (default 100) */
    int print_frequency; /* -1: adaptive check steps as in HPRQPParams (default) */
    int use_scaling;     /* Ruiz + Pock-Chambolle (default 1) */
    int device_number;   /* CUDA device (default 0) */
    int verbose;         /* unused, reserved */
} HPRQPBatchParams;

void hprqp_batch_params_set_defaults(HPRQPBatchParams *params);

/* Preprocess every instance (the single-QP builder's rules) and upload the
 * batch to the device.  The inputs are copied; the handle owns its data. */
HPRQPStatus hprqp_batch_create(size_t num_instances, const size_t *var_offsets, const size_t *row_offsets,
                               const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c,
                               const double *AL, const double *AU, const double *l, const double *u,
                               const double *obj_constants, int device_number, HPRQPBatch **out);

/* Solve all instances (inputs already on the device): persistent kernels,
 * one instance per CTA, taken from a work queue with two ends (half the CTAs
 * take the largest instance left, half the smallest).  In a batch of more
 * than two instances per SM, the instances of at most 640 variables and 640
 * rows with few nonzeros run in a launch of 640-thread CTAs started first,
 * the others in a launch of 1024-thread CTAs beside it; the shape is fixed
 * per instance, so an instance's result does not depend on the rest of the
 * batch or on timing.  Returns when the solve has ended.  May be called
 * repeatedly; every call starts from the original data, at zero or at the
 * point set by hprqp_batch_set_warm_start. */
HPRQPStatus hprqp_batch_solve(HPRQPBatch *batch, const HPRQPBatchParams *params);

/* Start the following hprqp_batch_solve calls from a given point instead of
 * zero (an addition: the reference always starts from zero, its iterates
 * being zero-filled at allocation, reference src/gpu/context.cu:75-96).
 * x0 and w0: total variables; y0: the caller's total rows (rows removed by
 * preprocessing are ignored).  w0 == NULL uses x0, y0 == NULL uses zero;
 * x0 == NULL clears the warm start.  The typical point is the x, y, w of a
 * solve of a nearby batch (hprqp_batch_get_results), e.g. the previous step
 * of a training loop.  Each instance starts its iterates and Halpern anchors
 * there (scaled like the data); the point is never accepted as optimal
 * before the first step.  sigma0 (one per instance, or NULL): the starting
 * step-size ratio sigma, e.g. hprqp_batch_get_sigma of that solve; entries
 * <= 0, and NULL, keep the reference's data-based sigma0 (reference
 * src/gpu/control.cu:196-200).  Non-finite entries:
 * HPRQP_STATUS_INVALID_ARGUMENT.  The values are copied. */
HPRQPStatus hprqp_batch_set_warm_start(HPRQPBatch *batch, const double *x0, const double *y0, const double *w0,
                                       const double *sigma0);

/* Ask the hprqp_batch_solve running on this batch (from another host
 * thread) to stop early -- an addition; the reference's only stop besides
 * convergence and max_iter is its time limit (src/shared/solver_backend.c:
 * 432-513), and an aborted instance ends the same way: an instance being
 * solved stops within 16 iterations with HPRQP_STATUS_TIME_LIMIT and its
 * current iterates, residuals recomputed; an instance not started yet (also
 * one started after time_limit has passed) is not set up and reports
 * HPRQP_STATUS_TIME_LIMIT at iteration 0 with zero vectors and infinite
 * residual and gap.  The solve then returns HPRQP_STATUS_OK as usual.  The
 * request stays set until a solve has ended, so a request made just before
 * hprqp_batch_solve starts stops that solve. */
HPRQPStatus hprqp_batch_request_abort(HPRQPBatch *batch);

/* sigma of each instance at the end of the last hprqp_batch_solve. */
HPRQPStatus hprqp_batch_get_sigma(const HPRQPBatch *batch, double *sigma);

/* Seconds each instance of the last hprqp_batch_solve took on its CTA, from
 * loading its data to writing its results (device clock; instances run
 * concurrently, so these do not add up to the launch time).  The per-solve
 * time a dataset table reports for a batched run. */
HPRQPStatus hprqp_batch_get_times(const HPRQPBatch *batch, double *seconds);

/* SpMV lane-group width of every matrix (an addition; the reference picks
 * between cuSPARSE and its own kernel per matrix by timing them,
 * src/gpu/iteration.cu:1287-1382).  Inside the solve kernel each row of Q,
 * A and A' is summed by a group of 1, 2, 4, 8, 16 or 32 lanes; by default
 * the width of each matrix of each instance is chosen when the batch is
 * created, from that matrix's row lengths (a cost model of the rounds,
 * passes and shuffles of the product).  hprqp_batch_set_spmv_lanes(b, w)
 * forces width w on every matrix (w = 0 restores the chosen widths; other
 * values: HPRQP_STATUS_INVALID_ARGUMENT); every width gives the same
 * iterates up to rounding.  hprqp_batch_get_spmv_lanes writes 3 widths per
 * instance (Q, A, A') in instance order. */
HPRQPStatus hprqp_batch_set_spmv_lanes(HPRQPBatch *batch, int lanes);
HPRQPStatus hprqp_batch_get_spmv_lanes(const HPRQPBatch *batch, int *lanes);

/* Device time of the last hprqp_batch_solve kernel, milliseconds. */
double hprqp_batch_last_solve_ms(const HPRQPBatch *batch);
size_t hprqp_batch_num_instances(const HPRQPBatch *batch);

/* Copy results to host arrays (any pointer may be NULL).  Per instance:
 * status (HPRQPStatus), iter, primal objective, KKT residual, relative gap.
 * Packed like the inputs: x, z, w (total variables) and y (total rows; rows
 * removed by preprocessing -- empty or free on both sides -- get 0). */
HPRQPStatus hprqp_batch_get_results(const HPRQPBatch *batch, int *status, size_t *iter, double *primal_obj,
                                    double *residual, double *gap, double *x, double *y, double *z, double *w);

/* Gradients of a scalar loss L(x*, y*) with respect to the problem data, by
 * implicit differentiation of the KKT conditions on the active set of the
 * last hprqp_batch_solve: variables with z != 0 sit at a bound (z > 0 lower,
 * z < 0 upper), rows with y != 0 at a bound (y > 0 lower, y < 0 upper);
 * strict complementarity is assumed.  Any output pointer may be NULL.
 * Packing as in hprqp_batch_create:
 *   dc, dl, du     total variables;  dAL, dAU  total rows (the caller's rows;
 *                  an equality row reports its whole gradient on the active
 *                  side, so dAL + dAU is the gradient of moving both sides);
 *   dQ_values      one value per nonzero of the caller's Q (the solver uses
 *                  (Q + Q')/2, so entry (i,j) gets -(lam_i x_j + lam_j x_i)/2);
 *   dA_values      one value per nonzero of the caller's A;
 *   minres_iters, minres_relres   per instance. */
typedef struct HPRQPBatchGradients {
    double *dc;
    double *dl;
    double *du;
    double *dAL;
    double *dAU;
    double *dQ_values;
    double *dA_values;
    int *minres_iters;
    double *minres_relres;
} HPRQPBatchGradients;

/* grad_x: dL/dx* (total variables); grad_y: dL/dy* (total rows) or NULL;
 * tol: relative MINRES residual (<= 0 selects 1e-12).  The adjoint systems
 * are solved on the device, one instance per CTA; the gradients are
 * assembled on the host. */
HPRQPStatus hprqp_batch_backward(HPRQPBatch *batch, const double *grad_x, const double *grad_y, double tol,
                                 HPRQPBatchGradients *gradients);

/* Device time of the last adjoint kernel, milliseconds. */
double hprqp_batch_last_backward_ms(const HPRQPBatch *batch);

void hprqp_batch_destroy(HPRQPBatch *batch);

/* One-call form: create + solve + get_results + destroy.  A batch of 1024
 * instances or more is built and launched in two parts -- first its smallest
 * instances, up to 15 % of the nonzeros, then the rest -- so that the host's
 * preprocessing and upload of the rest overlap the GPU's solve of the first
 * part, and the small instances, whose iteration counts vary most, start
 * early; the results are the same, bit for bit, as those of a handle created
 * with hprqp_batch_create and solved with hprqp_batch_solve, and time_limit
 * applies to each part's launch. */
HPRQPStatus hprqp_solve_batch(size_t num_instances, const size_t *var_offsets, const size_t *row_offsets,
                              const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c, const double *AL,
                              const double *AU, const double *l, const double *u, const double *obj_constants,
                              const HPRQPBatchParams *params, int *status, size_t *iter, double *primal_obj,
                              double *residual, double *gap, double *x, double *y, double *z, double *w);

#ifdef __cplusplus
}
#endif

#endif
