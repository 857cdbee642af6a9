/*
 * hprqp_diff.h -- implicit-differentiation adjoint of a single solve.
 *
 * Additions: the reference (PolyU-IOR/HPR-QP-C) has no adjoint.  The forward
 * solve is exactly solve_gpu (reference include/hprqp.h:38; same algorithm,
 * same results), except that its device state -- the scaled matrices, the
 * scaling vectors and the final iterate -- is kept for hprqp_backward instead
 * of being freed.  The backward pass solves, on the device, by MINRES,
 *     [[Q_FF, A_RF'], [A_RF, 0]] [lam_F; mu_R] = [gx_F; -gy_R]
 * with F the variables off their bounds (z == 0) and R the rows at a bound
 * (y != 0), using the same SpMV kernels as the solve, and assembles the
 * gradients on the host.  Meant for large single problems; many small ones
 * are differentiated by hprqp_batch_backward (hprqp_batch.h).
 *
 * Everything is in the space of the model passed to the solve (the output of
 * build_from_QAbc: symmetrised Q, the kept rows of A), like HPRQPResults.
 * Models with second-order cones are solved but not differentiated
 * (hprqp_backward returns HPRQP_STATUS_NOT_IMPLEMENTED for them).
 */
#ifndef HPRQP_DIFF_H
#define HPRQP_DIFF_H

#include <stddef.h>

#include "shared/types.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct HPRQPSolveState HPRQPSolveState;

/* solve_gpu that also returns a state for hprqp_backward (on OPTIMAL,
 * MAX_ITER or TIME_LIMIT; *state is NULL otherwise).  The model must stay
 * alive and unchanged until the state is destroyed. */
HPRQPStatus hprqp_solve_for_backward(const HPRQPModel *model, const HPRQPParams *params, HPRQPResults *results,
                                     HPRQPSolveState **state);

/* Gradients of a scalar loss L(x*, y*).  Any array pointer may be NULL.
 *   dc, dl, du      n entries;   dAL, dAU   m entries (an equality row
 *                   reports its whole gradient on its active side);
 *   dQ_values       one value per nonzero of model->Q (stored symmetric:
 *                   entry (i,j) gets -(lam_i x_j + lam_j x_i)/2);
 *   dA_values       one value per nonzero of model->A: -mu_r x_j + lam_j y_r;
 *   lam, mu         the adjoint solution (n and m entries). */
typedef struct HPRQPGradients {
    double *dc;
    double *dl;
    double *du;
    double *dAL;
    double *dAU;
    double *dQ_values;
    double *dA_values;
    double *lam;
    double *mu;
    long long minres_iters;
    double minres_relres;
    double backward_seconds; /* wall time of the call */
} HPRQPGradients;

/* grad_x: dL/dx* (n); grad_y: dL/dy* (m) or NULL; tol: relative MINRES
 * residual (<= 0 selects 1e-12); max_iter: MINRES iterations (0 selects
 * 4 (n + m) + 100). */
HPRQPStatus hprqp_backward(HPRQPSolveState *state, const double *grad_x, const double *grad_y, double tol,
                           long long max_iter, HPRQPGradients *gradients);

void hprqp_solve_state_destroy(HPRQPSolveState *state);

#ifdef __cplusplus
}
#endif

#endif
