/* Convex quadratic constraints.  Same entry points and meaning as
 * include/shared/qcqp.h of the reference (src/shared/qcqp.c): each
 * constraint  C_i x + 1/2 x' D_i x + constant_i <= 0  (D_i = R_i' R_i) is
 * lifted to one second-order cone over the rows  -C_i, -C_i, sqrt(2) R_i
 * with rhs  constant_i - 1, constant_i + 1, 0,  placed after the linear rows
 * of A, and the model is built by build_from_QAbc_soc (then solved by the
 * cone path of solve_gpu).  No constraints (C with zero rows): build_from_QAbc. */
#ifndef HPRQP_QCQP_H
#define HPRQP_QCQP_H

#include "shared/types.h"

#ifdef __cplusplus
extern "C" {
#endif

/* R: the stacked factors, rows [offsets[i], offsets[i+1]) for constraint i
 * (offsets: C->nrow + 1 entries, offsets[0] = 0, last = R->nrow). */
HPRQPStatus build_from_QAbc_qc_factors(const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c,
                                       const double *AL, const double *AU, const double *l, const double *u,
                                       double obj_constant, const HPRQPMatrixCSR *C, const double *constant,
                                       const HPRQPMatrixCSR *R, const size_t *offsets, HPRQPModel *model);

/* D: row i holds the diagonal of D_i (entries >= 0; negative: invalid). */
HPRQPStatus build_from_QAbc_qc_diagonal(const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c,
                                        const double *AL, const double *AU, const double *l, const double *u,
                                        double obj_constant, const HPRQPMatrixCSR *C, const double *constant,
                                        const HPRQPMatrixCSR *D, HPRQPModel *model);

#ifdef __cplusplus
}
#endif

#endif
