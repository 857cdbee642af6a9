/* Model building.  Same entry points and meaning as include/shared/build.h
 * of the reference (src/shared/build.c, src/shared/mps_qp.cpp:208-326). */
#ifndef HPRQP_BUILD_H
#define HPRQP_BUILD_H

#include "shared/types.h"

#ifdef __cplusplus
extern "C" {
#endif

void model_init(HPRQPModel *model);
void model_free(HPRQPModel *model);
HPRQPStatus model_copy(HPRQPModel *dest, const HPRQPModel *src);
/* = build_from_QAbc: copy, validate, symmetrise Q, drop empty and free rows */
HPRQPStatus build_model_from_arrays(const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c,
                                    const double *AL, const double *AU, const double *l, const double *u,
                                    double obj_constant, HPRQPModel *model);
/* = build_from_mps */
HPRQPStatus build_model_from_mps(const char *mps_path, HPRQPModel *model);
HPRQPStatus build_from_QAbc_soc(const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c,
                                const double *AL, const double *AU, const double *l, const double *u,
                                double obj_constant, const HPRQPSOCSpec *soc, HPRQPModel *model);
/* the cone blocks of a model: offsets strictly increasing and ending at n
 * (m), free cone variables, cone rows free with a finite rhs, rhs zero on
 * the linear rows */
HPRQPStatus model_validate_soc(const HPRQPModel *model);
/* In place, on a model that owns its data (reference build.c:339-400):
 * validate, replace Q by (Q + Q')/2 without entries |q| <= 1e-15, drop
 * empty rows and rows free on both sides (not in cone models), rebuild A'. */
HPRQPStatus preprocess_model(HPRQPModel *model);

#ifdef __cplusplus
}
#endif

#endif
