/*
 * hprqp.h -- the drop-in C entry points of the B200 HPR-QP engine.
 *
 * Each declaration replaces the function of the same name in the reference
 * project's include/hprqp.h (PolyU-IOR/HPR-QP-C), with the same signature
 * and meaning:
 *   model_init / model_free / model_copy      hprqp.h:14-16 (src/shared/build.c:402-502)
 *   build_from_QAbc                           hprqp.h:17-24 (src/shared/build.c:608-621)
 *   build_from_QAbc_soc                       hprqp.h:26-30 (src/shared/build.c:39-99, second-order cones)
 *   build_from_mps                            hprqp.h:31    (src/shared/mps_qp.cpp:208-326, free-format MPS
 *                                                            with QUADOBJ/QMATRIX and diagonal QCMATRIX rows)
 *   params_set_defaults / results_init/free   hprqp.h:33-35 (src/shared/solver.c:133-177)
 *   print_model_info / print_params_info      hprqp.h:36-37 (src/shared/solver_backend.c:240-271)
 *   solve_gpu                                 hprqp.h:38    (src/gpu/solver.cu:127-232)
 *   solve                                     hprqp.h:39    (src/shared/solver.c:245-260)
 *
 * Differences a caller can observe:
 *   - there is no CPU backend: solve() with params->use_gpu == 0 returns
 *     HPRQP_STATUS_NOT_IMPLEMENTED (and says so on stderr);
 *   - CPU polishing and the equality-Gram metric do not exist; their
 *     parameters are accepted and ignored (the reference with
 *     --polishing 0 --gram off);
 *   - second-order cones (build_from_QAbc_soc), MPS input (build_from_mps)
 *     and convex quadratic constraints (include/shared/qcqp.h, lifted to
 *     rotated Lorentz cones) are supported by solve_gpu; the batch API and
 *     the adjoints (hprqp_batch.h, hprqp_diff.h) take QPs without cones.
 */
#ifndef HPRQP_H
#define HPRQP_H

#ifdef __cplusplus
extern "C" {
#endif

#include "gpu/gpu.h"
#include "shared/sparse.h"
#include "shared/types.h"

void model_init(HPRQPModel *model);
void model_free(HPRQPModel *model);
HPRQPStatus model_copy(HPRQPModel *dest, const HPRQPModel *src);
HPRQPStatus build_from_QAbc(const HPRQPMatrixCSR *Q,
                            const HPRQPMatrixCSR *A,
                            const double *c,
                            const double *AL,
                            const double *AU,
                            const double *l,
                            const double *u,
                            double obj_constant,
                            HPRQPModel *model);
HPRQPStatus build_from_QAbc_soc(const HPRQPMatrixCSR *Q,
                                const HPRQPMatrixCSR *A,
                                const double *c, const double *AL, const double *AU,
                                const double *l, const double *u, double obj_constant,
                                const HPRQPSOCSpec *soc, HPRQPModel *model);
HPRQPStatus build_from_mps(const char *mps_path, HPRQPModel *model);

void params_set_defaults(HPRQPParams *params);
void results_init(HPRQPResults *results);
void results_free(HPRQPResults *results);
void print_model_info(const HPRQPModel *model);
void print_params_info(const HPRQPParams *params);
HPRQPStatus solve_gpu(const HPRQPModel *model, const HPRQPParams *params, HPRQPResults *results);
HPRQPStatus solve(const HPRQPModel *model, const HPRQPParams *params, HPRQPResults *results);

#ifdef __cplusplus
}
#endif

#endif
