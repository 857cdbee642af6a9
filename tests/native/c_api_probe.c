/* A C caller of the host-side entry points (compiled as pedantic C99 by the
 * CPU tests): the headers must be valid C, and the builders usable without a
 * GPU.  Prints one JSON line. */
#include <math.h>
#include <stdio.h>

#include "gpu/gpu.h"
#include "hprqp.h"
#include "hprqp_b200.h"
#include "hprqp_batch.h"
#include "hprqp_binding.h"
#include "hprqp_diff.h"
#include "shared/build.h"
#include "shared/qcqp.h"
#include "shared/sparse.h"
#include "shared/vector.h"

int main(int argc, char **argv)
{
    /* argv[1]: an MPS file for build_from_mps (optional) */
    /* min x0^2 + x1^2 - x0  s.t.  x0 + x1 <= 1,  x0^2 + 2 x1^2 - 0.5 <= 0 */
    size_t q_rp[] = {0, 1, 2}, q_ci[] = {0, 1}, a_rp[] = {0, 2}, a_ci[] = {0, 1};
    double q_v[] = {2.0, 2.0}, a_v[] = {1.0, 1.0};
    HPRQPMatrixCSR Q = {2, 2, 2, q_rp, q_ci, q_v, 0}, A = {1, 2, 2, a_rp, a_ci, a_v, 0};
    double c[] = {-1.0, 0.0}, AL[] = {-INFINITY}, AU[] = {1.0}, l[] = {-INFINITY, -INFINITY}, u[] = {INFINITY, INFINITY};
    size_t c_rp[] = {0, 0}, c_ci[] = {0}, d_rp[] = {0, 2}, d_ci[] = {0, 1};
    double c_v[] = {0.0}, d_v[] = {2.0, 4.0}, constant[] = {-0.5};
    HPRQPMatrixCSR C = {1, 2, 0, c_rp, c_ci, c_v, 0}, D = {1, 2, 2, d_rp, d_ci, d_v, 0};
    HPRQPModel qp, qcqp;
    model_init(&qp);
    model_init(&qcqp);
    HPRQPStatus s1 = build_from_QAbc(&Q, &A, c, AL, AU, l, u, 0.0, &qp);
    HPRQPStatus s2 = build_from_QAbc_qc_diagonal(&Q, &A, c, AL, AU, l, u, 0.0, &C, constant, &D, &qcqp);
    HPRQPStatus s3 = preprocess_model(&qp);
    double y[1];
    HPRQPStatus s4 = matrix_csr_matvec(&A, a_v, y);
    /* second-order cones: (x0, x1) in a 2-dimensional Lorentz cone, and the
       one row as a row cone of size 1 with rhs 0 (offsets end at n and m;
       cone variables and cone rows are unbounded) */
    size_t var_off[] = {0, 2}, row_off[] = {0, 1};
    double rhs[] = {0.0};
    HPRQPSOCSpec soc = {1, var_off, 1, row_off, rhs};
    HPRQPModel socm, mps;
    model_init(&socm);
    model_init(&mps);
    double ALs[] = {-INFINITY}, AUs[] = {INFINITY};
    HPRQPStatus s5 = build_from_QAbc_soc(&Q, &A, c, ALs, AUs, l, u, 0.0, &soc, &socm);
    HPRQPStatus s6 = argc > 1 ? build_from_mps(argv[1], &mps) : HPRQP_STATUS_INVALID_ARGUMENT;
    HPRQPBindingModel *mb = NULL;
    int bind_mps = argc > 1 ? (int)hprqp_model_create(&mb) : -1;
    if (argc > 1 && bind_mps == 0) bind_mps = (int)hprqp_model_read_from_mps(mb, argv[1]);
    size_t mps_n_bind = mb ? hprqp_model_num_variables(mb) : 0;
    hprqp_model_destroy(mb);
    /* the binding ABI, as the reference's tests/test_binding_api.c drives it;
       without a GPU the solve fails loudly */
    HPRQPBindingModel *bm = NULL;
    HPRQPBindingParams *bp = NULL;
    HPRQPBindingResults *br = NULL;
    int bind = hprqp_model_create(&bm) | hprqp_params_create(&bp) | hprqp_results_create(&br);
    bind |= hprqp_model_build_from_qabc_csr(bm, 2, 2, 2, q_rp, q_ci, q_v, 1, 2, 2, a_rp, a_ci, a_v, c, AL, AU, l,
                                            u, 0.0);
    bind |= hprqp_params_set_verbose(bp, 0);
    size_t bn = hprqp_model_num_variables(bm), bmr = hprqp_model_num_constraints(bm);
    int solve = (int)hprqp_optimize(bm, bp, br);
    hprqp_results_destroy(br);
    hprqp_params_destroy(bp);
    hprqp_model_destroy(bm);
    printf("{\"build\": %d, \"qc\": %d, \"pre\": %d, \"matvec\": %d, \"y\": %g, \"m_qp\": %zu, \"m_qc\": %zu, "
           "\"cones\": %zu, \"dot\": %g, \"soc\": %d, \"bind\": %d, \"bn\": %zu, \"bm\": %zu, "
           "\"solve\": %d, \"gpu\": %d, \"soc_build\": %d, \"soc_var_cones\": %zu, \"soc_row_cones\": %zu, "
           "\"mps\": %d, \"mps_n\": %zu, \"mps_m\": %zu, \"mps_nnz_q\": %zu, \"bind_mps\": %d, "
           "\"bind_mps_n\": %zu}\n",
           (int)s1, (int)s2, (int)s3, (int)s4, y[0], qp.A.nrow, qcqp.A.nrow, qcqp.num_row_cones,
           vec_dot(a_v, a_v, 2), (int)model_validate_soc(&qcqp), bind, bn, bmr, solve,
           gpu_backend_available(), (int)s5, socm.num_var_cones, socm.num_row_cones, (int)s6, mps.Q.ncol,
           mps.A.nrow, mps.Q.nnz, bind_mps, mps_n_bind);
    model_free(&socm);
    model_free(&mps);
    model_free(&qp);
    model_free(&qcqp);
    return 0;
}
