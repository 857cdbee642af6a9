// Convex quadratic constraints as second-order cones (reference
// include/shared/qcqp.h, src/shared/qcqp.c:16-99).
//
// Constraint i:  C_i x + 1/2 x' R_i' R_i x + constant_i <= 0.  With
// s = -C_i x - constant_i, the rotated-cone identity
//     (1 + s)^2 - (s - 1)^2 = 4 s  >=  2 |R_i x|^2
// turns it into one Lorentz cone over the rows
//     t  = -C_i x - (constant_i - 1),   v0 = -C_i x - (constant_i + 1),
//     v  = sqrt(2) R_i x,               |(v0, v)| <= t,
// i.e. rows A_i x - rhs_i in K with A_i = [-C_i; -C_i; sqrt(2) R_i] and
// rhs_i = [constant_i - 1; constant_i + 1; 0].  The cone rows follow the
// linear rows (free bounds), so the model goes through build_from_QAbc_soc.
// The entry values are formed exactly as the reference forms them (so the
// models agree bit for bit): -c for the head rows, sqrt(2.0) * r for the
// factor rows, sqrt(d) for a diagonal D = R'R.
#include "hprqp.h"
#include "shared/build.h"
#include "shared/qcqp.h"
#include "shared/sparse.h"

#include <cmath>
#include <cstdint>
#include <vector>

namespace {

bool finite_csr(const HPRQPMatrixCSR *m)
{
    if (!m || !matrix_csr_is_valid(m)) return false;
    for (size_t k = 0; k < m->nnz; ++k)
        if (!std::isfinite(m->values[k])) return false;
    return true;
}

}  // namespace

extern "C" {

HPRQPStatus build_from_QAbc_qc_factors(const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c,
                                       const double *AL, const double *AU, const double *l, const double *u,
                                       double obj_constant, const HPRQPMatrixCSR *C, const double *constant,
                                       const HPRQPMatrixCSR *R, const size_t *offsets, HPRQPModel *model)
{
    if (!Q || !A || !model || !finite_csr(C) || !finite_csr(R) || !matrix_csr_is_valid(A) || C->ncol != Q->ncol ||
        R->ncol != Q->ncol || A->ncol != Q->ncol)
        return HPRQP_STATUS_INVALID_ARGUMENT;
    const size_t nq = C->nrow, m = A->nrow, n = Q->ncol;
    if (nq == 0) return build_from_QAbc(Q, A, c, AL, AU, l, u, obj_constant, model);
    if (!constant || !offsets || offsets[0] != 0 || offsets[nq] != R->nrow || (m && (!AL || !AU)))
        return HPRQP_STATUS_INVALID_ARGUMENT;
    for (size_t i = 0; i < nq; ++i)
        if (!std::isfinite(constant[i]) || offsets[i] > offsets[i + 1] || offsets[i + 1] > R->nrow)
            return HPRQP_STATUS_INVALID_ARGUMENT;
    if (R->nrow > SIZE_MAX - m || nq > (SIZE_MAX - m - R->nrow) / 2 || R->nnz > SIZE_MAX - A->nnz ||
        C->nnz > (SIZE_MAX - A->nnz - R->nnz) / 2)
        return HPRQP_STATUS_INVALID_ARGUMENT;
    const size_t rows = m + 2 * nq + R->nrow;
    std::vector<size_t> rp(rows + 1), ci, cones(nq + 1);
    std::vector<double> v, al(rows, -INFINITY), au(rows, INFINITY), rhs(rows, 0.0);
    ci.reserve(A->nnz + 2 * C->nnz + R->nnz);
    v.reserve(ci.capacity());
    // linear rows first, unchanged
    for (size_t r = 0; r < m; ++r) {
        rp[r] = ci.size();
        for (size_t k = A->row_ptr[r]; k < A->row_ptr[r + 1]; ++k) {
            ci.push_back(A->col_ind[k]);
            v.push_back(A->values[k]);
        }
        al[r] = AL[r];
        au[r] = AU[r];
    }
    size_t row = m;
    for (size_t i = 0; i < nq; ++i) {
        cones[i] = row;
        for (int head = 0; head < 2; ++head, ++row) {
            rp[row] = ci.size();
            for (size_t k = C->row_ptr[i]; k < C->row_ptr[i + 1]; ++k) {
                ci.push_back(C->col_ind[k]);
                v.push_back(-C->values[k]);
            }
            rhs[row] = constant[i] + (head ? 1.0 : -1.0);
        }
        for (size_t f = offsets[i]; f < offsets[i + 1]; ++f, ++row) {
            rp[row] = ci.size();
            for (size_t k = R->row_ptr[f]; k < R->row_ptr[f + 1]; ++k) {
                ci.push_back(R->col_ind[k]);
                v.push_back(std::sqrt(2.0) * R->values[k]);
            }
        }
    }
    cones[nq] = row;
    rp[rows] = ci.size();
    size_t dummy_i = 0;
    double dummy_v = 0.0;
    HPRQPMatrixCSR lifted{rows, n, ci.size(), rp.data(), ci.empty() ? &dummy_i : ci.data(),
                          v.empty() ? &dummy_v : v.data(), 0};
    HPRQPSOCSpec spec{};
    spec.num_var_cones = 0;
    spec.var_offsets = nullptr;
    spec.num_row_cones = nq;
    spec.row_offsets = cones.data();
    spec.rhs = rhs.data();
    return build_from_QAbc_soc(Q, &lifted, c, al.data(), au.data(), l, u, obj_constant, &spec, model);
}

HPRQPStatus build_from_QAbc_qc_diagonal(const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c,
                                        const double *AL, const double *AU, const double *l, const double *u,
                                        double obj_constant, const HPRQPMatrixCSR *C, const double *constant,
                                        const HPRQPMatrixCSR *D, HPRQPModel *model)
{
    if (!Q || !finite_csr(D) || !C || C->nrow != D->nrow || C->ncol != D->ncol || D->ncol != Q->ncol)
        return HPRQP_STATUS_INVALID_ARGUMENT;
    // row i of D lists the diagonal of D_i; R_i gets one row sqrt(d) e_j per
    // positive entry
    std::vector<size_t> offsets(D->nrow + 1), rp(1, 0), ci;
    std::vector<double> v;
    for (size_t i = 0; i < D->nrow; ++i) {
        offsets[i] = ci.size();
        for (size_t k = D->row_ptr[i]; k < D->row_ptr[i + 1]; ++k) {
            const double d = D->values[k];
            if (d < 0.0) return HPRQP_STATUS_INVALID_ARGUMENT;
            if (d > 0.0) {
                ci.push_back(D->col_ind[k]);
                v.push_back(std::sqrt(d));
                rp.push_back(ci.size());
            }
        }
    }
    offsets[D->nrow] = ci.size();
    size_t dummy_i = 0;
    double dummy_v = 0.0;
    HPRQPMatrixCSR R{ci.size(), D->ncol, ci.size(), rp.data(), ci.empty() ? &dummy_i : ci.data(),
                     v.empty() ? &dummy_v : v.data(), 0};
    return build_from_QAbc_qc_factors(Q, A, c, AL, AU, l, u, obj_constant, C, constant, &R, offsets.data(), model);
}

}  // extern "C"
