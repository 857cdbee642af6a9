// Host model construction and preprocessing.
//
// Semantics follow the reference builder (src/shared/build.c:137-400,
// 504-621 and src/shared/sparse.c:21-181): Q is replaced by (Q + Q')/2 with
// entries of magnitude <= 1e-15 dropped before and after merging, rows of A
// that are empty or free on both sides are deleted, and the model is
// validated.  The implementation is this project's: the symmetrisation is a
// per-row merge of Q's row and Q''s row instead of a global sort of all
// entries, and the bounds/column-range checks run before anything is copied.
#include "hprqp.h"
#include "shared/build.h"
#include "shared/vector.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

extern "C" {

static void csr_reset(HPRQPMatrixCSR *m)
{
    m->nrow = m->ncol = m->nnz = 0;
    m->row_ptr = nullptr;
    m->col_ind = nullptr;
    m->values = nullptr;
    m->owns_data = 0;
}

HPRQPStatus matrix_csr_alloc(HPRQPMatrixCSR *m, size_t nrow, size_t ncol, size_t nnz)
{
    if (!m) return HPRQP_STATUS_INVALID_ARGUMENT;
    csr_reset(m);
    m->row_ptr = (size_t *)calloc(nrow + 1, sizeof(size_t));
    m->col_ind = (size_t *)calloc(nnz ? nnz : 1, sizeof(size_t));
    m->values = (double *)calloc(nnz ? nnz : 1, sizeof(double));
    if (!m->row_ptr || !m->col_ind || !m->values) {
        free(m->row_ptr);
        free(m->col_ind);
        free(m->values);
        csr_reset(m);
        return HPRQP_STATUS_ALLOCATION_FAILED;
    }
    m->nrow = nrow;
    m->ncol = ncol;
    m->nnz = nnz;
    m->owns_data = 1;
    return HPRQP_STATUS_OK;
}

void matrix_csr_free(HPRQPMatrixCSR *m)
{
    if (!m) return;
    if (m->owns_data) {
        free(m->row_ptr);
        free(m->col_ind);
        free(m->values);
    }
    csr_reset(m);
}

int matrix_csr_is_valid(const HPRQPMatrixCSR *m)
{
    if (!m || !m->row_ptr || !m->col_ind || !m->values) return 0;
    return m->row_ptr[0] == 0 && m->row_ptr[m->nrow] == m->nnz;
}

HPRQPStatus matrix_csr_copy(HPRQPMatrixCSR *d, const HPRQPMatrixCSR *s)
{
    if (!d || !s || !matrix_csr_is_valid(s)) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (d == s) return HPRQP_STATUS_OK;
    HPRQPStatus st = matrix_csr_alloc(d, s->nrow, s->ncol, s->nnz);
    if (st != HPRQP_STATUS_OK) return st;
    memcpy(d->row_ptr, s->row_ptr, (s->nrow + 1) * sizeof(size_t));
    if (s->nnz) {
        memcpy(d->col_ind, s->col_ind, s->nnz * sizeof(size_t));
        memcpy(d->values, s->values, s->nnz * sizeof(double));
    }
    return HPRQP_STATUS_OK;
}

// Stable counting-sort transpose (entries of a destination row keep source
// row order), as matrix_csr_transpose in src/shared/sparse.c:81-125.
HPRQPStatus matrix_csr_transpose(HPRQPMatrixCSR *d, const HPRQPMatrixCSR *s)
{
    if (!d || !s || !matrix_csr_is_valid(s)) return HPRQP_STATUS_INVALID_ARGUMENT;
    HPRQPStatus st = matrix_csr_alloc(d, s->ncol, s->nrow, s->nnz);
    if (st != HPRQP_STATUS_OK) return st;
    for (size_t k = 0; k < s->nnz; ++k) d->row_ptr[s->col_ind[k] + 1]++;
    for (size_t r = 0; r < d->nrow; ++r) d->row_ptr[r + 1] += d->row_ptr[r];
    std::vector<size_t> next(d->row_ptr, d->row_ptr + d->nrow);
    for (size_t r = 0; r < s->nrow; ++r)
        for (size_t k = s->row_ptr[r]; k < s->row_ptr[r + 1]; ++k) {
            const size_t pos = next[s->col_ind[k]]++;
            d->col_ind[pos] = r;
            d->values[pos] = s->values[k];
        }
    return HPRQP_STATUS_OK;
}

HPRQPStatus matrix_csr_matvec(const HPRQPMatrixCSR *m, const double *x, double *y)
{
    if (!matrix_csr_is_valid(m) || !x || !y) return HPRQP_STATUS_INVALID_ARGUMENT;
    for (size_t r = 0; r < m->nrow; ++r) {
        double s = 0.0;
        for (size_t k = m->row_ptr[r]; k < m->row_ptr[r + 1]; ++k) s += m->values[k] * x[m->col_ind[k]];
        y[r] = s;
    }
    return HPRQP_STATUS_OK;
}

HPRQPStatus matrix_csr_transpose_matvec(const HPRQPMatrixCSR *m, const double *x, double *y)
{
    if (!matrix_csr_is_valid(m) || !x || !y) return HPRQP_STATUS_INVALID_ARGUMENT;
    for (size_t c = 0; c < m->ncol; ++c) y[c] = 0.0;
    for (size_t r = 0; r < m->nrow; ++r)
        for (size_t k = m->row_ptr[r]; k < m->row_ptr[r + 1]; ++k) y[m->col_ind[k]] += m->values[k] * x[r];
    return HPRQP_STATUS_OK;
}

void model_init(HPRQPModel *model)
{
    if (model) memset(model, 0, sizeof(*model));
}

void model_free(HPRQPModel *model)
{
    if (!model) return;
    if (model->owns_data) {
        matrix_csr_free(&model->Q);
        matrix_csr_free(&model->A);
        matrix_csr_free(&model->AT);
        free(model->c);
        free(model->AL);
        free(model->AU);
        free(model->l);
        free(model->u);
        free(model->var_cone_offsets);
        free(model->row_cone_offsets);
        free(model->soc_rhs);
    }
    model_init(model);
}

static size_t *copy_offsets(const size_t *src, size_t count);

static double *copy_vec(const double *src, size_t n)
{
    if (n == 0) return nullptr;
    double *d = (double *)malloc(n * sizeof(double));
    if (d) memcpy(d, src, n * sizeof(double));
    return d;
}

HPRQPStatus model_copy(HPRQPModel *dest, const HPRQPModel *src)
{
    if (!dest || !src || !src->owns_data) return HPRQP_STATUS_INVALID_ARGUMENT;
    model_free(dest);
    dest->owns_data = 1;
    const size_t n = src->Q.ncol, m = src->A.nrow;
    HPRQPStatus st;
    if ((st = matrix_csr_copy(&dest->Q, &src->Q)) || (st = matrix_csr_copy(&dest->A, &src->A)) ||
        (st = matrix_csr_copy(&dest->AT, &src->AT))) {
        model_free(dest);
        return st;
    }
    dest->c = copy_vec(src->c, n);
    dest->l = copy_vec(src->l, n);
    dest->u = copy_vec(src->u, n);
    dest->AL = copy_vec(src->AL, m);
    dest->AU = copy_vec(src->AU, m);
    if ((n && (!dest->c || !dest->l || !dest->u)) || (m && (!dest->AL || !dest->AU))) {
        model_free(dest);
        return HPRQP_STATUS_ALLOCATION_FAILED;
    }
    dest->obj_constant = src->obj_constant;
    if (src->num_var_cones) {
        dest->var_cone_offsets = copy_offsets(src->var_cone_offsets, src->num_var_cones);
        dest->num_var_cones = src->num_var_cones;
    }
    if (src->num_row_cones) {
        dest->row_cone_offsets = copy_offsets(src->row_cone_offsets, src->num_row_cones);
        dest->soc_rhs = copy_vec(src->soc_rhs, m);
        dest->num_row_cones = src->num_row_cones;
    }
    if ((src->num_var_cones && !dest->var_cone_offsets) ||
        (src->num_row_cones && (!dest->row_cone_offsets || !dest->soc_rhs))) {
        model_free(dest);
        return HPRQP_STATUS_ALLOCATION_FAILED;
    }
    return HPRQP_STATUS_OK;
}

// (Q + Q') * factor, dropping |entry| <= tol before and after merging.
static HPRQPStatus symmetrize(HPRQPMatrixCSR *out, const HPRQPMatrixCSR *q, double factor, double tol)
{
    const size_t n = q->nrow;
    HPRQPMatrixCSR qt;
    csr_reset(&qt);
    HPRQPStatus st = matrix_csr_transpose(&qt, q);
    if (st != HPRQP_STATUS_OK) return st;
    struct E {
        size_t col;
        int src;   // 0: from Q's row, 1: from Q''s row (fixed merge order)
        size_t k;  // position inside the source row
        double v;
    };
    std::vector<size_t> rp(n + 1, 0);
    std::vector<size_t> cols;
    std::vector<double> vals;
    cols.reserve(2 * q->nnz);
    vals.reserve(2 * q->nnz);
    std::vector<E> row;
    for (size_t i = 0; i < n; ++i) {
        row.clear();
        for (size_t k = q->row_ptr[i]; k < q->row_ptr[i + 1]; ++k) {
            const double v = factor * q->values[k];
            if (std::fabs(v) > tol) row.push_back({q->col_ind[k], 0, k, v});
        }
        for (size_t k = qt.row_ptr[i]; k < qt.row_ptr[i + 1]; ++k) {
            const double v = factor * qt.values[k];
            if (std::fabs(v) > tol) row.push_back({qt.col_ind[k], 1, k, v});
        }
        std::sort(row.begin(), row.end(), [](const E &a, const E &b) {
            if (a.col != b.col) return a.col < b.col;
            if (a.src != b.src) return a.src < b.src;
            return a.k < b.k;
        });
        size_t p = 0;
        while (p < row.size()) {
            size_t e = p;
            double s = row[p].v;
            while (e + 1 < row.size() && row[e + 1].col == row[p].col) s += row[++e].v;
            if (std::fabs(s) > tol && s != 0.0) {
                cols.push_back(row[p].col);
                vals.push_back(s);
            }
            p = e + 1;
        }
        rp[i + 1] = cols.size();
    }
    matrix_csr_free(&qt);
    st = matrix_csr_alloc(out, n, q->ncol, cols.size());
    if (st != HPRQP_STATUS_OK) return st;
    memcpy(out->row_ptr, rp.data(), (n + 1) * sizeof(size_t));
    if (!cols.empty()) {
        memcpy(out->col_ind, cols.data(), cols.size() * sizeof(size_t));
        memcpy(out->values, vals.data(), vals.size() * sizeof(double));
    }
    return HPRQP_STATUS_OK;
}

static bool csr_indices_ok(const HPRQPMatrixCSR *m)
{
    for (size_t r = 0; r < m->nrow; ++r)
        if (m->row_ptr[r + 1] < m->row_ptr[r]) return false;
    for (size_t k = 0; k < m->nnz; ++k)
        if (m->col_ind[k] >= m->ncol) return false;
    return true;
}

static HPRQPStatus build_impl(const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c, const double *AL,
                              const double *AU, const double *l, const double *u, double obj_constant,
                              bool keep_all_rows, HPRQPModel *model)
{
    // argument checks: src/shared/build.c:513-531, 339-379
    if (!Q || !A || !model || !c || !l || !u) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (!matrix_csr_is_valid(Q) || !matrix_csr_is_valid(A)) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (Q->nrow != Q->ncol || Q->nrow != A->ncol) return HPRQP_STATUS_INVALID_ARGUMENT;
    const size_t n = A->ncol, m = A->nrow;
    if (m > 0 && (!AL || !AU)) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (!csr_indices_ok(Q) || !csr_indices_ok(A)) return HPRQP_STATUS_INVALID_ARGUMENT;
    for (size_t k = 0; k < Q->nnz; ++k)
        if (!std::isfinite(Q->values[k])) return HPRQP_STATUS_INVALID_ARGUMENT;
    for (size_t k = 0; k < A->nnz; ++k)
        if (!std::isfinite(A->values[k])) return HPRQP_STATUS_INVALID_ARGUMENT;
    for (size_t i = 0; i < n; ++i)
        if (!std::isfinite(c[i]) || std::isnan(l[i]) || std::isnan(u[i]) || l[i] > u[i])
            return HPRQP_STATUS_INVALID_ARGUMENT;
    for (size_t r = 0; r < m; ++r)
        if (std::isnan(AL[r]) || std::isnan(AU[r]) || AL[r] > AU[r]) return HPRQP_STATUS_INVALID_ARGUMENT;

    model_free(model);
    model->owns_data = 1;
    HPRQPStatus st = symmetrize(&model->Q, Q, 0.5, 1e-15);
    if (st != HPRQP_STATUS_OK) {
        model_free(model);
        return st;
    }
    // delete empty rows and rows free on both sides: build.c:254-337
    size_t kept = 0, kept_nnz = 0;
    for (size_t r = 0; r < m; ++r) {
        const size_t len = A->row_ptr[r + 1] - A->row_ptr[r];
        const bool free_row = std::isinf(AL[r]) && AL[r] < 0 && std::isinf(AU[r]) && AU[r] > 0;
        if (keep_all_rows || (len > 0 && !free_row)) {
            ++kept;
            kept_nnz += len;
        }
    }
    st = matrix_csr_alloc(&model->A, kept, n, kept_nnz);
    if (st != HPRQP_STATUS_OK) {
        model_free(model);
        return st;
    }
    model->AL = kept ? (double *)malloc(kept * sizeof(double)) : nullptr;
    model->AU = kept ? (double *)malloc(kept * sizeof(double)) : nullptr;
    model->c = copy_vec(c, n);
    model->l = copy_vec(l, n);
    model->u = copy_vec(u, n);
    if ((kept && (!model->AL || !model->AU)) || (n && (!model->c || !model->l || !model->u))) {
        model_free(model);
        return HPRQP_STATUS_ALLOCATION_FAILED;
    }
    size_t row = 0, pos = 0;
    for (size_t r = 0; r < m; ++r) {
        const size_t len = A->row_ptr[r + 1] - A->row_ptr[r];
        const bool free_row = std::isinf(AL[r]) && AL[r] < 0 && std::isinf(AU[r]) && AU[r] > 0;
        if (!keep_all_rows && (len == 0 || free_row)) continue;
        model->AL[row] = AL[r];
        model->AU[row] = AU[r];
        memcpy(model->A.col_ind + pos, A->col_ind + A->row_ptr[r], len * sizeof(size_t));
        memcpy(model->A.values + pos, A->values + A->row_ptr[r], len * sizeof(double));
        pos += len;
        model->A.row_ptr[++row] = pos;
    }
    st = matrix_csr_transpose(&model->AT, &model->A);
    if (st != HPRQP_STATUS_OK) {
        model_free(model);
        return st;
    }
    model->obj_constant = obj_constant;
    return HPRQP_STATUS_OK;
}

HPRQPStatus build_from_QAbc(const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c, const double *AL,
                            const double *AU, const double *l, const double *u, double obj_constant,
                            HPRQPModel *model)
{
    return build_impl(Q, A, c, AL, AU, l, u, obj_constant, false, model);
}

// Second-order cones (reference include/shared/types.h:35-48, build.c:39-99,
// 398): cones are contiguous suffix blocks of the variables and of the rows,
// given by strictly increasing offsets that end at n (m); cone variables have
// bounds (-inf, inf); on cone rows AL = -inf, AU = inf and the affine part is
// A x - rhs in K; rhs is zero on the linear rows.  Rows are not deleted.
static bool cone_offsets_ok(size_t count, const size_t *off, size_t length)
{
    if (count == 0) return true;
    if (!off || count > length || off[0] >= length || off[count] != length) return false;
    for (size_t k = 0; k < count; ++k)
        if (off[k] >= off[k + 1] || off[k + 1] > length) return false;
    return true;
}

static HPRQPStatus validate_cones(const HPRQPModel *model)
{
    const size_t n = model->Q.ncol, m = model->A.nrow;
    if (!cone_offsets_ok(model->num_var_cones, model->var_cone_offsets, n) ||
        !cone_offsets_ok(model->num_row_cones, model->row_cone_offsets, m))
        return HPRQP_STATUS_INVALID_ARGUMENT;
    if (model->num_var_cones && (!model->l || !model->u)) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (model->num_row_cones && (!model->AL || !model->AU)) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (model->num_var_cones)
        for (size_t i = model->var_cone_offsets[0]; i < n; ++i)
            if (model->l[i] != -INFINITY || model->u[i] != INFINITY) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (model->num_row_cones) {
        if (!model->soc_rhs) return HPRQP_STATUS_INVALID_ARGUMENT;
        for (size_t r = 0; r < m; ++r) {
            if (!std::isfinite(model->soc_rhs[r])) return HPRQP_STATUS_INVALID_ARGUMENT;
            if (r < model->row_cone_offsets[0]) {
                if (model->soc_rhs[r] != 0.0) return HPRQP_STATUS_INVALID_ARGUMENT;
            } else if (model->AL[r] != -INFINITY || model->AU[r] != INFINITY) {
                return HPRQP_STATUS_INVALID_ARGUMENT;
            }
        }
    }
    return HPRQP_STATUS_OK;
}

static size_t *copy_offsets(const size_t *src, size_t count)
{
    size_t *d = (size_t *)malloc((count + 1) * sizeof(size_t));
    if (d) memcpy(d, src, (count + 1) * sizeof(size_t));
    return d;
}

HPRQPStatus build_from_QAbc_soc(const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c,
                                const double *AL, const double *AU, const double *l, const double *u,
                                double obj_constant, const HPRQPSOCSpec *soc, HPRQPModel *model)
{
    const bool cones = soc && (soc->num_var_cones || soc->num_row_cones);
    if (!cones) return build_from_QAbc(Q, A, c, AL, AU, l, u, obj_constant, model);
    if (!Q || !A || !model) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (!cone_offsets_ok(soc->num_var_cones, soc->var_offsets, Q->ncol) ||
        !cone_offsets_ok(soc->num_row_cones, soc->row_offsets, A->nrow) || (soc->num_row_cones && !soc->rhs))
        return HPRQP_STATUS_INVALID_ARGUMENT;
    HPRQPStatus st = build_impl(Q, A, c, AL, AU, l, u, obj_constant, true, model);
    if (st != HPRQP_STATUS_OK) return st;
    if (soc->num_var_cones) {
        model->var_cone_offsets = copy_offsets(soc->var_offsets, soc->num_var_cones);
        if (!model->var_cone_offsets) {
            model_free(model);
            return HPRQP_STATUS_ALLOCATION_FAILED;
        }
        model->num_var_cones = soc->num_var_cones;
    }
    if (soc->num_row_cones) {
        model->row_cone_offsets = copy_offsets(soc->row_offsets, soc->num_row_cones);
        model->soc_rhs = copy_vec(soc->rhs, A->nrow);
        if (!model->row_cone_offsets || !model->soc_rhs) {
            model_free(model);
            return HPRQP_STATUS_ALLOCATION_FAILED;
        }
        model->num_row_cones = soc->num_row_cones;
    }
    st = validate_cones(model);
    if (st != HPRQP_STATUS_OK) model_free(model);
    return st;
}

// The reference's lower-level builder entry points (include/shared/build.h,
// src/shared/build.c:39-99, 339-400, 594-600): build_model_from_arrays is
// build_from_QAbc; preprocess_model redoes the builder's checks and
// reductions on a model that already owns its arrays.
HPRQPStatus build_model_from_arrays(const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c,
                                    const double *AL, const double *AU, const double *l, const double *u,
                                    double obj_constant, HPRQPModel *model)
{
    return build_impl(Q, A, c, AL, AU, l, u, obj_constant, false, model);
}

HPRQPStatus model_validate_soc(const HPRQPModel *model)
{
    return model ? validate_cones(model) : HPRQP_STATUS_INVALID_ARGUMENT;
}

HPRQPStatus preprocess_model(HPRQPModel *model)
{
    if (!model || !model->owns_data || !matrix_csr_is_valid(&model->AT)) return HPRQP_STATUS_INVALID_ARGUMENT;
    HPRQPStatus st = validate_cones(model);
    if (st != HPRQP_STATUS_OK) return st;
    const bool cones = model->num_var_cones || model->num_row_cones;
    // rebuild from the model's own arrays (cone models keep every row), then
    // hand the cone blocks over unchanged
    HPRQPModel out;
    model_init(&out);
    st = build_impl(&model->Q, &model->A, model->c, model->AL, model->AU, model->l, model->u, model->obj_constant,
                    cones, &out);
    if (st != HPRQP_STATUS_OK) return st;
    out.num_var_cones = model->num_var_cones;
    out.var_cone_offsets = model->var_cone_offsets;
    out.num_row_cones = model->num_row_cones;
    out.row_cone_offsets = model->row_cone_offsets;
    out.soc_rhs = model->soc_rhs;
    model->var_cone_offsets = model->row_cone_offsets = nullptr;
    model->soc_rhs = nullptr;
    model_free(model);
    *model = out;
    return HPRQP_STATUS_OK;
}

// vector helpers (include/shared/vector.h; reference src/shared/vector.c)
void vec_fill(double *x, size_t n, double value) { std::fill(x, x + n, value); }

void vec_copy(double *dest, const double *src, size_t n) { std::copy(src, src + n, dest); }

void vec_axpby(double *y, const double *x, size_t n, double a, double b)
{
    for (size_t i = 0; i < n; ++i) y[i] = a * x[i] + b * y[i];
}

double vec_dot(const double *x, const double *y, size_t n)
{
    double s = 0.0;
    for (size_t i = 0; i < n; ++i) s += x[i] * y[i];
    return s;
}

double vec_norm2(const double *x, size_t n) { return std::sqrt(vec_dot(x, x, n)); }

double vec_norm_inf(const double *x, size_t n)
{
    double m = 0.0;
    for (size_t i = 0; i < n; ++i)
        if (std::fabs(x[i]) > m) m = std::fabs(x[i]);
    return m;
}

void vec_project_box(double *y, const double *x, const double *lower, const double *upper, size_t n)
{
    for (size_t i = 0; i < n; ++i) y[i] = std::min(std::max(x[i], lower[i]), upper[i]);
}

// build_from_mps lives in mps.cpp

}  // extern "C"
