// Opaque-handle C ABI (hprqp_binding.h).  Same contract as the reference's
// src/shared/binding.c:19-346: handles are created/destroyed in pairs, the
// model builder takes raw size_t CSR arrays (NULL allowed for empty parts),
// results are read back through getters.
#include "hprqp_binding.h"

#include "hprqp.h"

#include <cstdlib>

struct HPRQPBindingModel {
    HPRQPModel model;
};

struct HPRQPBindingParams {
    HPRQPParams params;
};

struct HPRQPBindingResults {
    HPRQPResults results;
    size_t n;
    size_t m;
    HPRQPStatus status;
};

extern "C" {

const char *hprqp_status_name(HPRQPStatus status)
{
    switch (status) {
    case HPRQP_STATUS_OK:
        return "OK";
    case HPRQP_STATUS_INVALID_ARGUMENT:
        return "INVALID_ARGUMENT";
    case HPRQP_STATUS_ALLOCATION_FAILED:
        return "ALLOCATION_FAILED";
    case HPRQP_STATUS_NOT_IMPLEMENTED:
        return "NOT_IMPLEMENTED";
    case HPRQP_STATUS_MAX_ITER:
        return "MAX_ITER";
    case HPRQP_STATUS_TIME_LIMIT:
        return "TIME_LIMIT";
    case HPRQP_STATUS_OPTIMAL:
        return "OPTIMAL";
    case HPRQP_STATUS_CONTINUE:
        return "CONTINUE";
    default:
        return "UNKNOWN";
    }
}

int hprqp_gpu_backend_available(void) { return gpu_backend_available(); }

HPRQPStatus hprqp_model_create(HPRQPBindingModel **out)
{
    if (!out) return HPRQP_STATUS_INVALID_ARGUMENT;
    HPRQPBindingModel *m = (HPRQPBindingModel *)malloc(sizeof(*m));
    if (!m) return HPRQP_STATUS_ALLOCATION_FAILED;
    model_init(&m->model);
    *out = m;
    return HPRQP_STATUS_OK;
}

void hprqp_model_destroy(HPRQPBindingModel *m)
{
    if (!m) return;
    model_free(&m->model);
    free(m);
}

HPRQPStatus hprqp_model_read_from_mps(HPRQPBindingModel *m, const char *path)
{
    if (!m || !path) return HPRQP_STATUS_INVALID_ARGUMENT;
    return build_from_mps(path, &m->model);
}

static HPRQPStatus csr_view(HPRQPMatrixCSR *v, size_t nrow, size_t ncol, size_t nnz, const size_t *rp,
                            const size_t *ci, const double *val, size_t *empty_idx, double *empty_val)
{
    if ((nrow > 0 && !rp) || (nnz > 0 && (!ci || !val))) return HPRQP_STATUS_INVALID_ARGUMENT;
    v->nrow = nrow;
    v->ncol = ncol;
    v->nnz = nnz;
    v->row_ptr = (size_t *)(rp ? rp : empty_idx);
    v->col_ind = (size_t *)(ci ? ci : empty_idx);
    v->values = (double *)(val ? val : empty_val);
    v->owns_data = 0;
    return HPRQP_STATUS_OK;
}

HPRQPStatus hprqp_model_build_from_qabc_csr(HPRQPBindingModel *model, size_t q_nrow, size_t q_ncol,
                                            size_t q_nnz, const size_t *q_row_ptr, const size_t *q_col_ind,
                                            const double *q_values, size_t a_nrow, size_t a_ncol,
                                            size_t a_nnz, const size_t *a_row_ptr, const size_t *a_col_ind,
                                            const double *a_values, const double *c, const double *AL,
                                            const double *AU, const double *l, const double *u,
                                            double obj_constant)
{
    if (!model || !c || !l || !u) return HPRQP_STATUS_INVALID_ARGUMENT;
    HPRQPMatrixCSR q, a;
    size_t qe = 0, ae = 0;
    double qv = 0.0, av = 0.0;
    HPRQPStatus st = csr_view(&q, q_nrow, q_ncol, q_nnz, q_row_ptr, q_col_ind, q_values, &qe, &qv);
    if (st != HPRQP_STATUS_OK) return st;
    st = csr_view(&a, a_nrow, a_ncol, a_nnz, a_row_ptr, a_col_ind, a_values, &ae, &av);
    if (st != HPRQP_STATUS_OK) return st;
    return build_from_QAbc(&q, &a, c, AL, AU, l, u, obj_constant, &model->model);
}

size_t hprqp_model_num_variables(const HPRQPBindingModel *m) { return m ? m->model.Q.ncol : 0; }
size_t hprqp_model_num_constraints(const HPRQPBindingModel *m) { return m ? m->model.A.nrow : 0; }

HPRQPStatus hprqp_params_create(HPRQPBindingParams **out)
{
    if (!out) return HPRQP_STATUS_INVALID_ARGUMENT;
    HPRQPBindingParams *p = (HPRQPBindingParams *)malloc(sizeof(*p));
    if (!p) return HPRQP_STATUS_ALLOCATION_FAILED;
    params_set_defaults(&p->params);
    *out = p;
    return HPRQP_STATUS_OK;
}

void hprqp_params_destroy(HPRQPBindingParams *p) { free(p); }

HPRQPStatus hprqp_params_set_defaults(HPRQPBindingParams *p)
{
    if (!p) return HPRQP_STATUS_INVALID_ARGUMENT;
    params_set_defaults(&p->params);
    return HPRQP_STATUS_OK;
}

#define HPR_SETTER(name, type)                                                  \
    HPRQPStatus hprqp_params_set_##name(HPRQPBindingParams *p, type value)      \
    {                                                                           \
        if (!p) return HPRQP_STATUS_INVALID_ARGUMENT;                           \
        p->params.name = value;                                                 \
        return HPRQP_STATUS_OK;                                                 \
    }
HPR_SETTER(stoptol, double)
HPR_SETTER(max_iter, size_t)
HPR_SETTER(use_gpu, int)
HPR_SETTER(device_number, int)
HPR_SETTER(time_limit, double)
HPR_SETTER(check_iter, size_t)
HPR_SETTER(print_frequency, int)
HPR_SETTER(use_scaling, int)
HPR_SETTER(verbose, int)
HPR_SETTER(spmv_mode_q, HPRQPSpmvMode)
HPR_SETTER(spmv_mode_a, HPRQPSpmvMode)
#undef HPR_SETTER

HPRQPStatus hprqp_results_create(HPRQPBindingResults **out)
{
    if (!out) return HPRQP_STATUS_INVALID_ARGUMENT;
    HPRQPBindingResults *r = (HPRQPBindingResults *)malloc(sizeof(*r));
    if (!r) return HPRQP_STATUS_ALLOCATION_FAILED;
    results_init(&r->results);
    r->n = r->m = 0;
    r->status = HPRQP_STATUS_OK;
    *out = r;
    return HPRQP_STATUS_OK;
}

void hprqp_results_destroy(HPRQPBindingResults *r)
{
    if (!r) return;
    results_free(&r->results);
    free(r);
}

HPRQPStatus hprqp_optimize(const HPRQPBindingModel *model, const HPRQPBindingParams *params,
                           HPRQPBindingResults *r)
{
    if (!model || !params || !r) return HPRQP_STATUS_INVALID_ARGUMENT;
    results_free(&r->results);
    r->n = model->model.Q.ncol;
    r->m = model->model.A.nrow;
    r->status = solve(&model->model, &params->params, &r->results);
    return r->status;
}

HPRQPStatus hprqp_results_status(const HPRQPBindingResults *r)
{
    return r ? r->status : HPRQP_STATUS_INVALID_ARGUMENT;
}
size_t hprqp_results_num_variables(const HPRQPBindingResults *r) { return r ? r->n : 0; }
size_t hprqp_results_num_constraints(const HPRQPBindingResults *r) { return r ? r->m : 0; }
size_t hprqp_results_iter(const HPRQPBindingResults *r) { return r ? r->results.iter : 0; }
size_t hprqp_results_iter_4(const HPRQPBindingResults *r) { return r ? r->results.iter_4 : 0; }
size_t hprqp_results_iter_6(const HPRQPBindingResults *r) { return r ? r->results.iter_6 : 0; }
double hprqp_results_time(const HPRQPBindingResults *r) { return r ? r->results.time : 0.0; }
double hprqp_results_time_4(const HPRQPBindingResults *r) { return r ? r->results.time_4 : 0.0; }
double hprqp_results_time_6(const HPRQPBindingResults *r) { return r ? r->results.time_6 : 0.0; }
double hprqp_results_objective(const HPRQPBindingResults *r) { return r ? r->results.primal_obj : 0.0; }
double hprqp_results_residual(const HPRQPBindingResults *r) { return r ? r->results.residuals : 0.0; }
double hprqp_results_gap(const HPRQPBindingResults *r) { return r ? r->results.gap : 0.0; }
const double *hprqp_results_x_data(const HPRQPBindingResults *r) { return r ? r->results.x : nullptr; }
const double *hprqp_results_y_data(const HPRQPBindingResults *r) { return r ? r->results.y : nullptr; }
const double *hprqp_results_z_data(const HPRQPBindingResults *r) { return r ? r->results.z : nullptr; }
const double *hprqp_results_w_data(const HPRQPBindingResults *r) { return r ? r->results.w : nullptr; }

}  // extern "C"
