// Host outer loop of the HPR method and the reference-compatible entry
// points (solve, solve_gpu, params_set_defaults, results_*, print_*).
//
// The loop reproduces the control flow of the reference's
// solve_with_backend (src/shared/solver_backend.c:338-569): residual checks
// every check_iter iterations and at the adaptive print steps, restart rules
// (src/cpu/control.c:231-305), sigma update, restart, and milestone
// bookkeeping, so that iteration counts are comparable one to one.  Every
// vector operation runs on the device through engine.h; the host only
// handles scalars.
#include "engine.h"
#include "hprqp.h"

#include <cuda_runtime.h>

#include <chrono>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

namespace {

double now_s()
{
    using namespace std::chrono;
    return duration<double>(steady_clock::now().time_since_epoch()).count();
}

size_t adaptive_print_step(size_t iter)
{
    size_t step = 10;
    if (iter == 0) return step;
    while (iter / step >= 100 && step <= SIZE_MAX / 10) step *= 10;
    return step;
}

bool should_print(const HPRQPParams *p, size_t iter, double elapsed)
{
    if (p->print_frequency == -1 &&
        (iter % adaptive_print_step(iter) == 0 || iter == p->max_iter || elapsed > p->time_limit))
        return true;
    if (p->print_frequency > 0 &&
        (iter % (size_t)p->print_frequency == 0 || iter == p->max_iter || elapsed > p->time_limit))
        return true;
    return false;
}

int should_check_next(const HPRQPParams *p, const HPRQPRestart *r, size_t next)
{
    int t = 0;
    if (p->check_iter > 0 && next % p->check_iter == 0) t = 1;
    if (r->restart_flag > 0) t = 1;
    if (p->print_frequency == -1 && next % adaptive_print_step(next) == 0) t = 1;
    if (p->print_frequency > 0 && next % (size_t)p->print_frequency == 0) t = 1;
    return t;
}

void restart_init(HPRQPRestart *r)
{
    memset(r, 0, sizeof(*r));
    r->first_restart = 1;
    r->save_gap = r->current_gap = r->last_gap = r->best_gap = INFINITY;
    r->best_sigma = 1.0;
    r->weighted_norm = INFINITY;
}

// restart rules: sufficient (gap <= 0.2 last), necessary (<= 0.8 last and
// growing), long (inner >= {0.2|0.5} iter); first restart at check_iter.
void restart_check(HPRQPRestart *r, size_t iter, size_t check_iter, double sigma)
{
    if (check_iter == 0) return;
    r->restart_flag = 0;
    if (r->first_restart) {
        if (iter == check_iter) {
            r->first_restart = 0;
            r->restart_flag = 1;
            r->weighted_norm = r->current_gap;
            r->best_gap = r->current_gap;
            r->best_sigma = sigma;
        }
        return;
    }
    if (iter % check_iter != 0) return;
    if (r->current_gap < 0.0) r->current_gap = 1e-6;
    if (r->current_gap <= 0.2 * r->last_gap) {
        r->sufficient += 1;
        r->restart_flag = 1;
    }
    if (r->current_gap <= 0.8 * r->last_gap && r->current_gap > r->save_gap) {
        r->necessary += 1;
        r->restart_flag = 2;
    }
    const double fact =
        (r->weighted_norm > 0.0 && r->current_gap / r->weighted_norm > 1e-1) ? 0.5 : 0.2;
    if ((double)r->inner >= fact * (double)iter) {
        r->long_restart += 1;
        r->restart_flag = 3;
    }
    if (r->best_gap > r->current_gap) {
        r->best_gap = r->current_gap;
        r->best_sigma = sigma;
    }
    r->save_gap = r->current_gap;
}

void restart_post(HPRQPRestart *r, size_t iter, size_t check_iter, double gap)
{
    const bool at_check = check_iter > 0 && (iter + 1) % check_iter == 0;
    if (r->restart_flag > 0 || at_check) {
        if (r->restart_flag > 0) r->last_gap = gap;
        if (at_check) r->current_gap = gap;
    }
}

void print_log(size_t iter, const HPRQPResiduals *r, double sigma, double elapsed)
{
    printf("%5zu    %3.2e    %3.2e    %+7.6e    %+7.6e    %3.2e    %3.2e    %6.2f\n", iter, r->err_Rp_org_bar,
           r->err_Rd_org_bar, r->primal_obj_bar, r->dual_obj_bar, r->rel_gap_bar, sigma, elapsed);
}

const char *spmv_mode_name(HPRQPSpmvMode m)
{
    switch (m) {
    case HPRQP_SPMV_MODE_AUTO:
        return "auto";
    case HPRQP_SPMV_MODE_CUSPARSE:
        return "cusparse";
    case HPRQP_SPMV_MODE_CUSTOMIZED:
        return "customized";
    default:
        return "unknown";
    }
}

}  // namespace

extern "C" {

void params_set_defaults(HPRQPParams *p)
{
    // src/shared/solver.c:133-157
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->stoptol = 1e-8;
    p->max_iter = (size_t)INT_MAX;
    p->use_gpu = 1;
    p->device_number = 0;
    p->time_limit = 3600.0;
    p->check_iter = 100;
    p->print_frequency = -1;
    p->use_scaling = 1;
    p->verbose = 1;
    p->spmv_mode_q = HPRQP_SPMV_MODE_AUTO;
    p->spmv_mode_a = HPRQP_SPMV_MODE_AUTO;
    p->gram_mode = HPRQP_GRAM_AUTO;
    p->polishing = 1;
    p->polish_max_attempts = 12;
    p->polish_episode_seconds = 20.0;
    p->polish_total_seconds = 0.0;
    p->polish_memory_bytes = (size_t)8 * 1024 * 1024 * 1024;
}

void results_init(HPRQPResults *r)
{
    if (r) memset(r, 0, sizeof(*r));
}

void results_free(HPRQPResults *r)
{
    if (!r) return;
    free(r->x);
    free(r->y);
    free(r->z);
    free(r->w);
    results_init(r);
}

void print_model_info(const HPRQPModel *model)
{
    if (!model) return;
    printf("Model info:\n");
    printf("  variables: %zu\n", model->Q.ncol);
    printf("  constraints: %zu\n", model->A.nrow);
    printf("  nnz(Q): %zu\n", model->Q.nnz);
    printf("  nnz(A): %zu\n", model->A.nnz);
}

void print_params_info(const HPRQPParams *p)
{
    if (!p) return;
    printf("Parameter info:\n");
    printf("  stoptol: %.12g\n", p->stoptol);
    printf("  use_gpu: %s\n", p->use_gpu ? "on" : "off");
    printf("  device_number: %d\n", p->device_number);
    printf("  max_iter: %zu\n", p->max_iter);
    printf("  time_limit: %.12g\n", p->time_limit);
    printf("  check_iter: %zu\n", p->check_iter);
    printf("  print_frequency: %d\n", p->print_frequency);
    printf("  use_scaling: %s\n", p->use_scaling ? "on" : "off");
    printf("  verbose: %s\n", p->verbose ? "on" : "off");
    printf("  spmv mode Q: %s\n", spmv_mode_name(p->spmv_mode_q));
    printf("  spmv mode A: %s\n", spmv_mode_name(p->spmv_mode_a));
}

int gpu_backend_available(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return 0;
    }
    for (int d = 0; d < n; ++d) {
        cudaDeviceProp prop;
        if (cudaGetDeviceProperties(&prop, d) == cudaSuccess && prop.major == 10) return 1;
    }
    return 0;
}

}  // extern "C"

// solve_gpu, optionally handing the engine (scaled problem and final
// iterate) to the caller for the adjoint instead of destroying it.
HPRQPStatus hpr::solve_gpu_keep(const HPRQPModel *model, const HPRQPParams *params, HPRQPResults *results,
                                hpr::Engine **keep)
{
    if (keep) *keep = nullptr;
    const double t_begin = now_s();
    if (!model || !params || !results) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (params->gram_mode < HPRQP_GRAM_OFF || params->gram_mode > HPRQP_GRAM_REQUEST)
        return HPRQP_STATUS_INVALID_ARGUMENT;
    results_init(results);
    if (!matrix_csr_is_valid(&model->Q) || !matrix_csr_is_valid(&model->A) || !matrix_csr_is_valid(&model->AT) ||
        model->Q.ncol != model->A.ncol || !model->c || !model->l || !model->u ||
        (model->A.nrow > 0 && (!model->AL || !model->AU)))
        return HPRQP_STATUS_INVALID_ARGUMENT;
    if (params->verbose) {
        print_model_info(model);
        print_params_info(params);
    }
    if (!keep && hpr::single_cta_eligible(model, params)) {
        // the whole solve in one CTA of the batch kernel; the log comes back
        // with the results and is printed like the host loop prints it
        std::vector<double> log;
        if (params->verbose) log.resize(hpr::kSingleCtaLogCap * 8);
        size_t nlog = 0;
        const HPRQPStatus ret = hpr::solve_single_cta(model, params, results, params->verbose ? log.data() : nullptr,
                                                      hpr::kSingleCtaLogCap, &nlog);
        if (params->verbose && nlog > 0) {
            printf("HPRQP SOLVER starts (GPU mode, sm_100a engine, one CTA)...\n");
            printf(" iter     errRp        errRd         p_obj           d_obj          gap        sigma       time\n");
            for (size_t i = 0; i < nlog; ++i) {
                const double *r = log.data() + 8 * i;
                HPRQPResiduals res;
                memset(&res, 0, sizeof(res));
                res.err_Rp_org_bar = r[1];
                res.err_Rd_org_bar = r[2];
                res.primal_obj_bar = r[3];
                res.dual_obj_bar = r[4];
                res.rel_gap_bar = r[5];
                print_log((size_t)r[0], &res, r[6], r[7]);
            }
        }
        results->total_time = now_s() - t_begin;
        return ret;
    }
    hpr::Engine *eng = nullptr;
    hpr::SetupInfo info;
    memset(&info, 0, sizeof(info));
    HPRQPStatus st = hpr::engine_create(model, params, &eng, &info);
    if (st != HPRQP_STATUS_OK) {
        results->total_time = now_s() - t_begin;
        return st;
    }
    const size_t n = info.n, m = info.m;

    // ---- solve_with_backend (src/shared/solver_backend.c:338-569) ----
    HPRQPResiduals res;
    memset(&res, 0, sizeof(res));
    HPRQPRestart rst;
    restart_init(&rst);
    const double t0 = now_s();
    HPRQPStatus ret = HPRQP_STATUS_OK;
    int first_4 = 1, first_6 = 1;
    size_t iter_4 = 0, iter_6 = 0;
    double time_4 = 0.0, time_6 = 0.0;
    auto milestones = [&](size_t it) {
        if (first_4 && res.KKTx_and_gap_org_bar < 1e-4) {
            iter_4 = it;
            time_4 = now_s() - t0;
            first_4 = 0;
        }
        if (first_6 && res.KKTx_and_gap_org_bar < 1e-6) {
            iter_6 = it;
            time_6 = now_s() - t0;
            first_6 = 0;
        }
    };
    HPRQPStatus final_status = HPRQP_STATUS_MAX_ITER;
    size_t iter = 0;
    double sigma = info.sigma;
    st = hpr::engine_residuals(eng, &res, 0);
    if (st != HPRQP_STATUS_OK) {
        ret = st;
        goto done;
    }
    milestones(0);
    if (params->verbose) {
        printf("HPRQP SOLVER starts (GPU mode, sm_100a engine)...\n");
        printf(" iter     errRp        errRd         p_obj           d_obj          gap        sigma       time\n");
        print_log(0, &res, sigma, now_s() - t0);
    }
    rst.best_sigma = sigma;
    for (iter = 0;; ++iter) {
        bool print_yes = false;
        const double el = now_s() - t0;
        if (iter > 0) {
            print_yes = should_print(params, iter, el);
            if ((params->check_iter > 0 && iter % params->check_iter == 0) || print_yes) {
                st = hpr::engine_residuals(eng, &res, iter);
                if (st != HPRQP_STATUS_OK) {
                    ret = st;
                    goto done;
                }
                milestones(iter);
            } else {
                res.is_updated = 0;
            }
        }
        if (res.KKTx_and_gap_org_bar < params->stoptol) final_status = HPRQP_STATUS_OPTIMAL;
        else if (iter == params->max_iter) final_status = HPRQP_STATUS_MAX_ITER;
        else if (el > params->time_limit) final_status = HPRQP_STATUS_TIME_LIMIT;
        else final_status = HPRQP_STATUS_CONTINUE;

        restart_check(&rst, iter, params->check_iter, sigma);
        st = hpr::engine_update_sigma(eng, &rst, &res, &sigma);
        if (st != HPRQP_STATUS_OK) {
            ret = st;
            goto done;
        }
        if (rst.restart_flag > 0) {
            st = hpr::engine_restart_apply(eng);
            if (st != HPRQP_STATUS_OK) {
                ret = st;
                goto done;
            }
            rst.last_gap = rst.current_gap;
            rst.save_gap = INFINITY;
            rst.times += 1;
            rst.inner = 0;
        }
        if (params->verbose && (print_yes || final_status != HPRQP_STATUS_CONTINUE))
            print_log(iter, &res, sigma, now_s() - t0);
        if (final_status != HPRQP_STATUS_CONTINUE) break;

        const int to_check = should_check_next(params, &rst, iter + 1);
        st = hpr::engine_iteration_step(eng, rst.inner, to_check);
        if (st != HPRQP_STATUS_OK) {
            ret = st;
            goto done;
        }
        if (rst.restart_flag > 0 || (params->check_iter > 0 && (iter + 1) % params->check_iter == 0)) {
            double gap = 0.0;
            st = hpr::engine_m_norm(eng, &gap);
            if (st != HPRQP_STATUS_OK) {
                ret = st;
                goto done;
            }
            if (!std::isfinite(gap)) {
                ret = HPRQP_STATUS_INVALID_ARGUMENT;
                goto done;
            }
            restart_post(&rst, iter, params->check_iter, gap);
        }
        rst.inner += 1;
    }
    {
        // collect_results: src/shared/solver_backend.c:289-336
        const double elapsed = now_s() - t0;
        results->x = n ? (double *)calloc(n, sizeof(double)) : nullptr;
        results->w = n ? (double *)calloc(n, sizeof(double)) : nullptr;
        results->z = n ? (double *)calloc(n, sizeof(double)) : nullptr;
        results->y = m ? (double *)calloc(m, sizeof(double)) : nullptr;
        if ((n && (!results->x || !results->w || !results->z)) || (m && !results->y)) {
            results_free(results);
            ret = HPRQP_STATUS_ALLOCATION_FAILED;
            goto done;
        }
        st = hpr::engine_copy_output(eng, results->x, results->w, results->z, results->y);
        if (st != HPRQP_STATUS_OK) {
            results_free(results);
            ret = st;
            goto done;
        }
        results->iter = iter;
        results->time = elapsed;
        results->iter_4 = iter_4 == 0 ? iter : iter_4;
        results->iter_6 = iter_6 == 0 ? iter : iter_6;
        results->time_4 = time_4 == 0.0 ? elapsed : time_4;
        results->time_6 = time_6 == 0.0 ? elapsed : time_6;
        results->primal_obj = res.primal_obj_bar;
        results->residuals = res.KKTx_and_gap_org_bar;
        results->gap = res.rel_gap_bar;
        results->status = final_status;
        ret = final_status;
    }
done:
    if (keep && (ret == HPRQP_STATUS_OPTIMAL || ret == HPRQP_STATUS_MAX_ITER || ret == HPRQP_STATUS_TIME_LIMIT))
        *keep = eng;
    else
        hpr::engine_destroy(eng);
    results->total_time = now_s() - t_begin;
    return ret;
}

extern "C" {

HPRQPStatus solve_gpu(const HPRQPModel *model, const HPRQPParams *params, HPRQPResults *results)
{
    return hpr::solve_gpu_keep(model, params, results, nullptr);
}

HPRQPStatus solve(const HPRQPModel *model, const HPRQPParams *params, HPRQPResults *results)
{
    // src/shared/solver.c:245-260, without the CPU branch
    if (!params || !model || !results) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (!params->use_gpu) {
        results_init(results);
        fprintf(stderr, "hprqp-b200: use_gpu=0 requested, but this library has no CPU backend\n");
        return HPRQP_STATUS_NOT_IMPLEMENTED;
    }
    return solve_gpu(model, params, results);
}

}  // extern "C"
