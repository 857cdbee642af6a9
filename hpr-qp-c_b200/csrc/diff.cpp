// Implicit-differentiation adjoint of a single solve (include/hprqp_diff.h).
// The device side (MINRES on the scaled active-set KKT operator) is
// engine_adjoint in engine.cu; this file keeps the solve's state and turns
// the adjoint solution into gradients of the problem data.
#include "hprqp_diff.h"

#include <algorithm>
#include <cstdio>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

#include "engine.h"
#include "hprqp.h"

struct HPRQPSolveState {
    hpr::Engine *eng = nullptr;
    const HPRQPModel *model = nullptr;
    std::vector<double> x, y, z;
};

// rows [r0, r1) of y = M v, M host CSR
static void csr_rows(const HPRQPMatrixCSR &M, const double *v, double *y, size_t r0, size_t r1)
{
    for (size_t r = r0; r < r1; ++r) {
        double s = 0.0;
        for (size_t e = M.row_ptr[r]; e < M.row_ptr[r + 1]; ++e) s += M.values[e] * v[M.col_ind[e]];
        y[r] = s;
    }
}

template <class F>
static void parallel_rows(size_t count, F &&f)
{
    const unsigned nth = std::max(1u, std::min(std::thread::hardware_concurrency(), 16u));
    if (count < 4096 || nth == 1) {
        f(0, count);
        return;
    }
    std::vector<std::thread> th;
    const size_t chunk = (count + nth - 1) / nth;
    for (unsigned t = 0; t < nth; ++t) {
        const size_t a = std::min(count, t * chunk), b = std::min(count, a + chunk);
        if (a < b) th.emplace_back([&f, a, b] { f(a, b); });
    }
    for (auto &t : th) t.join();
}

extern "C" {

HPRQPStatus hprqp_solve_for_backward(const HPRQPModel *model, const HPRQPParams *params, HPRQPResults *results,
                                     HPRQPSolveState **state)
{
    if (!state) return HPRQP_STATUS_INVALID_ARGUMENT;
    *state = nullptr;
    hpr::Engine *eng = nullptr;
    const HPRQPStatus st = hpr::solve_gpu_keep(model, params, results, &eng);
    if (!eng) return st;
    HPRQPSolveState *s = new HPRQPSolveState();
    s->eng = eng;
    s->model = model;
    const size_t n = model->Q.ncol, m = model->A.nrow;
    s->x.assign(results->x, results->x + n);
    s->z.assign(results->z, results->z + n);
    if (m) s->y.assign(results->y, results->y + m);
    *state = s;
    return st;
}

HPRQPStatus hprqp_backward(HPRQPSolveState *s, const double *grad_x, const double *grad_y, double tol,
                           long long max_iter, HPRQPGradients *g)
{
    if (!s || !s->eng || !grad_x || !g) return HPRQP_STATUS_INVALID_ARGUMENT;
    const auto t0 = std::chrono::steady_clock::now();
    const HPRQPModel &M = *s->model;
    if (M.num_var_cones || M.num_row_cones) {
        fprintf(stderr, "hprqp-b200: hprqp_backward does not differentiate through second-order cones\n");
        return HPRQP_STATUS_NOT_IMPLEMENTED;
    }
    const size_t n = M.Q.ncol, m = M.A.nrow;
    if (!(tol > 0.0)) tol = 1e-12;
    if (max_iter <= 0) max_iter = 4 * (long long)(n + m) + 100;
    std::vector<double> lam(std::max<size_t>(n, 1)), mu(std::max<size_t>(m, 1));
    long long its = 0;
    double rel = 0.0;
    HPRQPStatus st = hpr::engine_adjoint(s->eng, grad_x, grad_y, tol, max_iter, lam.data(), mu.data(), &its, &rel);
    if (st != HPRQP_STATUS_OK) return st;
    // Q lam and A' mu with the model's (unscaled) matrices
    std::vector<double> qlam(std::max<size_t>(n, 1)), atmu(std::max<size_t>(n, 1), 0.0);
    parallel_rows(n, [&](size_t a, size_t b) { csr_rows(M.Q, lam.data(), qlam.data(), a, b); });
    if (m) parallel_rows(n, [&](size_t a, size_t b) { csr_rows(M.AT, mu.data(), atmu.data(), a, b); });
    const double *x = s->x.data(), *y = s->y.data(), *z = s->z.data();
    for (size_t i = 0; i < n; ++i) {
        if (g->dc) g->dc[i] = -lam[i];
        const double db = grad_x[i] - qlam[i] - atmu[i];
        if (g->dl) g->dl[i] = z[i] > 0.0 ? db : 0.0;
        if (g->du) g->du[i] = z[i] < 0.0 ? db : 0.0;
    }
    for (size_t r = 0; r < m; ++r) {
        if (g->dAL) g->dAL[r] = y[r] > 0.0 ? mu[r] : 0.0;
        if (g->dAU) g->dAU[r] = y[r] < 0.0 ? mu[r] : 0.0;
    }
    if (g->dQ_values)
        parallel_rows(n, [&](size_t a, size_t b) {
            for (size_t i = a; i < b; ++i)
                for (size_t e = M.Q.row_ptr[i]; e < M.Q.row_ptr[i + 1]; ++e) {
                    const size_t j = M.Q.col_ind[e];
                    g->dQ_values[e] = -0.5 * (lam[i] * x[j] + lam[j] * x[i]);
                }
        });
    if (g->dA_values)
        parallel_rows(m, [&](size_t a, size_t b) {
            for (size_t r = a; r < b; ++r)
                for (size_t e = M.A.row_ptr[r]; e < M.A.row_ptr[r + 1]; ++e) {
                    const size_t j = M.A.col_ind[e];
                    g->dA_values[e] = -mu[r] * x[j] + lam[j] * y[r];
                }
        });
    if (g->lam) memcpy(g->lam, lam.data(), n * sizeof(double));
    if (g->mu && m) memcpy(g->mu, mu.data(), m * sizeof(double));
    g->minres_iters = its;
    g->minres_relres = rel;
    g->backward_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return HPRQP_STATUS_OK;
}

void hprqp_solve_state_destroy(HPRQPSolveState *s)
{
    if (!s) return;
    hpr::engine_destroy(s->eng);
    delete s;
}

}  // extern "C"
