// Internal interface between the host outer loop (solver.cpp) and the CUDA
// engine (engine.cu).  Not installed; no CUDA types cross this header.
#pragma once

#include <cstddef>
#include <cstdint>

#include "shared/types.h"

namespace hpr {

struct Engine;  // device-resident problem + iterate state (engine.cu)

struct SetupInfo {
    double sigma;
    double lambda_max_A;
    double lambda_max_Q;
    int Q_is_diag;
    int noC;
    size_t n, m;
    HPRQPScaling scaling_scalars;  // only the scalar fields are filled
};

// Upload, scale (Ruiz x10 + Pock-Chambolle), power iteration, sigma0.
// Mirrors solve_gpu's setup sequence (reference src/gpu/solver.cu:167-210).
HPRQPStatus engine_create(const HPRQPModel *model, const HPRQPParams *params, Engine **out,
                          SetupInfo *info);
void engine_destroy(Engine *e);

// Backend operations with the semantics of the reference's
// HPRQPSolverBackendOps (src/shared/solver_backend.h:18-36).
HPRQPStatus engine_residuals(Engine *e, HPRQPResiduals *res, size_t iter);
HPRQPStatus engine_iteration_step(Engine *e, size_t inner, int to_check);
HPRQPStatus engine_m_norm(Engine *e, double *out);
HPRQPStatus engine_update_sigma(Engine *e, const HPRQPRestart *rst, const HPRQPResiduals *res,
                                double *sigma_out);
HPRQPStatus engine_restart_apply(Engine *e);
HPRQPStatus engine_copy_output(Engine *e, double *x, double *w, double *z, double *y);
double engine_sigma(const Engine *e);

// Diagnostics used by tests and the benchmark.
struct ScaleDump {
    double *row_norm, *col_norm, *q_val, *a_val, *at_val, *c, *l, *u, *AL, *AU;
    double norm_b_org, norm_c_org, norm_b, norm_c;
};
HPRQPStatus engine_dump_scaling(Engine *e, ScaleDump *d);

// Replace the engine's (x_bar, y_bar, z_bar) by a caller-given iterate in
// original space (host arrays; scaled on the device).
HPRQPStatus engine_set_bars(Engine *e, const double *x, const double *y, const double *z);

// Implicit-differentiation adjoint of the finished solve held by e: MINRES
// on the scaled active-set KKT operator (variables with z_bar == 0, rows with
// y_bar != 0).  gx (n) and gy (m, may be NULL) are host arrays in the model's
// space; lam (n) and mu (m) receive the adjoint solution in original space.
HPRQPStatus engine_adjoint(Engine *e, const double *gx, const double *gy, double tol, long long maxit,
                           double *lam, double *mu, long long *iters, double *relres);

// solve_gpu that hands its engine (scaled problem + final iterate) to the
// caller instead of destroying it (*keep is set only on a terminal status).
HPRQPStatus solve_gpu_keep(const HPRQPModel *model, const HPRQPParams *params, HPRQPResults *results,
                           Engine **keep);

// Small single QPs: the whole solve in one CTA of the batch kernel (one
// launch, no host round trips per iteration).  single_cta_eligible() says
// whether solve_gpu takes this path for a model and parameters; the solve
// fills results like the host loop (iterations, milestones, loop time,
// objective, residuals, x, y, z, w) and, when log is given, appends one
// record of 8 doubles per printed iteration (iter, errRp, errRd, primal obj,
// dual obj, gap, sigma, loop seconds).
constexpr size_t kSingleCtaLogCap = 100000;  // printed iterations the device log holds
bool single_cta_eligible(const HPRQPModel *model, const HPRQPParams *params);
HPRQPStatus solve_single_cta(const HPRQPModel *model, const HPRQPParams *params, HPRQPResults *results,
                             double *log_records, size_t log_cap, size_t *log_count);

// Kernel launch counter (process-wide, all engine kernels).
uint64_t launch_count();
void count_launch(uint64_t k = 1);

}  // namespace hpr
