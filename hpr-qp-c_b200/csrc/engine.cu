// CUDA engine for the plain (one QP per call) HPR path on sm_100a.
//
// The state lives in device memory for the whole solve.  One HPR step is four
// row-block SpMV kernels with fused epilogues (non-noC) or three (noC), the
// same decomposition as the reference's "customized" path
// (src/gpu/iteration.cu:699-1127) but with row blocks instead of
// thread-per-row dots.  Scalars that change during a solve (sigma, the
// Halpern counter) live in a small device struct so the step can be captured
// once in a CUDA graph and replayed.
#include "engine.h"
#include "rowblock.cuh"

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

namespace cg = cooperative_groups;

namespace hpr {

// --------------------------------------------------------------------------
// launch accounting
// --------------------------------------------------------------------------
static std::atomic<uint64_t> g_launches{0};
uint64_t launch_count() { return g_launches.load(); }
void count_launch(uint64_t k) { g_launches.fetch_add(k); }

static bool trace_on()
{
    static int on = -1;
    if (on < 0) {
        const char *v = getenv("HPRQP_B200_TRACE");
        on = (v && v[0] == '1') ? 1 : 0;
    }
    return on == 1;
}
#define HPR_TRACE(...)                                  \
    do {                                                \
        if (trace_on()) {                               \
            fprintf(stderr, "[hprqp-b200] " __VA_ARGS__); \
            fputc('\n', stderr);                       \
            fflush(stderr);                             \
        }                                               \
    } while (0)

#define HPR_CK(call)                                                                         \
    do {                                                                                     \
        cudaError_t err__ = (call);                                                          \
        if (err__ != cudaSuccess) {                                                          \
            fprintf(stderr, "hprqp-b200: CUDA error %s at %s:%d\n", cudaGetErrorString(err__), \
                    __FILE__, __LINE__);                                                     \
            return HPRQP_STATUS_NOT_IMPLEMENTED;                                             \
        }                                                                                    \
    } while (0)

// --------------------------------------------------------------------------
// device state
// --------------------------------------------------------------------------
struct Ctl {
    double sigma;
    double lambda_A;
    double lambda_Q;
    double pad0;
    long long inner;       // Halpern counter read by the 2nd..last kernel of a step
    long long inner_next;  // read by the first kernel of a step, which latches it
};

struct DState {
    int n = 0, m = 0;
    int q_is_diag = 0, noC = 0;
    DCsr Q, A, AT;
    double *c, *l, *u, *AL, *AU, *row_norm, *col_norm;
    double *x, *x_bar, *x_hat, *w, *w_bar, *y, *y_bar, *Ax, *ATy, *ATy_bar, *ATdy, *Qw, *Qw_bar, *Qx,
        *dQw, *QATdy, *dx, *dy, *dw, *s, *z_bar, *tempv, *diag_Q, *fact1, *fact2, *fact, *fact_M,
        *last_x, *last_y, *last_Qw, *last_w, *last_ATy;
    double *pz, *pq, *ptmp, *fac_r, *fac_c;  // setup scratch
    Ctl *ctl;
    // second-order cones (0 when none): cone offsets, linear lengths, scaled rhs
    int nvc = 0, nrc = 0, lin_n = 0, lin_m = 0;
    int *vco = nullptr, *rco = nullptr;
    double *rhs = nullptr;
};

struct Scal {
    double sigma, lA, lQ, h1, h2;
};

__device__ __forceinline__ Scal load_scal(const Ctl *c, bool first)
{
    Scal s;
    s.sigma = c->sigma;
    s.lA = c->lambda_A;
    s.lQ = c->lambda_Q;
    const long long k = first ? c->inner_next : c->inner;
    s.h1 = 1.0 / ((double)k + 2.0);
    s.h2 = 1.0 - s.h1;
    return s;
}

__device__ __forceinline__ double clampd(double v, double lo, double hi)
{
    return v < lo ? lo : (v > hi ? hi : v);
}

template <int N>
struct EpiBase {
    static constexpr int NRED = N;
    double *partials = nullptr;
    __device__ void init(Acc<N> &a) const
    {
#pragma unroll
        for (int k = 0; k < (N > 0 ? N : 1); ++k) a.v[k] = 0.0;
    }
    __host__ __device__ void ops(int *o) const
    {
        for (int k = 0; k < N; ++k) o[k] = kSum;
    }
    __device__ void extra(Acc<N> &) const {}
};

// first kernel of a step: latch inner_next -> inner
__device__ __forceinline__ void latch_inner(Ctl *c)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) c->inner = c->inner_next;
}
// last kernel of a step: inner_next = inner + 1
__device__ __forceinline__ void bump_inner(Ctl *c)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) c->inner_next = c->inner + 1;
}

// ---- one HPR step, non-noC ------------------------------------------------

// K1: Qw = Q w fused with the x / w_bar update.
// Reference kernels: gpu_update_zxw1_custom_{full,partial}_kernel,
// src/gpu/iteration.cu:282-370.
template <bool FULL>
struct EpiZXW1 : EpiBase<0> {
    DState S;
    __device__ void row(int i, double qw, Acc<0> &) const
    {
        const Scal k = load_scal(S.ctl, true);
        const double f2s = 1.0 / (1.0 + k.sigma * k.lQ), f1s = 1.0 - f2s;
        const double xi = S.x[i], wi = S.w[i];
        const double tmp = -qw + S.ATy[i] - S.c[i];
        const double z_raw = xi + k.sigma * tmp;
        const double xb = clampd(z_raw, S.l[i], S.u[i]);
        const double xh = 2.0 * xb - xi;
        const double wb = S.q_is_diag ? S.fact1[i] * wi + S.fact2[i] * xh : f1s * wi + f2s * xh;
        S.Qw[i] = qw;
        S.x_hat[i] = xh;
        if (FULL) {
            S.x_bar[i] = xb;
            S.z_bar[i] = (xb - z_raw) / k.sigma;
            S.dx[i] = xb - xi;
        }
        S.x[i] = k.h2 * xh + k.h1 * S.last_x[i];
        S.w_bar[i] = wb;
    }
    __device__ void extra(Acc<0> &) const { latch_inner(S.ctl); }
};

// K2: tempv = x_hat + sigma (Qw - Q w_bar).
// Reference: gpu_compute_tempv_custom_kernel, src/gpu/iteration.cu:386-403.
struct EpiTempv : EpiBase<0> {
    DState S;
    bool bump = false;
    __device__ void row(int i, double qwb, Acc<0> &) const
    {
        const double sigma = S.ctl->sigma;
        S.tempv[i] = S.x_hat[i] + sigma * (S.Qw[i] - qwb);
    }
    __device__ void extra(Acc<0> &) const
    {
        if (bump) bump_inner(S.ctl);
    }
};

// K3: Ax = A tempv fused with the projection onto [AL, AU] and the Halpern
// y update.  Reference: gpu_update_y_custom_{full,partial}_kernel,
// src/gpu/iteration.cu:505-571.
template <bool FULL>
struct EpiY : EpiBase<0> {
    DState S;
    bool bump = false;
    __device__ void row(int i, double ax, Acc<0> &) const
    {
        const Scal k = load_scal(S.ctl, false);
        const double f1 = k.lA * k.sigma, f2 = 1.0 / f1;
        const double yi = S.y[i];
        const double s_raw = ax - f1 * yi;
        const double sp = clampd(s_raw, S.AL[i], S.AU[i]);
        const double yb = f2 * (sp - s_raw);
        const double yh = 2.0 * yb - yi;
        S.y_bar[i] = yb;
        if (FULL) {
            S.Ax[i] = ax;
            S.dy[i] = yb - yi;
            S.s[i] = sp;
        }
        S.y[i] = k.h2 * yh + k.h1 * S.last_y[i];
    }
    __device__ void extra(Acc<0> &) const
    {
        if (bump) bump_inner(S.ctl);
    }
};

// K4: ATy_bar = A' y_bar fused with the w_bar correction and the Halpern
// averaging of w and A'y.  Reference: gpu_update_w2_custom_{full,partial}_kernel,
// src/gpu/iteration.cu:632-697.
template <bool FULL>
struct EpiW2 : EpiBase<0> {
    DState S;
    __device__ void row(int i, double atyb, Acc<0> &) const
    {
        const Scal k = load_scal(S.ctl, false);
        const double fs = k.sigma / (1.0 + k.sigma * k.lQ);
        const double f = S.q_is_diag ? S.fact[i] : fs;
        const double aty = S.ATy[i], wi = S.w[i];
        const double wbn = S.w_bar[i] + f * (atyb - aty);
        if (FULL) {
            S.dw[i] = wbn - wi;
            S.ATdy[i] = atyb - aty;
            S.w_bar[i] = wbn;
            S.ATy_bar[i] = atyb;
        }
        S.w[i] = k.h1 * S.last_w[i] + k.h2 * (2.0 * wbn - wi);
        S.ATy[i] = k.h1 * S.last_ATy[i] + k.h2 * (2.0 * atyb - aty);
    }
    __device__ void extra(Acc<0> &) const { bump_inner(S.ctl); }
};

// ---- one HPR step, noC (>= 80% free variables) ----------------------------

// K1n: ATy = A' y fused with the noC x / w update.
// Reference: gpu_update_zxw1_noC_{full,partial}_kernel, iteration.cu:190-280.
template <bool FULL>
struct EpiZXW1noC : EpiBase<0> {
    DState S;
    __device__ void row(int i, double aty, Acc<0> &) const
    {
        const Scal k = load_scal(S.ctl, true);
        const double f2s = 1.0 / (1.0 + k.sigma * k.lQ), f1s = 1.0 - f2s;
        const double xi = S.x[i], wi = S.w[i];
        S.ATy[i] = aty;
        const double tmp = -S.Qw[i] + aty - S.c[i];
        const double z_raw = xi + k.sigma * tmp;
        const double xb = clampd(z_raw, S.l[i], S.u[i]);
        const double xh = 2.0 * xb - xi;
        const double wb = S.q_is_diag ? S.fact1[i] * wi + S.fact2[i] * xh : f1s * wi + f2s * xh;
        const double wh = 2.0 * wb - wi;
        if (FULL) {
            S.x_bar[i] = xb;
            S.z_bar[i] = (xb - z_raw) / k.sigma;
            S.dx[i] = xb - xi;
            S.dw[i] = wb - wi;
        }
        S.x_hat[i] = xh;
        S.x[i] = k.h2 * xh + k.h1 * S.last_x[i];
        S.w_bar[i] = wb;
        S.w[i] = k.h2 * wh + k.h1 * S.last_w[i];
    }
    __device__ void extra(Acc<0> &) const { latch_inner(S.ctl); }
};

// K2n: Qw_bar = Q w_bar fused with the Halpern Qw update and tempv.
// Reference: gpu_compute_tempv_custom_noc_kernel + gpu_finalize_qw_noC_kernel,
// iteration.cu:405-447.
struct EpiQwNoC : EpiBase<0> {
    DState S;
    bool bump = false;
    __device__ void row(int i, double qwb, Acc<0> &) const
    {
        const Scal k = load_scal(S.ctl, false);
        const double qw = S.Qw[i];
        S.Qw_bar[i] = qwb;
        S.Qw[i] = k.h2 * (2.0 * qwb - qw) + k.h1 * S.last_Qw[i];
        S.tempv[i] = S.x_hat[i] + k.sigma * (qw - qwb);
    }
    __device__ void extra(Acc<0> &) const
    {
        if (bump) bump_inner(S.ctl);
    }
};

// ---- plain products -------------------------------------------------------

struct EpiStore : EpiBase<0> {
    double *out;
    __device__ void row(int i, double v, Acc<0> &) const { out[i] = v; }
};

// ---- second-order cones (reference src/gpu/soc_common.cuh,
// soc_iteration.cuh, soc_residuals.cuh) ------------------------------------
// Cones are contiguous suffix blocks: variables [vco[0], n), rows [rco[0], m).

// out = projection of in onto [lo, up] on [0, lin) and onto the Lorentz
// cones {(t, v) : |v| <= t} of the blocks; one warp per cone, the norm of v
// taken as max|v| * sqrt(sum (v_j / max|v|)^2) so squares cannot overflow.
__global__ void k_soc_project(const double *in, double *out, const double *lo, const double *up, int lin,
                              const int *off, int ncones)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    for (int i = tid; i < lin; i += nth) out[i] = clampd(in[i], lo[i], up[i]);
    const int lane = threadIdx.x & 31, wid = tid >> 5, nw = nth >> 5;
    for (int k = wid; k < ncones; k += nw) {
        const int b = off[k], e = off[k + 1];
        const double t = in[b];
        double mx = 0.0;
        for (int j = b + 1 + lane; j < e; j += 32) mx = fmax(mx, fabs(in[j]));
        mx = warp_max(mx);
        double sum = 0.0;
        if (mx > 0.0)
            for (int j = b + 1 + lane; j < e; j += 32) {
                const double q = in[j] / mx;
                sum += q * q;
            }
        sum = warp_sum(sum);
        const double nrm = mx * sqrt(sum);
        if (nrm <= t) {
            for (int j = b + lane; j < e; j += 32) out[j] = in[j];
        } else if (nrm <= -t) {
            for (int j = b + lane; j < e; j += 32) out[j] = 0.0;
        } else {
            const double alpha = 0.5 + 0.5 * (t / nrm);
            if (lane == 0) out[b] = 0.5 * nrm + 0.5 * t;
            for (int j = b + 1 + lane; j < e; j += 32) out[j] = alpha * in[j];
        }
    }
}

// scaling factors: the block maximum on every cone, so that a positive scalar
// scales each cone (which leaves the cone invariant)
__global__ void k_cone_block_max(double *f, const int *off, int ncones)
{
    const int tid = blockIdx.x * blockDim.x + threadIdx.x, nth = gridDim.x * blockDim.x;
    const int lane = threadIdx.x & 31, wid = tid >> 5, nw = nth >> 5;
    for (int k = wid; k < ncones; k += nw) {
        double mx = 0.0;
        for (int j = off[k] + lane; j < off[k + 1]; j += 32) mx = fmax(mx, f[j]);
        mx = warp_max(mx);
        for (int j = off[k] + lane; j < off[k + 1]; j += 32) f[j] = mx;
    }
}

// S1: Qw = Q w; tempv = x + sigma (-Qw + A'y - c) (the point to project)
struct EpiSocX1 : EpiBase<0> {
    DState S;
    __device__ void row(int i, double qw, Acc<0> &) const
    {
        const double sigma = S.ctl->sigma;
        S.Qw[i] = qw;
        S.tempv[i] = S.x[i] + sigma * (-qw + S.ATy[i] - S.c[i]);
    }
    __device__ void extra(Acc<0> &) const { latch_inner(S.ctl); }
};

// S3 (over n): x_bar = proj(tempv) is in place; z_bar, x_hat, Halpern x, w_bar
struct EpiSocXFinish : EpiBase<0> {
    DState S;
    __device__ void row(int i, double, Acc<0> &) const
    {
        const Scal k = load_scal(S.ctl, false);
        const double x = S.x[i], xb = S.x_bar[i], xh = 2.0 * xb - x;
        const double f2 = S.q_is_diag ? S.fact2[i] : 1.0 / (1.0 + k.sigma * k.lQ);
        const double f1 = S.q_is_diag ? S.fact1[i] : 1.0 - f2;
        S.dx[i] = xb - x;
        S.z_bar[i] = (xb - S.tempv[i]) / k.sigma;
        S.x_hat[i] = xh;
        S.x[i] = k.h1 * S.last_x[i] + k.h2 * xh;
        S.w_bar[i] = f1 * S.w[i] + f2 * xh;
    }
};

// S5: Ax = A tempv; Rp = Ax - rhs - tau y (the point to project), in pz
struct EpiSocY1 : EpiBase<0> {
    DState S;
    __device__ void row(int i, double ax, Acc<0> &) const
    {
        const double tau = S.ctl->sigma * S.ctl->lambda_A;
        S.Ax[i] = ax;
        S.pz[i] = ax - (S.rhs ? S.rhs[i] : 0.0) - tau * S.y[i];
    }
};

// S7 (over m): s = proj(Rp) is in place; y_bar, dy, Halpern y
struct EpiSocYFinish : EpiBase<0> {
    DState S;
    __device__ void row(int i, double, Acc<0> &) const
    {
        const Scal k = load_scal(S.ctl, false);
        const double tau = k.sigma * k.lA;
        const double y = S.y[i], yb = (S.s[i] - S.pz[i]) / tau;
        S.dy[i] = yb - y;
        S.y_bar[i] = yb;
        S.y[i] = k.h1 * S.last_y[i] + k.h2 * (2.0 * yb - y);
    }
};

// residuals: A x_bar - rhs into pq; slot: max|Ax rs|
struct EpiSocResA : EpiBase<1> {
    DState S;
    __host__ __device__ void ops(int *o) const { o[0] = kMax; }
    __device__ void row(int i, double ax, Acc<1> &a) const
    {
        S.pq[i] = ax - (S.rhs ? S.rhs[i] : 0.0);
        a.v[0] = fmax(a.v[0], fabs(ax * S.row_norm[i]));
    }
};

// residuals (over m): proj(Ax - rhs) is in pz; slots: max|Rp|, y_bar.s, y_bar.rhs
struct EpiSocRp : EpiBase<3> {
    DState S;
    __host__ __device__ void ops(int *o) const
    {
        o[0] = kMax;
        o[1] = kSum;
        o[2] = kSum;
    }
    __device__ void row(int i, double, Acc<3> &a) const
    {
        a.v[0] = fmax(a.v[0], fabs((S.pz[i] - S.pq[i]) * S.row_norm[i]));
        a.v[1] += S.y_bar[i] * S.s[i];
        if (S.rhs) a.v[2] += S.y_bar[i] * S.rhs[i];
    }
};

// residuals (over n): proj(x_bar) is in ptmp; slot: max|proj - x_bar| / cs
struct EpiSocViol : EpiBase<1> {
    DState S;
    __host__ __device__ void ops(int *o) const { o[0] = kMax; }
    __device__ void row(int i, double, Acc<1> &a) const
    {
        a.v[0] = fmax(a.v[0], fabs((S.ptmp[i] - S.x_bar[i]) / S.col_norm[i]));
    }
};

// ---- residuals (reference src/gpu/residuals.cu:81-183) ---------------------

// A x_bar: Ax, s = proj(Ax), Rp; slots: max|Rp|, max|Ax*rs|, sum ybar*s
struct EpiResA : EpiBase<3> {
    DState S;
    __host__ __device__ void ops(int *o) const
    {
        o[0] = kMax;
        o[1] = kMax;
        o[2] = kSum;
    }
    __device__ void row(int i, double ax, Acc<3> &a) const
    {
        const double proj = clampd(ax, S.AL[i], S.AU[i]);
        const double sf = S.row_norm[i];
        S.Ax[i] = ax;
        S.s[i] = proj;
        a.v[0] = fmax(a.v[0], fabs((proj - ax) * sf));
        a.v[1] = fmax(a.v[1], fabs(ax * sf));
        a.v[2] += S.y_bar[i] * proj;
    }
};

// Q x_bar: Qx and Rd; slots: max|Rd|, max|Qx cs|, max|ATy cs|, c.x, x.Qx,
// z.x, bound violation (iteration 0 only)
struct EpiResQ : EpiBase<7> {
    DState S;
    int iter0 = 0;
    __host__ __device__ void ops(int *o) const
    {
        o[0] = kMax;
        o[1] = kMax;
        o[2] = kMax;
        o[3] = kSum;
        o[4] = kSum;
        o[5] = kSum;
        o[6] = kMax;
    }
    __device__ void row(int i, double qx, Acc<7> &a) const
    {
        const double sf = S.col_norm[i];
        const double xb = S.x_bar[i], aty = S.ATdy[i];
        S.Qx[i] = qx;
        const double rd = (qx + S.c[i] - aty - S.z_bar[i]) * sf;
        a.v[0] = fmax(a.v[0], fabs(rd));
        a.v[1] = fmax(a.v[1], fabs(qx * sf));
        a.v[2] = fmax(a.v[2], fabs(aty * sf));
        a.v[3] += S.c[i] * xb;
        a.v[4] += xb * qx;
        a.v[5] += S.z_bar[i] * xb;
        if (iter0) {
            const double lo = S.l[i] - xb, hi = xb - S.u[i];
            double v = 0.0;
            if (lo > 0.0) v += lo;
            if (hi > 0.0) v += hi;
            a.v[6] = fmax(a.v[6], fabs(v * (1.0 / sf)));
        }
    }
};

// ---- M-norm (reference src/gpu/control.cu:243-332) -------------------------

// Q dw: slots dx.dx, dQw.dx, dQw.dQw, dw.dQw
struct EpiMQdw : EpiBase<4> {
    DState S;
    __device__ void row(int i, double v, Acc<4> &a) const
    {
        S.dQw[i] = v;
        const double dx = S.dx[i];
        a.v[0] += dx * dx;
        a.v[1] += v * dx;
        a.v[2] += v * v;
        a.v[3] += S.dw[i] * v;
    }
};

// A' dy: slots ATdy.dx, dy.dy (grid-stride extra over m)
struct EpiMATdy : EpiBase<2> {
    DState S;
    __device__ void row(int i, double v, Acc<2> &a) const
    {
        S.ATdy[i] = v;
        a.v[0] += v * S.dx[i];
    }
    __device__ void extra(Acc<2> &a) const
    {
        for (int i = blockIdx.x * kThreads + threadIdx.x; i < S.m; i += gridDim.x * kThreads) {
            const double d = S.dy[i];
            a.v[1] += d * d;
        }
    }
};

// Q ATdy: slots dQw.ATdy, ATdy.QATdy, (ATdy*fact_M).QATdy
struct EpiMQATdy : EpiBase<3> {
    DState S;
    __device__ void row(int i, double v, Acc<3> &a) const
    {
        S.QATdy[i] = v;
        const double at = S.ATdy[i];
        a.v[0] += S.dQw[i] * at;
        a.v[1] += at * v;
        if (S.q_is_diag) a.v[2] += (at * S.fact_M[i]) * v;
    }
};

// ---- sigma update (reference src/gpu/control.cu:334-529) -------------------

// differences against the restart anchors; slots dx.dx, dy.dy
struct EpiSigDiff : EpiBase<2> {
    DState S;
    __device__ void row(int i, double, Acc<2> &a) const
    {
        if (i < S.n) {
            const double dx = S.x_bar[i] - S.last_x[i];
            S.dx[i] = dx;
            S.dw[i] = S.w_bar[i] - S.last_w[i];
            a.v[0] += dx * dx;
            if (S.m > 0) S.ATdy[i] = S.ATy_bar[i] - S.last_ATy[i];
        }
        if (i < S.m) {
            const double dy = S.y_bar[i] - S.last_y[i];
            S.dy[i] = dy;
            a.v[1] += dy * dy;
        }
    }
};

// Q dw: slots dQw.ATdy (m>0), dQw.dQw, dw.dQw
struct EpiSigQdw : EpiBase<3> {
    DState S;
    __device__ void row(int i, double v, Acc<3> &a) const
    {
        S.dQw[i] = v;
        if (S.m > 0) a.v[0] += v * S.ATdy[i];
        a.v[1] += v * v;
        a.v[2] += S.dw[i] * v;
    }
};

// Q ATdy: slot ATdy.QATdy
struct EpiSigQATdy : EpiBase<1> {
    DState S;
    __device__ void row(int i, double v, Acc<1> &a) const
    {
        S.QATdy[i] = v;
        a.v[0] += S.ATdy[i] * v;
    }
};

// ---- restart (reference src/gpu/control.cu:531-591) -----------------------

// ATy_bar = A' y_bar, anchors <- bars
struct EpiRestart : EpiBase<0> {
    DState S;
    __device__ void row(int i, double atyb, Acc<0> &) const
    {
        const double xb = S.x_bar[i], wb = S.w_bar[i];
        S.x[i] = xb;
        S.last_x[i] = xb;
        S.w[i] = wb;
        S.last_w[i] = wb;
        if (S.m > 0) {
            S.ATy_bar[i] = atyb;
            S.ATy[i] = atyb;
            S.last_ATy[i] = atyb;
        }
        if (S.noC) {
            const double q = S.Qw_bar[i];
            S.Qw[i] = q;
            S.last_Qw[i] = q;
        }
    }
    __device__ void extra(Acc<0> &) const
    {
        for (int i = blockIdx.x * kThreads + threadIdx.x; i < S.m; i += gridDim.x * kThreads) {
            const double yb = S.y_bar[i];
            S.y[i] = yb;
            S.last_y[i] = yb;
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            S.ctl->inner = 0;
            S.ctl->inner_next = 0;
        }
    }
};

// ---- generic vector reductions --------------------------------------------

// slots: sum v^2 (v = vec)
struct EpiSumSq : EpiBase<1> {
    const double *vec;
    __device__ void row(int i, double, Acc<1> &a) const
    {
        const double v = vec[i];
        a.v[0] += v * v;
    }
};

// power iteration: q = z * inv_norm (inv read from device scalar)
struct EpiScaleCopy : EpiBase<0> {
    double *q;
    const double *z;
    double inv;
    __device__ void row(int i, double, Acc<0> &) const { q[i] = z[i] * inv; }
};

// power iteration: z = M q product with slots q.z, z.z
struct EpiPowProd : EpiBase<2> {
    double *z;
    const double *q;
    __device__ void row(int i, double v, Acc<2> &a) const
    {
        z[i] = v;
        a.v[0] += q[i] * v;
        a.v[1] += v * v;
    }
};

// power iteration: q = z - lambda q; slot: sum q^2
struct EpiPowResid : EpiBase<1> {
    double *q;
    const double *z;
    double lambda;
    __device__ void row(int i, double, Acc<1> &a) const
    {
        const double r = z[i] - lambda * q[i];
        q[i] = r;
        a.v[0] += r * r;
    }
};

// bound measures before/after scaling: slots max bm, sum bm^2, max|c|, sum c^2
struct EpiNorms : EpiBase<4> {
    DState S;
    __host__ __device__ void ops(int *o) const
    {
        o[0] = kMax;
        o[1] = kSum;
        o[2] = kMax;
        o[3] = kSum;
    }
    __device__ void row(int i, double, Acc<4> &a) const
    {
        if (i < S.m) {
            const double al = S.AL[i], au = S.AU[i];
            const double lo = isinf(al) ? 0.0 : fabs(al), hi = isinf(au) ? 0.0 : fabs(au);
            const double bm = lo > hi ? lo : hi;
            a.v[0] = fmax(a.v[0], bm);
            a.v[1] += bm * bm;
        }
        if (i < S.n) {
            const double c = S.c[i];
            a.v[2] = fmax(a.v[2], fabs(c));
            a.v[3] += c * c;
        }
    }
};

// free-variable count (noC detection, reference control.cu:23-34, 122-154)
struct EpiFreeCount : EpiBase<1> {
    DState S;
    __device__ void row(int i, double, Acc<1> &a) const
    {
        if (isinf(S.l[i]) && isinf(S.u[i])) a.v[0] += 1.0;
    }
};

struct EpiUnscale : EpiBase<0> {
    DState S;
    double *ox, *ow, *oz, *oy;
    __device__ void row(int i, double, Acc<0> &) const
    {
        if (i < S.n) {
            const double cn = S.col_norm[i];
            ox[i] = S.x_bar[i] / cn;
            ow[i] = S.w_bar[i] / cn;
            oz[i] = S.z_bar[i] * cn;
        }
        if (i < S.m) oy[i] = S.y_bar[i] / S.row_norm[i];
    }
};

struct EpiDiagFactors : EpiBase<0> {
    DState S;
    double sigma;
    __device__ void row(int i, double, Acc<0> &) const
    {
        const double inv = 1.0 / (1.0 + sigma * S.diag_Q[i]);
        S.fact2[i] = inv;
        S.fact[i] = sigma * inv;
        S.fact1[i] = sigma * S.diag_Q[i] * inv;
        S.fact_M[i] = sigma * sigma * inv;
    }
};

// --------------------------------------------------------------------------
// finalize: fold per-CTA partials in fixed order
// --------------------------------------------------------------------------
struct FinalizeSet {
    const double *partials;
    int nblocks, nred, opsmask;  // bit k set: slot k is a max
    double *out;
};
struct FinalizeArgs {
    FinalizeSet set[4];
};

__global__ void __launch_bounds__(kThreads) k_finalize(const FinalizeArgs args)
{
    const FinalizeSet fs = args.set[blockIdx.x];
    __shared__ double s_w[kWarps];
    for (int k = 0; k < fs.nred; ++k) {
        const bool is_max = (fs.opsmask >> k) & 1;
        double t = 0.0;
        for (int b = threadIdx.x; b < fs.nblocks; b += kThreads) {
            const double v = fs.partials[(size_t)b * fs.nred + k];
            t = is_max ? fmax(t, v) : t + v;
        }
        t = is_max ? warp_max(t) : warp_sum(t);
        if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = t;
        __syncthreads();
        if (threadIdx.x == 0) {
            double r = s_w[0];
            for (int w = 1; w < kWarps; ++w) r = is_max ? fmax(r, s_w[w]) : r + s_w[w];
            fs.out[k] = r;
        }
        __syncthreads();
    }
}

// --------------------------------------------------------------------------
// setup kernels (warp per row, grid-stride)
// --------------------------------------------------------------------------
__device__ __forceinline__ double row_absreduce(const int *rp, const double *v, int r, int lane, bool sum)
{
    double acc = 0.0;
    for (int k = rp[r] + lane; k < rp[r + 1]; k += 32) {
        const double a = fabs(v[k]);
        acc = sum ? acc + a : fmax(acc, a);
    }
    return sum ? warp_sum(acc) : warp_max(acc);
}

// column factors: sqrt of max/sum |.| over A' row j and Q row j
// (reference gpu_compute_row_{max,sum}_abs_with_q_kernel, scale.cu:15-90)
__global__ void k_col_factors(const DState S, int use_sum, double *cf)
{
    const int lane = threadIdx.x & 31;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int j = wid; j < S.n; j += nw) {
        double a = S.m > 0 ? row_absreduce(S.AT.rp, S.AT.v, j, lane, use_sum) : 0.0;
        const double b = row_absreduce(S.Q.rp, S.Q.v, j, lane, use_sum);
        a = use_sum ? a + b : fmax(a, b);
        if (lane == 0) cf[j] = a > 0.0 ? sqrt(a) : 1.0;
    }
}

__global__ void k_row_factors(const DState S, int use_sum, double *rf)
{
    const int lane = threadIdx.x & 31;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int r = wid; r < S.m; r += nw) {
        const double a = row_absreduce(S.A.rp, S.A.v, r, lane, use_sum);
        if (lane == 0) rf[r] = a > 0.0 ? sqrt(a) : 1.0;
    }
}

// scale rows of M by 1/rs[row] (multiplication by the reciprocal), then
// columns by division with cs[col]; same two roundings as the reference's
// gpu_scale_rows_csr_kernel + gpu_scale_cols_csr_kernel (scale.cu:113-150)
__device__ __forceinline__ void scale_row(const DCsr &M, int r, int lane, const double *rs, const double *cs)
{
    const double inv = 1.0 / rs[r];
    for (int k = M.rp[r] + lane; k < M.rp[r + 1]; k += 32) {
        double v = M.v[k] * inv;
        v /= cs[M.ci[k]];
        M.v[k] = v;
    }
}

__global__ void k_apply_n(const DState S, const double *cf, const double *rf)
{
    const int lane = threadIdx.x & 31;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int j = wid; j < S.n; j += nw) {
        scale_row(S.Q, j, lane, cf, cf);
        if (S.m > 0) scale_row(S.AT, j, lane, cf, rf);
        if (lane == 0) {
            S.col_norm[j] *= cf[j];
            S.c[j] /= cf[j];
            S.l[j] *= cf[j];
            S.u[j] *= cf[j];
        }
    }
}

__global__ void k_apply_m(const DState S, const double *cf, const double *rf)
{
    const int lane = threadIdx.x & 31;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int r = wid; r < S.m; r += nw) {
        scale_row(S.A, r, lane, rf, cf);
        if (lane == 0) {
            S.row_norm[r] *= rf[r];
            S.AL[r] /= rf[r];
            S.AU[r] /= rf[r];
            if (S.rhs) S.rhs[r] /= rf[r];
        }
    }
}

// Q diagonal extraction; slots: max |offdiag|, max |diag|
// (reference gpu_extract_diag_kernel, eigs.cu:50-82)
struct DiagOut {
    double *partials;
};
__global__ void k_extract_diag(const DState S, double *partials)
{
    const int lane = threadIdx.x & 31;
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    Acc<2> acc;
    acc.v[0] = acc.v[1] = 0.0;
    for (int r = wid; r < S.n; r += nw) {
        double d = 0.0, off = 0.0;
        for (int k = S.Q.rp[r] + lane; k < S.Q.rp[r + 1]; k += 32) {
            if (S.Q.ci[k] == r) d += S.Q.v[k];
            else off = fmax(off, fabs(S.Q.v[k]));
        }
        d = warp_sum(d);
        off = warp_max(off);
        if (lane == 0) S.diag_Q[r] = d;
        acc.v[0] = fmax(acc.v[0], off);
        acc.v[1] = fmax(acc.v[1], fabs(d));
    }
    const int ops[2] = {kMax, kMax};
    block_reduce_store<2>(acc, ops, partials + (size_t)blockIdx.x * 2);
}

__global__ void k_probe(double *z, int len)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < len; i += gridDim.x * blockDim.x)
        z[i] = 1.0 + ((double)i + 1.0) / ((double)len + 1.0);
}

__global__ void k_set_ctl(Ctl *c, double sigma, double lA, double lQ, int reset_inner)
{
    c->sigma = sigma;
    c->lambda_A = lA;
    c->lambda_Q = lQ;
    if (reset_inner) {
        c->inner = 0;
        c->inner_next = 0;
    }
}

// Golden-section search of a*x + b/x + x^2 * sum_i ATdy_i QATdy_i / (1 + x d_i)
// over [1e-12, 1e12] for a diagonal Q, all probes in one cooperative launch
// (every CTA folds the same partials in the same order, so all CTAs take the
// same branch).  Reference: src/gpu/control.cu:429-489 (a host loop of up to
// 200 kernel + blocking cuBLAS dot pairs).
__global__ void __launch_bounds__(kThreads) k_golden_diag(const DState S, double a, double b, double *partials,
                                                          double *result)
{
    cg::grid_group grid = cg::this_grid();
    __shared__ double s_w[kWarps];
    __shared__ double s_f;
    const int nb = gridDim.x;
    auto eval = [&](double xprobe, int parity) -> double {
        double t = 0.0;
        for (int i = blockIdx.x * kThreads + threadIdx.x; i < S.n; i += nb * kThreads)
            t += S.ATdy[i] * (S.QATdy[i] / (1.0 + xprobe * S.diag_Q[i]));
        t = warp_sum(t);
        if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = t;
        __syncthreads();
        if (threadIdx.x == 0) {
            double r = 0.0;
            for (int w = 0; w < kWarps; ++w) r += s_w[w];
            partials[parity * nb + blockIdx.x] = r;
        }
        grid.sync();
        if (threadIdx.x < 32) {
            double r = 0.0;
            for (int k = threadIdx.x; k < nb; k += 32) r += partials[parity * nb + k];
            r = warp_sum(r);
            if (threadIdx.x == 0) s_f = a * xprobe + b / xprobe + xprobe * xprobe * r;
        }
        __syncthreads();
        return s_f;
    };
    double left = 1e-12, right = 1e12;
    const double phi = (sqrt(5.0) - 1.0) / 2.0;
    double x1 = right - phi * (right - left), x2 = left + phi * (right - left);
    int parity = 0;
    double f1 = eval(x1, parity);
    parity ^= 1;
    double f2 = eval(x2, parity);
    parity ^= 1;
    for (int it = 0; it < 200; ++it) {
        if (fabs(right - left) <= 1e-12 * fmax(1.0, fabs(left))) break;
        if (f1 > f2) {
            left = x1;
            x1 = x2;
            f1 = f2;
            x2 = left + phi * (right - left);
            f2 = eval(x2, parity);
        } else {
            right = x2;
            x2 = x1;
            f2 = f1;
            x1 = right - phi * (right - left);
            f1 = eval(x1, parity);
        }
        parity ^= 1;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *result = f1 < f2 ? x1 : x2;
}

// --------------------------------------------------------------------------
// host side
// --------------------------------------------------------------------------
struct HostOut {
    double v[64];
};

struct Engine {
    DState S;
    int device = 0;
    int num_sms = 148;
    cudaStream_t stream = nullptr;
    void *dev_block = nullptr;  // all device allocations
    double *partials = nullptr;
    size_t partials_len = 0;
    HostOut *hout = nullptr;    // pinned, mapped
    HostOut *dout = nullptr;    // device alias of hout
    std::vector<void *> allocs;
    double sigma = 1.0, lambda_A = 0.0, lambda_Q = 0.0;
    double obj_constant = 0.0, norm_b_org = 0.0, norm_c_org = 0.0;
    // graphs of one step, partial / full
    cudaGraphExec_t step_graph[2] = {nullptr, nullptr};
    uint64_t step_launches[2] = {0, 0};
    bool use_graphs = true;
};

template <class T>
static HPRQPStatus dalloc(Engine *e, T **p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    void *ptr = nullptr;
    cudaError_t err = cudaMalloc(&ptr, count * sizeof(T));
    if (err != cudaSuccess) {
        fprintf(stderr, "hprqp-b200: cudaMalloc(%zu bytes) failed: %s\n", count * sizeof(T),
                cudaGetErrorString(err));
        return HPRQP_STATUS_ALLOCATION_FAILED;
    }
    e->allocs.push_back(ptr);
    *p = (T *)ptr;
    return HPRQP_STATUS_OK;
}

static HPRQPStatus upload_csr(Engine *e, const HPRQPMatrixCSR &h, DCsr &d)
{
    if (h.nnz > (size_t)INT32_MAX - 64 || h.nrow > (size_t)INT32_MAX - 64 || h.ncol > (size_t)INT32_MAX)
        return HPRQP_STATUS_NOT_IMPLEMENTED;  // int32 device indices (reference cuda_common.h:29-50)
    d.nrow = (int)h.nrow;
    d.ncol = (int)h.ncol;
    d.nnz = (int)h.nnz;
    const size_t npad = padded_nnz(h.nnz);
    std::vector<int> rp(h.nrow + 1), ci(npad, 0);
    for (size_t r = 0; r <= h.nrow; ++r) rp[r] = (int)h.row_ptr[r];
    for (size_t k = 0; k < h.nnz; ++k) ci[k] = (int)h.col_ind[k];
    TilePlan plan;
    build_tile_plan(rp, plan);
    std::vector<unsigned char> heads;
    build_heads(rp, heads);
    HPRQPStatus st;
    const size_t nt = plan.tiles.size(), nc = plan.chunks.size(), nl = plan.long_rows.size();
    if ((st = dalloc(e, &d.rp, rp.size())) || (st = dalloc(e, &d.ci, npad)) || (st = dalloc(e, &d.v, npad)) ||
        (st = dalloc(e, &d.heads, heads.size())) || (st = dalloc(e, &d.tiles, nt ? nt : 1)) ||
        (st = dalloc(e, &d.chunks, nc ? nc : 1)) || (st = dalloc(e, &d.long_rows, nl ? nl : 1)) ||
        (st = dalloc(e, &d.chunk_partial, nc ? nc : 1)) || (st = dalloc(e, &d.err, 1)))
        return st;
    d.staged = choose_staged(rp, ci);
    d.ntiles = (int)nt;
    d.nchunks = (int)nc;
    d.nlong = (int)nl;
    d.grid_main = std::max(1, (d.ntiles + kWarps - 1) / kWarps);
    d.grid_chunk = (d.nchunks + kWarps - 1) / kWarps;
    d.grid_long = d.nlong ? (d.nlong + kThreads - 1) / kThreads : 0;
    HPR_CK(cudaMemsetAsync(d.err, 0, sizeof(int), e->stream));
    HPR_CK(cudaMemcpyAsync(d.rp, rp.data(), rp.size() * sizeof(int), cudaMemcpyHostToDevice, e->stream));
    HPR_CK(cudaMemcpyAsync(d.ci, ci.data(), ci.size() * sizeof(int), cudaMemcpyHostToDevice, e->stream));
    HPR_CK(cudaMemsetAsync(d.v + h.nnz, 0, (npad - h.nnz) * sizeof(double), e->stream));  // zero padding
    if (h.nnz)
        HPR_CK(cudaMemcpyAsync(d.v, h.values, h.nnz * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    HPR_CK(cudaMemcpyAsync(d.heads, heads.data(), heads.size(), cudaMemcpyHostToDevice, e->stream));
    if (nt)
        HPR_CK(cudaMemcpyAsync(d.tiles, plan.tiles.data(), nt * sizeof(int4), cudaMemcpyHostToDevice, e->stream));
    if (nc)
        HPR_CK(cudaMemcpyAsync(d.chunks, plan.chunks.data(), nc * sizeof(int4), cudaMemcpyHostToDevice, e->stream));
    if (nl)
        HPR_CK(cudaMemcpyAsync(d.long_rows, plan.long_rows.data(), nl * sizeof(int2), cudaMemcpyHostToDevice,
                               e->stream));
    // the host vectors die at return: make the copies complete first
    HPR_CK(cudaStreamSynchronize(e->stream));
    return HPRQP_STATUS_OK;
}

static int ew_grid(const Engine *e, int len)
{
    int g = (len + kThreads - 1) / kThreads;
    return std::max(1, std::min(g, e->num_sms * 4));
}

template <class Epi>
static void launch_rb_at(Engine *e, const DCsr &M, const double *x, Epi epi, size_t poff)
{
    if (M.nrow == 0) return;
    epi.partials = e->partials + poff;
    if (M.nchunks) {
        k_chunks<<<M.grid_chunk, kThreads, 0, e->stream>>>(M, x);
        count_launch();
    }
    if (M.staged) k_spmv_staged<Epi><<<M.grid_main, kThreads, 0, e->stream>>>(M, x, epi);
    else k_spmv<Epi><<<M.grid_main, kThreads, 0, e->stream>>>(M, x, epi);
    count_launch();
    if (M.nlong) {
        k_long_epi<Epi><<<M.grid_long, kThreads, 0, e->stream>>>(M, epi);
        count_launch();
    }
}

template <class Epi>
static void launch_rb(Engine *e, const DCsr &M, const double *x, Epi epi)
{
    launch_rb_at(e, M, x, epi, 0);
}

template <class Epi>
static int launch_ew(Engine *e, int len, Epi epi, int partial_offset = 0)
{
    if (len <= 0) return 0;
    const int g = ew_grid(e, len);
    if (Epi::NRED > 0) epi.partials = e->partials + partial_offset;
    k_elementwise<Epi><<<g, kThreads, 0, e->stream>>>(len, epi);
    count_launch();
    return g;
}

static int opsmask_of(const int *ops, int n)
{
    int m = 0;
    for (int k = 0; k < n; ++k)
        if (ops[k] == kMax) m |= 1 << k;
    return m;
}

// finalize up to 4 partial sets into hout->v[out_off...]
struct FinSpec {
    size_t partial_offset;
    int nblocks, nred, opsmask, out_off;
};
static HPRQPStatus finalize(Engine *e, const FinSpec *specs, int count, bool sync)
{
    FinalizeArgs args;
    memset(&args, 0, sizeof(args));
    for (int k = 0; k < count; ++k) {
        args.set[k].partials = e->partials + specs[k].partial_offset;
        args.set[k].nblocks = specs[k].nblocks;
        args.set[k].nred = specs[k].nred;
        args.set[k].opsmask = specs[k].opsmask;
        args.set[k].out = e->dout->v + specs[k].out_off;
    }
    k_finalize<<<count, kThreads, 0, e->stream>>>(args);
    count_launch();
    if (sync) HPR_CK(cudaStreamSynchronize(e->stream));
    return HPRQP_STATUS_OK;
}

template <class Epi>
static FinSpec spec_of(int nblocks, int out_off, size_t poff = 0)
{
    Epi tmp;
    int ops[Epi::NRED > 0 ? Epi::NRED : 1];
    tmp.ops(ops);
    return FinSpec{poff, nblocks, Epi::NRED, opsmask_of(ops, Epi::NRED), out_off};
}


// ---- power iteration (reference src/gpu/eigs.cu:185-383) -------------------
static HPRQPStatus power_iteration(Engine *e, bool is_a, double *lambda_out)
{
    DState &S = e->S;
    const int len = is_a ? S.m : S.n;
    *lambda_out = 0.0;
    if (len == 0) return HPRQP_STATUS_OK;
    if (!is_a && S.Q.nnz == 0) return HPRQP_STATUS_OK;
    double *z = S.pz, *q = S.pq;
    k_probe<<<ew_grid(e, len), kThreads, 0, e->stream>>>(z, len);
    count_launch();
    // ||z||^2 of the probe
    {
        EpiSumSq ep;
        ep.vec = z;
        const int g = launch_ew(e, len, ep);
        FinSpec f = spec_of<EpiSumSq>(g, 0);
        HPRQPStatus st = finalize(e, &f, 1, true);
        if (st) return st;
    }
    double zz = e->hout->v[0];
    double lambda = 1.0;
    for (int it = 0; it < 5000; ++it) {
        const double qn = sqrt(zz);
        if (qn <= 1e-16) {
            lambda = 0.0;
            break;
        }
        EpiScaleCopy sc;
        sc.q = q;
        sc.z = z;
        sc.inv = 1.0 / qn;
        launch_ew(e, len, sc);
        EpiPowProd pp;
        pp.z = z;
        pp.q = q;
        int nb;
        if (is_a) {
            EpiStore st;
            st.out = S.ptmp;
            launch_rb(e, S.AT, q, st);
            launch_rb(e, S.A, S.ptmp, pp);
            nb = S.A.npart();
        } else {
            launch_rb(e, S.Q, q, pp);
            nb = S.Q.npart();
        }
        FinSpec f = spec_of<EpiPowProd>(nb, 0);
        HPRQPStatus st = finalize(e, &f, 1, true);
        if (st) return st;
        lambda = e->hout->v[0];
        zz = e->hout->v[1];
        const double zn = sqrt(zz);
        EpiPowResid pr;
        pr.q = q;
        pr.z = z;
        pr.lambda = lambda;
        const int g = launch_ew(e, len, pr);
        FinSpec f2 = spec_of<EpiPowResid>(g, 2);
        st = finalize(e, &f2, 1, true);
        if (st) return st;
        const double err = sqrt(e->hout->v[2]);
        if (err / (zn + fabs(lambda) + 1e-16) < 1e-4) break;
    }
    *lambda_out = lambda < 0.0 ? 0.0 : lambda;
    return HPRQP_STATUS_OK;
}

static void free_engine_memory(Engine *e)
{
    for (int k = 0; k < 2; ++k)
        if (e->step_graph[k]) cudaGraphExecDestroy(e->step_graph[k]);
    for (void *p : e->allocs) cudaFree(p);
    e->allocs.clear();
    if (e->hout) cudaFreeHost(e->hout);
    if (e->stream) cudaStreamDestroy(e->stream);
}

void engine_destroy(Engine *e)
{
    if (!e) return;
    free_engine_memory(e);
    delete e;
}

static HPRQPStatus launch_step(Engine *e, int to_check);

HPRQPStatus engine_create(const HPRQPModel *model, const HPRQPParams *params, Engine **out, SetupInfo *info)
{
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        fprintf(stderr, "hprqp-b200: no CUDA device available; this engine has no CPU fallback\n");
        return HPRQP_STATUS_NOT_IMPLEMENTED;
    }
    if (params->device_number < 0 || params->device_number >= ndev) return HPRQP_STATUS_INVALID_ARGUMENT;
    Engine *e = new Engine();
    e->device = params->device_number;
    HPRQPStatus st = HPRQP_STATUS_OK;
#define E_CK(call)                                                                                   \
    do {                                                                                             \
        cudaError_t err__ = (call);                                                                  \
        if (err__ != cudaSuccess) {                                                                  \
            fprintf(stderr, "hprqp-b200: CUDA error %s at %s:%d\n", cudaGetErrorString(err__), __FILE__, \
                    __LINE__);                                                                       \
            engine_destroy(e);                                                                       \
            return HPRQP_STATUS_NOT_IMPLEMENTED;                                                     \
        }                                                                                            \
    } while (0)
#define E_ST(expr)                 \
    do {                           \
        st = (expr);               \
        if (st != HPRQP_STATUS_OK) { \
            engine_destroy(e);     \
            return st;             \
        }                          \
    } while (0)
    HPR_TRACE("create: set device");
    E_CK(cudaSetDevice(e->device));
    E_CK(cudaDeviceGetAttribute(&e->num_sms, cudaDevAttrMultiProcessorCount, e->device));
    E_CK(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    E_CK(cudaHostAlloc((void **)&e->hout, sizeof(HostOut), cudaHostAllocMapped));
    E_CK(cudaHostGetDevicePointer((void **)&e->dout, e->hout, 0));
    memset(e->hout, 0, sizeof(HostOut));

    HPR_TRACE("create: host alloc ok");
    DState &S = e->S;
    const int n = (int)model->Q.ncol, m = (int)model->A.nrow;
    if (model->Q.ncol > (size_t)INT32_MAX / 2 || model->A.nrow > (size_t)INT32_MAX / 2) {
        engine_destroy(e);
        return HPRQP_STATUS_NOT_IMPLEMENTED;
    }
    S.n = n;
    S.m = m;
    E_ST(upload_csr(e, model->Q, S.Q));
    E_ST(upload_csr(e, model->A, S.A));
    E_ST(upload_csr(e, model->AT, S.AT));
    HPR_TRACE("create: csr uploaded");
    // vectors
    double **nvecs[] = {&S.c, &S.l, &S.u, &S.col_norm, &S.x, &S.x_bar, &S.x_hat, &S.w, &S.w_bar, &S.ATy,
                        &S.ATy_bar, &S.ATdy, &S.Qw, &S.Qw_bar, &S.Qx, &S.dQw, &S.QATdy, &S.dx, &S.dw,
                        &S.z_bar, &S.tempv, &S.diag_Q, &S.fact1, &S.fact2, &S.fact, &S.fact_M, &S.last_x,
                        &S.last_Qw, &S.last_w, &S.last_ATy, &S.ptmp, &S.fac_c};
    double **mvecs[] = {&S.AL, &S.AU, &S.row_norm, &S.y, &S.y_bar, &S.Ax, &S.dy, &S.s, &S.last_y, &S.fac_r};
    const size_t nn = (size_t)std::max(n, 1), mm = (size_t)std::max(m, 1);
    const size_t nmax = std::max(nn, mm);
    const size_t n_al = (nn + 31) & ~size_t(31), m_al = (mm + 31) & ~size_t(31), x_al = (nmax + 31) & ~size_t(31);
    const size_t nv = sizeof(nvecs) / sizeof(nvecs[0]), mv = sizeof(mvecs) / sizeof(mvecs[0]);
    double *block = nullptr;
    E_ST(dalloc(e, &block, nv * n_al + mv * m_al + 2 * x_al));
    E_CK(cudaMemsetAsync(block, 0, (nv * n_al + mv * m_al + 2 * x_al) * sizeof(double), e->stream));
    for (size_t k = 0; k < nv; ++k) *nvecs[k] = block + k * n_al;
    for (size_t k = 0; k < mv; ++k) *mvecs[k] = block + nv * n_al + k * m_al;
    S.pz = block + nv * n_al + mv * m_al;
    S.pq = S.pz + x_al;
    E_ST(dalloc(e, &S.ctl, 1));
    E_CK(cudaMemsetAsync(S.ctl, 0, sizeof(Ctl), e->stream));
    int max_blocks = std::max({S.Q.npart(), S.A.npart(), S.AT.npart(), e->num_sms * 4, 1});
    e->partials_len = (size_t)max_blocks * 8 * 2;
    E_ST(dalloc(e, &e->partials, e->partials_len));
    HPR_TRACE("create: buffers allocated");
    // problem vectors
    E_CK(cudaMemcpyAsync(S.c, model->c, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    E_CK(cudaMemcpyAsync(S.l, model->l, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    E_CK(cudaMemcpyAsync(S.u, model->u, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    if (m > 0) {
        E_CK(cudaMemcpyAsync(S.AL, model->AL, m * sizeof(double), cudaMemcpyHostToDevice, e->stream));
        E_CK(cudaMemcpyAsync(S.AU, model->AU, m * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    }
    // second-order cones: offsets (int), linear lengths, rhs
    S.lin_n = n;
    S.lin_m = m;
    if (model->num_var_cones || model->num_row_cones) {
        auto up_off = [&](const size_t *off, size_t count, int **dst) -> HPRQPStatus {
            std::vector<int> h(count + 1);
            for (size_t k = 0; k <= count; ++k) h[k] = (int)off[k];
            HPRQPStatus st2 = dalloc(e, dst, count + 1);
            if (st2) return st2;
            HPR_CK(cudaMemcpy(*dst, h.data(), (count + 1) * sizeof(int), cudaMemcpyHostToDevice));
            return HPRQP_STATUS_OK;
        };
        if (model->num_var_cones) {
            E_ST(up_off(model->var_cone_offsets, model->num_var_cones, &S.vco));
            S.nvc = (int)model->num_var_cones;
            S.lin_n = (int)model->var_cone_offsets[0];
        }
        if (model->num_row_cones) {
            E_ST(up_off(model->row_cone_offsets, model->num_row_cones, &S.rco));
            S.nrc = (int)model->num_row_cones;
            S.lin_m = (int)model->row_cone_offsets[0];
            E_ST(dalloc(e, &S.rhs, (size_t)m));
            E_CK(cudaMemcpy(S.rhs, model->soc_rhs, m * sizeof(double), cudaMemcpyHostToDevice));
        }
    }
    {
        std::vector<double> ones(nmax, 1.0);
        E_CK(cudaMemcpyAsync(S.col_norm, ones.data(), n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
        if (m > 0)
            E_CK(cudaMemcpyAsync(S.row_norm, ones.data(), m * sizeof(double), cudaMemcpyHostToDevice, e->stream));
        E_CK(cudaStreamSynchronize(e->stream));
    }

    HPR_TRACE("create: vectors uploaded");
    // ---- scaling: reference src/gpu/scale.cu:332-560 --------------------
    EpiNorms en;
    en.S = S;
    {
        const int g = launch_ew(e, (int)nmax, en);
        FinSpec f = spec_of<EpiNorms>(g, 0);
        E_ST(finalize(e, &f, 1, true));
    }
    e->norm_b_org = m > 0 ? e->hout->v[0] : 0.0;
    if (S.rhs)
        for (int r = 0; r < m; ++r) e->norm_b_org = std::max(e->norm_b_org, std::fabs(model->soc_rhs[r]));
    e->norm_c_org = e->hout->v[2];
    e->obj_constant = model->obj_constant;
    info->scaling_scalars.norm_b_org = e->norm_b_org;
    info->scaling_scalars.norm_c_org = e->norm_c_org;
    if (params->use_scaling) {
        const int wgrid = std::max(1, std::min((int)((nmax * 32 + kThreads - 1) / kThreads), e->num_sms * 8));
        for (int pass = 0; pass < 11; ++pass) {
            const int use_sum = pass == 10;
            k_col_factors<<<wgrid, kThreads, 0, e->stream>>>(S, use_sum, S.fac_c);
            count_launch();
            if (m > 0) {
                k_row_factors<<<wgrid, kThreads, 0, e->stream>>>(S, use_sum, S.fac_r);
                count_launch();
            }
            if (S.nvc) {
                k_cone_block_max<<<wgrid, kThreads, 0, e->stream>>>(S.fac_c, S.vco, S.nvc);
                count_launch();
            }
            if (S.nrc) {
                k_cone_block_max<<<wgrid, kThreads, 0, e->stream>>>(S.fac_r, S.rco, S.nrc);
                count_launch();
            }
            k_apply_n<<<wgrid, kThreads, 0, e->stream>>>(S, S.fac_c, S.fac_r);
            count_launch();
            if (m > 0) {
                k_apply_m<<<wgrid, kThreads, 0, e->stream>>>(S, S.fac_c, S.fac_r);
                count_launch();
            }
        }
        E_CK(cudaGetLastError());
    }
    {
        const int g = launch_ew(e, (int)nmax, en);
        FinSpec f = spec_of<EpiNorms>(g, 0);
        E_ST(finalize(e, &f, 1, true));
    }
    HPR_TRACE("create: scaled");
    double norm_b = m > 0 ? sqrt(e->hout->v[1]) : 0.0;
    const double norm_c = sqrt(e->hout->v[3]);
    if (S.rhs) {
        std::vector<double> rs(m), rn(m);
        E_CK(cudaMemcpy(rs.data(), S.rhs, m * sizeof(double), cudaMemcpyDeviceToHost));
        double ss = 0.0;
        for (int r = 0; r < m; ++r) ss += rs[r] * rs[r];
        norm_b = std::max(norm_b, sqrt(ss));
    }
    info->scaling_scalars.norm_b = norm_b;
    info->scaling_scalars.norm_c = norm_c;
    info->scaling_scalars.b_scale = 1.0;
    info->scaling_scalars.c_scale = 1.0;

    // ---- workspace setup: reference src/gpu/control.cu:156-241 ------------
    double sigma = 1.0;
    if (norm_b > 1e-16 && norm_c > 1e-16 && norm_b < 1e16 && norm_c < 1e16) sigma = norm_b / norm_c;
    {
        EpiFreeCount fc;
        fc.S = S;
        const int g = launch_ew(e, n, fc);
        if (g > 0) {
            FinSpec f = spec_of<EpiFreeCount>(g, 0);
            E_ST(finalize(e, &f, 1, true));
            S.noC = 5.0 * e->hout->v[0] > 4.0 * (double)n;
        }
    }
    HPR_TRACE("create: noC done");
    double lambda_Q = 0.0, lambda_A = 0.0;
    {
        const int wgrid = std::max(1, std::min((int)((nn * 32 + kThreads - 1) / kThreads), e->num_sms * 8));
        k_extract_diag<<<wgrid, kThreads, 0, e->stream>>>(S, e->partials);
        count_launch();
        FinSpec f{0, wgrid, 2, 3, 0};
        E_ST(finalize(e, &f, 1, true));
        S.q_is_diag = e->hout->v[0] <= 1e-15;
        if (S.q_is_diag) lambda_Q = e->hout->v[1];
    }
    HPR_TRACE("create: diag done");
    if (!S.q_is_diag) {
        E_ST(power_iteration(e, false, &lambda_Q));
        lambda_Q *= 1.05;
    }
    HPR_TRACE("create: lambda_Q done");
    E_ST(power_iteration(e, true, &lambda_A));
    lambda_A *= 1.05;
    if (S.nvc || S.nrc) {
        // reference control.cu:216-220: no noC step on cone models; a constant
        // affine cone is meaningful even when A is zero
        S.noC = 0;
        if (m > 0 && lambda_A <= 0.0) lambda_A = 1.0;
    }
    // the power iteration used pz/pq/ptmp only; iterate vectors are still zero
    e->sigma = sigma;
    e->lambda_A = lambda_A;
    e->lambda_Q = lambda_Q;
    k_set_ctl<<<1, 1, 0, e->stream>>>(S.ctl, sigma, lambda_A, lambda_Q, 1);
    count_launch();
    if (S.q_is_diag) {
        EpiDiagFactors df;
        df.S = S;
        df.sigma = sigma;
        launch_ew(e, n, df);
    }
    E_CK(cudaStreamSynchronize(e->stream));
    E_CK(cudaGetLastError());

    info->sigma = sigma;
    info->lambda_max_A = lambda_A;
    info->lambda_max_Q = lambda_Q;
    info->Q_is_diag = S.q_is_diag;
    info->noC = S.noC;
    info->n = n;
    info->m = m;
    const char *env = getenv("HPRQP_B200_GRAPHS");
    e->use_graphs = !(env && env[0] == '0');
    *out = e;
    return HPRQP_STATUS_OK;
#undef E_CK
#undef E_ST
}

double engine_sigma(const Engine *e) { return e->sigma; }

// ---- one step ----------------------------------------------------------------
// one HPR step on a cone model (reference gpu_soc_iteration_step,
// src/gpu/soc_iteration.cuh:45-83): always the full writes
static void enqueue_soc_step(Engine *e)
{
    DState &S = e->S;
    const int pg = std::max(1, std::min(e->num_sms * 8, (std::max(S.n, S.m) + kThreads - 1) / kThreads));
    EpiSocX1 k1;
    k1.S = S;
    launch_rb(e, S.Q, S.w, k1);
    k_soc_project<<<pg, kThreads, 0, e->stream>>>(S.tempv, S.x_bar, S.l, S.u, S.lin_n, S.vco, S.nvc);
    count_launch();
    EpiSocXFinish fx;
    fx.S = S;
    launch_ew(e, S.n, fx);
    EpiTempv k2;
    k2.S = S;
    launch_rb(e, S.Q, S.w_bar, k2);
    if (S.m > 0) {
        EpiSocY1 k3;
        k3.S = S;
        launch_rb(e, S.A, S.tempv, k3);
        k_soc_project<<<pg, kThreads, 0, e->stream>>>(S.pz, S.s, S.AL, S.AU, S.lin_m, S.rco, S.nrc);
        count_launch();
        EpiSocYFinish fy;
        fy.S = S;
        launch_ew(e, S.m, fy);
    }
    EpiW2<true> k4;
    k4.S = S;
    launch_rb(e, S.AT, S.y_bar, k4);
}

static void enqueue_step(Engine *e, int to_check)
{
    DState &S = e->S;
    if (S.nvc || S.nrc) {
        enqueue_soc_step(e);
        return;
    }
    if (S.noC) {
        if (to_check) {
            EpiZXW1noC<true> k1;
            k1.S = S;
            launch_rb(e, S.AT, S.y, k1);
        } else {
            EpiZXW1noC<false> k1;
            k1.S = S;
            launch_rb(e, S.AT, S.y, k1);
        }
        EpiQwNoC k2;
        k2.S = S;
        k2.bump = S.m == 0;
        launch_rb(e, S.Q, S.w_bar, k2);
        if (S.m > 0) {
            if (to_check) {
                EpiY<true> k3;
                k3.S = S;
                k3.bump = true;
                launch_rb(e, S.A, S.tempv, k3);
            } else {
                EpiY<false> k3;
                k3.S = S;
                k3.bump = true;
                launch_rb(e, S.A, S.tempv, k3);
            }
        }
        return;
    }
    if (to_check) {
        EpiZXW1<true> k1;
        k1.S = S;
        launch_rb(e, S.Q, S.w, k1);
    } else {
        EpiZXW1<false> k1;
        k1.S = S;
        launch_rb(e, S.Q, S.w, k1);
    }
    if (S.m > 0) {
        EpiTempv k2;
        k2.S = S;
        launch_rb(e, S.Q, S.w_bar, k2);
        if (to_check) {
            EpiY<true> k3;
            k3.S = S;
            launch_rb(e, S.A, S.tempv, k3);
        } else {
            EpiY<false> k3;
            k3.S = S;
            launch_rb(e, S.A, S.tempv, k3);
        }
    }
    if (to_check) {
        EpiW2<true> k4;
        k4.S = S;
        launch_rb(e, S.AT, S.y_bar, k4);
    } else {
        EpiW2<false> k4;
        k4.S = S;
        launch_rb(e, S.AT, S.y_bar, k4);
    }
}


static HPRQPStatus launch_step(Engine *e, int to_check)
{
    to_check = to_check ? 1 : 0;
    if (!e->use_graphs) {
        enqueue_step(e, to_check);
        return HPRQP_STATUS_OK;
    }
    if (!e->step_graph[to_check]) {
        cudaGraph_t g;
        const uint64_t before = launch_count();
        HPR_CK(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
        enqueue_step(e, to_check);
        HPR_CK(cudaStreamEndCapture(e->stream, &g));
        e->step_launches[to_check] = launch_count() - before;
        g_launches.store(before);  // captured launches are counted at replay
        HPR_CK(cudaGraphInstantiate(&e->step_graph[to_check], g, 0));
        cudaGraphDestroy(g);
    }
    HPR_CK(cudaGraphLaunch(e->step_graph[to_check], e->stream));
    count_launch(e->step_launches[to_check]);
    return HPRQP_STATUS_OK;
}

HPRQPStatus engine_iteration_step(Engine *e, size_t inner, int to_check)
{
    (void)inner;  // the Halpern counter is tracked on the device (Ctl)
    return launch_step(e, to_check);
}

// ---- residuals ------------------------------------------------------------------
// residuals of a cone model (reference gpu_soc_compute_residuals,
// src/gpu/soc_residuals.cuh:28-77): s of the last step paired with y_bar,
// y_bar.rhs in the dual objective, errRp from the projection of A x_bar - rhs,
// and the distance of x_bar to its domain at every check
static HPRQPStatus engine_residuals_soc(Engine *e, HPRQPResiduals *res)
{
    DState &S = e->S;
    memset(res, 0, sizeof(*res));
    const int pg = std::max(1, std::min(e->num_sms * 8, (std::max(S.n, S.m) + kThreads - 1) / kThreads));
    const size_t off_q = 0, off_a = (size_t)std::max(S.Q.npart(), 1) * 7;
    const size_t off_rp = off_a + (size_t)std::max(S.A.npart(), 1);
    if (S.m > 0) {
        EpiStore st;
        st.out = S.ATdy;
        launch_rb(e, S.AT, S.y_bar, st);
    } else {
        HPR_CK(cudaMemsetAsync(S.ATdy, 0, (size_t)S.n * sizeof(double), e->stream));
    }
    EpiResQ rq;
    rq.S = S;
    rq.iter0 = 0;
    launch_rb_at(e, S.Q, S.x_bar, rq, off_q);
    FinSpec specs[4];
    int ns = 0;
    specs[ns++] = spec_of<EpiResQ>(S.Q.npart(), 8, off_q);
    if (S.m > 0) {
        EpiSocResA ra;
        ra.S = S;
        launch_rb_at(e, S.A, S.x_bar, ra, off_a);
        specs[ns++] = spec_of<EpiSocResA>(S.A.npart(), 0, off_a);
        k_soc_project<<<pg, kThreads, 0, e->stream>>>(S.pq, S.pz, S.AL, S.AU, S.lin_m, S.rco, S.nrc);
        count_launch();
        EpiSocRp rp;
        rp.S = S;
        const int g = launch_ew(e, S.m, rp, (int)off_rp);
        specs[ns++] = spec_of<EpiSocRp>(g, 16, off_rp);
    }
    const size_t off_v = off_rp + (size_t)e->num_sms * 4 * 3;
    k_soc_project<<<pg, kThreads, 0, e->stream>>>(S.x_bar, S.ptmp, S.l, S.u, S.lin_n, S.vco, S.nvc);
    count_launch();
    EpiSocViol vi;
    vi.S = S;
    const int gv = launch_ew(e, S.n, vi, (int)off_v);
    if (gv > 0) specs[ns++] = spec_of<EpiSocViol>(gv, 20, off_v);
    HPRQPStatus st = finalize(e, specs, ns, true);
    if (st) return st;
    const double *v = e->hout->v;
    const double max_rd = v[8], max_qx = v[9], max_aty = v[10], c_dot_x = v[11], x_dot_qx = v[12],
                 z_dot_x = v[13];
    const double max_ax = S.m > 0 ? v[0] : 0.0, max_rp = S.m > 0 ? v[16] : 0.0;
    const double y_dot_s = S.m > 0 ? v[17] : 0.0, y_dot_rhs = S.m > 0 ? v[18] : 0.0;
    const double violation = gv > 0 ? v[20] : 0.0;
    res->primal_obj_bar = (c_dot_x + 0.5 * x_dot_qx) + e->obj_constant;
    res->dual_obj_bar = (-0.5 * x_dot_qx + z_dot_x + y_dot_s + y_dot_rhs) + e->obj_constant;
    res->rel_gap_bar = fabs(res->primal_obj_bar - res->dual_obj_bar) /
                       (1.0 + fmax(fabs(res->primal_obj_bar), fabs(res->dual_obj_bar)));
    res->err_Rd_org_bar = max_rd / (1.0 + fmax(e->norm_c_org, fmax(max_aty, max_qx)));
    if (S.m > 0) res->err_Rp_org_bar = max_rp / (1.0 + fmax(e->norm_b_org, max_ax));
    res->err_Rp_org_bar = fmax(res->err_Rp_org_bar, violation);
    res->KKTx_and_gap_org_bar = fmax(res->err_Rp_org_bar, fmax(res->err_Rd_org_bar, res->rel_gap_bar));
    res->is_updated = 1;
    return HPRQP_STATUS_OK;
}

HPRQPStatus engine_residuals(Engine *e, HPRQPResiduals *res, size_t iter)
{
    DState &S = e->S;
    if (S.nvc || S.nrc) return engine_residuals_soc(e, res);
    memset(res, 0, sizeof(*res));
    const size_t off_a = 0, off_q = (size_t)std::max(S.A.npart(), 1) * 3;
    int nspec = 0;
    FinSpec specs[2];
    if (S.m > 0) {
        EpiStore st;
        st.out = S.ATdy;
        launch_rb(e, S.AT, S.y_bar, st);
        EpiResA ra;
        ra.S = S;
        launch_rb_at(e, S.A, S.x_bar, ra, off_a);
        specs[nspec++] = spec_of<EpiResA>(S.A.npart(), 0, off_a);
    } else {
        HPR_CK(cudaMemsetAsync(S.ATdy, 0, (size_t)S.n * sizeof(double), e->stream));
    }
    EpiResQ rq;
    rq.S = S;
    rq.iter0 = iter == 0;
    launch_rb_at(e, S.Q, S.x_bar, rq, off_q);
    specs[nspec++] = spec_of<EpiResQ>(S.Q.npart(), 8, off_q);
    HPRQPStatus st = finalize(e, specs, nspec, true);
    if (st) return st;
    const double *v = e->hout->v;
    double max_rp = 0, max_ax = 0, y_dot_s = 0;
    if (S.m > 0) {
        max_rp = v[0];
        max_ax = v[1];
        y_dot_s = v[2];
    }
    const double max_rd = v[8], max_qx = v[9], max_aty = v[10], c_dot_x = v[11], x_dot_qx = v[12],
                 z_dot_x = v[13], bound_v = v[14];
    // formulas of src/gpu/residuals.cu:367-411 (b_scale = c_scale = 1)
    res->primal_obj_bar = (c_dot_x + 0.5 * x_dot_qx) + e->obj_constant;
    res->dual_obj_bar = (-0.5 * x_dot_qx + z_dot_x + y_dot_s) + e->obj_constant;
    res->rel_gap_bar = fabs(res->primal_obj_bar - res->dual_obj_bar) /
                       (1.0 + fmax(fabs(res->primal_obj_bar), fabs(res->dual_obj_bar)));
    res->err_Rd_org_bar = max_rd / (1.0 + fmax(e->norm_c_org, fmax(max_aty, max_qx)));
    if (S.m > 0) res->err_Rp_org_bar = max_rp / (1.0 + fmax(e->norm_b_org, max_ax));
    if (iter == 0 && bound_v > res->err_Rp_org_bar) res->err_Rp_org_bar = bound_v;
    res->KKTx_and_gap_org_bar = fmax(res->err_Rp_org_bar, fmax(res->err_Rd_org_bar, res->rel_gap_bar));
    res->is_updated = 1;
    return HPRQP_STATUS_OK;
}

// ---- M-norm ---------------------------------------------------------------------
HPRQPStatus engine_m_norm(Engine *e, double *out)
{
    DState &S = e->S;
    const size_t o1 = 0, o2 = (size_t)S.Q.npart() * 4, o3 = o2 + (size_t)std::max(S.AT.npart(), 1) * 2;
    EpiMQdw a;
    a.S = S;
    launch_rb_at(e, S.Q, S.dw, a, o1);
    FinSpec specs[3];
    int ns = 0;
    specs[ns++] = spec_of<EpiMQdw>(S.Q.npart(), 0, o1);
    if (S.m > 0) {
        EpiMATdy b;
        b.S = S;
        launch_rb_at(e, S.AT, S.dy, b, o2);
        specs[ns++] = spec_of<EpiMATdy>(S.AT.npart(), 8, o2);
        EpiMQATdy c;
        c.S = S;
        launch_rb_at(e, S.Q, S.ATdy, c, o3);
        specs[ns++] = spec_of<EpiMQATdy>(S.Q.npart(), 16, o3);
    }
    HPRQPStatus st = finalize(e, specs, ns, true);
    if (st) return st;
    const double *v = e->hout->v;
    const double sigma = e->sigma, lA = e->lambda_A, lQ = e->lambda_Q;
    const double dx_sq = v[0], dqw_dx = v[1], dqw_sq = v[2], dw_dqw = v[3];
    double m1 = 0.0, m3 = 0.0;
    double m2 = (1.0 / sigma) * dx_sq;
    m2 -= 2.0 * dqw_dx;
    if (S.m > 0) {
        const double atdy_dx = v[8], dy_sq = v[9], dqw_atdy = v[16], atdy_qatdy = v[17], diag_term = v[18];
        m1 = sigma * lA * dy_sq;
        m1 -= 2.0 * sigma * dqw_atdy;
        m2 += 2.0 * atdy_dx;
        if (S.q_is_diag) {
            m3 = diag_term;
            m1 += sigma * dqw_sq;
        } else {
            m3 = (sigma * sigma) / (1.0 + sigma * lQ) * atdy_qatdy;
            m1 += sigma * lQ * dw_dqw;
        }
    } else if (!S.q_is_diag) {
        m1 = sigma * lQ * dw_dqw;
    }
    m2 += m1 > 0.0 ? m1 : 0.0;
    *out = sqrt((m2 > 0.0 ? m2 : 0.0) + (m3 > 0.0 ? m3 : 0.0));
    return HPRQP_STATUS_OK;
}

// ---- sigma update -----------------------------------------------------------------
static double golden_scalar(double a, double b, double c, double d)
{
    // reference src/gpu/cuda_common.h:115-147
    double left = 1e-12, right = 1e12;
    const double ip = (sqrt(5.0) - 1.0) / 2.0, ip2 = (3.0 - sqrt(5.0)) / 2.0;
    auto f = [&](double x) { return a * x + b / x + c * x * x / (1.0 + d * x); };
    double x1 = left + ip2 * (right - left), x2 = left + ip * (right - left);
    double f1 = f(x1), f2 = f(x2);
    for (int it = 0; it < 256; ++it) {
        if (fabs(right - left) <= 1e-13 * fmax(1.0, fmax(fabs(left), fabs(right)))) break;
        if (f1 > f2) {
            left = x1;
            x1 = x2;
            f1 = f2;
            x2 = left + ip * (right - left);
            f2 = f(x2);
        } else {
            right = x2;
            x2 = x1;
            f2 = f1;
            x1 = left + ip2 * (right - left);
            f1 = f(x1);
        }
    }
    return 0.5 * (left + right);
}

static double clamp_h(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }

HPRQPStatus engine_update_sigma(Engine *e, const HPRQPRestart *rst, const HPRQPResiduals *res, double *sigma_out)
{
    DState &S = e->S;
    *sigma_out = e->sigma;
    if (rst->restart_flag < 1) return HPRQP_STATUS_OK;
    const double sigma_old = e->sigma, lA = e->lambda_A, lQ = e->lambda_Q;
    EpiSigDiff d;
    d.S = S;
    const int g = launch_ew(e, std::max(S.n, S.m), d, 0);
    const size_t o2 = (size_t)g * 2, o3 = o2 + (size_t)S.Q.npart() * 3;
    EpiSigQdw q1;
    q1.S = S;
    launch_rb_at(e, S.Q, S.dw, q1, o2);
    FinSpec specs[3];
    int ns = 0;
    specs[ns++] = spec_of<EpiSigDiff>(g, 0, 0);
    specs[ns++] = spec_of<EpiSigQdw>(S.Q.npart(), 8, o2);
    if (S.m > 0) {
        EpiSigQATdy q2;
        q2.S = S;
        launch_rb_at(e, S.Q, S.ATdy, q2, o3);
        specs[ns++] = spec_of<EpiSigQATdy>(S.Q.npart(), 16, o3);
    }
    HPRQPStatus st = finalize(e, specs, ns, true);
    if (st) return st;
    const double *v = e->hout->v;
    const double dx_sq = v[0], dy_sq = v[1], dqw_atdy = v[8], dqw_sq = v[9], dw_dqw = v[10];
    double a = 0.0, b = dx_sq, c_term = 0.0, d_term = 0.0;
    if (S.m > 0) {
        a = lA * dy_sq;
        a -= 2.0 * dqw_atdy;
    }
    if (S.q_is_diag) {
        a += dqw_sq;
    } else {
        a += lQ * dw_dqw;
        if (S.m > 0) {
            c_term = v[16];
            d_term = lQ;
        }
    }
    a = fmax(a, 1e-12);
    b = fmax(b, 1e-12);
    double est;
    if (S.q_is_diag && S.m > 0) {
        // cooperative grid: one CTA per SM
        int per_sm = 0;
        HPR_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_golden_diag, kThreads, 0));
        int grid = std::max(1, std::min(e->num_sms * std::max(per_sm, 1), (S.n + kThreads - 1) / kThreads));
        grid = std::min(grid, e->num_sms * std::max(per_sm, 1));
        double *partials = e->partials;
        double *result = e->dout->v + 30;
        DState Sv = S;
        void *args[] = {(void *)&Sv, (void *)&a, (void *)&b, (void *)&partials, (void *)&result};
        HPR_CK(cudaLaunchCooperativeKernel((void *)k_golden_diag, grid, kThreads, args, 0, e->stream));
        count_launch();
        HPR_CK(cudaStreamSynchronize(e->stream));
        est = e->hout->v[30];
    } else if (!S.q_is_diag && S.m > 0) {
        est = golden_scalar(a, b, c_term > 0.0 ? c_term : 0.0, d_term > 0.0 ? d_term : 0.0);
    } else {
        est = sqrt(b / a);
    }
    est = clamp_h(est, 1e-12, 1e12);
    const double fact = (rst->best_gap > 0.0 && std::isfinite(rst->best_gap))
                            ? exp(-0.05 * (rst->current_gap / rst->best_gap))
                            : 1.0;
    const double cand = exp(fact * log(est) + (1.0 - fact) * log(rst->best_sigma > 0.0 ? rst->best_sigma : sigma_old));
    double kappa = 1.0;
    const double t1 = fmax(fmin(res->err_Rd_org_bar, res->err_Rp_org_bar), fmin(res->rel_gap_bar, rst->current_gap));
    if (t1 <= 9e-10 && res->err_Rp_org_bar > 0.0) {
        const double ratio = res->err_Rd_org_bar / res->err_Rp_org_bar;
        kappa = t1 > 5e-10 ? clamp_h(sqrt(ratio), 1e-2, 100.0) : clamp_h(ratio, 1e-2, 100.0);
    }
    e->sigma = clamp_h(kappa * cand, 1e-12, 1e12);
    k_set_ctl<<<1, 1, 0, e->stream>>>(S.ctl, e->sigma, lA, lQ, 0);
    count_launch();
    if (S.q_is_diag && fabs(e->sigma - sigma_old) > 1e-15) {
        EpiDiagFactors df;
        df.S = S;
        df.sigma = e->sigma;
        launch_ew(e, S.n, df);
    }
    HPR_CK(cudaGetLastError());
    *sigma_out = e->sigma;
    return HPRQP_STATUS_OK;
}

HPRQPStatus engine_restart_apply(Engine *e)
{
    DState &S = e->S;
    EpiRestart r;
    r.S = S;
    launch_rb(e, S.AT, S.y_bar, r);
    if (S.n == 0) {
        // no rows to carry the epilogue: reset the counter directly
        k_set_ctl<<<1, 1, 0, e->stream>>>(S.ctl, e->sigma, e->lambda_A, e->lambda_Q, 1);
        count_launch();
    }
    HPR_CK(cudaGetLastError());
    return HPRQP_STATUS_OK;
}

HPRQPStatus engine_copy_output(Engine *e, double *x, double *w, double *z, double *y)
{
    DState &S = e->S;
    const int n = S.n, m = S.m;
    double *buf = nullptr;
    HPRQPStatus st = dalloc(e, &buf, (size_t)3 * std::max(n, 1) + std::max(m, 1));
    if (st) return st;
    EpiUnscale u;
    u.S = S;
    u.ox = buf;
    u.ow = buf + std::max(n, 1);
    u.oz = buf + 2 * (size_t)std::max(n, 1);
    u.oy = buf + 3 * (size_t)std::max(n, 1);
    launch_ew(e, std::max(n, m), u);
    if (n > 0) {
        HPR_CK(cudaMemcpyAsync(x, u.ox, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
        HPR_CK(cudaMemcpyAsync(w, u.ow, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
        HPR_CK(cudaMemcpyAsync(z, u.oz, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    }
    if (m > 0) HPR_CK(cudaMemcpyAsync(y, u.oy, m * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    HPR_CK(cudaStreamSynchronize(e->stream));
    return HPRQP_STATUS_OK;
}

// ---- implicit-differentiation adjoint on the device-wide kernels ------------
// MINRES on P Ks P with Ks = [[Q_s, A_s'], [A_s, 0]] (the scaled matrices of
// the finished solve), P the 0/1 active-set mask (z_bar == 0 on variables,
// y_bar != 0 on rows).  Vectors are [n-part | m-part] of length n + m.
struct EpiAdjInit : EpiBase<1> {  // v <- D^-1 P [gx; -gy], acc += v^2  (len n + m)
    int n;
    const double *zb, *yb, *cn, *rn, *gx, *gy;
    double *v;
    __device__ void row(int i, double, Acc<1> &a) const
    {
        double t;
        if (i < n) t = zb[i] == 0.0 ? gx[i] / cn[i] : 0.0;
        else t = (gy && yb[i - n] != 0.0) ? -gy[i - n] / rn[i - n] : 0.0;
        v[i] = t;
        a.v[0] += t * t;
    }
};
struct EpiAdjScale : EpiBase<0> {
    double *v;
    double s;
    __device__ void row(int i, double, Acc<0> &) const { v[i] *= s; }
};
struct EpiAdjM : EpiBase<1> {  // vn_m = P_m (A_s v_n), acc += v_m . vn_m
    const double *yb, *vm;
    double *vnm;
    __device__ void row(int r, double a, Acc<1> &acc) const
    {
        const double t = yb[r] != 0.0 ? a : 0.0;
        vnm[r] = t;
        acc.v[0] += vm[r] * t;
    }
};
struct EpiAdjN : EpiBase<1> {  // vn_n = P_n (Q_s v_n + A_s' v_m), acc += v_n . vn_n
    const double *zb, *tmp, *vn;
    double *vnn;
    __device__ void row(int i, double s, Acc<1> &acc) const
    {
        const double t = zb[i] == 0.0 ? (tmp ? tmp[i] + s : s) : 0.0;
        vnn[i] = t;
        acc.v[0] += vn[i] * t;
    }
};
struct EpiAdjLanczos : EpiBase<1> {  // vn <- vn - alpha v - beta vo, acc += vn^2  (len n + m)
    double *vn;
    const double *v, *vo;
    double alpha, beta;
    __device__ void row(int i, double, Acc<1> &a) const
    {
        const double t = vn[i] - alpha * v[i] - beta * vo[i];
        vn[i] = t;
        a.v[0] += t * t;
    }
};
struct EpiAdjStep : EpiBase<0> {  // direction update, solution update, Lanczos normalisation
    const double *v, *wo, *w;
    double *wn, *sol, *vn;
    double r2, r3, inv_r1, step, inv_b;
    __device__ void row(int i, double, Acc<0> &) const
    {
        const double d = (v[i] - r3 * wo[i] - r2 * w[i]) * inv_r1;
        wn[i] = d;
        sol[i] += step * d;
        vn[i] *= inv_b;
    }
};
struct EpiAdjOut : EpiBase<0> {  // lambda = sol_n / col_norm, mu = sol_m / row_norm
    int n;
    const double *sol, *cn, *rn;
    double *out;
    __device__ void row(int i, double, Acc<0> &) const { out[i] = i < n ? sol[i] / cn[i] : sol[i] / rn[i - n]; }
};

HPRQPStatus engine_adjoint(Engine *e, const double *gx, const double *gy, double tol, long long maxit,
                           double *lam, double *mu, long long *iters, double *relres)
{
    DState &S = e->S;
    const int n = S.n, m = S.m, len = n + m;
    HPR_CK(cudaSetDevice(e->device));
    if (len == 0) {
        *iters = 0;
        *relres = 0.0;
        return HPRQP_STATUS_OK;
    }
    double *blk = nullptr;
    HPRQPStatus st = dalloc(e, &blk, (size_t)9 * len + 2);
    if (st) return st;
    double *vb[3] = {blk, blk + len, blk + 2 * (size_t)len};
    double *wb[3] = {blk + 3 * (size_t)len, blk + 4 * (size_t)len, blk + 5 * (size_t)len};
    double *sol = blk + 6 * (size_t)len, *tmp = blk + 7 * (size_t)len, *g = blk + 8 * (size_t)len;
    HPR_CK(cudaMemsetAsync(blk, 0, (size_t)9 * len * sizeof(double), e->stream));
    if (n) HPR_CK(cudaMemcpyAsync(g, gx, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    if (m && gy) HPR_CK(cudaMemcpyAsync(g + n, gy, m * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    double *vo = vb[0], *v = vb[1], *vn = vb[2], *wo = wb[0], *w = wb[1], *wn = wb[2];
    // right-hand side and beta0
    EpiAdjInit ini;
    ini.n = n;
    ini.zb = S.z_bar;
    ini.yb = S.y_bar;
    ini.cn = S.col_norm;
    ini.rn = S.row_norm;
    ini.gx = g;
    ini.gy = gy ? g + n : nullptr;
    ini.v = v;
    int gsz = launch_ew(e, len, ini, 0);
    FinSpec f0 = spec_of<EpiAdjInit>(gsz, 0, 0);
    if ((st = finalize(e, &f0, 1, true))) return st;
    const double beta0 = sqrt(e->hout->v[0]);
    double beta = beta0, eta = beta0, c_old = 1.0, c = 1.0, s_old = 0.0, s = 0.0;
    long long it = 0;
    if (beta0 > 0.0) {
        EpiAdjScale sc;
        sc.v = v;
        sc.s = 1.0 / beta0;
        launch_ew(e, len, sc);
        const size_t pa = 0, pat = (size_t)std::max(S.A.npart(), 1);
        for (it = 0; it < maxit; ++it) {
            // vn = P Ks P v, alpha = v . vn
            FinSpec fa[2];
            int nf = 0;
            if (m > 0) {
                EpiStore q;
                q.out = tmp;
                launch_rb(e, S.Q, v, q);
                EpiAdjM am;
                am.yb = S.y_bar;
                am.vm = v + n;
                am.vnm = vn + n;
                launch_rb_at(e, S.A, v, am, pa);
                fa[nf++] = spec_of<EpiAdjM>(S.A.npart(), 0, pa);
                EpiAdjN an;
                an.zb = S.z_bar;
                an.tmp = tmp;
                an.vn = v;
                an.vnn = vn;
                launch_rb_at(e, S.AT, v + n, an, pat);
                fa[nf++] = spec_of<EpiAdjN>(S.AT.npart(), 1, pat);
            } else {
                EpiAdjN an;
                an.zb = S.z_bar;
                an.tmp = nullptr;
                an.vn = v;
                an.vnn = vn;
                launch_rb_at(e, S.Q, v, an, pa);
                fa[nf++] = spec_of<EpiAdjN>(S.Q.npart(), 0, pa);
            }
            if ((st = finalize(e, fa, nf, true))) return st;
            const double alpha = e->hout->v[0] + (nf > 1 ? e->hout->v[1] : 0.0);
            EpiAdjLanczos lz;
            lz.vn = vn;
            lz.v = v;
            lz.vo = vo;
            lz.alpha = alpha;
            lz.beta = beta;
            gsz = launch_ew(e, len, lz, 0);
            FinSpec fb = spec_of<EpiAdjLanczos>(gsz, 0, 0);
            if ((st = finalize(e, &fb, 1, true))) return st;
            const double beta_new = sqrt(e->hout->v[0]);
            // Givens QR of the new tridiagonal column (Paige-Saunders)
            const double r1h = c * alpha - c_old * s * beta;
            const double r1 = sqrt(r1h * r1h + beta_new * beta_new);
            const double r2 = s * alpha + c_old * c * beta;
            const double r3 = s_old * beta;
            const double c_new = r1 > 0.0 ? r1h / r1 : 1.0;
            const double s_new = r1 > 0.0 ? beta_new / r1 : 0.0;
            EpiAdjStep up;
            up.v = v;
            up.wo = wo;
            up.w = w;
            up.wn = wn;
            up.sol = sol;
            up.vn = vn;
            up.r2 = r2;
            up.r3 = r3;
            up.inv_r1 = r1 > 0.0 ? 1.0 / r1 : 0.0;
            up.step = c_new * eta;
            up.inv_b = beta_new > 0.0 ? 1.0 / beta_new : 0.0;
            launch_ew(e, len, up);
            eta = -s_new * eta;
            double *t0 = vo;
            vo = v;
            v = vn;
            vn = t0;
            t0 = wo;
            wo = w;
            w = wn;
            wn = t0;
            beta = beta_new;
            c_old = c;
            c = c_new;
            s_old = s;
            s = s_new;
            if (fabs(eta) <= tol * beta0 || beta_new == 0.0) {
                ++it;
                break;
            }
        }
    }
    EpiAdjOut o;
    o.n = n;
    o.sol = sol;
    o.cn = S.col_norm;
    o.rn = S.row_norm;
    o.out = tmp;  // reuse: n + m entries
    launch_ew(e, len, o);
    if (n) HPR_CK(cudaMemcpyAsync(lam, tmp, n * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    if (m) HPR_CK(cudaMemcpyAsync(mu, tmp + n, m * sizeof(double), cudaMemcpyDeviceToHost, e->stream));
    HPR_CK(cudaStreamSynchronize(e->stream));
    HPR_CK(cudaGetLastError());
    *iters = it;
    *relres = beta0 > 0.0 ? fabs(eta) / beta0 : 0.0;
    return HPRQP_STATUS_OK;
}

// ---- caller-given iterate (diagnostics) ---------------------------------------
struct EpiSetBars : EpiBase<0> {  // scaled space: x_bar = x cn, z_bar = z / cn, y_bar = y rn
    int n, m;
    const double *x, *y, *z, *cn, *rn;
    double *xb, *yb, *zb;
    __device__ void row(int i, double, Acc<0> &) const
    {
        if (i < n) {
            xb[i] = x[i] * cn[i];
            zb[i] = z[i] / cn[i];
        }
        if (i < m) yb[i] = y[i] * rn[i];
    }
};

HPRQPStatus engine_set_bars(Engine *e, const double *x, const double *y, const double *z)
{
    DState &S = e->S;
    const int n = S.n, m = S.m;
    double *buf = nullptr;
    HPRQPStatus st = dalloc(e, &buf, (size_t)2 * std::max(n, 1) + std::max(m, 1));
    if (st) return st;
    if (n) HPR_CK(cudaMemcpyAsync(buf, x, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    if (n) HPR_CK(cudaMemcpyAsync(buf + n, z, n * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    if (m) HPR_CK(cudaMemcpyAsync(buf + 2 * (size_t)n, y, m * sizeof(double), cudaMemcpyHostToDevice, e->stream));
    EpiSetBars sb;
    sb.n = n;
    sb.m = m;
    sb.x = buf;
    sb.z = buf + n;
    sb.y = buf + 2 * (size_t)n;
    sb.cn = S.col_norm;
    sb.rn = S.row_norm;
    sb.xb = S.x_bar;
    sb.yb = S.y_bar;
    sb.zb = S.z_bar;
    launch_ew(e, std::max(n, m), sb);
    HPR_CK(cudaStreamSynchronize(e->stream));
    return HPRQP_STATUS_OK;
}

HPRQPStatus engine_dump_scaling(Engine *e, ScaleDump *d)
{
    DState &S = e->S;
    auto cp = [&](double *dst, const double *src, size_t cnt) -> cudaError_t {
        if (!dst || cnt == 0) return cudaSuccess;
        return cudaMemcpyAsync(dst, src, cnt * sizeof(double), cudaMemcpyDeviceToHost, e->stream);
    };
    HPR_CK(cp(d->row_norm, S.row_norm, S.m));
    HPR_CK(cp(d->col_norm, S.col_norm, S.n));
    HPR_CK(cp(d->q_val, S.Q.v, S.Q.nnz));
    HPR_CK(cp(d->a_val, S.A.v, S.A.nnz));
    HPR_CK(cp(d->at_val, S.AT.v, S.AT.nnz));
    HPR_CK(cp(d->c, S.c, S.n));
    HPR_CK(cp(d->l, S.l, S.n));
    HPR_CK(cp(d->u, S.u, S.n));
    HPR_CK(cp(d->AL, S.AL, S.m));
    HPR_CK(cp(d->AU, S.AU, S.m));
    HPR_CK(cudaStreamSynchronize(e->stream));
    return HPRQP_STATUS_OK;
}

}  // namespace hpr

// --------------------------------------------------------------------------
// diagnostics (hprqp_b200.h)
// --------------------------------------------------------------------------
#include "hprqp_b200.h"

namespace hpr {

constexpr int kBoundSpan = 2048;  // entries per warp of k_gather_bound

// The floor of any CSR product with this sparsity pattern: every index and
// value streamed once and every x[col] gathered, with no row structure at
// all (one warp per kBoundSpan consecutive entries, eight loads in flight
// per lane); out[warp] = sum of v[k] * x[ci[k]] over its entries.
__global__ void __launch_bounds__(kThreads) k_gather_bound(const int *__restrict__ ci, const double *__restrict__ v,
                                                           const double *__restrict__ x, int nnz, double *out)
{
    const int warp = (blockIdx.x * kThreads + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    const int k0 = warp * kBoundSpan, k1 = min(k0 + kBoundSpan, nnz);
    double s = 0.0;
    for (int k = k0 + lane; k < k1; k += 32 * kSpmvWinU) {
        int c[kSpmvWinU];
        double w[kSpmvWinU];
#pragma unroll
        for (int u = 0; u < kSpmvWinU; ++u) {
            const int kk = k + 32 * u;
            c[u] = kk < k1 ? __ldcs(ci + kk) : -1;
            w[u] = kk < k1 ? __ldcs(v + kk) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kSpmvWinU; ++u)
            if (c[u] >= 0) s = fma(w[u], __ldg(x + c[u]), s);
    }
    s = warp_sum(s);
    if (lane == 0 && k0 < nnz) out[warp] = s;
}

// bound == false: y = M x with the engine's tile kernels; bound == true:
// k_gather_bound over the same arrays, *checksum = the sum of all products
static HPRQPStatus spmv_standalone(size_t nrow, size_t ncol, size_t nnz, const size_t *row_ptr,
                                   const size_t *col_ind, const double *values, const double *x, double *y,
                                   int reps, double *ms, bool bound = false, double *checksum = nullptr)
{
    if (!bound && nrow && !y) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (bound && !checksum) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (!row_ptr || (nnz && (!col_ind || !values)) || (ncol && !x) || reps < 1)
        return HPRQP_STATUS_INVALID_ARGUMENT;
    if (row_ptr[0] != 0 || row_ptr[nrow] != nnz) return HPRQP_STATUS_INVALID_ARGUMENT;
    for (size_t r = 0; r < nrow; ++r)
        if (row_ptr[r + 1] < row_ptr[r]) return HPRQP_STATUS_INVALID_ARGUMENT;
    for (size_t k = 0; k < nnz; ++k)
        if (col_ind[k] >= ncol) return HPRQP_STATUS_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        fprintf(stderr, "hprqp-b200: no CUDA device available; this engine has no CPU fallback\n");
        return HPRQP_STATUS_NOT_IMPLEMENTED;
    }
    Engine *e = new Engine();
    HPRQPStatus st = HPRQP_STATUS_OK;
    auto fail = [&](HPRQPStatus s) {
        engine_destroy(e);
        return s;
    };
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess)
        return fail(HPRQP_STATUS_NOT_IMPLEMENTED);
    HPRQPMatrixCSR h;
    h.nrow = nrow;
    h.ncol = ncol;
    h.nnz = nnz;
    h.row_ptr = (size_t *)row_ptr;
    h.col_ind = (size_t *)col_ind;
    h.values = (double *)values;
    h.owns_data = 0;
    DCsr M;
    if ((st = upload_csr(e, h, M))) return fail(st);
    double *dx = nullptr, *dy = nullptr;
    char *flush = nullptr;
    const size_t flush_bytes = (size_t)256 << 20;
    if ((st = dalloc(e, &dx, ncol)) || (st = dalloc(e, &dy, nrow)) || (st = dalloc(e, &flush, flush_bytes)))
        return fail(st);
    if (ncol && cudaMemcpy(dx, x, ncol * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess)
        return fail(HPRQP_STATUS_NOT_IMPLEMENTED);
    EpiStore ep;
    ep.out = dy;
    const int bound_warps = (int)((nnz + kBoundSpan - 1) / kBoundSpan);
    const int bound_grid = std::max(1, (bound_warps + kWarps - 1) / kWarps);
    double *dpart = nullptr;
    if (bound && (st = dalloc(e, &dpart, (size_t)std::max(bound_warps, 1)))) return fail(st);
    auto product = [&]() {
        if (bound) {
            k_gather_bound<<<bound_grid, kThreads, 0, e->stream>>>(M.ci, M.v, dx, M.nnz, dpart);
            count_launch();
        } else {
            launch_rb(e, M, dx, ep);
        }
    };
    cudaEvent_t ev0, ev1;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    double total_ms = 0.0;
    // matrices smaller than 2 x L2 would be timed from L2: evict them first
    const bool do_flush = nnz * 12 + nrow * 4 < ((size_t)256 << 20);
    // one untimed launch first (module loading, first-touch of the buffers)
    product();
    for (int r = 0; r < reps; ++r) {
        if (do_flush) cudaMemsetAsync(flush, r & 0xff, flush_bytes, e->stream);
        cudaEventRecord(ev0, e->stream);
        product();
        cudaEventRecord(ev1, e->stream);
        cudaEventSynchronize(ev1);
        float t = 0.f;
        cudaEventElapsedTime(&t, ev0, ev1);
        total_ms += t;
    }
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    if (!bound && nrow && cudaMemcpy(y, dy, nrow * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
        return fail(HPRQP_STATUS_NOT_IMPLEMENTED);
    if (bound) {
        std::vector<double> part((size_t)bound_warps);
        if (bound_warps &&
            cudaMemcpy(part.data(), dpart, part.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess)
            return fail(HPRQP_STATUS_NOT_IMPLEMENTED);
        double t = 0.0;
        for (double p : part) t += p;
        *checksum = t;
    }
    if (cudaGetLastError() != cudaSuccess) return fail(HPRQP_STATUS_NOT_IMPLEMENTED);
    if (ms) *ms = total_ms / reps;
    engine_destroy(e);
    return HPRQP_STATUS_OK;
}

}  // namespace hpr

extern "C" {

HPRQPStatus hprqp_b200_spmv(size_t nrow, size_t ncol, size_t nnz, const size_t *row_ptr, const size_t *col_ind,
                            const double *values, const double *x, double *y, int reps, double *ms_per_spmv)
{
    return hpr::spmv_standalone(nrow, ncol, nnz, row_ptr, col_ind, values, x, y, reps, ms_per_spmv);
}

HPRQPStatus hprqp_b200_gather_bound(size_t nrow, size_t ncol, size_t nnz, const size_t *row_ptr,
                                    const size_t *col_ind, const double *values, const double *x, int reps,
                                    double *ms_per_pass, double *checksum)
{
    return hpr::spmv_standalone(nrow, ncol, nnz, row_ptr, col_ind, values, x, nullptr, reps, ms_per_pass, true,
                                checksum);
}

HPRQPStatus hprqp_b200_setup(const HPRQPModel *model, const HPRQPParams *params, double *out9, double *row_norm,
                             double *col_norm, double *q_val, double *a_val, double *at_val, double *c, double *l,
                             double *u, double *AL, double *AU)
{
    if (!model || !params || !out9) return HPRQP_STATUS_INVALID_ARGUMENT;
    hpr::Engine *e = nullptr;
    hpr::SetupInfo info;
    memset(&info, 0, sizeof(info));
    HPRQPStatus st = hpr::engine_create(model, params, &e, &info);
    if (st != HPRQP_STATUS_OK) return st;
    out9[0] = info.sigma;
    out9[1] = info.lambda_max_A;
    out9[2] = info.lambda_max_Q;
    out9[3] = info.Q_is_diag;
    out9[4] = info.noC;
    out9[5] = info.scaling_scalars.norm_b_org;
    out9[6] = info.scaling_scalars.norm_c_org;
    out9[7] = info.scaling_scalars.norm_b;
    out9[8] = info.scaling_scalars.norm_c;
    hpr::ScaleDump d{row_norm, col_norm, q_val, a_val, at_val, c, l, u, AL, AU, 0, 0, 0, 0};
    st = hpr::engine_dump_scaling(e, &d);
    hpr::engine_destroy(e);
    return st;
}

HPRQPStatus hprqp_b200_residuals(const HPRQPModel *model, const HPRQPParams *params, const double *x,
                                 const double *y, const double *z, size_t iter, HPRQPResiduals *out)
{
    if (!model || !params || !x || !z || !out || (model->A.nrow > 0 && !y)) return HPRQP_STATUS_INVALID_ARGUMENT;
    hpr::Engine *e = nullptr;
    hpr::SetupInfo info;
    memset(&info, 0, sizeof(info));
    HPRQPStatus st = hpr::engine_create(model, params, &e, &info);
    if (st != HPRQP_STATUS_OK) return st;
    st = hpr::engine_set_bars(e, x, y, z);
    if (st == HPRQP_STATUS_OK) st = hpr::engine_residuals(e, out, iter);
    hpr::engine_destroy(e);
    return st;
}

uint64_t hprqp_b200_launch_count(void) { return hpr::launch_count(); }

}  // extern "C"
