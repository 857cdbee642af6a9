// Batched HPR-QP solver: persistent kernels solve thousands of independent
// QPs.
//
// Each CTA takes instances from a global work queue with two ends (even
// CTAs take the largest instance left, odd CTAs the smallest, take_instance)
// and runs the complete method for
// its instance: Ruiz + Pock-Chambolle scaling, power iterations, HPR steps,
// residual checks, restarts and the sigma update, with the control logic of
// the reference's outer loop (src/shared/solver_backend.c:338-569,
// src/cpu/control.c:231-411) executed by thread 0 on CTA-shared scalars and
// every vector operation spread over the CTA.  Convergence, restarts and
// sigma are therefore per instance, and an instance that converges frees
// its CTA for the next one immediately.
//
// Inside a CTA, y = M x gives every warp a contiguous range of rows and
// runs it as a CSR-vector product: a group of g lanes shares a row (32/g
// rows per pass), each lane reads the row as 16-byte-aligned quads of
// entries, and the group folds its partial sums with g-1 shuffles.  The
// group width g of each matrix (Q, A, A') of each instance is chosen on the
// host when the batch is packed, from that matrix's sequence of row
// lengths, by a cost model of the rounds, passes and shuffles every warp
// would run (the per-instance SpMV autotuner, choose_lane_group).  The choice
// is structural, so an instance sums in the same order in every solve; every
// reduction is folded in a fixed order, so each instance's result is
// independent of which CTA solved it.
#include "engine.h"
#include "hprqp_batch.h"
#include "hprqp.h"
#include "rowblock.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <thread>
#include <vector>

namespace hpr {

// Two CTA shapes, chosen per batch: 1024 threads and one CTA (one instance)
// per SM -- measured on the 4096-QP batch with the quad-load SpMV: 851
// solves/s, against 705 for 512 threads x 2 CTAs per SM (148 instances in
// flight keep more of their matrices in L2 than 296, and each instance gets
// twice the warps) -- except for batches of one to two instances per SM,
// which run in one wave of 512-thread CTAs (256 QPs of n = 500: forward
// 118 ms against 126 ms, adjoint 15.7 ms against 21.1 ms).
#ifndef HPR_BATCH_LD
#define HPR_BATCH_LD __ldg  // instance matrices are re-read every iteration: keep them in L2
#endif
#ifndef HPR_BATCH_VEC_SMEM
#define HPR_BATCH_VEC_SMEM 1
#endif
constexpr int kBigCta = 1024, kMidCta = 640, kSmallCta = 512;
constexpr int ctas_per_sm(int bt) { return bt >= 1024 ? 1 : 1024 / bt; }
// In a batch of 1024-thread CTAs, an instance with n, m <= kMidCta (every
// vector loop one entry per thread) and work (nnz(Q) + 2 nnz(A) + n of the
// preprocessed model) at most kMidCtaMaxWork is solved by a 640-thread CTA
// (96 registers against 64, one CTA per SM either way), in a launch of its
// own started first (batch_launch).  Per-iteration times on the 4096-QP
// batch recipe: 640 threads 18-24 % faster for n < 640, even or slower
// above (each vector loop takes two passes), 7-15 % slower for work above
// 40,000; 768 and 512 threads gave smaller and larger versions of the same
// trade.  The rule is per instance, so an instance takes the same shape in
// every batch of 1024-thread CTAs.
constexpr long long kMidCtaMaxWork = 30000;
// dynamic shared memory per CTA: the gathered vectors move to shared memory
// when they fit and the pool leaves L1 large (batch_launch), else they stay
// in global memory (L1-cached)
constexpr size_t smem_limit(int bt) { return ctas_per_sm(bt) == 1 ? 200 * 1024 : 110 * 1024; }
// shared memory per SM up to which the gathered vectors use a pool (batch_launch)
constexpr size_t kPoolPerSm = 64 * 1024, kReservedSmemPerCta = 1024;

struct BInst {
    long long q_nz, a_nz, at_nz;  // first entry of the instance's matrices
    int q_rp, a_rp, at_rp;        // first row pointer
    int var, row;                 // first variable / row in the packed vectors
    int n, m;
    int q_lg, a_lg, at_lg;        // log2 of the SpMV lane-group width of Q, A, A' (0..5)
    double obj_constant;
};

struct BatchArgs {
    int K;
    const BInst *inst;
    const int *order;
    unsigned long long *counter;  // the work queue's two ends (take_instance)
    const int *q_rp, *q_ci, *a_rp, *a_ci, *at_rp, *at_ci;
    const double *q_v0, *a_v0, *at_v0, *c0, *l0, *u0, *AL0, *AU0;
    double *q_v, *a_v, *at_v;  // scaled copies
    double *ws;                // per-CTA workspace
    size_t ws_stride;
    int nmax, mmax;
    int vec_smem;              // 1: the gathered vectors live in shared memory
    // parameters
    double stoptol;
    long long max_iter;
    double time_limit;
    int check_iter;
    int print_frequency;
    int use_scaling;
    unsigned long long t_start;  // globaltimer at launch (ns), set by CTA 0
    // host-mapped flag set by hprqp_batch_request_abort (nonzero: stop);
    // read by thread 0 of each CTA when an instance starts and every
    // kAbortPoll iterations
    const int *abort_flag;
    // outputs (packed like the inputs)
    double *x, *y, *z, *w;
    int *status;
    long long *iters;
    double *pobj, *resid, *gap;
    int *restarts;
    unsigned long long *phase_clk;  // optional [grid x 8] clock64 totals per phase
    unsigned char *active_x;  // 1 = variable at a bound (for the adjoint)
    unsigned char *active_r;  // 1 = row at a bound
    double *col_norm_out, *row_norm_out;  // scaling of each instance (for the adjoint)
    // optional starting point in the caller's (unscaled) variables, packed
    // like the outputs; nullptr = start from zero as the reference does
    const double *x_start, *w_start, *y_start;
    const double *sigma_start;  // per instance, optional (<= 0: from the data)
    double *sigma_out;          // per instance: sigma at the end of the solve
    double *seconds_out;        // per instance: device time from its start to its end on its CTA
    // single-QP solves (solve_gpu of a small model runs as a batch of one):
    // the time limit counts from the start of the instance's iteration loop,
    // as the host loop's does (after setup); optional milestone, loop-time
    // and log outputs
    int time_from_loop;
    long long *iter4_out, *iter6_out;  // first checked iteration with KKT < 1e-4 / 1e-6 (-1: none)
    double *time4_out, *time6_out;     // loop seconds at those iterations
    double *loop_seconds_out;          // loop seconds at the end
    double *log_buf;                   // kLogFields doubles per printed iteration (instance 0 only)
    int log_cap;
    int *log_count;
};

// optional per-CTA phase clocks: 0 load+scale, 1 setup norms/diag, 2 power
// iterations, 3 steps, 4 residuals, 5 m-norm, 6 sigma+restart, 7 total
#define PHASE_T0() long long _pt0 = clock64()
#define PHASE_ADD(k)                                                                       \
    do {                                                                                   \
        if (B.phase_clk && threadIdx.x == 0)                                               \
            B.phase_clk[blockIdx.x * 8 + (k)] += (unsigned long long)(clock64() - _pt0);   \
        _pt0 = clock64();                                                                  \
    } while (0)

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

constexpr int kAbortPoll = 16;  // iterations between reads of the host abort flag
// one log record: iter, errRp, errRd, primal obj, dual obj, gap, sigma, loop seconds
constexpr int kLogFields = 8;

// the host's abort request (a system-scope read of host-mapped memory)
__device__ __forceinline__ bool abort_requested(const int *flag)
{
    if (!flag) return false;
    int v;
    asm volatile("ld.relaxed.sys.global.s32 %0, [%1];" : "=r"(v) : "l"(flag) : "memory");
    return v != 0;
}

// local CSR view of one instance's matrix
struct LCsr {
    int nrow;
    const int *rp;
    const int *ci;
    const double *v;
    int lg;  // log2 of the lanes that share a row in cta_spmv
};

__device__ __forceinline__ double clampd(double v, double lo, double hi)
{
    return v < lo ? lo : (v > hi ? hi : v);
}

// fold per-thread values over the CTA; every thread gets the results
template <int N, int kBW>
__device__ __forceinline__ void cta_allreduce(double (&v)[N], const int (&ops)[N], double (*s_red)[8],
                                              double *s_out)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < N; ++k) {
        const double r = ops[k] == kMax ? warp_max(v[k]) : warp_sum(v[k]);
        if (lane == 0) s_red[warp][k] = r;
    }
    __syncthreads();
    if (threadIdx.x < N) {
        const int k = threadIdx.x;
        double t = s_red[0][k];
        for (int w = 1; w < kBW; ++w) t = ops[k] == kMax ? fmax(t, s_red[w][k]) : t + s_red[w][k];
        s_out[k] = t;
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < N; ++k) v[k] = s_out[k];
}

// Rows of a matrix with nrow rows that warp `warp` owns in cta_spmv: one
// contiguous range per warp, balanced to within one row.  It depends on
// nrow only, so products with Q and A' (both n rows) call their epilogues
// for a row on the same thread.
template <int kBW>
__device__ __forceinline__ void warp_rows(int nrow, int warp, int &r0, int &r1)
{
    const int per = (nrow + kBW - 1) / kBW;
    r0 = min(warp * per, nrow);
    r1 = min(r0 + per, nrow);
}

// y = M x; f(row, y_row) is called by the lane that owns the row, on 32
// consecutive rows per warp at a time (coalesced epilogues).
//
// Each warp walks its rows in chunks of 32: the chunk's row pointers are
// read once (one per lane), then passes of 32/g rows run with g lanes per
// row.  A row's entries are read as 16-byte-aligned quads (one int4 of
// column indices and two double2 of values; every instance's entries start
// on a 4-entry boundary and the arrays carry 4 entries of tail padding):
// lane j of the group takes quads j, j+g, ... of the aligned span that
// covers the row, masks the entries outside the row, and adds v * x[col]
// into its own sum in entry order.  The group folds its g sums with an
// xor-shuffle tree and the row's value moves to the lane that owns the row.
// The summation order depends on g only.
template <int BT, class F>
__device__ __forceinline__ void cta_spmv(const LCsr &M, const double *x, F &&f)
{
    constexpr int kBW = BT / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int lg = M.lg, g = 1 << lg, sh = 5 - lg, rpp = 32 >> lg;
    const int gl = lane & (g - 1), grp = lane >> lg;
    const int4 *ci4 = reinterpret_cast<const int4 *>(M.ci);
    const double2 *v2 = reinterpret_cast<const double2 *>(M.v);
    int w0, w1;
    warp_rows<kBW>(M.nrow, warp, w0, w1);
    for (int c0 = w0; c0 < w1; c0 += 32) {
        const int nr = min(32, w1 - c0);
        const int my_b = lane < nr ? M.rp[c0 + lane] : 0;
        const int my_e = lane < nr ? M.rp[c0 + lane + 1] : 0;
        double mine = 0.0;
        const int passes = (nr + rpp - 1) >> sh;
        for (int p = 0; p < passes; ++p) {
            const int rr = (p << sh) + grp;  // row of the chunk this group sums (< 32)
            const int b = __shfl_sync(0xffffffffu, my_b, rr);
            const int e = __shfl_sync(0xffffffffu, my_e, rr);
            double s = 0.0;
            if (rr < nr) {
                const int q1 = (e + 3) >> 2;
                for (int q = (b >> 2) + gl; q < q1; q += g) {
                    const int4 c = HPR_BATCH_LD(ci4 + q);
                    const double2 va = HPR_BATCH_LD(v2 + 2 * q), vb = HPR_BATCH_LD(v2 + 2 * q + 1);
                    // every entry masked (a branch for the quads inside the
                    // row measured 10 % slower: the lanes of a group diverge)
                    const int k0 = 4 * q;
                    if (k0 >= b && k0 < e) s = fma(va.x, x[c.x], s);
                    if (k0 + 1 >= b && k0 + 1 < e) s = fma(va.y, x[c.y], s);
                    if (k0 + 2 >= b && k0 + 2 < e) s = fma(vb.x, x[c.z], s);
                    if (k0 + 3 >= b && k0 + 3 < e) s = fma(vb.y, x[c.w], s);
                }
            }
            for (int o = g >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            // rows p*rpp .. p*rpp+rpp-1 of the chunk sit on lanes 0, g, 2g, ...
            const double val = __shfl_sync(0xffffffffu, s, (lane & (rpp - 1)) << lg);
            if ((lane >> sh) == p) mine = val;
        }
        if (lane < nr) f(c0 + lane, mine);
    }
}

// CTA-shared control state of the instance being solved
struct CtaState {
    double sigma, lA, lQ;
    int q_is_diag, noC;
    int n, m;
    // restart (HPRQPRestart, include/shared/types.h:177-193)
    int restart_flag, first_restart;
    double last_gap, current_gap, save_gap, weighted_norm, best_gap, best_sigma;
    long long inner, times;
    // residuals (HPRQPResiduals)
    double rp, rd, kkt, pobj, dobj, gap;
    double norm_b_org, norm_c_org, obj_constant;
    int to_check, do_res, stop, final_status;
    int aborted;  // the host asked the batch to stop (sticky for the instance)
    int print_yes, got4, got6;
    double red[16];
    double scal[8];
};

struct Vecs {
    double *c, *l, *u, *col_norm, *x, *x_bar, *x_hat, *w, *w_bar, *ATy, *ATy_bar, *ATdy, *Qw, *Qw_bar, *Qx,
        *dQw, *QATdy, *dx, *dw, *z_bar, *tempv, *diag_Q, *fact1, *fact2, *fact, *fact_M, *last_x, *last_Qw,
        *last_w, *last_ATy, *fac_c, *pn;
    double *AL, *AU, *row_norm, *y, *y_bar, *Ax, *dy, *s, *last_y, *fac_r, *pz, *pq;
};

constexpr int kBatchNVecs = 32, kBatchMVecs = 12;

static __device__ Vecs carve(double *base, int nmax, int mmax, double *smem_pool)
{
    Vecs V;
    double **nv[kBatchNVecs] = {&V.c,      &V.l,      &V.u,      &V.col_norm, &V.x,     &V.x_bar,  &V.x_hat,
                                &V.w,      &V.w_bar,  &V.ATy,    &V.ATy_bar,  &V.ATdy,  &V.Qw,     &V.Qw_bar,
                                &V.Qx,     &V.dQw,    &V.QATdy,  &V.dx,       &V.dw,    &V.z_bar,  &V.tempv,
                                &V.diag_Q, &V.fact1,  &V.fact2,  &V.fact,     &V.fact_M, &V.last_x, &V.last_Qw,
                                &V.last_w, &V.last_ATy, &V.fac_c, &V.pn};
    double **mv[kBatchMVecs] = {&V.AL, &V.AU, &V.row_norm, &V.y,     &V.y_bar, &V.Ax,
                                &V.dy, &V.s,  &V.last_y,   &V.fac_r, &V.pz,    &V.pq};
    const int na = (nmax + 31) & ~31, ma = (mmax + 31) & ~31;
    for (int k = 0; k < kBatchNVecs; ++k) *nv[k] = base + (size_t)k * na;
    for (int k = 0; k < kBatchMVecs; ++k) *mv[k] = base + (size_t)kBatchNVecs * na + (size_t)k * ma;
    if (smem_pool) {
        // the gather sources of the step, the residuals and the power iteration
        V.w = smem_pool;
        V.w_bar = smem_pool + na;
        V.tempv = smem_pool + 2 * na;
        V.x_bar = smem_pool + 3 * na;
        V.y_bar = smem_pool + 4 * na;
        V.y = smem_pool + 4 * na + ma;
    }
    return V;
}

template <int kBW>
__device__ __forceinline__ void scale_rows(const LCsr &M, double *vals, const double *rs, const double *cs)
{
    // v *= 1/rs[row]; v /= cs[col]  (reference scale.cu:113-150 roundings)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int r = warp; r < M.nrow; r += kBW) {
        const double inv = 1.0 / rs[r];
        for (int k = M.rp[r] + lane; k < M.rp[r + 1]; k += 32) {
            double v = vals[k] * inv;
            v /= cs[M.ci[k]];
            vals[k] = v;
        }
    }
}

__device__ __forceinline__ double row_abs(const LCsr &M, int r, bool sum)
{
    const int lane = threadIdx.x & 31;
    double acc = 0.0;
    for (int k = M.rp[r] + lane; k < M.rp[r + 1]; k += 32) {
        const double a = fabs(M.v[k]);
        acc = sum ? acc + a : fmax(acc, a);
    }
    return sum ? warp_sum(acc) : warp_max(acc);
}

// Power iteration (reference src/gpu/eigs.cu:185-383), CTA-wide.
template <int BT>
static __device__ double cta_power(const LCsr &A, const LCsr &AT, const LCsr &Q, bool is_a, int len, double *z,
                            double *q, double *tmp, double (*s_red)[8], double *s_out)
{
    constexpr int kBT = BT, kBW = BT / 32;
    if (len == 0) return 0.0;
    const int tid = threadIdx.x;
    for (int i = tid; i < len; i += kBT) z[i] = 1.0 + ((double)i + 1.0) / ((double)len + 1.0);
    double v1[1] = {0.0};
    const int ops1[1] = {kSum};
    for (int i = tid; i < len; i += kBT) v1[0] += z[i] * z[i];
    __syncthreads();
    cta_allreduce<1, kBW>(v1, ops1, s_red, s_out);
    double zz = v1[0], lambda = 1.0;
    bool q_ready = false;  // q = z / |z| was already written by the last residual pass
    for (int it = 0; it < 5000; ++it) {
        const double qn = sqrt(zz);
        if (qn <= 1e-16) {
            lambda = 0.0;
            break;
        }
        if (!q_ready) {
            const double inv = 1.0 / qn;
            for (int i = tid; i < len; i += kBT) q[i] = z[i] * inv;
            __syncthreads();
        }
        double v2[2] = {0.0, 0.0};
        const int ops2[2] = {kSum, kSum};
        if (is_a) {
            cta_spmv<kBT>(AT, q, [&](int r, double s) { tmp[r] = s; });
            __syncthreads();
            cta_spmv<kBT>(A, tmp, [&](int r, double s) {
                z[r] = s;
                v2[0] += q[r] * s;
                v2[1] += s * s;
            });
        } else {
            cta_spmv<kBT>(Q, q, [&](int r, double s) {
                z[r] = s;
                v2[0] += q[r] * s;
                v2[1] += s * s;
            });
        }
        __syncthreads();
        cta_allreduce<2, kBW>(v2, ops2, s_red, s_out);
        lambda = v2[0];
        zz = v2[1];
        const double zn = sqrt(zz);
        // the residual |z - lambda q| and, in the same pass, the next
        // iteration's q = z / |z| (the same products as a separate pass; not
        // used when the residual test stops the iteration)
        q_ready = zn > 1e-16;
        const double inv_next = q_ready ? 1.0 / zn : 0.0;
        double v3[1] = {0.0};
        for (int i = tid; i < len; i += kBT) {
            const double r = z[i] - lambda * q[i];
            if (q_ready) q[i] = z[i] * inv_next;
            v3[0] += r * r;
        }
        cta_allreduce<1, kBW>(v3, ops1, s_red, s_out);
        if (sqrt(v3[0]) / (zn + fabs(lambda) + 1e-16) < 1e-4) break;
    }
    return lambda < 0.0 ? 0.0 : lambda;
}

// The next instance for this CTA, or -1 when every instance is taken.
// `order` lists the instances largest first (nonzeros); even CTAs take from
// its front, odd CTAs from its back.  Iteration counts vary most among the
// small instances (a few run a hundred times the median count), and such a
// straggler taken last would run alone at the end of the launch; from the
// back it starts at once, while the large instances, whose counts vary
// little, are still taken largest first.  One 64-bit counter holds both
// ends (low half: taken from the front, high half: from the back), so one
// atomic both claims an index and checks that the two ends have not met;
// the claims that succeed hand out each index exactly once.
static __device__ __forceinline__ int take_instance(unsigned long long *counter, const int *order, int K)
{
    const bool back = blockIdx.x & 1;
    const unsigned long long old = atomicAdd(counter, back ? (1ull << 32) : 1ull);
    const unsigned long long front_taken = old & 0xffffffffull, back_taken = old >> 32;
    if (front_taken + back_taken >= (unsigned long long)K) return -1;
    return order[back ? K - 1 - (int)back_taken : (int)front_taken];
}

static __device__ __forceinline__ size_t adaptive_step_d(long long iter)
{
    long long step = 10;
    if (iter == 0) return step;
    while (iter / step >= 100) step *= 10;
    return step;
}

// a % d == 0 for the iteration counters of thread 0, in 32-bit arithmetic
// while both fit (every practical count; 64-bit division is a long software
// sequence that the whole CTA would wait for at the next barrier)
static __device__ __forceinline__ bool divides(long long a, long long d)
{
    if (a >= 0 && d > 0 && a <= 0x7fffffffLL && d <= 0x7fffffffLL) return (unsigned)a % (unsigned)d == 0u;
    return a % d == 0;
}

// iter lies on the reference's adaptive print grid (src/shared/solver_backend.c
// print steps: every 10 below 1000, every 100 below 10000, ...)
static __device__ __forceinline__ bool on_print_grid(long long iter)
{
    if (iter >= 0 && iter <= 0x7fffffffLL) {
        const unsigned it = (unsigned)iter;
        unsigned step = 10;
        while (it / step >= 100u && step <= 100000000u) step *= 10;
        return it % step == 0u;
    }
    return iter % (long long)adaptive_step_d(iter) == 0;
}

template <int BT>
__global__ void __launch_bounds__(BT, ctas_per_sm(BT)) k_batch_solve(const BatchArgs B)
{
    constexpr int kBT = BT, kBW = BT / 32;
    extern __shared__ __align__(16) double dyn_smem[];
    __shared__ CtaState S;
    __shared__ double s_red[kBW][8];
    __shared__ double s_out[8];
    __shared__ int s_inst, s_skip;
    const int tid = threadIdx.x;
    Vecs V = carve(B.ws + (size_t)blockIdx.x * B.ws_stride, B.nmax, B.mmax, B.vec_smem ? dyn_smem : nullptr);

    for (;;) {
        if (tid == 0) {
            s_inst = take_instance(B.counter, B.order, B.K);
            // an instance taken after the batch's time limit or after an
            // abort request is not set up: it reports TIME_LIMIT at iteration
            // 0 with zero vectors and infinite residuals
            // (a single-QP solve counts its time limit from its own loop)
            s_skip = s_inst >= 0 && (abort_requested(B.abort_flag) ||
                                     (!B.time_from_loop &&
                                      1e-9 * (double)(globaltimer_ns() - B.t_start) > B.time_limit));
        }
        __syncthreads();
        const int k = s_inst;
        const bool skip = s_skip;
        __syncthreads();
        if (k < 0) break;
        const BInst I = B.inst[k];
        const int n = I.n, m = I.m;
        if (skip) {
            for (int i = tid; i < n; i += kBT) {
                B.x[I.var + i] = B.w[I.var + i] = B.z[I.var + i] = 0.0;
                if (B.active_x) B.active_x[I.var + i] = 0;
                B.col_norm_out[I.var + i] = 1.0;
            }
            for (int i = tid; i < m; i += kBT) {
                B.y[I.row + i] = 0.0;
                if (B.active_r) B.active_r[I.row + i] = 0;
                B.row_norm_out[I.row + i] = 1.0;
            }
            if (tid == 0) {
                B.status[k] = 5;
                B.iters[k] = 0;
                B.pobj[k] = 0.0;
                B.resid[k] = INFINITY;
                B.gap[k] = INFINITY;
                B.restarts[k] = 0;
                B.sigma_out[k] = 0.0;
                B.seconds_out[k] = 0.0;
            }
            __syncthreads();
            continue;
        }
        const unsigned long long inst_t0 = globaltimer_ns();
        LCsr Q{n, B.q_rp + I.q_rp, B.q_ci + I.q_nz, B.q_v + I.q_nz, I.q_lg};
        LCsr A{m, B.a_rp + I.a_rp, B.a_ci + I.a_nz, B.a_v + I.a_nz, I.a_lg};
        LCsr AT{n, B.at_rp + I.at_rp, B.at_ci + I.at_nz, B.at_v + I.at_nz, I.at_lg};
        double *qv = B.q_v + I.q_nz, *av = B.a_v + I.a_nz, *atv = B.at_v + I.at_nz;
        const int q_nnz = Q.rp[n], a_nnz = m > 0 ? A.rp[m] : 0;

        PHASE_T0();
        const long long _ptot = clock64();
        // ---- load (scaled copies start as the originals) --------------------
        for (int i = tid; i < q_nnz; i += kBT) qv[i] = B.q_v0[I.q_nz + i];
        for (int i = tid; i < a_nnz; i += kBT) {
            av[i] = B.a_v0[I.a_nz + i];
            atv[i] = B.at_v0[I.at_nz + i];
        }
        for (int i = tid; i < n; i += kBT) {
            V.c[i] = B.c0[I.var + i];
            V.l[i] = B.l0[I.var + i];
            V.u[i] = B.u0[I.var + i];
            V.col_norm[i] = 1.0;
        }
        for (int i = tid; i < m; i += kBT) {
            V.AL[i] = B.AL0[I.row + i];
            V.AU[i] = B.AU0[I.row + i];
            V.row_norm[i] = 1.0;
        }
        __syncthreads();
        // norms of the original data: max bound measure, max |c|
        {
            double v[2] = {0.0, 0.0};
            const int ops[2] = {kMax, kMax};
            for (int i = tid; i < m; i += kBT) {
                const double lo = isinf(V.AL[i]) ? 0.0 : fabs(V.AL[i]), hi = isinf(V.AU[i]) ? 0.0 : fabs(V.AU[i]);
                v[0] = fmax(v[0], lo > hi ? lo : hi);
            }
            for (int i = tid; i < n; i += kBT) v[1] = fmax(v[1], fabs(V.c[i]));
            cta_allreduce<2, kBW>(v, ops, s_red, s_out);
            if (tid == 0) {
                S.norm_b_org = v[0];
                S.norm_c_org = v[1];
            }
        }
        // ---- scaling: Ruiz x10 + Pock-Chambolle (reference scale.cu:332-560)
        if (B.use_scaling) {
            const int lane = tid & 31, warp = tid >> 5;
            for (int pass = 0; pass < 11; ++pass) {
                const bool use_sum = pass == 10;
                for (int j = warp; j < n; j += kBW) {
                    double a = m > 0 ? row_abs(AT, j, use_sum) : 0.0;
                    const double b = row_abs(Q, j, use_sum);
                    a = use_sum ? a + b : fmax(a, b);
                    if (lane == 0) V.fac_c[j] = a > 0.0 ? sqrt(a) : 1.0;
                }
                for (int r = warp; r < m; r += kBW) {
                    const double a = row_abs(A, r, use_sum);
                    if (lane == 0) V.fac_r[r] = a > 0.0 ? sqrt(a) : 1.0;
                }
                __syncthreads();
                scale_rows<kBW>(Q, qv, V.fac_c, V.fac_c);
                if (m > 0) {
                    scale_rows<kBW>(A, av, V.fac_r, V.fac_c);
                    scale_rows<kBW>(AT, atv, V.fac_c, V.fac_r);
                }
                for (int i = tid; i < n; i += kBT) {
                    const double f = V.fac_c[i];
                    V.col_norm[i] *= f;
                    V.c[i] /= f;
                    V.l[i] *= f;
                    V.u[i] *= f;
                }
                for (int i = tid; i < m; i += kBT) {
                    const double f = V.fac_r[i];
                    V.row_norm[i] *= f;
                    V.AL[i] /= f;
                    V.AU[i] /= f;
                }
                __syncthreads();
            }
        }
        PHASE_ADD(0);
        // ---- setup: sigma0, noC, Q diagonal, eigenvalues (control.cu:156-241)
        {
            double v[4] = {0.0, 0.0, 0.0, 0.0};
            const int ops[4] = {kSum, kSum, kSum, kMax};
            for (int i = tid; i < m; i += kBT) {
                const double lo = isinf(V.AL[i]) ? 0.0 : fabs(V.AL[i]), hi = isinf(V.AU[i]) ? 0.0 : fabs(V.AU[i]);
                const double bm = lo > hi ? lo : hi;
                v[0] += bm * bm;
            }
            for (int i = tid; i < n; i += kBT) {
                v[1] += V.c[i] * V.c[i];
                if (isinf(V.l[i]) && isinf(V.u[i])) v[2] += 1.0;
            }
            // Q diagonal and largest off-diagonal magnitude
            const int lane = tid & 31, warp = tid >> 5;
            double offmax = 0.0, diagmax = 0.0;
            for (int r = warp; r < n; r += kBW) {
                double d = 0.0, off = 0.0;
                for (int kk = Q.rp[r] + lane; kk < Q.rp[r + 1]; kk += 32) {
                    if (Q.ci[kk] == r) d += Q.v[kk];
                    else off = fmax(off, fabs(Q.v[kk]));
                }
                d = warp_sum(d);
                off = warp_max(off);
                if (lane == 0) V.diag_Q[r] = d;
                offmax = fmax(offmax, off);
                diagmax = fmax(diagmax, fabs(d));
            }
            v[3] = offmax;
            cta_allreduce<4, kBW>(v, ops, s_red, s_out);
            double v2[1] = {diagmax};
            const int ops2[1] = {kMax};
            cta_allreduce<1, kBW>(v2, ops2, s_red, s_out);
            if (tid == 0) {
                const double nb = sqrt(v[0]), nc = sqrt(v[1]);
                S.sigma = (nb > 1e-16 && nc > 1e-16 && nb < 1e16 && nc < 1e16) ? nb / nc : 1.0;
                if (B.sigma_start && B.sigma_start[k] > 0.0) S.sigma = clampd(B.sigma_start[k], 1e-12, 1e12);
                S.noC = n > 0 && 5.0 * v[2] > 4.0 * (double)n;
                S.q_is_diag = v[3] <= 1e-15;
                S.lQ = S.q_is_diag ? v2[0] : 0.0;
                S.n = n;
                S.m = m;
                S.obj_constant = I.obj_constant;
            }
            __syncthreads();
        }
        PHASE_ADD(1);
        if (!S.q_is_diag) {
            const double lq = (q_nnz > 0) ? cta_power<kBT>(A, AT, Q, false, n, V.pn, V.tempv, V.Qx, s_red, s_out) : 0.0;
            if (tid == 0) S.lQ = lq * 1.05;
        }
        {
            // the products' sources in the slots of y_bar and w (in the
            // shared-memory pool when there is one), which the starting
            // iterates below overwrite
            const double la = m > 0 ? cta_power<kBT>(A, AT, Q, true, m, V.pz, V.y_bar, V.w, s_red, s_out) : 0.0;
            if (tid == 0) S.lA = la * 1.05;
        }
        __syncthreads();
        PHASE_ADD(2);
        // starting iterates (zero, or the warm start scaled into the solver's
        // variables: x_s = x * col_norm, y_s = y * row_norm, the inverse of
        // the output map below; the Halpern anchors start at the same point);
        // diagonal factors
        const bool warm = B.x_start != nullptr;
        for (int i = tid; i < n; i += kBT) {
            const double xs = warm ? B.x_start[I.var + i] * V.col_norm[i] : 0.0;
            const double ws = warm ? B.w_start[I.var + i] * V.col_norm[i] : 0.0;
            V.x[i] = V.x_bar[i] = V.x_hat[i] = V.last_x[i] = xs;
            V.w[i] = V.w_bar[i] = V.last_w[i] = ws;
            V.ATy[i] = V.ATy_bar[i] = V.ATdy[i] = V.Qw[i] = V.Qw_bar[i] = V.Qx[i] = 0.0;
            V.dQw[i] = V.QATdy[i] = V.dx[i] = V.dw[i] = V.z_bar[i] = V.tempv[i] = 0.0;
            V.last_Qw[i] = V.last_ATy[i] = 0.0;
            if (S.q_is_diag) {
                const double inv = 1.0 / (1.0 + S.sigma * V.diag_Q[i]);
                V.fact2[i] = inv;
                V.fact[i] = S.sigma * inv;
                V.fact1[i] = S.sigma * V.diag_Q[i] * inv;
                V.fact_M[i] = S.sigma * S.sigma * inv;
            }
        }
        for (int i = tid; i < m; i += kBT) {
            V.y[i] = V.y_bar[i] = V.last_y[i] = warm ? B.y_start[I.row + i] * V.row_norm[i] : 0.0;
            V.Ax[i] = V.dy[i] = V.s[i] = 0.0;
        }
        __syncthreads();
        if (warm) {
            // the products the step carries with the iterates: A'y, and Q w
            // on the noC path (reference iteration.cu:831-920)
            if (m > 0)
                cta_spmv<kBT>(AT, V.y, [&](int i, double s) { V.ATy[i] = V.ATy_bar[i] = V.last_ATy[i] = s; });
            if (S.noC) cta_spmv<kBT>(Q, V.w, [&](int i, double s) { V.Qw[i] = V.Qw_bar[i] = V.last_Qw[i] = s; });
        }
        if (tid == 0) {
            S.restart_flag = 0;
            S.first_restart = 1;
            S.save_gap = S.current_gap = S.last_gap = S.best_gap = INFINITY;
            S.weighted_norm = INFINITY;
            S.best_sigma = S.sigma;
            S.inner = 0;
            S.times = 0;
            S.aborted = 0;
        }
        __syncthreads();

        // ---- residuals (reference residuals.cu:81-183) ----------------------
        auto residuals = [&](long long iter) {
            if (m > 0) cta_spmv<kBT>(AT, V.y_bar, [&](int r, double s) { V.ATdy[r] = s; });
            else
                for (int i = tid; i < n; i += kBT) V.ATdy[i] = 0.0;
            double a[3] = {0.0, 0.0, 0.0};
            const int opa[3] = {kMax, kMax, kSum};
            if (m > 0)
                cta_spmv<kBT>(A, V.x_bar, [&](int r, double ax) {
                    const double proj = clampd(ax, V.AL[r], V.AU[r]);
                    const double sf = V.row_norm[r];
                    V.Ax[r] = ax;
                    V.s[r] = proj;
                    a[0] = fmax(a[0], fabs((proj - ax) * sf));
                    a[1] = fmax(a[1], fabs(ax * sf));
                    a[2] += V.y_bar[r] * proj;
                });
            __syncthreads();
            double q[7] = {0, 0, 0, 0, 0, 0, 0};
            const int opq[7] = {kMax, kMax, kMax, kSum, kSum, kSum, kMax};
            cta_spmv<kBT>(Q, V.x_bar, [&](int r, double qx) {
                const double sf = V.col_norm[r];
                const double xb = V.x_bar[r], aty = V.ATdy[r];
                V.Qx[r] = qx;
                const double rd = (qx + V.c[r] - aty - V.z_bar[r]) * sf;
                q[0] = fmax(q[0], fabs(rd));
                q[1] = fmax(q[1], fabs(qx * sf));
                q[2] = fmax(q[2], fabs(aty * sf));
                q[3] += V.c[r] * xb;
                q[4] += xb * qx;
                q[5] += V.z_bar[r] * xb;
                if (iter == 0) {
                    const double lo = V.l[r] - xb, hi = xb - V.u[r];
                    double vv = 0.0;
                    if (lo > 0.0) vv += lo;
                    if (hi > 0.0) vv += hi;
                    q[6] = fmax(q[6], fabs(vv * (1.0 / sf)));
                }
            });
            cta_allreduce<3, kBW>(a, opa, s_red, s_out);
            cta_allreduce<7, kBW>(q, opq, s_red, s_out);
            if (tid == 0) {
                S.pobj = (q[3] + 0.5 * q[4]) + S.obj_constant;
                S.dobj = (-0.5 * q[4] + q[5] + a[2]) + S.obj_constant;
                S.gap = fabs(S.pobj - S.dobj) / (1.0 + fmax(fabs(S.pobj), fabs(S.dobj)));
                S.rd = q[0] / (1.0 + fmax(S.norm_c_org, fmax(q[2], q[1])));
                S.rp = m > 0 ? a[0] / (1.0 + fmax(S.norm_b_org, a[1])) : 0.0;
                if (iter == 0 && q[6] > S.rp) S.rp = q[6];
                S.kkt = fmax(S.rp, fmax(S.rd, S.gap));
            }
            __syncthreads();
        };

        // ---- one HPR step (reference iteration.cu:1386-1442) ------------------
        auto step = [&](int full) {
            const double sigma = S.sigma, lA = S.lA, lQ = S.lQ;
            const double h1 = 1.0 / ((double)S.inner + 2.0), h2 = 1.0 - h1;
            const double f2s = 1.0 / (1.0 + sigma * lQ), f1s = 1.0 - f2s;
            const int diag = S.q_is_diag;
            if (S.noC) {
                auto upd = [&](int i, double aty) {
                    const double xi = V.x[i], wi = V.w[i];
                    V.ATy[i] = aty;
                    const double z_raw = xi + sigma * (-V.Qw[i] + aty - V.c[i]);
                    const double xb = clampd(z_raw, V.l[i], V.u[i]);
                    const double xh = 2.0 * xb - xi;
                    const double wb = diag ? V.fact1[i] * wi + V.fact2[i] * xh : f1s * wi + f2s * xh;
                    if (full) {
                        V.x_bar[i] = xb;
                        V.z_bar[i] = (xb - z_raw) / sigma;
                        V.dx[i] = xb - xi;
                        V.dw[i] = wb - wi;
                    }
                    V.x_hat[i] = xh;
                    V.x[i] = h2 * xh + h1 * V.last_x[i];
                    V.w_bar[i] = wb;
                    V.w[i] = h2 * (2.0 * wb - wi) + h1 * V.last_w[i];
                };
                if (m > 0) cta_spmv<kBT>(AT, V.y, upd);
                else
                    for (int i = tid; i < n; i += kBT) upd(i, 0.0);
                __syncthreads();
                cta_spmv<kBT>(Q, V.w_bar, [&](int i, double qwb) {
                    const double qw = V.Qw[i];
                    V.Qw_bar[i] = qwb;
                    V.Qw[i] = h2 * (2.0 * qwb - qw) + h1 * V.last_Qw[i];
                    V.tempv[i] = V.x_hat[i] + sigma * (qw - qwb);
                });
                __syncthreads();
            } else {
                cta_spmv<kBT>(Q, V.w, [&](int i, double qw) {
                    const double xi = V.x[i], wi = V.w[i];
                    const double z_raw = xi + sigma * (-qw + V.ATy[i] - V.c[i]);
                    const double xb = clampd(z_raw, V.l[i], V.u[i]);
                    const double xh = 2.0 * xb - xi;
                    V.Qw[i] = qw;
                    V.x_hat[i] = xh;
                    if (full) {
                        V.x_bar[i] = xb;
                        V.z_bar[i] = (xb - z_raw) / sigma;
                        V.dx[i] = xb - xi;
                    }
                    V.x[i] = h2 * xh + h1 * V.last_x[i];
                    V.w_bar[i] = diag ? V.fact1[i] * wi + V.fact2[i] * xh : f1s * wi + f2s * xh;
                });
                __syncthreads();
                if (m > 0) {
                    cta_spmv<kBT>(Q, V.w_bar,
                             [&](int i, double qwb) { V.tempv[i] = V.x_hat[i] + sigma * (V.Qw[i] - qwb); });
                    __syncthreads();
                }
            }
            if (m > 0) {
                const double f1 = lA * sigma, f2 = 1.0 / f1;
                cta_spmv<kBT>(A, V.tempv, [&](int i, double ax) {
                    const double yi = V.y[i];
                    const double s_raw = ax - f1 * yi;
                    const double sp = clampd(s_raw, V.AL[i], V.AU[i]);
                    const double yb = f2 * (sp - s_raw);
                    V.y_bar[i] = yb;
                    if (full) {
                        V.Ax[i] = ax;
                        V.dy[i] = yb - yi;
                        V.s[i] = sp;
                    }
                    V.y[i] = h2 * (2.0 * yb - yi) + h1 * V.last_y[i];
                });
                __syncthreads();
            }
            if (!S.noC) {
                const double fs = sigma / (1.0 + sigma * lQ);
                auto w2 = [&](int i, double atyb) {
                    const double f = diag ? V.fact[i] : fs;
                    const double aty = V.ATy[i], wi = V.w[i];
                    const double wbn = V.w_bar[i] + f * (atyb - aty);
                    if (full) {
                        V.dw[i] = wbn - wi;
                        V.ATdy[i] = atyb - aty;
                        V.w_bar[i] = wbn;
                        V.ATy_bar[i] = atyb;
                    }
                    V.w[i] = h1 * V.last_w[i] + h2 * (2.0 * wbn - wi);
                    V.ATy[i] = h1 * V.last_ATy[i] + h2 * (2.0 * atyb - aty);
                };
                if (m > 0) cta_spmv<kBT>(AT, V.y_bar, w2);
                else
                    for (int i = tid; i < n; i += kBT) w2(i, 0.0);
                __syncthreads();
            }
        };

        // ---- M-norm (reference control.cu:243-332) ---------------------------
        auto m_norm = [&]() -> double {
            double a[4] = {0, 0, 0, 0};
            const int ops4[4] = {kSum, kSum, kSum, kSum};
            cta_spmv<kBT>(Q, V.dw, [&](int i, double v) {
                V.dQw[i] = v;
                const double dx = V.dx[i];
                a[0] += dx * dx;
                a[1] += v * dx;
                a[2] += v * v;
                a[3] += V.dw[i] * v;
            });
            __syncthreads();
            double b[2] = {0, 0}, c3[3] = {0, 0, 0};
            const int ops2[2] = {kSum, kSum}, ops3[3] = {kSum, kSum, kSum};
            if (m > 0) {
                cta_spmv<kBT>(AT, V.dy, [&](int i, double v) {
                    V.ATdy[i] = v;
                    b[0] += v * V.dx[i];
                });
                for (int i = tid; i < m; i += kBT) b[1] += V.dy[i] * V.dy[i];
                __syncthreads();
                cta_spmv<kBT>(Q, V.ATdy, [&](int i, double v) {
                    V.QATdy[i] = v;
                    const double at = V.ATdy[i];
                    c3[0] += V.dQw[i] * at;
                    c3[1] += at * v;
                    if (S.q_is_diag) c3[2] += (at * V.fact_M[i]) * v;
                });
            }
            cta_allreduce<4, kBW>(a, ops4, s_red, s_out);
            cta_allreduce<2, kBW>(b, ops2, s_red, s_out);
            cta_allreduce<3, kBW>(c3, ops3, s_red, s_out);
            const double sigma = S.sigma, lA = S.lA, lQ = S.lQ;
            double m1 = 0.0, m3 = 0.0, m2 = (1.0 / sigma) * a[0];
            m2 -= 2.0 * a[1];
            if (m > 0) {
                m1 = sigma * lA * b[1];
                m1 -= 2.0 * sigma * c3[0];
                m2 += 2.0 * b[0];
                if (S.q_is_diag) {
                    m3 = c3[2];
                    m1 += sigma * a[2];
                } else {
                    m3 = (sigma * sigma) / (1.0 + sigma * lQ) * c3[1];
                    m1 += sigma * lQ * a[3];
                }
            } else if (!S.q_is_diag) {
                m1 = sigma * lQ * a[3];
            }
            m2 += m1 > 0.0 ? m1 : 0.0;
            return sqrt((m2 > 0.0 ? m2 : 0.0) + (m3 > 0.0 ? m3 : 0.0));
        };

        // ---- sigma update (reference control.cu:334-529) ----------------------
        auto sigma_update = [&]() {
            const double sigma_old = S.sigma, lA = S.lA, lQ = S.lQ;
            double d[2] = {0, 0};
            const int ops2[2] = {kSum, kSum};
            for (int i = tid; i < n; i += kBT) {
                const double dx = V.x_bar[i] - V.last_x[i];
                V.dx[i] = dx;
                V.dw[i] = V.w_bar[i] - V.last_w[i];
                d[0] += dx * dx;
                if (m > 0) V.ATdy[i] = V.ATy_bar[i] - V.last_ATy[i];
            }
            for (int i = tid; i < m; i += kBT) {
                const double dy = V.y_bar[i] - V.last_y[i];
                V.dy[i] = dy;
                d[1] += dy * dy;
            }
            __syncthreads();
            double e3[3] = {0, 0, 0}, f1v[1] = {0};
            const int ops3[3] = {kSum, kSum, kSum}, ops1[1] = {kSum};
            cta_spmv<kBT>(Q, V.dw, [&](int i, double v) {
                V.dQw[i] = v;
                if (m > 0) e3[0] += v * V.ATdy[i];
                e3[1] += v * v;
                e3[2] += V.dw[i] * v;
            });
            if (m > 0) {
                cta_spmv<kBT>(Q, V.ATdy, [&](int i, double v) {
                    V.QATdy[i] = v;
                    f1v[0] += V.ATdy[i] * v;
                });
            }
            cta_allreduce<2, kBW>(d, ops2, s_red, s_out);
            cta_allreduce<3, kBW>(e3, ops3, s_red, s_out);
            cta_allreduce<1, kBW>(f1v, ops1, s_red, s_out);
            double a = 0.0, b = d[0], c_term = 0.0, d_term = 0.0;
            if (m > 0) a = lA * d[1] - 2.0 * e3[0];
            if (S.q_is_diag) {
                a += e3[1];
            } else {
                a += lQ * e3[2];
                if (m > 0) {
                    c_term = f1v[0];
                    d_term = lQ;
                }
            }
            a = fmax(a, 1e-12);
            b = fmax(b, 1e-12);
            double est;
            if (S.q_is_diag && m > 0) {
                // golden section with a CTA-wide sum per probe
                double left = 1e-12, right = 1e12;
                const double phi = (sqrt(5.0) - 1.0) / 2.0;
                auto f = [&](double xp) {
                    double t[1] = {0.0};
                    for (int i = tid; i < n; i += kBT) t[0] += V.ATdy[i] * (V.QATdy[i] / (1.0 + xp * V.diag_Q[i]));
                    cta_allreduce<1, kBW>(t, ops1, s_red, s_out);
                    return a * xp + b / xp + xp * xp * t[0];
                };
                double x1 = right - phi * (right - left), x2 = left + phi * (right - left);
                double fa = f(x1), fb = f(x2);
                for (int it = 0; it < 200; ++it) {
                    if (fabs(right - left) <= 1e-12 * fmax(1.0, fabs(left))) break;
                    if (fa > fb) {
                        left = x1;
                        x1 = x2;
                        fa = fb;
                        x2 = left + phi * (right - left);
                        fb = f(x2);
                    } else {
                        right = x2;
                        x2 = x1;
                        fb = fa;
                        x1 = right - phi * (right - left);
                        fa = f(x1);
                    }
                }
                est = fa < fb ? x1 : x2;
            } else if (!S.q_is_diag && m > 0) {
                const double cc = c_term > 0.0 ? c_term : 0.0, dd = d_term > 0.0 ? d_term : 0.0;
                double left = 1e-12, right = 1e12;
                const double ip = (sqrt(5.0) - 1.0) / 2.0, ip2 = (3.0 - sqrt(5.0)) / 2.0;
                auto f = [&](double xp) { return a * xp + b / xp + cc * xp * xp / (1.0 + dd * xp); };
                double x1 = left + ip2 * (right - left), x2 = left + ip * (right - left);
                double fa = f(x1), fb = f(x2);
                for (int it = 0; it < 256; ++it) {
                    if (fabs(right - left) <= 1e-13 * fmax(1.0, fmax(fabs(left), fabs(right)))) break;
                    if (fa > fb) {
                        left = x1;
                        x1 = x2;
                        fa = fb;
                        x2 = left + ip * (right - left);
                        fb = f(x2);
                    } else {
                        right = x2;
                        x2 = x1;
                        fb = fa;
                        x1 = left + ip2 * (right - left);
                        fa = f(x1);
                    }
                }
                est = 0.5 * (left + right);
            } else {
                est = sqrt(b / a);
            }
            if (tid == 0) {
                est = clampd(est, 1e-12, 1e12);
                const double fact =
                    (S.best_gap > 0.0 && isfinite(S.best_gap)) ? exp(-0.05 * (S.current_gap / S.best_gap)) : 1.0;
                const double cand =
                    exp(fact * log(est) + (1.0 - fact) * log(S.best_sigma > 0.0 ? S.best_sigma : sigma_old));
                double kappa = 1.0;
                const double t1 = fmax(fmin(S.rd, S.rp), fmin(S.gap, S.current_gap));
                if (t1 <= 9e-10 && S.rp > 0.0) {
                    const double ratio = S.rd / S.rp;
                    kappa = t1 > 5e-10 ? clampd(sqrt(ratio), 1e-2, 100.0) : clampd(ratio, 1e-2, 100.0);
                }
                S.sigma = clampd(kappa * cand, 1e-12, 1e12);
                S.scal[0] = sigma_old;
            }
            __syncthreads();
            if (S.q_is_diag && fabs(S.sigma - S.scal[0]) > 1e-15) {
                const double sg = S.sigma;
                for (int i = tid; i < n; i += kBT) {
                    const double inv = 1.0 / (1.0 + sg * V.diag_Q[i]);
                    V.fact2[i] = inv;
                    V.fact[i] = sg * inv;
                    V.fact1[i] = sg * V.diag_Q[i] * inv;
                    V.fact_M[i] = sg * sg * inv;
                }
                __syncthreads();
            }
        };

        auto restart_apply = [&]() {
            for (int i = tid; i < n; i += kBT) {
                const double xb = V.x_bar[i], wb = V.w_bar[i];
                V.x[i] = V.last_x[i] = xb;
                V.w[i] = V.last_w[i] = wb;
                if (S.noC) V.Qw[i] = V.last_Qw[i] = V.Qw_bar[i];
            }
            for (int i = tid; i < m; i += kBT) V.y[i] = V.last_y[i] = V.y_bar[i];
            if (m > 0) {
                cta_spmv<kBT>(AT, V.y_bar, [&](int i, double s) { V.ATy_bar[i] = V.ATy[i] = V.last_ATy[i] = s; });
            }
            __syncthreads();
            if (tid == 0) {
                S.last_gap = S.current_gap;
                S.save_gap = INFINITY;
                S.times += 1;
                S.inner = 0;
            }
            __syncthreads();
        };

        // ---- outer loop (reference solver_backend.c:432-513) ------------------
        const unsigned long long loop_t0 = globaltimer_ns();  // used by thread 0
        // one log record of the current residuals (the host loop's print_log)
        auto log_record = [&](long long it) {
            if (!B.log_buf || k != 0) return;
            const int slot = *B.log_count;
            if (slot >= B.log_cap) return;
            double *r = B.log_buf + (size_t)slot * kLogFields;
            r[0] = (double)it;
            r[1] = S.rp;
            r[2] = S.rd;
            r[3] = S.pobj;
            r[4] = S.dobj;
            r[5] = S.gap;
            r[6] = S.sigma;
            r[7] = 1e-9 * (double)(globaltimer_ns() - loop_t0);
            *B.log_count = slot + 1;
        };
        // first checked iteration below 1e-4 / 1e-6 (the host loop's milestones)
        auto milestones = [&](long long it) {
            const double el = 1e-9 * (double)(globaltimer_ns() - loop_t0);
            if (!S.got4 && S.kkt < 1e-4) {
                S.got4 = 1;
                if (B.iter4_out) {
                    B.iter4_out[k] = it;
                    B.time4_out[k] = el;
                }
            }
            if (!S.got6 && S.kkt < 1e-6) {
                S.got6 = 1;
                if (B.iter6_out) {
                    B.iter6_out[k] = it;
                    B.time6_out[k] = el;
                }
            }
        };
        residuals(0);
        if (tid == 0) {
            S.got4 = S.got6 = 0;
            if (B.iter4_out) B.iter4_out[k] = B.iter6_out[k] = -1;
            milestones(0);
            log_record(0);
        }
        long long iter;
        for (iter = 0;; ++iter) {
            if (tid == 0) {
                const double el = 1e-9 * (double)(globaltimer_ns() - (B.time_from_loop ? loop_t0 : B.t_start));
                if (iter % kAbortPoll == 0 && !S.aborted && abort_requested(B.abort_flag)) S.aborted = 1;
                // an abort request stops the instance like the time limit
                const bool over = el > B.time_limit || S.aborted;
                int print_yes = 0;
                if (iter > 0) {
                    if (B.print_frequency == -1 &&
                        (on_print_grid(iter) || iter == B.max_iter || over))
                        print_yes = 1;
                    if (B.print_frequency > 0 && (divides(iter, B.print_frequency) || iter == B.max_iter || over))
                        print_yes = 1;
                }
                S.do_res = iter > 0 && ((B.check_iter > 0 && divides(iter, B.check_iter)) || print_yes);
                S.print_yes = print_yes;
                S.scal[1] = el;
            }
            __syncthreads();
            PHASE_ADD(3);
            if (S.do_res) residuals(iter);
            PHASE_ADD(4);
            if (tid == 0) {
                const double el = S.scal[1];
                if (S.do_res) milestones(iter);
                int fs;
                // a warm start is not an HPR iterate: its y and z need not lie
                // in the normal cones the residual formulas assume, so it is
                // not accepted as optimal before the first step
                if (S.kkt < B.stoptol && !(warm && iter == 0)) fs = 6;
                else if (iter == B.max_iter) fs = 4;
                else if (el > B.time_limit || S.aborted) fs = 5;
                else fs = 7;
                S.final_status = fs;
                // restart_check (src/cpu/control.c:231-282)
                const long long ci = B.check_iter;
                if (ci > 0) {
                    S.restart_flag = 0;
                    if (S.first_restart) {
                        if (iter == ci) {
                            S.first_restart = 0;
                            S.restart_flag = 1;
                            S.weighted_norm = S.current_gap;
                            S.best_gap = S.current_gap;
                            S.best_sigma = S.sigma;
                        }
                    } else if (divides(iter, ci)) {
                        if (S.current_gap < 0.0) S.current_gap = 1e-6;
                        if (S.current_gap <= 0.2 * S.last_gap) S.restart_flag = 1;
                        if (S.current_gap <= 0.8 * S.last_gap && S.current_gap > S.save_gap) S.restart_flag = 2;
                        const double f =
                            (S.weighted_norm > 0.0 && S.current_gap / S.weighted_norm > 1e-1) ? 0.5 : 0.2;
                        if ((double)S.inner >= f * (double)iter) S.restart_flag = 3;
                        if (S.best_gap > S.current_gap) {
                            S.best_gap = S.current_gap;
                            S.best_sigma = S.sigma;
                        }
                        S.save_gap = S.current_gap;
                    }
                }
            }
            __syncthreads();
            if (S.restart_flag > 0) {
                sigma_update();
                restart_apply();
            }
            PHASE_ADD(6);
            if (tid == 0 && (S.print_yes || S.final_status != 7)) log_record(iter);
            if (S.final_status != 7) break;
            if (tid == 0) {
                const long long nx = iter + 1;
                int t = 0;
                if (B.check_iter > 0 && divides(nx, B.check_iter)) t = 1;
                if (S.restart_flag > 0) t = 1;
                if (B.print_frequency == -1 && on_print_grid(nx)) t = 1;
                if (B.print_frequency > 0 && divides(nx, B.print_frequency)) t = 1;
                S.to_check = t;
            }
            __syncthreads();
            step(S.to_check);
            PHASE_ADD(3);
            const bool at_check = B.check_iter > 0 && divides(iter + 1, B.check_iter);
            if (S.restart_flag > 0 || at_check) {
                const double g = m_norm();
                if (tid == 0) {
                    if (S.restart_flag > 0) S.last_gap = g;
                    if (at_check) S.current_gap = g;
                    if (!isfinite(g)) S.final_status = 1;
                }
                __syncthreads();
                PHASE_ADD(5);
                if (S.final_status == 1) break;
            }
            if (tid == 0) S.inner += 1;
            __syncthreads();
        }

        // ---- output (reference workspace.cu:427-511) ---------------------------
        for (int i = tid; i < n; i += kBT) {
            const double cn = V.col_norm[i];
            B.x[I.var + i] = V.x_bar[i] / cn;
            B.w[I.var + i] = V.w_bar[i] / cn;
            B.z[I.var + i] = V.z_bar[i] * cn;
            if (B.active_x) B.active_x[I.var + i] = V.z_bar[i] != 0.0;
            B.col_norm_out[I.var + i] = cn;
        }
        for (int i = tid; i < m; i += kBT) {
            B.y[I.row + i] = V.y_bar[i] / V.row_norm[i];
            if (B.active_r) B.active_r[I.row + i] = V.y_bar[i] != 0.0;
            B.row_norm_out[I.row + i] = V.row_norm[i];
        }
        if (B.phase_clk && tid == 0) B.phase_clk[blockIdx.x * 8 + 7] += (unsigned long long)(clock64() - _ptot);
        if (tid == 0) {
            B.status[k] = S.final_status;
            B.iters[k] = iter;
            B.pobj[k] = S.pobj;
            B.resid[k] = S.kkt;
            B.gap[k] = S.gap;
            B.restarts[k] = (int)S.times;
            B.sigma_out[k] = S.sigma;
            B.seconds_out[k] = 1e-9 * (double)(globaltimer_ns() - inst_t0);
            if (B.loop_seconds_out) B.loop_seconds_out[k] = 1e-9 * (double)(globaltimer_ns() - loop_t0);
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// implicit-differentiation adjoint: MINRES on the active-set KKT operator
// ---------------------------------------------------------------------------
// For each instance, with F = {i : z_i == 0} (variables off their bounds)
// and R = {r : y_r != 0} (rows at a bound), solve
//     [[Q_FF, A_RF'], [A_RF, 0]] [lam_F; mu_R] = [gx_F; -gy_R]
// matrix-free.  The solve runs on the scaled matrices the last
// hprqp_batch_solve left on the device: with D = diag(col_norm, row_norm),
// K = D Ks D, so Ks (D lam) = D^-1 rhs and lam = D^-1 sol.  The operator is
// applied as P Ks P with P the 0/1 active-set mask (read from z and y), so
// every Krylov vector stays inside the active subspace.  MINRES is the
// Paige-Saunders recurrence (Lanczos three-term step + Givens QR of the
// tridiagonal), one instance per CTA; the three Lanczos vectors, which are
// the SpMV gather sources, live in shared memory when they fit.
struct AdjArgs {
    int K;
    const BInst *inst;
    const int *order;
    unsigned long long *counter;  // the work queue's two ends (take_instance)
    const int *q_rp, *q_ci, *a_rp, *a_ci, *at_rp, *at_ci;
    const double *q_v, *a_v, *at_v;             // scaled matrices left by the last solve
    const double *col_norm, *row_norm, *z, *y;  // per instance, packed
    const double *gx, *gy;                      // loss gradients (packed; gy may be null)
    double *lam_x, *lam_y;                      // outputs: lambda, mu (original space)
    int *iters;
    double *relres;
    double tol;
    int maxit_factor;
    double *ws;
    size_t ws_stride;
    int nmax, mmax;
    int lanczos_smem;  // 1: the Lanczos vectors live in shared memory
};

constexpr int kAdjGlobalN = 5, kAdjGlobalM = 4;  // sol, w_old, w, w_new (+ Q v) per CTA in global memory
constexpr int kAdjLanczos = 3;                   // v_old, v, v_new (n and m parts)

template <int BT>
__global__ void __launch_bounds__(BT, ctas_per_sm(BT)) k_batch_adjoint(const AdjArgs B)
{
    constexpr int kBT = BT, kBW = BT / 32;
    extern __shared__ __align__(16) double dyn_smem[];
    __shared__ double s_red[kBW][8];
    __shared__ double s_out[8];
    __shared__ int s_inst;
    const int tid = threadIdx.x;
    const int na = (B.nmax + 31) & ~31, ma = (B.mmax + 31) & ~31;
    double *g = B.ws + (size_t)blockIdx.x * B.ws_stride;
    double *lz = B.lanczos_smem ? dyn_smem : g + kAdjGlobalN * (size_t)na + kAdjGlobalM * (size_t)ma;
    for (;;) {
        if (tid == 0) {
            s_inst = take_instance(B.counter, B.order, B.K);
        }
        __syncthreads();
        const int k = s_inst;
        __syncthreads();
        if (k < 0) break;
        const BInst I = B.inst[k];
        const int n = I.n, m = I.m;
        const LCsr Q{n, B.q_rp + I.q_rp, B.q_ci + I.q_nz, B.q_v + I.q_nz, I.q_lg};
        const LCsr A{m, B.a_rp + I.a_rp, B.a_ci + I.a_nz, B.a_v + I.a_nz, I.a_lg};
        const LCsr AT{n, B.at_rp + I.at_rp, B.at_ci + I.at_nz, B.at_v + I.at_nz, I.at_lg};
        const double *cn = B.col_norm + I.var, *rn = B.row_norm + I.row;
        const double *zk = B.z + I.var, *yk = B.y + I.row;
        double *sol_n = g, *wo_n = g + na, *w_n = g + 2 * na, *wn_n = g + 3 * na, *tmp = g + 4 * na;
        double *gm = g + kAdjGlobalN * (size_t)na;
        double *sol_m = gm, *wo_m = gm + ma, *w_m = gm + 2 * ma, *wn_m = gm + 3 * ma;
        double *vo_n = lz, *v_n = lz + na, *vn_n = lz + 2 * na;
        double *vo_m = lz + 3 * na, *v_m = lz + 3 * na + ma, *vn_m = lz + 3 * na + 2 * ma;
        const int ops1[1] = {kSum};
        double b2[1] = {0.0};
        for (int i = tid; i < n; i += kBT) {
            const double rhs = zk[i] == 0.0 ? B.gx[I.var + i] / cn[i] : 0.0;  // D^-1 P rhs
            v_n[i] = rhs;
            b2[0] += rhs * rhs;
            sol_n[i] = vo_n[i] = wo_n[i] = w_n[i] = 0.0;
        }
        for (int r = tid; r < m; r += kBT) {
            const double rhs = (B.gy && yk[r] != 0.0) ? -B.gy[I.row + r] / rn[r] : 0.0;
            v_m[r] = rhs;
            b2[0] += rhs * rhs;
            sol_m[r] = vo_m[r] = wo_m[r] = w_m[r] = 0.0;
        }
        cta_allreduce<1, kBW>(b2, ops1, s_red, s_out);
        const double beta0 = sqrt(b2[0]);
        double beta = beta0, eta = beta0;
        double c_old = 1.0, c = 1.0, s_old = 0.0, s = 0.0;
        int it = 0;
        if (beta0 > 0.0) {
            const double inv = 1.0 / beta0;
            for (int i = tid; i < n; i += kBT) v_n[i] *= inv;
            for (int r = tid; r < m; r += kBT) v_m[r] *= inv;
            __syncthreads();
            const int maxit = B.maxit_factor * (n + m) + 100;
            for (it = 0; it < maxit; ++it) {
                // v_new = P Ks P v.  Q and A' have the same number of rows, so
                // cta_spmv calls their epilogues for row i on the same thread
                // and tmp[i] is written and read by that thread.
                if (m > 0) {
                    cta_spmv<kBT>(Q, v_n, [&](int i, double q) { tmp[i] = q; });
                    cta_spmv<kBT>(A, v_n, [&](int r, double a) { vn_m[r] = yk[r] != 0.0 ? a : 0.0; });
                    cta_spmv<kBT>(AT, v_m,
                             [&](int i, double at) { vn_n[i] = zk[i] == 0.0 ? tmp[i] + at : 0.0; });
                } else {
                    cta_spmv<kBT>(Q, v_n, [&](int i, double q) { vn_n[i] = zk[i] == 0.0 ? q : 0.0; });
                }
                __syncthreads();
                double al[1] = {0.0};
                for (int i = tid; i < n; i += kBT) al[0] += v_n[i] * vn_n[i];
                for (int r = tid; r < m; r += kBT) al[0] += v_m[r] * vn_m[r];
                cta_allreduce<1, kBW>(al, ops1, s_red, s_out);
                const double alpha = al[0];
                double bn[1] = {0.0};
                for (int i = tid; i < n; i += kBT) {
                    const double t = vn_n[i] - alpha * v_n[i] - beta * vo_n[i];
                    vn_n[i] = t;
                    bn[0] += t * t;
                }
                for (int r = tid; r < m; r += kBT) {
                    const double t = vn_m[r] - alpha * v_m[r] - beta * vo_m[r];
                    vn_m[r] = t;
                    bn[0] += t * t;
                }
                cta_allreduce<1, kBW>(bn, ops1, s_red, s_out);
                const double beta_new = sqrt(bn[0]);
                // Givens QR of the new tridiagonal column
                const double r1h = c * alpha - c_old * s * beta;
                const double r1 = sqrt(r1h * r1h + beta_new * beta_new);
                const double r2 = s * alpha + c_old * c * beta;
                const double r3 = s_old * beta;
                const double c_new = r1 > 0.0 ? r1h / r1 : 1.0;
                const double s_new = r1 > 0.0 ? beta_new / r1 : 0.0;
                const double inv_r1 = r1 > 0.0 ? 1.0 / r1 : 0.0;
                const double step = c_new * eta;
                const double inv_b = beta_new > 0.0 ? 1.0 / beta_new : 0.0;
                for (int i = tid; i < n; i += kBT) {
                    const double wn = (v_n[i] - r3 * wo_n[i] - r2 * w_n[i]) * inv_r1;
                    wn_n[i] = wn;
                    sol_n[i] += step * wn;
                    vn_n[i] *= inv_b;
                }
                for (int r = tid; r < m; r += kBT) {
                    const double wn = (v_m[r] - r3 * wo_m[r] - r2 * w_m[r]) * inv_r1;
                    wn_m[r] = wn;
                    sol_m[r] += step * wn;
                    vn_m[r] *= inv_b;
                }
                eta = -s_new * eta;
                __syncthreads();
                // rotate v_old <- v <- v_new and w_old <- w <- w_new
                double *t0 = vo_n;
                vo_n = v_n;
                v_n = vn_n;
                vn_n = t0;
                t0 = vo_m;
                vo_m = v_m;
                v_m = vn_m;
                vn_m = t0;
                t0 = wo_n;
                wo_n = w_n;
                w_n = wn_n;
                wn_n = t0;
                t0 = wo_m;
                wo_m = w_m;
                w_m = wn_m;
                wn_m = t0;
                beta = beta_new;
                c_old = c;
                c = c_new;
                s_old = s;
                s = s_new;
                if (fabs(eta) <= B.tol * beta0 || beta_new == 0.0) {
                    ++it;
                    break;
                }
            }
        }
        for (int i = tid; i < n; i += kBT) B.lam_x[I.var + i] = sol_n[i] / cn[i];
        for (int r = tid; r < m; r += kBT) B.lam_y[I.row + r] = sol_m[r] / rn[r];
        if (tid == 0) {
            B.iters[k] = it;
            B.relres[k] = beta0 > 0.0 ? fabs(eta) / beta0 : 0.0;
        }
        __syncthreads();
    }
}

__global__ void k_batch_clock(unsigned long long *t)
{
    *t = globaltimer_ns();
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
#define B_CK(call)                                                                                     \
    do {                                                                                               \
        cudaError_t err__ = (call);                                                                    \
        if (err__ != cudaSuccess) {                                                                    \
            fprintf(stderr, "hprqp-b200 batch: CUDA error %s at %s:%d\n", cudaGetErrorString(err__), __FILE__, \
                    __LINE__);                                                                         \
            return HPRQP_STATUS_NOT_IMPLEMENTED;                                                       \
        }                                                                                              \
    } while (0)

}  // namespace hpr

// std::vector storage without value-initialisation: the packing arrays are
// fully written by the packing threads, so zero-filling gigabytes first is waste
template <class T>
struct NoInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = NoInitAlloc<U>;
    };
    NoInitAlloc() = default;
    template <class U>
    NoInitAlloc(const NoInitAlloc<U> &) noexcept {}
    template <class U>
    void construct(U *p) noexcept
    {
        ::new ((void *)p) U;
    }
    template <class U, class... Args>
    void construct(U *p, Args &&...args)
    {
        ::new ((void *)p) U(std::forward<Args>(args)...);
    }
};
template <class T>
using HostVec = std::vector<T, NoInitAlloc<T>>;

struct HPRQPBatch {
    int device = 0;
    int num_sms = 148;
    int cta_threads = 1024;  // threads per CTA of the solve and adjoint kernels (kBigCta or kSmallCta)
    // kBigCta batches: the last k_mid instances of the solve's work order
    // (mid_cta_instance) are solved by kMidCta CTAs in a launch of their own
    // on `stream`, the others by kBigCta CTAs on stream_mid
    size_t k_mid = 0;
    cudaStream_t stream = nullptr, stream_mid = nullptr;
    int ws_slots = 0, phase_slots = 0;  // per-CTA workspaces and phase counters allocated
    size_t K = 0;
    std::vector<size_t> var_off, row_off;          // original packing (caller's layout)
    std::vector<int> n_k, m_k;                      // preprocessed sizes
    std::vector<std::vector<size_t>> kept_rows;     // per instance: original local row of each kept row
    std::vector<hpr::BInst> inst;
    std::vector<int> tuned_lg;  // autotuned lane-group widths (log2), Q, A, A' per instance
    int forced_lanes = 0;       // hprqp_batch_set_spmv_lanes: 0 = autotuned
    hpr::BInst *d_inst = nullptr;
    size_t total_n = 0, total_m = 0, total_m_orig = 0;
    int nmax = 0, mmax = 0;
    std::vector<void *> allocs;
    hpr::BatchArgs args{};
    double last_ms = 0.0;
    bool solved = false;
    // the caller's CSR index arrays of Q and A (the adjoint writes one value per caller nonzero)
    std::vector<size_t> q_rp_in, q_ci_in, a_rp_in, a_ci_in;
    bool has_caller_csr = false;
    // adjoint buffers, allocated by the first hprqp_batch_backward
    double *adj_gx = nullptr, *adj_gy = nullptr, *adj_lx = nullptr, *adj_ly = nullptr, *adj_rel = nullptr;
    double *adj_ws = nullptr;
    int *adj_it = nullptr;
    unsigned long long *adj_counter = nullptr;
    size_t adj_ws_count = 0;
    double last_adjoint_ms = 0.0;
    // warm start (device packing: total variables, kept rows), set by
    // hprqp_batch_set_warm_start
    double *start_x = nullptr, *start_w = nullptr, *start_y = nullptr, *start_sigma = nullptr;
    unsigned long long *d_t0 = nullptr, *d_phase = nullptr;
    // abort request: one int in host-mapped pinned memory, read by the kernel
    int *h_abort = nullptr, *d_abort = nullptr;
    // host copies of the preprocessed models (kept for the adjoint)
    std::vector<HPRQPModel> models;
};

namespace hpr {

template <class T>
static HPRQPStatus balloc(HPRQPBatch *b, T **p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    void *ptr = nullptr;
    if (cudaMalloc(&ptr, count * sizeof(T)) != cudaSuccess) {
        fprintf(stderr, "hprqp-b200 batch: cudaMalloc(%zu bytes) failed\n", count * sizeof(T));
        return HPRQP_STATUS_ALLOCATION_FAILED;
    }
    b->allocs.push_back(ptr);
    *p = (T *)ptr;
    return HPRQP_STATUS_OK;
}

// Several device arrays carved out of one allocation (256-byte aligned
// slices): a batch's arrays are created together and freed together, and
// one cudaMalloc instead of forty keeps small batches (and solve_gpu of a
// small model) cheap to set up.
class Carver {
public:
    template <class T>
    Carver &add(T **p, size_t count)
    {
        req_.push_back({(void **)p, std::max<size_t>(count, 1) * sizeof(T)});
        return *this;
    }
    HPRQPStatus commit(HPRQPBatch *b)
    {
        size_t total = 0;
        for (auto &r : req_) total += (r.second + 255) & ~size_t(255);
        char *base = nullptr;
        HPRQPStatus st = balloc(b, &base, total);
        if (st != HPRQP_STATUS_OK) return st;
        size_t off = 0;
        for (auto &r : req_) {
            *r.first = base + off;
            off += (r.second + 255) & ~size_t(255);
        }
        return HPRQP_STATUS_OK;
    }

private:
    std::vector<std::pair<void **, size_t>> req_;
};

static void batch_free(HPRQPBatch *b)
{
    for (void *p : b->allocs) cudaFree(p);
    b->allocs.clear();
    if (b->h_abort) cudaFreeHost(b->h_abort);
    b->h_abort = b->d_abort = nullptr;
    for (auto &m : b->models) model_free(&m);
    b->models.clear();
    if (b->stream) cudaStreamDestroy(b->stream);
    if (b->stream_mid) cudaStreamDestroy(b->stream_mid);
    b->stream = b->stream_mid = nullptr;
}

// The per-instance SpMV autotuner: the lane-group width of cta_spmv for one
// matrix, from its row lengths.  For every width g = 1, 2, ..., 32 it walks
// the rows exactly as cta_spmv does (kBW contiguous warp ranges, chunks of
// 32 rows, passes of 32/g rows, rounds of one aligned quad per lane, the row
// with the most quads in a pass setting its rounds) and charges each warp
//     kChunkCost per chunk + per pass (kPassCost + log2(g) kShuffleCost
//     + rounds * kRoundCost);
// the warp with the largest charge sets the product's time, and the width
// with the smallest such time wins (ties: the wider group, whose loads are
// better coalesced).  A round is a 16-byte index load and two 16-byte value
// loads, four dependent gathers and FMAs; a shuffle step is one shuffle of a
// double; a pass moves two row pointers and writes the row sums; a chunk
// reads 33 row pointers and runs the caller's epilogue on its rows.  The
// weights are least-squares fits to the per-instance times of the 4096-QP
// batch recipe solved with each width forced (hprqp_batch_set_spmv_lanes),
// in arbitrary units: a pass costs half a round and a chunk four rounds.
constexpr double kRoundCost = 23.1, kShuffleCost = 0.59, kPassCost = 11.6, kChunkCost = 94.3;

static double lane_group_cost(const size_t *rp, int nrow, int lg, int kBW)
{
    const int g = 1 << lg, rpp = 32 >> lg;
    const int per = (nrow + kBW - 1) / kBW;
    double worst = 0.0;
    for (int w = 0; w < kBW; ++w) {
        const int w0 = std::min(w * per, nrow), w1 = std::min(w0 + per, nrow);
        double cost = 0.0;
        for (int c0 = w0; c0 < w1; c0 += 32) {
            const int nr = std::min(32, w1 - c0);
            cost += kChunkCost;
            for (int p0 = 0; p0 < nr; p0 += rpp) {
                size_t most = 0;
                for (int r = c0 + p0; r < std::min(c0 + p0 + rpp, c0 + nr); ++r)
                    if (rp[r + 1] > rp[r]) most = std::max(most, ((rp[r + 1] + 3) >> 2) - (rp[r] >> 2));
                const size_t rounds = (most + (size_t)g - 1) / (size_t)g;
                cost += kPassCost + lg * kShuffleCost + (double)rounds * kRoundCost;
            }
        }
        worst = std::max(worst, cost);
    }
    return worst;
}

static int choose_lane_group(const size_t *rp, int nrow, int warps)
{
    int best = 0;
    double best_cost = 0.0;
    for (int lg = 0; lg <= 5; ++lg) {
        const double c = lane_group_cost(rp, nrow, lg, warps);
        if (lg == 0 || c <= best_cost) {
            best = lg;
            best_cost = c;
        }
    }
    return best;
}

// extract instance k of a block-diagonal CSR (rows [r0, r1), columns
// [c0, c1)) as a local CSR view into freshly allocated arrays
static HPRQPStatus extract_block(const HPRQPMatrixCSR *M, size_t r0, size_t r1, size_t c0, size_t c1,
                                 std::vector<size_t> &rp, std::vector<size_t> &ci, std::vector<double> &v)
{
    rp.assign(r1 - r0 + 1, 0);
    ci.clear();
    v.clear();
    for (size_t r = r0; r < r1; ++r) {
        for (size_t k = M->row_ptr[r]; k < M->row_ptr[r + 1]; ++k) {
            const size_t c = M->col_ind[k];
            if (c < c0 || c >= c1) return HPRQP_STATUS_INVALID_ARGUMENT;  // not block diagonal
            ci.push_back(c - c0);
            v.push_back(M->values[k]);
        }
        rp[r - r0 + 1] = ci.size();
    }
    return HPRQP_STATUS_OK;
}

}  // namespace hpr

extern "C" {

void hprqp_batch_params_set_defaults(HPRQPBatchParams *p)
{
    if (!p) return;
    memset(p, 0, sizeof(*p));
    p->stoptol = 1e-6;
    p->max_iter = (size_t)INT_MAX;
    p->time_limit = 3600.0;
    p->check_iter = 100;
    p->print_frequency = -1;
    p->use_scaling = 1;
    p->device_number = 0;
}

// an instance's work measure: nonzeros the products of one HPR step stream,
// plus its variables
static long long instance_work(const HPRQPModel &M)
{
    return (long long)M.Q.nnz + 2 * (long long)M.A.nnz + (long long)M.Q.ncol;
}

// whether an instance of a batch of 1024-thread CTAs is solved by a kMidCta CTA
static bool mid_cta_instance(const HPRQPModel &M)
{
    using namespace hpr;
    return M.Q.ncol <= (size_t)kMidCta && M.A.nrow <= (size_t)kMidCta && instance_work(M) <= kMidCtaMaxWork;
}

static HPRQPStatus batch_create_impl(size_t K, const size_t *var_offsets, const size_t *row_offsets,
                                     const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c,
                                     const double *AL, const double *AU, const double *l, const double *u,
                                     const double *obj_constants, int device_number, bool keep_caller_csr,
                                     HPRQPBatch **out, bool abortable = true, size_t k_begin = 0,
                                     size_t k_count = 0, int cta_threads = 0, const size_t *subset = nullptr)
{
    // instances [k_begin, k_begin + k_count) of the caller's batch (k_count 0:
    // all of them), or, when subset is given, the k_count instances
    // subset[0..k_count) (distinct caller indices; k_begin unused); the batch
    // packs them one after the other in that order
    using namespace hpr;
    if (!out || !var_offsets || !row_offsets || !Q || !A || !c || !l || !u || K == 0)
        return HPRQP_STATUS_INVALID_ARGUMENT;
    *out = nullptr;
    if (!matrix_csr_is_valid(Q) || !matrix_csr_is_valid(A) || Q->nrow != Q->ncol || A->ncol != Q->ncol ||
        var_offsets[0] != 0 || row_offsets[0] != 0 || var_offsets[K] != Q->nrow || row_offsets[K] != A->nrow)
        return HPRQP_STATUS_INVALID_ARGUMENT;
    if (A->nrow > 0 && (!AL || !AU)) return HPRQP_STATUS_INVALID_ARGUMENT;
    for (size_t k = 0; k < K; ++k)
        if (var_offsets[k + 1] < var_offsets[k] || row_offsets[k + 1] < row_offsets[k])
            return HPRQP_STATUS_INVALID_ARGUMENT;
    if (subset) {
        if (k_count == 0 || k_count > K || keep_caller_csr) return HPRQP_STATUS_INVALID_ARGUMENT;
        for (size_t j = 0; j < k_count; ++j)
            if (subset[j] >= K) return HPRQP_STATUS_INVALID_ARGUMENT;
        k_begin = 0;
    }
    if (k_count == 0) k_count = K - k_begin;
    if (k_begin >= K || k_count > K - k_begin || (keep_caller_csr && k_count != K))
        return HPRQP_STATUS_INVALID_ARGUMENT;
    const size_t kb = k_begin;
    // the caller's index of instance k of this batch
    auto caller = [&](size_t k) { return subset ? subset[k] : kb + k; };
    K = k_count;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        fprintf(stderr, "hprqp-b200: no CUDA device available; this engine has no CPU fallback\n");
        return HPRQP_STATUS_NOT_IMPLEMENTED;
    }
    if (device_number < 0 || device_number >= ndev) return HPRQP_STATUS_INVALID_ARGUMENT;
    int sms = 148;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_number) != cudaSuccess) {
        cudaGetLastError();
        sms = 148;
    }

    const char *trc = getenv("HPRQP_B200_BATCH_TRACE");
    const bool ctrace = trc && trc[0] == '1';
    auto cnow = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
    const double c0 = cnow();
    HPRQPBatch *b = new HPRQPBatch();
    b->K = K;
    b->device = device_number;
    // 512-thread CTAs (two per SM) when one wave of them holds the whole
    // batch and one wave of 1024-thread CTAs does not
    b->cta_threads = (K > (size_t)sms && K <= (size_t)2 * sms) ? kSmallCta : kBigCta;
    if (cta_threads == kSmallCta || cta_threads == kBigCta) b->cta_threads = cta_threads;
    b->var_off.assign(K + 1, 0);
    b->row_off.assign(K + 1, 0);
    for (size_t k = 0; k < K; ++k) {
        const size_t kk = caller(k);
        b->var_off[k + 1] = b->var_off[k] + (var_offsets[kk + 1] - var_offsets[kk]);
        b->row_off[k + 1] = b->row_off[k] + (row_offsets[kk + 1] - row_offsets[kk]);
    }
    b->total_m_orig = b->row_off[K];
    b->models.resize(K);
    for (auto &mm : b->models) model_init(&mm);
    b->kept_rows.resize(K);
    if (keep_caller_csr) {  // the adjoint maps gradients to the caller's nonzeros
        b->q_rp_in.assign(Q->row_ptr, Q->row_ptr + Q->nrow + 1);
        b->q_ci_in.assign(Q->col_ind, Q->col_ind + Q->nnz);
        b->a_rp_in.assign(A->row_ptr, A->row_ptr + A->nrow + 1);
        b->a_ci_in.assign(A->col_ind, A->col_ind + A->nnz);
    }
    b->has_caller_csr = keep_caller_csr;
    // ---- per-instance build + preprocess (the single-QP builder), threaded
    std::vector<HPRQPStatus> st_k(K, HPRQP_STATUS_OK);
    const unsigned nth = (unsigned)std::max<size_t>(1, std::min<size_t>(std::min(std::thread::hardware_concurrency(), 32u), K));
    auto worker = [&](unsigned tix) {
        std::vector<size_t> qrp, qci, arp, aci;
        std::vector<double> qv, av;
        for (size_t k = tix; k < K; k += nth) {
            const size_t kk = caller(k);
            const size_t v0 = var_offsets[kk], v1 = var_offsets[kk + 1], r0 = row_offsets[kk], r1 = row_offsets[kk + 1];
            HPRQPStatus st = extract_block(Q, v0, v1, v0, v1, qrp, qci, qv);
            if (st == HPRQP_STATUS_OK) st = extract_block(A, r0, r1, v0, v1, arp, aci, av);
            if (st != HPRQP_STATUS_OK) {
                st_k[k] = st;
                continue;
            }
            size_t e_idx = 0;
            double e_val = 0.0;
            HPRQPMatrixCSR q{v1 - v0, v1 - v0, qci.size(), qrp.data(), qci.empty() ? &e_idx : qci.data(),
                             qv.empty() ? &e_val : qv.data(), 0};
            HPRQPMatrixCSR a{r1 - r0, v1 - v0, aci.size(), arp.data(), aci.empty() ? &e_idx : aci.data(),
                             av.empty() ? &e_val : av.data(), 0};
            st = build_from_QAbc(&q, &a, c + v0, r1 > r0 ? AL + r0 : nullptr, r1 > r0 ? AU + r0 : nullptr, l + v0,
                                 u + v0, obj_constants ? obj_constants[kk] : 0.0, &b->models[k]);
            st_k[k] = st;
            if (st == HPRQP_STATUS_OK) {
                // record which original rows survived preprocessing
                auto &kr = b->kept_rows[k];
                kr.clear();
                for (size_t r = r0; r < r1; ++r) {
                    const size_t len = A->row_ptr[r + 1] - A->row_ptr[r];
                    const bool free_row = std::isinf(AL[r]) && AL[r] < 0 && std::isinf(AU[r]) && AU[r] > 0;
                    if (len > 0 && !free_row) kr.push_back(r - r0);
                }
            }
        }
    };
    {
        std::vector<std::thread> th;
        if (nth == 1) worker(0);
        else
            for (unsigned t = 0; t < nth; ++t) th.emplace_back(worker, t);
        for (auto &t : th) t.join();
    }
    for (size_t k = 0; k < K; ++k)
        if (st_k[k] != HPRQP_STATUS_OK) {
            HPRQPStatus st = st_k[k];
            batch_free(b);
            delete b;
            return st;
        }
    const double c1 = cnow();
    // ---- pack (int32 local indices)
    size_t qnz = 0, anz = 0, qrp = 0, arp = 0, atrp = 0, nv = 0, nr = 0;
    b->inst.resize(K);
    for (size_t k = 0; k < K; ++k) {
        const HPRQPModel &M = b->models[k];
        BInst &I = b->inst[k];
        I.q_nz = (long long)qnz;
        I.a_nz = (long long)anz;
        I.at_nz = (long long)anz;
        I.q_rp = (int)qrp;
        I.a_rp = (int)arp;
        I.at_rp = (int)atrp;
        I.var = (int)nv;
        I.row = (int)nr;
        I.n = (int)M.Q.ncol;
        I.m = (int)M.A.nrow;
        I.obj_constant = M.obj_constant;
        // every instance's entries start on a 4-entry (16-byte) boundary, so
        // cta_spmv can read aligned quads of indices and values
        qnz += (M.Q.nnz + 3) & ~size_t(3);
        anz += (M.A.nnz + 3) & ~size_t(3);
        qrp += M.Q.nrow + 1;
        arp += M.A.nrow + 1;
        atrp += M.AT.nrow + 1;
        nv += M.Q.ncol;
        nr += M.A.nrow;
        b->nmax = std::max(b->nmax, I.n);
        b->mmax = std::max(b->mmax, I.m);
    }
    if (qrp > (size_t)INT32_MAX || arp > (size_t)INT32_MAX || nv > (size_t)INT32_MAX || nr > (size_t)INT32_MAX) {
        batch_free(b);
        delete b;
        return HPRQP_STATUS_NOT_IMPLEMENTED;
    }
    b->total_n = nv;
    b->total_m = nr;
    // + 4: the last quad of the last instance stays inside the arrays
    qnz += 4;
    anz += 4;
    HostVec<int> h_qrp(qrp), h_arp(arp), h_atrp(atrp), h_qci(qnz), h_aci(anz), h_atci(anz);
    HostVec<double> h_qv(qnz), h_av(anz), h_atv(anz),
        h_c(std::max<size_t>(nv, 1)), h_l(std::max<size_t>(nv, 1)), h_u(std::max<size_t>(nv, 1)),
        h_AL(std::max<size_t>(nr, 1)), h_AU(std::max<size_t>(nr, 1));
    h_c[0] = h_l[0] = h_u[0] = h_AL[0] = h_AU[0] = 0.0;
    for (size_t e = qnz - 4; e < qnz; ++e) {
        h_qci[e] = 0;
        h_qv[e] = 0.0;
    }
    for (size_t e = anz - 4; e < anz; ++e) {
        h_aci[e] = h_atci[e] = 0;
        h_av[e] = h_atv[e] = 0.0;
    }
    b->tuned_lg.assign(3 * K, 0);
    auto pack_worker = [&](unsigned tix) {
    for (size_t k = tix; k < K; k += nth) {
        const HPRQPModel &M = b->models[k];
        BInst &I = b->inst[k];
        const int warps = (b->cta_threads == kBigCta && mid_cta_instance(M) ? kMidCta : b->cta_threads) / 32;
        I.q_lg = b->tuned_lg[3 * k] = choose_lane_group(M.Q.row_ptr, (int)M.Q.nrow, warps);
        I.a_lg = b->tuned_lg[3 * k + 1] = choose_lane_group(M.A.row_ptr, (int)M.A.nrow, warps);
        I.at_lg = b->tuned_lg[3 * k + 2] = choose_lane_group(M.AT.row_ptr, (int)M.AT.nrow, warps);
        for (size_t r = 0; r <= M.Q.nrow; ++r) h_qrp[I.q_rp + r] = (int)M.Q.row_ptr[r];
        for (size_t r = 0; r <= M.A.nrow; ++r) h_arp[I.a_rp + r] = (int)M.A.row_ptr[r];
        for (size_t r = 0; r <= M.AT.nrow; ++r) h_atrp[I.at_rp + r] = (int)M.AT.row_ptr[r];
        for (size_t e = 0; e < M.Q.nnz; ++e) {
            h_qci[I.q_nz + e] = (int)M.Q.col_ind[e];
            h_qv[I.q_nz + e] = M.Q.values[e];
        }
        for (size_t e = M.Q.nnz; e < ((M.Q.nnz + 3) & ~size_t(3)); ++e) {  // alignment padding
            h_qci[I.q_nz + e] = 0;
            h_qv[I.q_nz + e] = 0.0;
        }
        for (size_t e = 0; e < M.A.nnz; ++e) {
            h_aci[I.a_nz + e] = (int)M.A.col_ind[e];
            h_av[I.a_nz + e] = M.A.values[e];
            h_atci[I.at_nz + e] = (int)M.AT.col_ind[e];
            h_atv[I.at_nz + e] = M.AT.values[e];
        }
        for (size_t e = M.A.nnz; e < ((M.A.nnz + 3) & ~size_t(3)); ++e) {
            h_aci[I.a_nz + e] = h_atci[I.at_nz + e] = 0;
            h_av[I.a_nz + e] = h_atv[I.at_nz + e] = 0.0;
        }
        memcpy(&h_c[I.var], M.c, M.Q.ncol * sizeof(double));
        memcpy(&h_l[I.var], M.l, M.Q.ncol * sizeof(double));
        memcpy(&h_u[I.var], M.u, M.Q.ncol * sizeof(double));
        if (M.A.nrow) {
            memcpy(&h_AL[I.row], M.AL, M.A.nrow * sizeof(double));
            memcpy(&h_AU[I.row], M.AU, M.A.nrow * sizeof(double));
        }
    }
    };
    {
        std::vector<std::thread> pth;
        if (nth == 1) pack_worker(0);
        else
            for (unsigned t = 0; t < nth; ++t) pth.emplace_back(pack_worker, t);
        for (auto &t : pth) t.join();
    }
    const double c2 = cnow();
    // ---- device
    HPRQPStatus st = HPRQP_STATUS_OK;
    auto fail = [&](HPRQPStatus s) {
        batch_free(b);
        delete b;
        return s;
    };
    if (cudaSetDevice(device_number) != cudaSuccess ||
        cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, device_number) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&b->stream_mid, cudaStreamNonBlocking) != cudaSuccess)
        return fail(HPRQP_STATUS_NOT_IMPLEMENTED);
    BatchArgs &G = b->args;
    G.K = (int)K;
    int *d_qrp, *d_arp, *d_atrp, *d_qci, *d_aci, *d_atci;
    double *d_qv0, *d_av0, *d_atv0, *d_c, *d_l, *d_u, *d_AL, *d_AU;
    BInst *d_inst;
    int *d_order;
    unsigned long long *d_counter;
    Carver cv;
    cv.add(&d_qrp, qrp).add(&d_arp, arp).add(&d_atrp, atrp).add(&d_qci, h_qci.size()).add(&d_aci, h_aci.size());
    cv.add(&d_atci, h_atci.size()).add(&d_qv0, h_qv.size()).add(&d_av0, h_av.size()).add(&d_atv0, h_atv.size());
    cv.add(&G.q_v, h_qv.size()).add(&G.a_v, h_av.size()).add(&G.at_v, h_atv.size());
    cv.add(&d_c, h_c.size()).add(&d_l, h_l.size()).add(&d_u, h_u.size()).add(&d_AL, h_AL.size()).add(&d_AU, h_AU.size());
    cv.add(&d_inst, K).add(&d_order, 2 * K).add(&d_counter, 2);
    cv.add(&G.x, h_c.size()).add(&G.z, h_c.size()).add(&G.w, h_c.size()).add(&G.y, h_AL.size());
    cv.add(&G.status, K).add(&G.iters, K).add(&G.pobj, K).add(&G.resid, K).add(&G.gap, K).add(&G.restarts, K);
    cv.add(&G.sigma_out, K).add(&G.seconds_out, K).add(&G.active_x, h_c.size()).add(&G.active_r, h_AL.size());
    cv.add(&G.col_norm_out, h_c.size()).add(&G.row_norm_out, h_AL.size()).add(&b->d_t0, 1);
    if ((st = cv.commit(b))) return fail(st);
    // work orders, largest instances first: the adjoint's (second half of
    // d_order) over all instances; the solve's (first half) the same with,
    // in a kBigCta batch, the k_mid instances for kMidCta CTAs moved to its
    // end -- the kBigCta launch takes the first K - k_mid entries, the
    // kMidCta launch the rest, each as a queue with two ends
    std::vector<int> order(2 * K);
    std::iota(order.begin(), order.begin() + K, 0);
    std::stable_sort(order.begin(), order.begin() + K,
                     [&](int x, int y) { return instance_work(b->models[x]) > instance_work(b->models[y]); });
    std::copy(order.begin(), order.begin() + K, order.begin() + K);
    b->k_mid = 0;
    if (b->cta_threads == kBigCta) {
        std::stable_partition(order.begin(), order.begin() + K, [&](int k) { return !mid_cta_instance(b->models[k]); });
        for (size_t k = 0; k < K; ++k) b->k_mid += mid_cta_instance(b->models[k]);
    }
    auto up = [&](void *d, const void *h, size_t bytes) {
        return cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, b->stream) == cudaSuccess;
    };
    if (!up(d_qrp, h_qrp.data(), qrp * 4) || !up(d_arp, h_arp.data(), arp * 4) || !up(d_atrp, h_atrp.data(), atrp * 4) ||
        !up(d_qci, h_qci.data(), h_qci.size() * 4) || !up(d_aci, h_aci.data(), h_aci.size() * 4) ||
        !up(d_atci, h_atci.data(), h_atci.size() * 4) || !up(d_qv0, h_qv.data(), h_qv.size() * 8) ||
        !up(d_av0, h_av.data(), h_av.size() * 8) || !up(d_atv0, h_atv.data(), h_atv.size() * 8) ||
        !up(d_c, h_c.data(), h_c.size() * 8) || !up(d_l, h_l.data(), h_l.size() * 8) ||
        !up(d_u, h_u.data(), h_u.size() * 8) || !up(d_AL, h_AL.data(), h_AL.size() * 8) ||
        !up(d_AU, h_AU.data(), h_AU.size() * 8) || !up(d_inst, b->inst.data(), K * sizeof(BInst)) ||
        !up(d_order, order.data(), 2 * K * sizeof(int)) || cudaStreamSynchronize(b->stream) != cudaSuccess)
        return fail(HPRQP_STATUS_NOT_IMPLEMENTED);
    // the abort flag (host-mapped memory) exists only for batches a caller
    // holds a handle to: the one-call forms cannot be asked to stop
    if (abortable) {
        if (cudaHostAlloc((void **)&b->h_abort, sizeof(int), cudaHostAllocMapped) != cudaSuccess ||
            cudaHostGetDevicePointer((void **)&b->d_abort, b->h_abort, 0) != cudaSuccess)
            return fail(HPRQP_STATUS_NOT_IMPLEMENTED);
        __atomic_store_n(b->h_abort, 0, __ATOMIC_SEQ_CST);
    }
    G.abort_flag = b->d_abort;
    G.inst = d_inst;
    b->d_inst = d_inst;
    G.order = d_order;
    G.counter = d_counter;
    G.q_rp = d_qrp;
    G.a_rp = d_arp;
    G.at_rp = d_atrp;
    G.q_ci = d_qci;
    G.a_ci = d_aci;
    G.at_ci = d_atci;
    G.q_v0 = d_qv0;
    G.a_v0 = d_av0;
    G.at_v0 = d_atv0;
    G.c0 = d_c;
    G.l0 = d_l;
    G.u0 = d_u;
    G.AL0 = d_AL;
    G.AU0 = d_AU;
    G.nmax = std::max(b->nmax, 1);
    G.mmax = std::max(b->mmax, 1);
    if (ctrace)
        fprintf(stderr, "[hprqp-b200 batch] create: preprocess %.3f s, pack %.3f s, device %.3f s\n", c1 - c0, c2 - c1,
                cnow() - c2);
    *out = b;
    return HPRQP_STATUS_OK;
}

HPRQPStatus hprqp_batch_create(size_t K, const size_t *var_offsets, const size_t *row_offsets,
                               const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c, const double *AL,
                               const double *AU, const double *l, const double *u, const double *obj_constants,
                               int device_number, HPRQPBatch **out)
{
    return batch_create_impl(K, var_offsets, row_offsets, Q, A, c, AL, AU, l, u, obj_constants, device_number, true,
                             out);
}

}  // extern "C"

namespace hpr {

// a launched solve (batch_launch) waiting for batch_finish: one launch, or
// two (segments of the work order) timed from one start event
struct SolveLaunch {
    cudaEvent_t e0 = nullptr, e1[2] = {nullptr, nullptr};
    unsigned long long *d_phase = nullptr;
    int segments = 0;
    int bt[2] = {0, 0}, grid[2] = {0, 0};
    size_t smem[2] = {0, 0};
};

static void solve_launch_release(SolveLaunch &L)
{
    if (L.e0) cudaEventDestroy(L.e0);
    for (auto &e : L.e1)
        if (e) cudaEventDestroy(e);
    L.e0 = L.e1[0] = L.e1[1] = nullptr;
}

// Start the solve of a batch and return; the launches' events and optional
// phase clocks are in L.  A kBigCta batch with instances for kMidCta CTAs
// (mid_cta_instance) runs them first, in a kMidCta launch on the batch's
// stream, and the others in a kBigCta launch on stream_mid: the mid-size CTAs (one
// per SM) start every small instance at once -- the ones whose iteration
// counts vary most -- and the 1024-thread CTAs take the SMs as they finish.
static HPRQPStatus batch_launch(HPRQPBatch *b, const HPRQPBatchParams *p, SolveLaunch &L)
{
    B_CK(cudaSetDevice(b->device));
    BatchArgs &G = b->args;
    const size_t na = ((size_t)G.nmax + 31) & ~size_t(31), ma = ((size_t)G.mmax + 31) & ~size_t(31);
    const size_t vec_bytes = (4 * na + 2 * ma) * sizeof(double);  // the gathered vectors
    struct Seg {
        size_t first, count;  // entries of the work order
        int bt;
        cudaStream_t stream;
    };
    Seg seg[2];
    int ns = 0;
    const size_t k_big = b->K - b->k_mid;
    if (b->k_mid > 0) {
        seg[ns] = {k_big, b->k_mid, kMidCta, b->stream};
        ++ns;
    }
    if (k_big > 0) {
        seg[ns] = {0, k_big, b->cta_threads, ns == 0 ? b->stream : b->stream_mid};
        ++ns;
    }
    L.segments = ns;
    auto kern_of = [](int bt) {
        return bt == kBigCta ? k_batch_solve<kBigCta> : bt == kMidCta ? k_batch_solve<kMidCta> : k_batch_solve<kSmallCta>;
    };
    int vec_smem[2] = {0, 0}, slots = 0, off[2] = {0, 0};
    for (int s = 0; s < ns; ++s) {
        const int bt = seg[s].bt;
        auto kern = kern_of(bt);
        // The gathered vectors go to shared memory only while the carveout
        // that takes leaves most of the SM's 256 KB of unified L1 / shared
        // memory to L1, which holds the instance's other vectors and its
        // matrices: at most kPoolPerSm bytes of shared memory per SM (static
        // and reserved bytes of every resident CTA included).  Measured on
        // the 4096-QP batch (n up to 2000: 99.5 KB per SM with the pool) the
        // pool made the mid-size instances whose whole working set fits a
        // 248 KB L1 (n ~ 500) 5 % slower and the large ones 4 % faster; on
        // 296 large QPs (two CTAs per SM, 195 KB) it cost 12 %; on 256 QPs of
        // n = 500 (48 KB) it saved 12 %.
        cudaFuncAttributes fa;
        B_CK(cudaFuncGetAttributes(&fa, kern));
        const size_t pool_per_sm = (size_t)ctas_per_sm(bt) * (vec_bytes + fa.sharedSizeBytes + kReservedSmemPerCta);
        vec_smem[s] = HPR_BATCH_VEC_SMEM && vec_bytes <= smem_limit(bt) && pool_per_sm <= kPoolPerSm;
        L.smem[s] = vec_smem[s] ? vec_bytes : 0;
        B_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem[s]));
        int per_sm = 0;
        B_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, bt, L.smem[s]));
        L.bt[s] = bt;
        L.grid[s] = std::max(1, std::min((int)seg[s].count, b->num_sms * std::max(per_sm, 1)));
        off[s] = slots;
        slots += L.grid[s];
    }
    // per-CTA workspace of every launch (allocated lazily, kept for the next solves)
    const size_t stride = kBatchNVecs * na + kBatchMVecs * ma;
    if (!G.ws || G.ws_stride != stride || b->ws_slots < slots) {
        double *ws = nullptr;
        HPRQPStatus st = balloc(b, &ws, stride * (size_t)slots);
        if (st) return st;
        G.ws = ws;
        G.ws_stride = stride;
        b->ws_slots = slots;
    }
    G.stoptol = p->stoptol;
    G.max_iter = (long long)std::min<size_t>(p->max_iter, (size_t)LLONG_MAX);
    G.time_limit = p->time_limit;
    G.check_iter = (int)p->check_iter;
    G.print_frequency = p->print_frequency;
    G.use_scaling = p->use_scaling;
    unsigned long long *d_t0 = b->d_t0;
    B_CK(cudaMemsetAsync(G.counter, 0, 2 * sizeof(*G.counter), b->stream));
    k_batch_clock<<<1, 1, 0, b->stream>>>(d_t0);
    count_launch();
    unsigned long long h_t0 = 0;
    B_CK(cudaMemcpyAsync(&h_t0, d_t0, sizeof(h_t0), cudaMemcpyDeviceToHost, b->stream));
    B_CK(cudaStreamSynchronize(b->stream));
    G.t_start = h_t0;
    const char *pe = getenv("HPRQP_B200_BATCH_PHASES");
    unsigned long long *d_phase = nullptr;
    if (pe && pe[0] == '1') {
        if (!b->d_phase || b->phase_slots < slots) {
            HPRQPStatus st2 = balloc(b, &b->d_phase, (size_t)slots * 8);
            if (st2) return st2;
            b->phase_slots = slots;
        }
        d_phase = b->d_phase;
        B_CK(cudaMemsetAsync(d_phase, 0, (size_t)slots * 8 * sizeof(unsigned long long), b->stream));
    }
    L.d_phase = d_phase;
    B_CK(cudaEventCreate(&L.e0));
    for (int s = 0; s < ns; ++s) B_CK(cudaEventCreate(&L.e1[s]));
    B_CK(cudaEventRecord(L.e0, b->stream));
    cudaError_t err = cudaSuccess;
    for (int s = 0; s < ns && err == cudaSuccess; ++s) {
        BatchArgs A = G;
        A.K = (int)seg[s].count;
        A.order = G.order + seg[s].first;
        A.counter = G.counter + s;
        A.ws = G.ws + (size_t)off[s] * stride;
        A.vec_smem = vec_smem[s];
        A.phase_clk = d_phase ? d_phase + (size_t)off[s] * 8 : nullptr;
        if (seg[s].stream != b->stream) err = cudaStreamWaitEvent(seg[s].stream, L.e0, 0);
        if (err != cudaSuccess) break;
        kern_of(seg[s].bt)<<<L.grid[s], seg[s].bt, L.smem[s], seg[s].stream>>>(A);
        count_launch();
        err = cudaGetLastError();
        if (err == cudaSuccess) err = cudaEventRecord(L.e1[s], seg[s].stream);
    }
    if (err != cudaSuccess) {
        // nothing launched may still run when the caller frees the batch
        cudaStreamSynchronize(b->stream);
        cudaStreamSynchronize(b->stream_mid);
        B_CK(err);
    }
    return HPRQP_STATUS_OK;
}

// Wait for a launched solve, record its device time (start event to the end
// of the last launch), print the optional phase clocks.
static HPRQPStatus batch_finish(HPRQPBatch *b, SolveLaunch &L)
{
    B_CK(cudaSetDevice(b->device));
    cudaError_t err = cudaSuccess;
    float ms = 0.f;
    for (int s = 0; s < L.segments; ++s) {
        const cudaError_t e = cudaEventSynchronize(L.e1[s]);
        if (err == cudaSuccess) err = e;
        float t = 0.f;
        if (e == cudaSuccess && cudaEventElapsedTime(&t, L.e0, L.e1[s]) == cudaSuccess) ms = std::max(ms, t);
    }
    solve_launch_release(L);
    B_CK(err);
    B_CK(cudaGetLastError());
    b->last_ms = ms;
    b->solved = true;
    // an abort request ends with the solve it stopped
    if (b->h_abort) __atomic_store_n(b->h_abort, 0, __ATOMIC_SEQ_CST);
    if (L.d_phase) {
        int slots = 0;
        for (int s = 0; s < L.segments; ++s) slots += L.grid[s];
        std::vector<unsigned long long> h((size_t)slots * 8);
        B_CK(cudaMemcpy(h.data(), L.d_phase, h.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
        double tot[8] = {0};
        for (int g = 0; g < slots; ++g)
            for (int q = 0; q < 8; ++q) tot[q] += (double)h[(size_t)g * 8 + q];
        fprintf(stderr, "[hprqp-b200 batch phases, %% of CTA time] load+scale %.1f setup %.1f power %.1f steps %.1f "
                        "residuals %.1f m-norm %.1f sigma+restart %.1f (",
                100 * tot[0] / tot[7], 100 * tot[1] / tot[7], 100 * tot[2] / tot[7], 100 * tot[3] / tot[7],
                100 * tot[4] / tot[7], 100 * tot[5] / tot[7], 100 * tot[6] / tot[7]);
        for (int s = 0; s < L.segments; ++s)
            fprintf(stderr, "%s%d CTAs of %d threads, smem %zu", s ? "; " : "", L.grid[s], L.bt[s], L.smem[s]);
        fprintf(stderr, ")\n");
    }
    return HPRQP_STATUS_OK;
}

}  // namespace hpr

extern "C" {

HPRQPStatus hprqp_batch_solve(HPRQPBatch *b, const HPRQPBatchParams *p)
{
    using namespace hpr;
    if (!b || !p) return HPRQP_STATUS_INVALID_ARGUMENT;
    SolveLaunch L;
    HPRQPStatus st = batch_launch(b, p, L);
    if (st != HPRQP_STATUS_OK) {
        solve_launch_release(L);
        return st;
    }
    return batch_finish(b, L);
}

HPRQPStatus hprqp_batch_set_warm_start(HPRQPBatch *b, const double *x0, const double *y0, const double *w0,
                                       const double *sigma0)
{
    using namespace hpr;
    if (!b) return HPRQP_STATUS_INVALID_ARGUMENT;
    BatchArgs &G = b->args;
    if (!x0) {
        G.x_start = G.w_start = G.y_start = G.sigma_start = nullptr;
        return HPRQP_STATUS_OK;
    }
    if (sigma0)
        for (size_t k = 0; k < b->K; ++k)
            if (std::isnan(sigma0[k]) || std::isinf(sigma0[k])) return HPRQP_STATUS_INVALID_ARGUMENT;
    const size_t N = b->total_n, M = b->total_m;
    for (size_t i = 0; i < N; ++i)
        if (!std::isfinite(x0[i]) || (w0 && !std::isfinite(w0[i]))) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (y0)
        for (size_t i = 0; i < b->total_m_orig; ++i)
            if (!std::isfinite(y0[i])) return HPRQP_STATUS_INVALID_ARGUMENT;
    B_CK(cudaSetDevice(b->device));
    HPRQPStatus st;
    if (!b->start_x &&
        ((st = balloc(b, &b->start_x, N)) || (st = balloc(b, &b->start_w, N)) || (st = balloc(b, &b->start_y, M)) ||
         (st = balloc(b, &b->start_sigma, b->K))))
        return st;
    // y0 is given on the caller's rows: keep the rows the builder kept
    std::vector<double> hy(std::max<size_t>(M, 1), 0.0);
    if (y0)
        for (size_t k = 0; k < b->K; ++k) {
            const auto &kr = b->kept_rows[k];
            for (size_t r = 0; r < kr.size(); ++r) hy[b->inst[k].row + r] = y0[b->row_off[k] + kr[r]];
        }
    if (N) {
        B_CK(cudaMemcpyAsync(b->start_x, x0, N * sizeof(double), cudaMemcpyHostToDevice, b->stream));
        B_CK(cudaMemcpyAsync(b->start_w, w0 ? w0 : x0, N * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    }
    if (M) B_CK(cudaMemcpyAsync(b->start_y, hy.data(), M * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    if (sigma0)
        B_CK(cudaMemcpyAsync(b->start_sigma, sigma0, b->K * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    B_CK(cudaStreamSynchronize(b->stream));
    G.x_start = b->start_x;
    G.w_start = b->start_w;
    G.y_start = b->start_y;
    G.sigma_start = sigma0 ? b->start_sigma : nullptr;
    return HPRQP_STATUS_OK;
}

// copy K doubles of a per-instance output of the last solve to the host
static HPRQPStatus batch_download(const HPRQPBatch *b, const double *d, double *h)
{
    if (!b || !b->solved || !h) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (cudaMemcpyAsync(h, d, b->K * sizeof(double), cudaMemcpyDeviceToHost, b->stream) != cudaSuccess ||
        cudaStreamSynchronize(b->stream) != cudaSuccess)
        return HPRQP_STATUS_NOT_IMPLEMENTED;
    return HPRQP_STATUS_OK;
}

HPRQPStatus hprqp_batch_get_sigma(const HPRQPBatch *b, double *sigma)
{
    return batch_download(b, b ? b->args.sigma_out : nullptr, sigma);
}

HPRQPStatus hprqp_batch_get_times(const HPRQPBatch *b, double *seconds)
{
    return batch_download(b, b ? b->args.seconds_out : nullptr, seconds);
}

double hprqp_batch_last_solve_ms(const HPRQPBatch *b) { return b ? b->last_ms : 0.0; }

size_t hprqp_batch_num_instances(const HPRQPBatch *b) { return b ? b->K : 0; }

HPRQPStatus hprqp_batch_request_abort(HPRQPBatch *b)
{
    if (!b || !b->h_abort) return HPRQP_STATUS_INVALID_ARGUMENT;
    __atomic_store_n(b->h_abort, 1, __ATOMIC_SEQ_CST);
    return HPRQP_STATUS_OK;
}

HPRQPStatus hprqp_batch_set_spmv_lanes(HPRQPBatch *b, int lanes)
{
    using namespace hpr;
    if (!b || !(lanes == 0 || lanes == 1 || lanes == 2 || lanes == 4 || lanes == 8 || lanes == 16 || lanes == 32))
        return HPRQP_STATUS_INVALID_ARGUMENT;
    int lg = 0;
    while ((1 << lg) < lanes) ++lg;
    for (size_t k = 0; k < b->K; ++k) {
        BInst &I = b->inst[k];
        I.q_lg = lanes ? lg : b->tuned_lg[3 * k];
        I.a_lg = lanes ? lg : b->tuned_lg[3 * k + 1];
        I.at_lg = lanes ? lg : b->tuned_lg[3 * k + 2];
    }
    B_CK(cudaSetDevice(b->device));
    B_CK(cudaMemcpyAsync(b->d_inst, b->inst.data(), b->K * sizeof(BInst), cudaMemcpyHostToDevice, b->stream));
    B_CK(cudaStreamSynchronize(b->stream));
    b->forced_lanes = lanes;
    return HPRQP_STATUS_OK;
}

HPRQPStatus hprqp_batch_get_spmv_lanes(const HPRQPBatch *b, int *lanes)
{
    if (!b || !lanes) return HPRQP_STATUS_INVALID_ARGUMENT;
    for (size_t k = 0; k < b->K; ++k) {
        lanes[3 * k] = 1 << b->inst[k].q_lg;
        lanes[3 * k + 1] = 1 << b->inst[k].a_lg;
        lanes[3 * k + 2] = 1 << b->inst[k].at_lg;
    }
    return HPRQP_STATUS_OK;
}

HPRQPStatus hprqp_batch_get_results(const HPRQPBatch *b, int *status, size_t *iter, double *primal_obj,
                                    double *residual, double *gap, double *x, double *y, double *z, double *w)
{
    if (!b || !b->solved) return HPRQP_STATUS_INVALID_ARGUMENT;
    const hpr::BatchArgs &G = b->args;
    const size_t K = b->K;
    std::vector<long long> it(K);
    std::vector<int> stv(K);
    auto down = [&](void *h, const void *d, size_t bytes) {
        return cudaMemcpyAsync(h, d, bytes, cudaMemcpyDeviceToHost, b->stream) == cudaSuccess;
    };
    if (!down(stv.data(), G.status, K * sizeof(int)) || !down(it.data(), G.iters, K * sizeof(long long)))
        return HPRQP_STATUS_NOT_IMPLEMENTED;
    if ((primal_obj && !down(primal_obj, G.pobj, K * 8)) || (residual && !down(residual, G.resid, K * 8)) ||
        (gap && !down(gap, G.gap, K * 8)))
        return HPRQP_STATUS_NOT_IMPLEMENTED;
    std::vector<double> hx, hy;
    // x, z, w: preprocessing keeps every variable, so the packing matches the caller's
    if ((x && !down(x, G.x, b->total_n * 8)) || (z && !down(z, G.z, b->total_n * 8)) ||
        (w && !down(w, G.w, b->total_n * 8)))
        return HPRQP_STATUS_NOT_IMPLEMENTED;
    if (y) {
        hy.resize(std::max<size_t>(b->total_m, 1));
        if (!down(hy.data(), G.y, b->total_m * 8)) return HPRQP_STATUS_NOT_IMPLEMENTED;
    }
    if (cudaStreamSynchronize(b->stream) != cudaSuccess) return HPRQP_STATUS_NOT_IMPLEMENTED;
    for (size_t k = 0; k < K; ++k) {
        if (status) status[k] = stv[k];
        if (iter) iter[k] = (size_t)it[k];
    }
    if (y) {
        // scatter back to the caller's rows; rows removed by preprocessing get 0
        std::fill(y, y + b->total_m_orig, 0.0);
        for (size_t k = 0; k < K; ++k) {
            const auto &kr = b->kept_rows[k];
            for (size_t r = 0; r < kr.size(); ++r) y[b->row_off[k] + kr[r]] = hy[b->inst[k].row + r];
        }
    }
    return HPRQP_STATUS_OK;
}

HPRQPStatus hprqp_batch_backward(HPRQPBatch *b, const double *grad_x, const double *grad_y, double tol,
                                 HPRQPBatchGradients *out)
{
    using namespace hpr;
    if (!b || !grad_x || !out) return HPRQP_STATUS_INVALID_ARGUMENT;
    if (!b->solved || !b->has_caller_csr) {
        fprintf(stderr, "hprqp-b200: hprqp_batch_backward needs a completed hprqp_batch_solve\n");
        return HPRQP_STATUS_INVALID_ARGUMENT;
    }
    if (!(tol > 0.0)) tol = 1e-12;
    B_CK(cudaSetDevice(b->device));
    const size_t K = b->K, N = b->total_n, M = b->total_m;
    BatchArgs &G = b->args;
    HPRQPStatus st;
    // ---- device buffers (first call only)
    const size_t na = ((size_t)G.nmax + 31) & ~size_t(31), ma = ((size_t)G.mmax + 31) & ~size_t(31);
    const size_t lz_bytes = (size_t)kAdjLanczos * (na + ma) * sizeof(double);
    const int bt = b->cta_threads;
    auto kern = bt == kBigCta ? k_batch_adjoint<kBigCta> : k_batch_adjoint<kSmallCta>;
    const int lanczos_smem = lz_bytes <= smem_limit(bt);
    const size_t smem = lanczos_smem ? lz_bytes : 0;
    B_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 0;
    B_CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, bt, smem));
    const int grid = std::max(1, std::min((int)K, b->num_sms * std::max(per_sm, 1)));
    const size_t stride = kAdjGlobalN * na + kAdjGlobalM * ma + (lanczos_smem ? 0 : (size_t)kAdjLanczos * (na + ma));
    if (!b->adj_gx) {
        if ((st = balloc(b, &b->adj_gx, N)) || (st = balloc(b, &b->adj_gy, M)) || (st = balloc(b, &b->adj_lx, N)) ||
            (st = balloc(b, &b->adj_ly, M)) || (st = balloc(b, &b->adj_rel, K)) || (st = balloc(b, &b->adj_it, K)) ||
            (st = balloc(b, &b->adj_counter, 1)))
            return st;
    }
    if (b->adj_ws_count < stride * (size_t)grid) {
        if ((st = balloc(b, &b->adj_ws, stride * (size_t)grid))) return st;
        b->adj_ws_count = stride * (size_t)grid;
    }
    // ---- loss gradients in the device packing (rows: the rows kept by preprocessing)
    std::vector<double> gy_kept;
    if (grad_y) {
        gy_kept.assign(std::max<size_t>(M, 1), 0.0);
        for (size_t k = 0; k < K; ++k) {
            const auto &kr = b->kept_rows[k];
            for (size_t r = 0; r < kr.size(); ++r) gy_kept[b->inst[k].row + r] = grad_y[b->row_off[k] + kr[r]];
        }
        B_CK(cudaMemcpyAsync(b->adj_gy, gy_kept.data(), M * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    }
    std::vector<double> gx_dev(std::max<size_t>(N, 1), 0.0);
    for (size_t k = 0; k < K; ++k)
        memcpy(&gx_dev[b->inst[k].var], grad_x + b->var_off[k], (size_t)b->inst[k].n * sizeof(double));
    B_CK(cudaMemcpyAsync(b->adj_gx, gx_dev.data(), N * sizeof(double), cudaMemcpyHostToDevice, b->stream));
    B_CK(cudaMemsetAsync(b->adj_counter, 0, sizeof(*b->adj_counter), b->stream));
    AdjArgs A{};
    A.K = (int)K;
    A.inst = G.inst;
    A.order = G.order + K;  // the adjoint's work order: all instances, largest first
    A.counter = b->adj_counter;
    A.q_rp = G.q_rp;
    A.q_ci = G.q_ci;
    A.a_rp = G.a_rp;
    A.a_ci = G.a_ci;
    A.at_rp = G.at_rp;
    A.at_ci = G.at_ci;
    A.q_v = G.q_v;
    A.a_v = G.a_v;
    A.at_v = G.at_v;
    A.col_norm = G.col_norm_out;
    A.row_norm = G.row_norm_out;
    A.z = G.z;
    A.y = G.y;
    A.gx = b->adj_gx;
    A.gy = grad_y ? b->adj_gy : nullptr;
    A.lam_x = b->adj_lx;
    A.lam_y = b->adj_ly;
    A.iters = b->adj_it;
    A.relres = b->adj_rel;
    A.tol = tol;
    A.maxit_factor = 4;
    A.ws = b->adj_ws;
    A.ws_stride = stride;
    A.nmax = G.nmax;
    A.mmax = G.mmax;
    A.lanczos_smem = lanczos_smem;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, b->stream);
    kern<<<grid, bt, smem, b->stream>>>(A);
    count_launch();
    cudaEventRecord(e1, b->stream);
    cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    B_CK(err);
    B_CK(cudaGetLastError());
    b->last_adjoint_ms = ms;
    // ---- lambda, mu and the solution back on the host (device packing)
    std::vector<double> lx(std::max<size_t>(N, 1)), ly(std::max<size_t>(M, 1)), x(std::max<size_t>(N, 1)),
        z(std::max<size_t>(N, 1)), y(std::max<size_t>(M, 1)), rel(K);
    std::vector<int> its(K);
    B_CK(cudaMemcpyAsync(lx.data(), b->adj_lx, N * 8, cudaMemcpyDeviceToHost, b->stream));
    B_CK(cudaMemcpyAsync(ly.data(), b->adj_ly, M * 8, cudaMemcpyDeviceToHost, b->stream));
    B_CK(cudaMemcpyAsync(x.data(), G.x, N * 8, cudaMemcpyDeviceToHost, b->stream));
    B_CK(cudaMemcpyAsync(z.data(), G.z, N * 8, cudaMemcpyDeviceToHost, b->stream));
    B_CK(cudaMemcpyAsync(y.data(), G.y, M * 8, cudaMemcpyDeviceToHost, b->stream));
    B_CK(cudaMemcpyAsync(rel.data(), b->adj_rel, K * 8, cudaMemcpyDeviceToHost, b->stream));
    B_CK(cudaMemcpyAsync(its.data(), b->adj_it, K * 4, cudaMemcpyDeviceToHost, b->stream));
    B_CK(cudaStreamSynchronize(b->stream));
    if (out->minres_iters) memcpy(out->minres_iters, its.data(), K * sizeof(int));
    if (out->minres_relres) memcpy(out->minres_relres, rel.data(), K * sizeof(double));
    // ---- gradient assembly, per instance on host threads (caller's packing)
    const unsigned nth = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
    auto worker = [&](unsigned tix) {
        std::vector<double> qlam, atmu, mu_orig, y_orig;
        for (size_t k = tix; k < K; k += nth) {
            const HPRQPModel &Mk = b->models[k];
            const BInst &I = b->inst[k];
            const size_t n = Mk.Q.ncol, m = Mk.A.nrow, v0 = b->var_off[k], r0 = b->row_off[k];
            const size_t m_orig = b->row_off[k + 1] - r0;
            const double *lam = lx.data() + I.var, *mu = ly.data() + I.row, *xk = x.data() + I.var;
            const double *zk = z.data() + I.var, *yk = y.data() + I.row, *gk = grad_x + v0;
            // Q lam and A' mu with the preprocessed (symmetrised, unscaled) model
            qlam.assign(n, 0.0);
            atmu.assign(n, 0.0);
            for (size_t i = 0; i < n; ++i)
                for (size_t e = Mk.Q.row_ptr[i]; e < Mk.Q.row_ptr[i + 1]; ++e)
                    qlam[i] += Mk.Q.values[e] * lam[Mk.Q.col_ind[e]];
            for (size_t r = 0; r < m; ++r)
                for (size_t e = Mk.A.row_ptr[r]; e < Mk.A.row_ptr[r + 1]; ++e)
                    atmu[Mk.A.col_ind[e]] += Mk.A.values[e] * mu[r];
            for (size_t i = 0; i < n; ++i) {
                if (out->dc) out->dc[v0 + i] = -lam[i];
                const double db = gk[i] - qlam[i] - atmu[i];
                if (out->dl) out->dl[v0 + i] = zk[i] > 0.0 ? db : 0.0;
                if (out->du) out->du[v0 + i] = zk[i] < 0.0 ? db : 0.0;
            }
            mu_orig.assign(m_orig, 0.0);
            y_orig.assign(m_orig, 0.0);
            const auto &kr = b->kept_rows[k];
            for (size_t r = 0; r < kr.size(); ++r) {
                mu_orig[kr[r]] = mu[r];
                y_orig[kr[r]] = yk[r];
            }
            for (size_t r = 0; r < m_orig; ++r) {
                if (out->dAL) out->dAL[r0 + r] = y_orig[r] > 0.0 ? mu_orig[r] : 0.0;
                if (out->dAU) out->dAU[r0 + r] = y_orig[r] < 0.0 ? mu_orig[r] : 0.0;
            }
            // caller's Q entry (i, j) enters (Q + Q')/2 at (i, j) and (j, i)
            if (out->dQ_values)
                for (size_t i = 0; i < n; ++i)
                    for (size_t e = b->q_rp_in[v0 + i]; e < b->q_rp_in[v0 + i + 1]; ++e) {
                        const size_t j = b->q_ci_in[e] - v0;
                        out->dQ_values[e] = -0.5 * (lam[i] * xk[j] + lam[j] * xk[i]);
                    }
            // caller's A entry (r, j)
            if (out->dA_values)
                for (size_t r = 0; r < m_orig; ++r)
                    for (size_t e = b->a_rp_in[r0 + r]; e < b->a_rp_in[r0 + r + 1]; ++e) {
                        const size_t j = b->a_ci_in[e] - v0;
                        out->dA_values[e] = -mu_orig[r] * xk[j] + lam[j] * y_orig[r];
                    }
        }
    };
    std::vector<std::thread> th;
    for (unsigned t = 0; t < nth; ++t) th.emplace_back(worker, t);
    for (auto &t : th) t.join();
    return HPRQP_STATUS_OK;
}

double hprqp_batch_last_backward_ms(const HPRQPBatch *b) { return b ? b->last_adjoint_ms : 0.0; }

void hprqp_batch_destroy(HPRQPBatch *b)
{
    if (!b) return;
    hpr::batch_free(b);
    delete b;
}

}  // extern "C"

namespace hpr {

// The one-call form of a large batch in two parts, so that the host's
// preprocessing and upload of the second part run while the GPU solves the
// first.  The first part is the smallest instances, up to kFirstPartWork of
// the nonzeros: they are quick to build, so their launch starts early, and
// they are the ones whose iteration counts vary most (a small instance can
// run a hundred times the median count, and such a straggler, started late,
// would end the call late).  The rest is built and uploaded meanwhile and
// launched on its own stream (its CTAs take the SMs as the first launch's
// CTAs finish); each part's results are scattered back to the caller's
// packing.  Each instance is solved by one CTA of the shape a single launch
// would give it (batches this large take 1024-thread CTAs, and 640-thread
// CTAs for the instances mid_cta_instance picks, a rule on the instance
// alone), so the results equal a single launch's bit for bit; each launch
// keeps its own time limit.
constexpr size_t kSplitMinInstances = 1024;
constexpr double kFirstPartWork = 0.15;

// Results of a batch built from the caller's instances ids[0..K) (in that
// order), written to the caller's packed arrays.
static HPRQPStatus scatter_results(const HPRQPBatch *b, const std::vector<size_t> &ids, const size_t *var_offsets,
                                   const size_t *row_offsets, int *status, size_t *iter, double *primal_obj,
                                   double *residual, double *gap, double *x, double *y, double *z, double *w)
{
    const size_t K = ids.size(), nb = b->var_off[K], mb = b->row_off[K];
    std::vector<int> st_b(status ? K : 0);
    std::vector<size_t> it_b(iter ? K : 0);
    std::vector<double> po_b(primal_obj ? K : 0), re_b(residual ? K : 0), ga_b(gap ? K : 0);
    std::vector<double> x_b(x ? nb : 0), y_b(y ? mb : 0), z_b(z ? nb : 0), w_b(w ? nb : 0);
    auto ptr = [](auto &v, const void *want) { return want ? v.data() : nullptr; };
    HPRQPStatus st = hprqp_batch_get_results(b, ptr(st_b, status), ptr(it_b, iter), ptr(po_b, primal_obj),
                                             ptr(re_b, residual), ptr(ga_b, gap), ptr(x_b, x), ptr(y_b, y),
                                             ptr(z_b, z), ptr(w_b, w));
    if (st != HPRQP_STATUS_OK) return st;
    for (size_t j = 0; j < K; ++j) {
        const size_t k = ids[j];
        if (status) status[k] = st_b[j];
        if (iter) iter[k] = it_b[j];
        if (primal_obj) primal_obj[k] = po_b[j];
        if (residual) residual[k] = re_b[j];
        if (gap) gap[k] = ga_b[j];
        const size_t vj = b->var_off[j], nj = b->var_off[j + 1] - vj, rj = b->row_off[j],
                     mj = b->row_off[j + 1] - rj;
        if (x) memcpy(x + var_offsets[k], x_b.data() + vj, nj * sizeof(double));
        if (z) memcpy(z + var_offsets[k], z_b.data() + vj, nj * sizeof(double));
        if (w) memcpy(w + var_offsets[k], w_b.data() + vj, nj * sizeof(double));
        if (y) memcpy(y + row_offsets[k], y_b.data() + rj, mj * sizeof(double));
    }
    return HPRQP_STATUS_OK;
}

static HPRQPStatus solve_batch_in_two(size_t K, const size_t *var_offsets, const size_t *row_offsets,
                                      const HPRQPMatrixCSR *Q, const HPRQPMatrixCSR *A, const double *c,
                                      const double *AL, const double *AU, const double *l, const double *u,
                                      const double *obj_constants, const HPRQPBatchParams *params, int *status,
                                      size_t *iter, double *primal_obj, double *residual, double *gap, double *x,
                                      double *y, double *z, double *w, bool trace)
{
    auto now = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
    const double t0 = now();
    // the instances by nonzeros (the measure of the kernel's work queue),
    // smallest first; the first part takes them up to kFirstPartWork of the
    // total, each part keeps the caller's order
    std::vector<double> wk(K);
    double total = 0.0;
    for (size_t k = 0; k < K; ++k) {
        const size_t v0 = var_offsets[k], v1 = var_offsets[k + 1], r0 = row_offsets[k], r1 = row_offsets[k + 1];
        wk[k] = (double)(Q->row_ptr[v1] - Q->row_ptr[v0]) + 2.0 * (double)(A->row_ptr[r1] - A->row_ptr[r0]) +
                (double)(v1 - v0);
        total += wk[k];
    }
    std::vector<size_t> by_size(K);
    std::iota(by_size.begin(), by_size.end(), size_t(0));
    std::stable_sort(by_size.begin(), by_size.end(), [&](size_t a, size_t b) { return wk[a] < wk[b]; });
    size_t K1 = 0;
    for (double acc = 0.0; K1 < K - 1 && acc < kFirstPartWork * total; ++K1) acc += wk[by_size[K1]];
    K1 = std::max<size_t>(K1, 1);
    std::vector<size_t> ids[2];
    ids[0].assign(by_size.begin(), by_size.begin() + K1);
    ids[1].assign(by_size.begin() + K1, by_size.end());
    for (auto &v : ids) std::sort(v.begin(), v.end());
    HPRQPBatch *b[2] = {nullptr, nullptr};
    SolveLaunch L[2];
    HPRQPStatus st = HPRQP_STATUS_OK;
    int launched = 0;
    double t_create[2] = {0.0, 0.0};
    for (int part = 0; part < 2 && st == HPRQP_STATUS_OK; ++part) {
        const double tc = now();
        // both parts take the CTA shape the whole batch would take, so each
        // instance sums in the same order as in a single launch
        st = batch_create_impl(K, var_offsets, row_offsets, Q, A, c, AL, AU, l, u, obj_constants,
                               params->device_number, false, &b[part], false, 0, ids[part].size(), kBigCta,
                               ids[part].data());
        t_create[part] = now() - tc;
        if (st == HPRQP_STATUS_OK) st = batch_launch(b[part], params, L[part]);
        if (st == HPRQP_STATUS_OK) ++launched;
    }
    const double t1 = now();
    for (int part = 0; part < launched; ++part) {
        const HPRQPStatus s2 = batch_finish(b[part], L[part]);
        if (st == HPRQP_STATUS_OK) st = s2;
    }
    const double t2 = now();
    for (int part = 0; part < 2 && st == HPRQP_STATUS_OK; ++part)
        st = scatter_results(b[part], ids[part], var_offsets, row_offsets, status, iter, primal_obj, residual, gap, x,
                             y, z, w);
    const double t3 = now();
    for (int part = 0; part < 2; ++part) {
        if (part >= launched) solve_launch_release(L[part]);
        if (b[part]) hprqp_batch_destroy(b[part]);
    }
    if (trace)
        fprintf(stderr,
                "[hprqp-b200 batch] in two launches (%zu smallest + %zu instances): create %.3f + %.3f s, until both "
                "kernels end %.3f s, results %.3f s, destroy %.3f s\n",
                ids[0].size(), ids[1].size(), t_create[0], t_create[1], t2 - t1 + (t1 - t0 - t_create[0] - t_create[1]),
                t3 - t2, now() - t3);
    return st;
}

}  // namespace hpr

extern "C" {

HPRQPStatus hprqp_solve_batch(size_t K, const size_t *var_offsets, const size_t *row_offsets, const HPRQPMatrixCSR *Q,
                              const HPRQPMatrixCSR *A, const double *c, const double *AL, const double *AU,
                              const double *l, const double *u, const double *obj_constants,
                              const HPRQPBatchParams *params, int *status, size_t *iter, double *primal_obj,
                              double *residual, double *gap, double *x, double *y, double *z, double *w)
{
    if (!params) return HPRQP_STATUS_INVALID_ARGUMENT;
    const char *tr = getenv("HPRQP_B200_BATCH_TRACE");
    const bool trace = tr && tr[0] == '1';
    auto now = [] { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); };
    const double t0 = now();
    if (K >= hpr::kSplitMinInstances && Q && A && var_offsets && row_offsets && matrix_csr_is_valid(Q) &&
        matrix_csr_is_valid(A) && var_offsets[K] == Q->nrow && row_offsets[K] == A->nrow)
        return hpr::solve_batch_in_two(K, var_offsets, row_offsets, Q, A, c, AL, AU, l, u, obj_constants, params,
                                       status, iter, primal_obj, residual, gap, x, y, z, w, trace);
    HPRQPBatch *b = nullptr;
    HPRQPStatus st = batch_create_impl(K, var_offsets, row_offsets, Q, A, c, AL, AU, l, u, obj_constants,
                                       params->device_number, false, &b, false);
    if (st != HPRQP_STATUS_OK) return st;
    const double t1 = now();
    st = hprqp_batch_solve(b, params);
    const double t2 = now();
    if (st == HPRQP_STATUS_OK) st = hprqp_batch_get_results(b, status, iter, primal_obj, residual, gap, x, y, z, w);
    const double t3 = now();
    const double kernel_s = b->last_ms / 1e3;
    hprqp_batch_destroy(b);
    if (trace)
        fprintf(stderr, "[hprqp-b200 batch] create %.3f s, solve %.3f s (kernel %.3f s), results %.3f s, destroy %.3f s\n",
                t1 - t0, t2 - t1, kernel_s, t3 - t2, now() - t3);
    return st;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// small single QPs: solve_gpu as a batch of one
// ---------------------------------------------------------------------------
namespace hpr {

// Models whose products per iteration stay below this many nonzeros
// (2 nnz(Q) + 2 nnz(A)) run in one CTA of the batch kernel: a host-driven
// iteration costs four kernel launches and the device-wide passes of the
// plain engine, which small problems cannot fill.  Process-wide; set by
// hprqp_b200_set_single_cta_max_work.
static size_t g_single_cta_max_work = 200000;

static size_t log_records_needed(const HPRQPParams *p)
{
    if (!p->verbose) return 0;
    if (p->print_frequency > 0) return p->max_iter / (size_t)p->print_frequency + 4;
    if (p->print_frequency == -1) return 2048;  // adaptive steps: < 100 per decade of iterations
    return 4;
}

bool single_cta_eligible(const HPRQPModel *m, const HPRQPParams *p)
{
    if (!m || !p || m->num_var_cones || m->num_row_cones) return false;
    if (m->Q.ncol == 0 || m->Q.ncol > (size_t)INT32_MAX || m->A.nrow > (size_t)INT32_MAX) return false;
    if (2 * (m->Q.nnz + m->A.nnz) > g_single_cta_max_work) return false;
    return log_records_needed(p) <= kSingleCtaLogCap;
}

HPRQPStatus solve_single_cta(const HPRQPModel *model, const HPRQPParams *params, HPRQPResults *results,
                             double *log_records, size_t log_cap, size_t *log_count)
{
    if (log_count) *log_count = 0;
    const size_t n = model->Q.ncol, m = model->A.nrow;
    const size_t var_off[2] = {0, n}, row_off[2] = {0, m};
    HPRQPBatch *b = nullptr;
    // the model is already preprocessed; the builder's rules leave it unchanged
    HPRQPStatus st = batch_create_impl(1, var_off, row_off, &model->Q, &model->A, model->c, model->AL, model->AU,
                                       model->l, model->u, &model->obj_constant, params->device_number, false, &b,
                                       false);
    if (st != HPRQP_STATUS_OK) return st;
    BatchArgs &G = b->args;
    long long *d_i4 = nullptr, *d_i6 = nullptr;
    double *d_t = nullptr, *d_log = nullptr;
    int *d_logn = nullptr;
    const size_t cap = log_records ? std::min(log_cap, log_records_needed(params)) : 0;
    Carver cv;
    cv.add(&d_i4, 1).add(&d_i6, 1).add(&d_t, 3).add(&d_logn, 1);
    if (cap) cv.add(&d_log, cap * kLogFields);
    if ((st = cv.commit(b))) {
        hprqp_batch_destroy(b);
        return st;
    }
    auto cuda_fail = [&](cudaError_t e, int line) {
        fprintf(stderr, "hprqp-b200: CUDA error %s at %s:%d\n", cudaGetErrorString(e), __FILE__, line);
        hprqp_batch_destroy(b);
        return HPRQP_STATUS_NOT_IMPLEMENTED;
    };
    cudaError_t ce = cudaMemsetAsync(d_logn, 0, sizeof(int), b->stream);
    if (ce != cudaSuccess) return cuda_fail(ce, __LINE__);
    G.time_from_loop = 1;
    G.iter4_out = d_i4;
    G.iter6_out = d_i6;
    G.time4_out = d_t;
    G.time6_out = d_t + 1;
    G.loop_seconds_out = d_t + 2;
    G.log_buf = d_log;
    G.log_cap = (int)cap;
    G.log_count = d_logn;
    HPRQPBatchParams bp;
    hprqp_batch_params_set_defaults(&bp);
    bp.stoptol = params->stoptol;
    bp.max_iter = params->max_iter;
    bp.time_limit = params->time_limit;
    bp.check_iter = params->check_iter;
    bp.print_frequency = params->print_frequency;
    bp.use_scaling = params->use_scaling;
    bp.device_number = params->device_number;
    st = hprqp_batch_solve(b, &bp);
    if (st != HPRQP_STATUS_OK) {
        hprqp_batch_destroy(b);
        return st;
    }
    int status = 0;
    size_t iter = 0;
    double pobj = 0.0, resid = 0.0, gap = 0.0;
    results->x = (double *)calloc(n, sizeof(double));
    results->w = (double *)calloc(n, sizeof(double));
    results->z = (double *)calloc(n, sizeof(double));
    results->y = m ? (double *)calloc(m, sizeof(double)) : nullptr;
    if (!results->x || !results->w || !results->z || (m && !results->y)) {
        results_free(results);
        hprqp_batch_destroy(b);
        return HPRQP_STATUS_ALLOCATION_FAILED;
    }
    st = hprqp_batch_get_results(b, &status, &iter, &pobj, &resid, &gap, results->x, results->y, results->z,
                                 results->w);
    long long i4 = -1, i6 = -1;
    double t[3] = {0.0, 0.0, 0.0};
    int nlog = 0;
    if (st == HPRQP_STATUS_OK) {
        if ((ce = cudaMemcpy(&i4, d_i4, sizeof(i4), cudaMemcpyDeviceToHost)) != cudaSuccess ||
            (ce = cudaMemcpy(&i6, d_i6, sizeof(i6), cudaMemcpyDeviceToHost)) != cudaSuccess ||
            (ce = cudaMemcpy(t, d_t, sizeof(t), cudaMemcpyDeviceToHost)) != cudaSuccess ||
            (ce = cudaMemcpy(&nlog, d_logn, sizeof(int), cudaMemcpyDeviceToHost)) != cudaSuccess ||
            (nlog > 0 && (ce = cudaMemcpy(log_records, d_log, (size_t)nlog * kLogFields * sizeof(double),
                                          cudaMemcpyDeviceToHost)) != cudaSuccess)) {
            results_free(results);
            return cuda_fail(ce, __LINE__);
        }
    }
    hprqp_batch_destroy(b);
    if (st != HPRQP_STATUS_OK) {
        results_free(results);
        return st;
    }
    if (log_count) *log_count = (size_t)nlog;
    const double elapsed = t[2];
    // the host loop's bookkeeping: a milestone never reached (or reached at
    // iteration 0) reports the final iteration and time
    results->iter = iter;
    results->time = elapsed;
    results->iter_4 = i4 <= 0 ? iter : (size_t)i4;
    results->iter_6 = i6 <= 0 ? iter : (size_t)i6;
    results->time_4 = (i4 < 0 || t[0] == 0.0) ? elapsed : t[0];
    results->time_6 = (i6 < 0 || t[1] == 0.0) ? elapsed : t[1];
    results->primal_obj = pobj;
    results->residuals = resid;
    results->gap = gap;
    results->status = status;
    return (HPRQPStatus)status;
}

}  // namespace hpr

extern "C" size_t hprqp_b200_set_single_cta_max_work(size_t max_work)
{
    const size_t old = hpr::g_single_cta_max_work;
    hpr::g_single_cta_max_work = max_work;
    return old;
}
