// Row-block CSR SpMV with a fused per-row epilogue (sm_100a, FP64).
//
// Every HPR kernel is "y = M x, then an elementwise update of row i that
// consumes y_i" (reference kernels src/gpu/iteration.cu:110-697 fuse the
// same way with a thread-per-row dot).  Here a matrix is cut once, at setup,
// into row blocks: maximal runs of consecutive rows whose total nnz fits in
// kCap staged products (or a single longer row).  One CTA owns one block:
//
//   1. stream the block's values/column indices with coalesced, evict-first
//      loads (they are touched once per product), gather x through L1/L2
//      (x is the vector reused by every row), and stage the products in
//      shared memory;
//   2. reduce each row's products with a lane group whose width (1..32) is
//      the block's mean row length rounded down to a power of two, using
//      warp shuffles; rows longer than kCap use the whole CTA;
//   3. run the epilogue thread-per-row so its vector traffic is coalesced,
//      and fold optional reductions into a per-CTA partial (fixed order,
//      hence bit-reproducible run to run).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace hpr {

constexpr int kThreads = 256;
constexpr int kCap = 2048;     // staged products per row block
constexpr int kMaxRows = 1024; // rows per row block
constexpr int kWarps = kThreads / 32;

struct DCsr {
    int nrow = 0, ncol = 0, nnz = 0;
    int *rp = nullptr;
    int *ci = nullptr;
    double *v = nullptr;
    int2 *blocks = nullptr;  // row-block partition
    int nblocks = 0;
};

enum RedOp : int { kSum = 0, kMax = 1 };

__device__ __forceinline__ double ld_stream(const double *p) { return __ldcs(p); }
__device__ __forceinline__ int ld_stream(const int *p) { return __ldcs(p); }

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

__device__ __forceinline__ double warp_max(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Deterministic CTA sum (warp trees, then warp partials in order).
__device__ __forceinline__ double block_sum(double v, double *scratch /* >= kWarps */)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < kWarps; ++i) t += scratch[i];
    __syncthreads();
    return t;  // valid in thread 0
}

// Per-thread reduction accumulator with compile-time slot count.
template <int N>
struct Acc {
    double v[N > 0 ? N : 1];
};

// Fold per-thread accumulators of a CTA and write one partial per slot.
template <int N>
__device__ __forceinline__ void block_reduce_store(Acc<N> &acc, const int *ops, double *out)
{
    if constexpr (N > 0) {
        __shared__ double s_red[kWarps][N];
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int k = 0; k < N; ++k) {
            double v = ops[k] == kMax ? warp_max(acc.v[k]) : warp_sum(acc.v[k]);
            if (lane == 0) s_red[warp][k] = v;
        }
        __syncthreads();
        if (threadIdx.x < N) {
            const int k = threadIdx.x;
            double t = s_red[0][k];
            for (int w = 1; w < kWarps; ++w) t = ops[k] == kMax ? fmax(t, s_red[w][k]) : t + s_red[w][k];
            out[k] = t;
        }
    }
}

// Epilogue concept:
//   static constexpr int NRED;  __device__ void ops(int*) const;
//   __device__ void row(int i, double y_i, Acc<NRED>&) const;
//   __device__ void extra(Acc<NRED>&) const;   // optional grid-stride work
//   double *partials;                          // [gridDim.x * NRED]
template <class Epi>
__global__ void __launch_bounds__(kThreads) k_rowblock(const DCsr M, const double *__restrict__ xin,
                                                       const Epi epi)
{
    __shared__ double s_prod[kCap];
    __shared__ double s_sum[kMaxRows];
    __shared__ double s_scr[kWarps];
    const int tid = threadIdx.x;
    const int2 blk = M.blocks[blockIdx.x];
    const int r0 = blk.x, r1 = blk.y;
    const int k0 = M.rp[r0], k1 = M.rp[r1];
    const int nnz = k1 - k0, nrows = r1 - r0;

    if (nnz > kCap) {
        // one long row: the whole CTA streams it
        double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
        int k = k0 + tid;
        for (; k + 3 * kThreads < k1; k += 4 * kThreads) {
            const int c0 = ld_stream(M.ci + k), c1 = ld_stream(M.ci + k + kThreads);
            const int c2 = ld_stream(M.ci + k + 2 * kThreads), c3 = ld_stream(M.ci + k + 3 * kThreads);
            const double v0 = ld_stream(M.v + k), v1 = ld_stream(M.v + k + kThreads);
            const double v2 = ld_stream(M.v + k + 2 * kThreads), v3 = ld_stream(M.v + k + 3 * kThreads);
            s0 = fma(v0, __ldg(xin + c0), s0);
            s1 = fma(v1, __ldg(xin + c1), s1);
            s2 = fma(v2, __ldg(xin + c2), s2);
            s3 = fma(v3, __ldg(xin + c3), s3);
        }
        for (; k < k1; k += kThreads) s0 = fma(ld_stream(M.v + k), __ldg(xin + ld_stream(M.ci + k)), s0);
        const double t = block_sum((s0 + s1) + (s2 + s3), s_scr);
        if (tid == 0) s_sum[0] = t;
    } else {
        // 1. stage products
        for (int j0 = 0; j0 < nnz; j0 += 4 * kThreads) {
            int c[4];
            double v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int j = j0 + u * kThreads + tid;
                if (j < nnz) {
                    c[u] = ld_stream(M.ci + k0 + j);
                    v[u] = ld_stream(M.v + k0 + j);
                }
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int j = j0 + u * kThreads + tid;
                if (j < nnz) s_prod[j] = v[u] * __ldg(xin + c[u]);
            }
        }
        __syncthreads();
        // 2. per-row reduction with lane groups of width G
        const int avg = nrows > 0 ? nnz / nrows : 0;
        const int G = avg >= 32 ? 32 : avg >= 16 ? 16 : avg >= 8 ? 8 : avg >= 4 ? 4 : avg >= 2 ? 2 : 1;
        const int gl = tid & (G - 1);
        const int ngroups = kThreads / G;
        const int group = tid / G;
        const int rounds = (nrows + ngroups - 1) / ngroups;
        for (int rd = 0; rd < rounds; ++rd) {
            const int rr = rd * ngroups + group;
            double s = 0.0;
            if (rr < nrows) {
                const int a = M.rp[r0 + rr] - k0, b = M.rp[r0 + rr + 1] - k0;
                for (int j = a + gl; j < b; j += G) s += s_prod[j];
            }
            for (int o = G >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (gl == 0 && rr < nrows) s_sum[rr] = s;
        }
    }
    __syncthreads();
    // 3. epilogue, thread per row
    Acc<Epi::NRED> acc;
    epi.init(acc);
    for (int r = tid; r < nrows; r += kThreads) epi.row(r0 + r, s_sum[r], acc);
    epi.extra(acc);
    if constexpr (Epi::NRED > 0) {
        int ops[Epi::NRED > 0 ? Epi::NRED : 1];
        epi.ops(ops);
        block_reduce_store<Epi::NRED>(acc, ops, epi.partials + (size_t)blockIdx.x * Epi::NRED);
    }
}

// Plain elementwise kernel over max(n, m) with the same epilogue/reduction
// plumbing (no matrix).
template <class Epi>
__global__ void __launch_bounds__(kThreads) k_elementwise(int len, const Epi epi)
{
    Acc<Epi::NRED> acc;
    epi.init(acc);
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < len; i += gridDim.x * kThreads) epi.row(i, 0.0, acc);
    epi.extra(acc);
    if constexpr (Epi::NRED > 0) {
        int ops[Epi::NRED > 0 ? Epi::NRED : 1];
        epi.ops(ops);
        block_reduce_store<Epi::NRED>(acc, ops, epi.partials + (size_t)blockIdx.x * Epi::NRED);
    }
}

}  // namespace hpr
