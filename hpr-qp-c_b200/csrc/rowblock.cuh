// Warp-tiled CSR SpMV with a fused per-row epilogue (sm_100a, FP64).
//
// Every HPR kernel is "y = M x, then an elementwise update of row i that
// consumes y_i" (the reference fuses the same way with a thread-per-row dot,
// src/gpu/iteration.cu:282-697).  The cost of y = M x on B200 is the latency
// of the x[col] gathers (x lives in L2, the matrix streams from HBM), so the
// kernel is built to keep as many independent loads in flight as possible:
//
//   * each matrix is cut once, at setup, into warp tiles of up to 32
//     consecutive rows; a tile also fixes its lane-group width G (1..32), a
//     power of two near a quarter of the tile's mean row length, so each
//     lane of a group adds a few entries of its row;
//   * a warp walks its tile in 32/G-row passes; inside a row, a lane issues
//     four independent value/column/x loads per step (values and indices are
//     read once, with evict-first hints so they do not displace x in L2);
//   * the row sums are shuffled so that lane i holds row i, and the
//     epilogue runs on all 32 lanes for 32 consecutive rows: coalesced;
//   * rows longer than kLongRow are cut into kChunk-entry chunks, one warp
//     per chunk; a second tiny kernel adds a row's chunk partials in order
//     and runs its epilogue;
//   * reductions requested by an epilogue are folded per CTA in a fixed
//     order, so results are bit-reproducible run to run.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace hpr {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kLongRow = 4096;  // rows longer than this are chunked
constexpr int kChunk = 2048;    // entries per chunk of a long row
constexpr int kSoloRow = 256;   // rows at least this long get a tile of their own
#ifndef HPR_SPMV_MIN_BLOCKS
#define HPR_SPMV_MIN_BLOCKS 4  // CTAs per SM the register budget must allow
#endif

struct DCsr {
    int nrow = 0, ncol = 0, nnz = 0;
    int *rp = nullptr;
    int *ci = nullptr;
    double *v = nullptr;
    int4 *tiles = nullptr;  // {r0, r1, G, 0}
    int ntiles = 0;
    int4 *chunks = nullptr;  // {row, k0, k1, slot}
    int nchunks = 0;
    int2 *long_rows = nullptr;  // {row, first chunk slot}
    int nlong = 0;
    double *chunk_partial = nullptr;
    int *err = nullptr;
    int grid_main = 0;   // CTAs of k_spmv (8 tiles each)
    int grid_chunk = 0;  // CTAs of k_chunks (8 chunks each)
    int grid_long = 0;   // CTAs of k_long_epi
    int npart() const { return grid_main + grid_long; }
};

enum RedOp : int { kSum = 0, kMax = 1 };

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

// Deterministic CTA sum (warp trees, then warp partials in order); the
// result is valid in thread 0.
__device__ __forceinline__ double block_sum(double v, double *scratch)
{
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    double t = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < kWarps; ++i) t += scratch[i];
    __syncthreads();
    return t;
}

template <int N>
struct Acc {
    double v[N > 0 ? N : 1];
};

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

// sum of v[k] * x[ci[k]] over k = a + gl, a + gl + G, ... < e, four
// independent loads in flight per step
__device__ __forceinline__ double row_dot(const DCsr &M, const double *__restrict__ x, int a, int e, int gl,
                                          int G)
{
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int k = a + gl;
    for (; k + 3 * G < e; k += 4 * G) {
        const int c0 = __ldcs(M.ci + k), c1 = __ldcs(M.ci + k + G);
        const int c2 = __ldcs(M.ci + k + 2 * G), c3 = __ldcs(M.ci + k + 3 * G);
        const double v0 = __ldcs(M.v + k), v1 = __ldcs(M.v + k + G);
        const double v2 = __ldcs(M.v + k + 2 * G), v3 = __ldcs(M.v + k + 3 * G);
        s0 = fma(v0, __ldg(x + c0), s0);
        s1 = fma(v1, __ldg(x + c1), s1);
        s2 = fma(v2, __ldg(x + c2), s2);
        s3 = fma(v3, __ldg(x + c3), s3);
    }
    for (; k < e; k += G) s0 = fma(__ldcs(M.v + k), __ldg(x + __ldcs(M.ci + k)), s0);
    return (s0 + s1) + (s2 + s3);
}

// Epilogue concept:
//   static constexpr int NRED;  __host__ __device__ void ops(int*) const;
//   __device__ void init(Acc&) const; row(int i, double y_i, Acc&) const;
//   __device__ void extra(Acc&) const;        // once per CTA, main kernel only
//   double *partials;                         // [npart * NRED]
template <class Epi>
__global__ void __launch_bounds__(kThreads, HPR_SPMV_MIN_BLOCKS) k_spmv(const DCsr M, const double *__restrict__ xin, const Epi epi)
{
    Acc<Epi::NRED> acc;
    epi.init(acc);
    const int lane = threadIdx.x & 31;
    const int t = blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (t < M.ntiles) {
        const int4 T = M.tiles[t];
        const int r0 = T.x, nr = T.y - T.x, G = T.z;
        const int rpp = 32 / G;  // rows per pass
        const int gl = lane & (G - 1), grp = lane / G;
        const int passes = (nr + rpp - 1) / rpp;
        double mine = 0.0;  // sum of row r0 + lane
        for (int p = 0; p < passes; ++p) {
            const int rr = p * rpp + grp;
            double s = 0.0;
            if (rr < nr) s = row_dot(M, xin, __ldg(M.rp + r0 + rr), __ldg(M.rp + r0 + rr + 1), gl, G);
            for (int o = G >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            const double v = __shfl_sync(0xffffffffu, s, (lane % rpp) * G);
            if (lane / rpp == p) mine = v;
        }
        if (lane < nr) epi.row(r0 + lane, mine, acc);
    }
    epi.extra(acc);
    if constexpr (Epi::NRED > 0) {
        int ops[Epi::NRED > 0 ? Epi::NRED : 1];
        epi.ops(ops);
        block_reduce_store<Epi::NRED>(acc, ops, epi.partials + (size_t)blockIdx.x * Epi::NRED);
    }
}

// one warp per chunk of a long row: partial sums only
static __global__ void __launch_bounds__(kThreads) k_chunks(const DCsr M, const double *__restrict__ xin)
{
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * kWarps + (threadIdx.x >> 5);
    if (c >= M.nchunks) return;
    const int4 C = M.chunks[c];
    double s = row_dot(M, xin, C.y, C.z, lane, 32);
    s = warp_sum(s);
    if (lane == 0) M.chunk_partial[C.w] = s;
}

// long rows: add the chunk partials in order and run the epilogue
template <class Epi>
__global__ void __launch_bounds__(kThreads) k_long_epi(const DCsr M, const Epi epi)
{
    Acc<Epi::NRED> acc;
    epi.init(acc);
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < M.nlong) {
        const int2 lr = M.long_rows[i];
        const int c1 = i + 1 < M.nlong ? M.long_rows[i + 1].y : M.nchunks;
        double s = 0.0;
        for (int c = lr.y; c < c1; ++c) s += M.chunk_partial[c];
        epi.row(lr.x, s, acc);
    }
    if constexpr (Epi::NRED > 0) {
        int ops[Epi::NRED > 0 ? Epi::NRED : 1];
        epi.ops(ops);
        block_reduce_store<Epi::NRED>(acc, ops,
                                      epi.partials + (size_t)(M.grid_main + blockIdx.x) * Epi::NRED);
    }
}

// Elementwise kernel over max(n, m) with the same epilogue/reduction
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

// ---------------------------------------------------------------------------
// host: tile plan
// ---------------------------------------------------------------------------
struct TilePlan {
    std::vector<int4> tiles;
    std::vector<int4> chunks;
    std::vector<int2> long_rows;
};

inline int lane_group_for(long long nnz, int rows)
{
    const long long avg = rows > 0 ? nnz / rows : 0;
    int G = 1;
    while (G < 32 && 4LL * G * 2 <= avg) G *= 2;  // about four entries per lane
    return G;
}

inline void build_tile_plan(const std::vector<int> &rp, TilePlan &p)
{
    p = TilePlan();
    const int nrow = (int)rp.size() - 1;
    int r = 0;
    while (r < nrow) {
        const int len = rp[r + 1] - rp[r];
        if (len > kLongRow) {
            p.long_rows.push_back(make_int2(r, (int)p.chunks.size()));
            for (int k = rp[r]; k < rp[r + 1]; k += kChunk) {
                const int k1 = k + kChunk < rp[r + 1] ? k + kChunk : rp[r + 1];
                p.chunks.push_back(make_int4(r, k, k1, (int)p.chunks.size()));
            }
            ++r;
            continue;
        }
        if (len >= kSoloRow) {
            p.tiles.push_back(make_int4(r, r + 1, 32, 0));
            ++r;
            continue;
        }
        int r1 = r;
        while (r1 < nrow && r1 - r < 32 && rp[r1 + 1] - rp[r1] < kSoloRow) ++r1;
        p.tiles.push_back(make_int4(r, r1, lane_group_for(rp[r1] - rp[r], r1 - r), 0));
        r = r1;
    }
}

}  // namespace hpr
