// Tiled CSR SpMV with a fused per-row epilogue (sm_100a, FP64).
//
// Every HPR kernel is "y = M x, then an elementwise update of row i that
// consumes y_i" (the reference fuses the same way with a thread-per-row dot,
// src/gpu/iteration.cu:282-697).  The cost of y = M x on B200 is the latency
// of the matrix stream from HBM and of the x[col] gathers from L2, so the
// kernel keeps many independent loads in flight and never lets a short or
// long row idle a lane:
//
//   * each matrix is cut once, at setup, into warp tiles: consecutive rows,
//     at most kTileRows of them and at most kTileCap entries in total (a row
//     longer than kTileCap is cut into kTileCap-entry chunks, one warp per
//     chunk, and a second tiny kernel adds its chunk partials in order);
//   * a warp streams its tile's entries as 256-entry windows aligned to 8
//     entries: each lane owns 8 consecutive entries, loaded with 16-byte
//     vector loads, and the next window's loads are issued before the x
//     gathers of the current one are consumed;
//   * row starts come from a bitmap built at setup (one bit per entry), so a
//     lane sums its own entries in registers and writes the rows that start
//     and end inside it; a row crossing lanes is finished by one segmented
//     warp scan (segment flags from a ballot), and a carry links windows.
//     Shared memory holds only the tile's row sums: the x gathers and the
//     matrix stream are all the L1 traffic, which measured ~11% faster than
//     staging the products in shared memory for a segmented scan there;
//   * the row sums are indexed by the ordinal of the row among the tile's
//     non-empty rows, and the epilogue runs after the tile, lane i on rows
//     i and i + 32: coalesced;
//   * a matrix whose rows are mostly runs of consecutive columns (dense
//     blocks, e.g. the transpose of dense factor rows) runs k_spmv_staged
//     instead: strided lanes, so a run's gathers are coalesced, products
//     summed by a segmented scan in shared memory (choose_staged);
//   * reductions requested by an epilogue are folded per CTA in a fixed
//     order, so results are bit-reproducible run to run.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <vector>

namespace hpr {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kTileRows = 64;   // rows per warp tile (two per lane)
constexpr int kTileCap = 1024;  // entries per warp tile; longer rows are chunked
constexpr int kChunk = kTileCap;  // entries per chunk of a long row
constexpr int kSpmvWinU = 8;  // entries per lane per window (two int4 + four double2 loads)
constexpr int kSpmvWin = 32 * kSpmvWinU;  // entries per window
static_assert(kSpmvWinU == 8, "the window loads and the row-start bitmap assume 8 entries per lane");
// CTAs per SM the register budget must allow: 4 for k_spmv (64 registers;
// more warps hide the x-gather latency: 2-4% faster than 3 on the n=1e6
// QP's matrices), 3 for k_spmv_staged (its shared-memory scan spills at 64)
#ifndef HPR_SPMV_MIN_BLOCKS
#define HPR_SPMV_MIN_BLOCKS 4
#endif
#ifndef HPR_SPMV_STAGED_MIN_BLOCKS
#define HPR_SPMV_STAGED_MIN_BLOCKS 3
#endif

struct DCsr {
    int nrow = 0, ncol = 0, nnz = 0;
    int *rp = nullptr;
    int *ci = nullptr;
    double *v = nullptr;    // ci and v hold padded_nnz(nnz) entries, the padding zero
    int4 *tiles = nullptr;  // {r0, r1, entries, 0}
    int ntiles = 0;
    int4 *chunks = nullptr;  // {row, k0, k1, slot}
    int nchunks = 0;
    int2 *long_rows = nullptr;  // {row, first chunk slot}
    int nlong = 0;
    double *chunk_partial = nullptr;
    int *err = nullptr;
    unsigned char *heads = nullptr;  // bit j of heads[q]: entry 8q + j starts a non-empty row
    int staged = 0;      // 1: tiles run k_spmv_staged (rows of consecutive columns)
    int grid_main = 0;   // CTAs of k_spmv (one tile per warp)
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

// Row sums of one warp tile (rows r0 .. r0 + nr - 1, entries k0 .. k1 - 1,
// at most kTileRows rows and kTileCap entries) into srow[ordinal], where the
// ordinal of a non-empty row counts the non-empty rows before it in the tile.
//
// Windows start at k0 rounded down to a multiple of 8 (the arrays are padded
// to a multiple of 8 entries, so the vector loads stay in bounds); lane L
// owns entries base + 8L .. base + 8L + 7.  Bit j of heads[q] marks entry
// 8q + j as the first entry of a non-empty row.  A lane sums its entries in
// order, writes the rows that start and end inside it, and hands the open
// row across lanes with one segmented warp scan; the row still open at the
// end of a window is carried into the next one.
__device__ __forceinline__ void tile_rowsums(const DCsr &M, const double *__restrict__ x, int k0, int k1,
                                             double *srow)
{
    constexpr unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    double carry = 0.0;
    int ord_base = 0;
    int c[kSpmvWinU];
    double v[kSpmvWinU];
    unsigned hb = 0;
    auto load = [&](int base) {
        const int e = base + kSpmvWinU * lane;
        if (e < k1) {
            const int4 c0 = __ldcs(reinterpret_cast<const int4 *>(M.ci + e));
            const int4 c1 = __ldcs(reinterpret_cast<const int4 *>(M.ci + e + 4));
            const double2 v0 = __ldcs(reinterpret_cast<const double2 *>(M.v + e));
            const double2 v1 = __ldcs(reinterpret_cast<const double2 *>(M.v + e + 2));
            const double2 v2 = __ldcs(reinterpret_cast<const double2 *>(M.v + e + 4));
            const double2 v3 = __ldcs(reinterpret_cast<const double2 *>(M.v + e + 6));
            c[0] = c0.x, c[1] = c0.y, c[2] = c0.z, c[3] = c0.w;
            c[4] = c1.x, c[5] = c1.y, c[6] = c1.z, c[7] = c1.w;
            v[0] = v0.x, v[1] = v0.y, v[2] = v1.x, v[3] = v1.y;
            v[4] = v2.x, v[5] = v2.y, v[6] = v3.x, v[7] = v3.y;
            hb = __ldg(M.heads + (e >> 3));
        } else {
#pragma unroll
            for (int j = 0; j < kSpmvWinU; ++j) {
                c[j] = 0;
                v[j] = 0.0;
            }
            hb = 0;
        }
    };
    const int base0 = k0 & ~(kSpmvWinU - 1);
    if (base0 < k1) load(base0);
    for (int base = base0; base < k1; base += kSpmvWin) {
        const int e = base + kSpmvWinU * lane;
        int lo = k0 - e, hi = k1 - e;
        lo = lo < 0 ? 0 : (lo > kSpmvWinU ? kSpmvWinU : lo);
        hi = hi < 0 ? 0 : (hi > kSpmvWinU ? kSpmvWinU : hi);
        const unsigned vm = hi > lo ? (((1u << hi) - 1u) & ~((1u << lo) - 1u)) : 0u;
        double p[kSpmvWinU];
#pragma unroll
        for (int j = 0; j < kSpmvWinU; ++j) p[j] = ((vm >> j) & 1u) ? v[j] * __ldg(x + c[j]) : 0.0;
        const unsigned h = hb & vm;
        load(base + kSpmvWin);  // the next window's stream, in flight while this one is summed
        int before = 0, total = 0;
#pragma unroll
        for (int j = 0; j < kSpmvWinU; ++j) {
            const unsigned bj = __ballot_sync(FULL, (h >> j) & 1u);
            before += __popc(bj & lt);
            total += __popc(bj);
        }
        const int ord0 = ord_base + before;  // ordinal of this lane's first row start
        double run = 0.0, prefix = 0.0;
        int nh = 0;
#pragma unroll
        for (int j = 0; j < kSpmvWinU; ++j) {
            if ((h >> j) & 1u) {
                if (nh == 0) prefix = run;
                else srow[ord0 + nh - 1] = run;  // a row inside this lane
                ++nh;
                run = 0.0;
            }
            run += p[j];
        }
        // segmented inclusive scan over the lanes; a lane with a row start
        // begins a segment (flags come from one ballot, not from shuffles)
        const bool has = h != 0u;
        const unsigned hm = __ballot_sync(FULL, has);
        double s = (lane == 0 && !has) ? carry + run : run;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double u = __shfl_up_sync(FULL, s, o);
            const unsigned span = lane >= o ? ((lt | (1u << lane)) & ~((1u << (lane - o + 1)) - 1u)) : 0u;
            if (lane >= o && (hm & span) == 0u) s = u + s;
        }
        double ex = __shfl_up_sync(FULL, s, 1);
        if (lane == 0) ex = carry;
        if (has && ord0 > 0) srow[ord0 - 1] = ex + prefix;  // the row open before this lane's first start
        carry = __shfl_sync(FULL, s, 31);
        ord_base += total;
    }
    __syncwarp();
    if (lane == 0 && ord_base > 0) srow[ord_base - 1] = carry;  // the tile's last non-empty row
    __syncwarp();
}

// Epilogue concept:
//   static constexpr int NRED;  __host__ __device__ void ops(int*) const;
//   __device__ void init(Acc&) const; row(int i, double y_i, Acc&) const;
//   __device__ void extra(Acc&) const;        // once per CTA, main kernel only
//   double *partials;                         // [npart * NRED]
template <class Epi>
__global__ void __launch_bounds__(kThreads, HPR_SPMV_MIN_BLOCKS) k_spmv(const DCsr M, const double *__restrict__ xin, const Epi epi)
{
    __shared__ double s_row[kWarps][kTileRows];
    Acc<Epi::NRED> acc;
    epi.init(acc);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int t = blockIdx.x * kWarps + wid;
    if (t < M.ntiles) {
        const int4 T = M.tiles[t];
        const int r0 = T.x, nr = T.y - T.x;
        tile_rowsums(M, xin, __ldg(M.rp + r0), __ldg(M.rp + T.y), s_row[wid]);
        // ordinals of this lane's rows lane and lane + 32 among the tile's non-empty rows
        const unsigned lt = (1u << lane) - 1u;
        bool ne[2];
        unsigned bm[2];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int r = lane + 32 * j;
            ne[j] = r < nr && __ldg(M.rp + r0 + r + 1) > __ldg(M.rp + r0 + r);
            bm[j] = __ballot_sync(0xffffffffu, ne[j]);
        }
        const int ord[2] = {__popc(bm[0] & lt), __popc(bm[0]) + __popc(bm[1] & lt)};
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            const int r = lane + 32 * j;
            if (r < nr) epi.row(r0 + r, ne[j] ? s_row[wid][ord[j]] : 0.0, acc);
        }
    }
    epi.extra(acc);
    if constexpr (Epi::NRED > 0) {
        int ops[Epi::NRED > 0 ? Epi::NRED : 1];
        epi.ops(ops);
        block_reduce_store<Epi::NRED>(acc, ops, epi.partials + (size_t)blockIdx.x * Epi::NRED);
    }
}

// padded shared-memory slot of window entry i (conflict-free for both the
// strided writes and the lane-contiguous reads of the segmented scan)
__device__ __forceinline__ int win_slot(int i) { return i + (i >> 3); }

// Staged variant, for matrices whose rows hold runs of consecutive columns
// (dense blocks): lane L loads entries L, L + 32, ... of each 256-entry
// window, so the x gathers of a run are coalesced; the products go to shared
// memory and a segmented scan there (head flags from the tile's row starts,
// staged in shared memory) sums them per row into rowsum[0 .. nr - 1].
// rs[0 .. nr] are the tile's row starts in shared memory.
__device__ __forceinline__ void tile_rowsums_staged(const DCsr &M, const double *__restrict__ x, const int *rs, int nr,
                                             double *sv, unsigned char *sh, double *rowsum)
{
    constexpr int KR = kTileRows / 32;
    const int lane = threadIdx.x & 31;
    const int k0 = rs[0], k1 = rs[nr];
#pragma unroll
    for (int j = 0; j < KR; ++j) {
        const int r = lane + 32 * j;
        if (r < nr) rowsum[r] = 0.0;  // empty rows keep 0
    }
    double carry = 0.0;
    int c[kSpmvWinU];
    double v[kSpmvWinU];
#pragma unroll
    for (int u = 0; u < kSpmvWinU; ++u) {
        const int k = k0 + u * 32 + lane;
        c[u] = k < k1 ? __ldcs(M.ci + k) : 0;
        v[u] = k < k1 ? __ldcs(M.v + k) : 0.0;
    }
    for (int base = k0; base < k1; base += kSpmvWin) {
        const int nb = base + kSpmvWin;
        double p[kSpmvWinU];
#pragma unroll
        for (int u = 0; u < kSpmvWinU; ++u) p[u] = v[u] * __ldg(x + c[u]);
        // next window's stream, in flight while this one is summed
#pragma unroll
        for (int u = 0; u < kSpmvWinU; ++u) {
            const int k = nb + u * 32 + lane;
            c[u] = k < k1 ? __ldcs(M.ci + k) : 0;
            v[u] = k < k1 ? __ldcs(M.v + k) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kSpmvWinU; ++u) {
            const int i = u * 32 + lane;
            sv[win_slot(i)] = p[u];
            sh[i] = 0;
        }
        __syncwarp();
#pragma unroll
        for (int j = 0; j < KR; ++j) {
            const int r = lane + 32 * j;
            if (r < nr) {
                const int a = rs[r], e = rs[r + 1];
                if (a < e && a >= base && a < nb) sh[a - base] = 1;
            }
        }
        __syncwarp();
        // lane-contiguous segmented sums, lane 0 continuing the carried row
        double run = lane == 0 ? carry : 0.0;
        bool seg = false;
#pragma unroll
        for (int j = 0; j < kSpmvWinU; ++j) {
            const int i = lane * kSpmvWinU + j;
            const double q = sv[win_slot(i)];
            if (sh[i]) {
                run = q;
                seg = true;
            } else {
                run += q;
            }
            p[j] = run;
        }
        // segmented inclusive scan of the lane tails across the warp
        double tail = run;
        bool tseg = seg;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const double tl = __shfl_up_sync(0xffffffffu, tail, off);
            const bool fl = __shfl_up_sync(0xffffffffu, (int)tseg, off);
            if (lane >= off && !tseg) {
                tail = tl + tail;
                tseg = fl;
            }
        }
        double cin = __shfl_up_sync(0xffffffffu, tail, 1);
        if (lane == 0) cin = 0.0;
        __syncwarp();
        bool h = false;
#pragma unroll
        for (int j = 0; j < kSpmvWinU; ++j) {
            const int i = lane * kSpmvWinU + j;
            h = h || sh[i];
            if (!h) p[j] = cin + p[j];
            sv[win_slot(i)] = p[j];
        }
        carry = __shfl_sync(0xffffffffu, p[kSpmvWinU - 1], 31);
        __syncwarp();
        // rows that end in this window
#pragma unroll
        for (int j = 0; j < KR; ++j) {
            const int r = lane + 32 * j;
            if (r < nr) {
                const int a = rs[r], e = rs[r + 1];
                if (a < e && e - 1 >= base && e - 1 < nb) rowsum[r] = sv[win_slot(e - 1 - base)];
            }
        }
        __syncwarp();
    }
}

template <class Epi>
__global__ void __launch_bounds__(kThreads, HPR_SPMV_STAGED_MIN_BLOCKS) k_spmv_staged(const DCsr M, const double *__restrict__ xin, const Epi epi)
{
    __shared__ double s_val[kWarps][kSpmvWin + kSpmvWin / 8];
    __shared__ unsigned char s_head[kWarps][kSpmvWin];
    __shared__ int s_rs[kWarps][kTileRows + 1];
    __shared__ double s_row[kWarps][kTileRows];
    Acc<Epi::NRED> acc;
    epi.init(acc);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int t = blockIdx.x * kWarps + wid;
    if (t < M.ntiles) {
        const int4 T = M.tiles[t];
        const int r0 = T.x, nr = T.y - T.x;
        int *rs = s_rs[wid];
        for (int r = lane; r <= nr; r += 32) rs[r] = __ldg(M.rp + r0 + r);
        __syncwarp();
        tile_rowsums_staged(M, xin, rs, nr, s_val[wid], s_head[wid], s_row[wid]);
        __syncwarp();
#pragma unroll
        for (int j = 0; j < kTileRows / 32; ++j) {
            const int r = lane + 32 * j;
            if (r < nr) epi.row(r0 + r, s_row[wid][r], acc);
        }
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

// entries allocated for ci and v: a multiple of kSpmvWinU, plus one group
inline size_t padded_nnz(size_t nnz) { return ((nnz + kSpmvWinU - 1) / kSpmvWinU + 1) * kSpmvWinU; }

// row-start bitmap: bit j of byte q set when entry 8q + j is the first entry
// of a non-empty row; padded_nnz(nnz) / 8 bytes
inline void build_heads(const std::vector<int> &rp, std::vector<unsigned char> &heads)
{
    const size_t nrow = rp.size() - 1;
    heads.assign(padded_nnz((size_t)rp[nrow]) / kSpmvWinU, 0);
    for (size_t r = 0; r < nrow; ++r)
        if (rp[r + 1] > rp[r]) heads[(size_t)rp[r] >> 3] |= (unsigned char)(1u << (rp[r] & 7));
}

// Tile kernel of a matrix, fixed at setup from its structure so that every
// solve of a model sums in the same order: k_spmv_staged when at least half
// of the consecutive entry pairs inside rows are consecutive columns (dense
// blocks: its strided lanes then gather x coalesced), else k_spmv.
inline int choose_staged(const std::vector<int> &rp, const std::vector<int> &ci)
{
    size_t pairs = 0, runs = 0;
    for (size_t r = 0; r + 1 < rp.size(); ++r)
        for (int k = rp[r]; k + 1 < rp[r + 1]; ++k) {
            ++pairs;
            runs += ci[k + 1] == ci[k] + 1;
        }
    return pairs > 0 && 2 * runs >= pairs;
}

// Warp tiles: consecutive rows, at most kTileRows rows and kTileCap
// entries; a row longer than kTileCap becomes kChunk-entry chunks.
inline void build_tile_plan(const std::vector<int> &rp, TilePlan &p)
{
    p = TilePlan();
    const int nrow = (int)rp.size() - 1;
    int r = 0;
    while (r < nrow) {
        const int len = rp[r + 1] - rp[r];
        if (len > kTileCap) {
            p.long_rows.push_back(make_int2(r, (int)p.chunks.size()));
            for (int k = rp[r]; k < rp[r + 1]; k += kChunk) {
                const int k1 = k + kChunk < rp[r + 1] ? k + kChunk : rp[r + 1];
                p.chunks.push_back(make_int4(r, k, k1, (int)p.chunks.size()));
            }
            ++r;
            continue;
        }
        int r1 = r, nnz = 0;
        while (r1 < nrow && r1 - r < kTileRows) {
            const int l = rp[r1 + 1] - rp[r1];
            if (l > kTileCap || (nnz + l > kTileCap && r1 > r)) break;
            nnz += l;
            ++r1;
        }
        p.tiles.push_back(make_int4(r, r1, nnz, 0));
        r = r1;
    }
}

}  // namespace hpr
