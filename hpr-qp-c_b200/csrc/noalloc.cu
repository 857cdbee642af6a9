// Power iteration for lambda_max(A A') that allocates no device memory.
//
// Some callers cannot call cudaMalloc at all: a host application whose GPU
// memory is owned by another allocator (a framework's caching allocator or
// a preallocated arena that must account for every byte), or an embedded or
// real-time host that forbids device allocation after start-up.  They can still pass device buffers they own
// for the inputs.  This entry point serves them: the work vectors and the
// reduction partials of the power iteration live in a fixed file-scope
// device array instead of memory obtained at call time.
//
// The array holds kNoAllocDoubles doubles (8 MiB) and every GPU that loads
// this library keeps it until the process exits.  Its layout for one call is
// z[m] | q[m] | t[n] | partials[kPartSlots]; a call with 2m + n larger than
// kNoAllocDoubles - kPartSlots (1,046,526) is rejected with
// HPRQP_STATUS_INVALID_ARGUMENT and a message on stderr.  Every call reuses the same
// array: it does not start at zero (each region is fully written before it is
// read), and two calls that overlap on the GPU -- on different streams, or
// from different host threads -- would overwrite each other's vectors, so
// calls on one device must not overlap.
//
// Host code cannot use the array's name as a device address (it denotes a
// host-side shadow), so the first call on each device, with that device
// current, looks up the real address with cudaGetSymbolAddress and caches it
// together with the identity of the device's current CUDA context
// (cuCtxGetId).  A later call that finds another context on the device -- the
// caller ran cudaDeviceReset, or the primary context was released and created
// again, which reloads the module at a new address -- looks the address up
// again instead of using a stale one.  Make the first call on a device before
// any stream capture there: it may load this library's device code.
//
// The call selects `device` for its own work and restores the caller's
// current device before it returns, on every path.
#include "hprqp_b200.h"
#include "rowblock.cuh"

#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

namespace hpr_noalloc {

constexpr size_t kNoAllocDoubles = size_t(1) << 20;  // 8 MiB of scratch per device
constexpr int kT = 256;
constexpr int kMaxBlocks = 1024;
constexpr size_t kPartSlots = 2 * kMaxBlocks + 2;  // partials, then two result slots
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocDoubles];

struct ScratchSlot {
    double *addr;
    unsigned long long ctx_id;  // cuCtxGetId of the context the address belongs to
    bool has_id;
};
static ScratchSlot g_scratch_slot[kMaxDevices];
static std::mutex g_scratch_mutex;

static __global__ void k_probe(double *z, int len)
{
    for (int i = blockIdx.x * kT + threadIdx.x; i < len; i += gridDim.x * kT)
        z[i] = 1.0 + ((double)i + 1.0) / ((double)len + 1.0);
}

// per-CTA partial of sum(a[i] * b[i]) (and of sum(b[i]^2) when two slots)
__device__ __forceinline__ void store_partials(double s0, double s1, double *part, int two)
{
    __shared__ double w0[kT / 32], w1[kT / 32];
    s0 = hpr::warp_sum(s0);
    s1 = hpr::warp_sum(s1);
    if ((threadIdx.x & 31) == 0) {
        w0[threadIdx.x >> 5] = s0;
        w1[threadIdx.x >> 5] = s1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int w = 0; w < kT / 32; ++w) {
            t0 += w0[w];
            t1 += w1[w];
        }
        part[blockIdx.x] = t0;
        if (two) part[kMaxBlocks + blockIdx.x] = t1;
    }
}

static __global__ void k_sumsq(const double *v, int len, double *part)
{
    double s = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < len; i += gridDim.x * kT) s += v[i] * v[i];
    store_partials(s, 0.0, part, 0);
}

// fold the partials in block order; out[0] (and out[1]) on the device
static __global__ void k_fold(const double *part, int nb, int two, double *out)
{
    if (threadIdx.x == 0) {
        double t0 = 0.0, t1 = 0.0;
        for (int b = 0; b < nb; ++b) {
            t0 += part[b];
            if (two) t1 += part[kMaxBlocks + b];
        }
        out[0] = t0;
        if (two) out[1] = t1;
    }
}

static __global__ void k_scale(double *q, const double *z, int len, double inv)
{
    for (int i = blockIdx.x * kT + threadIdx.x; i < len; i += gridDim.x * kT) q[i] = z[i] * inv;
}

// y = M x, one warp per 32-row tile with a lane-group width chosen from the
// tile's mean row length; when `part` is set, also the per-CTA partials of
// q.y and y.y
static __global__ void k_spmv(const int *rp, const int *ci, const double *v, int nrow, const double *x, double *y,
                       const double *q, double *part)
{
    const int lane = threadIdx.x & 31;
    const int warps = gridDim.x * (kT / 32);
    double s_qy = 0.0, s_yy = 0.0;
    for (int t = blockIdx.x * (kT / 32) + (threadIdx.x >> 5); t * 32 < nrow; t += warps) {
        const int r0 = t * 32, nr = min(32, nrow - r0);
        const int nnz = rp[r0 + nr] - rp[r0];
        int G = 1;
        while (G < 32 && 8 * G <= nnz / nr) G *= 2;
        const int rpp = 32 / G, gl = lane & (G - 1), grp = lane / G;
        const int passes = (nr + rpp - 1) / rpp;
        double mine = 0.0;
        for (int p = 0; p < passes; ++p) {
            const int rr = p * rpp + grp;
            double s = 0.0;
            if (rr < nr) {
                for (int k = rp[r0 + rr] + gl; k < rp[r0 + rr + 1]; k += G) s = fma(v[k], x[ci[k]], s);
            }
            for (int o = G >> 1; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            const double val = __shfl_sync(0xffffffffu, s, (lane % rpp) * G);
            if (lane / rpp == p) mine = val;
        }
        if (lane < nr) {
            y[r0 + lane] = mine;
            if (part) {
                s_qy += q[r0 + lane] * mine;
                s_yy += mine * mine;
            }
        }
    }
    if (part) store_partials(s_qy, s_yy, part, 1);
}

static __global__ void k_resid(double *q, const double *z, int len, double lambda, double *part)
{
    double s = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < len; i += gridDim.x * kT) {
        const double r = z[i] - lambda * q[i];
        q[i] = r;
        s += r * r;
    }
    store_partials(s, 0.0, part, 0);
}

static int grid_for(long long work)
{
    long long g = (work + kT - 1) / kT;
    return (int)(g < 1 ? 1 : (g > kMaxBlocks ? kMaxBlocks : g));
}

// Identity of the current context (cuCtxGetId, reached through the runtime's
// driver entry points so the library links only cudart); false when the
// driver does not offer it.
static bool current_context_id(unsigned long long *id)
{
    using GetCurrentFn = CUresult (*)(CUcontext *);
    using GetIdFn = CUresult (*)(CUcontext, unsigned long long *);
    static GetCurrentFn get_current = nullptr;
    static GetIdFn get_id = nullptr;
    static bool looked_up = false;
    if (!looked_up) {
        void *f0 = nullptr, *f1 = nullptr;
        cudaDriverEntryPointQueryResult q0, q1;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f0, cudaEnableDefault, &q0) == cudaSuccess &&
            q0 == cudaDriverEntryPointSuccess && cudaGetDriverEntryPoint("cuCtxGetId", &f1, cudaEnableDefault, &q1) ==
                                                     cudaSuccess && q1 == cudaDriverEntryPointSuccess) {
            get_current = (GetCurrentFn)f0;
            get_id = (GetIdFn)f1;
        }
        cudaGetLastError();  // a missing entry point is not an error of this call
        looked_up = true;
    }
    if (!get_current || !get_id) return false;
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr) return false;
    return get_id(ctx, id) == CUDA_SUCCESS;
}

// Address of the scratch array on `device`, which must be current: looked up
// on the first call in each context of the device and cached with that
// context's id.  Without context ids (an old driver) it is looked up on
// every call.
static HPRQPStatus scratch_for(int device, double **out)
{
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    ScratchSlot &slot = g_scratch_slot[device];
    unsigned long long id = 0;
    const bool has_id = current_context_id(&id);
    if (!slot.addr || !has_id || !slot.has_id || slot.ctx_id != id) {
        double *ptr = nullptr;
        const cudaError_t err = cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch);
        if (err != cudaSuccess || ptr == nullptr) {
            fprintf(stderr, "hprqp-b200: cudaGetSymbolAddress of the no-allocation scratch failed: %s\n",
                    cudaGetErrorString(err));
            return HPRQP_STATUS_NOT_IMPLEMENTED;
        }
        slot.addr = ptr;
        slot.ctx_id = id;
        slot.has_id = has_id;
    }
    *out = slot.addr;
    return HPRQP_STATUS_OK;
}

// Makes `device` current for the duration of a call and gives the caller's
// current device back on every return path.
class DeviceGuard {
public:
    DeviceGuard() { ok_ = cudaGetDevice(&saved_) == cudaSuccess; }
    ~DeviceGuard()
    {
        if (ok_) cudaSetDevice(saved_);
    }
    DeviceGuard(const DeviceGuard &) = delete;
    DeviceGuard &operator=(const DeviceGuard &) = delete;

private:
    int saved_ = 0;
    bool ok_ = false;
};

#define NA_CK(call)                                                                                   \
    do {                                                                                              \
        cudaError_t err__ = (call);                                                                   \
        if (err__ != cudaSuccess) {                                                                   \
            fprintf(stderr, "hprqp-b200: CUDA error %s at %s:%d\n", cudaGetErrorString(err__), __FILE__, \
                    __LINE__);                                                                        \
            return HPRQP_STATUS_NOT_IMPLEMENTED;                                                      \
        }                                                                                             \
    } while (0)

static HPRQPStatus fetch(const double *dev, double *host, int count, cudaStream_t stream)
{
    NA_CK(cudaMemcpyAsync(host, dev, count * sizeof(double), cudaMemcpyDeviceToHost, stream));
    NA_CK(cudaStreamSynchronize(stream));
    return HPRQP_STATUS_OK;
}

static HPRQPStatus power_lambda(int device, size_t m, size_t n, const int *a_rp, const int *a_ci,
                                const double *a_v, const int *at_rp, const int *at_ci, const double *at_v,
                                void *stream_handle, double *lambda_out, int *iterations_out)
{
    if (!lambda_out || (m > 0 && (!a_rp || !a_ci || !a_v || !at_rp || !at_ci || !at_v)))
        return HPRQP_STATUS_INVALID_ARGUMENT;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess) {
        cudaGetLastError();
        fprintf(stderr, "hprqp-b200: no CUDA device available; this engine has no CPU fallback\n");
        return HPRQP_STATUS_NOT_IMPLEMENTED;
    }
    if (device < 0 || device >= ndev || device >= kMaxDevices) {
        fprintf(stderr, "hprqp-b200: hprqp_b200_power_lambda_noalloc: device %d does not exist (%d visible)\n",
                device, ndev);
        return HPRQP_STATUS_INVALID_ARGUMENT;
    }
    if (m > (size_t)INT32_MAX || n > (size_t)INT32_MAX || 2 * m + n > kNoAllocDoubles - kPartSlots) {
        fprintf(stderr,
                "hprqp-b200: hprqp_b200_power_lambda_noalloc: 2*m + n = %zu exceeds the fixed scratch of %zu "
                "doubles (use the allocating setup path for larger problems)\n",
                2 * m + n, kNoAllocDoubles - kPartSlots);
        return HPRQP_STATUS_INVALID_ARGUMENT;
    }
    *lambda_out = 0.0;
    if (iterations_out) *iterations_out = 0;
    if (m == 0) return HPRQP_STATUS_OK;
    DeviceGuard restore_device;
    NA_CK(cudaSetDevice(device));
    double *base = nullptr;
    HPRQPStatus st = scratch_for(device, &base);
    if (st != HPRQP_STATUS_OK) return st;
    cudaStream_t s = (cudaStream_t)stream_handle;
    const int mi = (int)m, ni = (int)n;
    double *z = base, *q = base + m, *t = base + 2 * m, *part = base + 2 * m + n;
    double *out = part + 2 * kMaxBlocks;
    const int gm = grid_for(mi);
    // one warp per 32-row tile, eight tiles per CTA
    const int g_at = grid_for(((long long)ni + 31) / 32 * 32);
    const int g_a = grid_for(((long long)mi + 31) / 32 * 32);
    double h[2] = {0.0, 0.0};
    k_probe<<<gm, kT, 0, s>>>(z, mi);
    k_sumsq<<<gm, kT, 0, s>>>(z, mi, part);
    k_fold<<<1, 32, 0, s>>>(part, gm, 0, out);
    if ((st = fetch(out, h, 1, s))) return st;
    double zz = h[0], lambda = 1.0;
    int it = 0;
    for (; it < 5000; ++it) {
        const double qn = sqrt(zz);
        if (qn <= 1e-16) {
            lambda = 0.0;
            break;
        }
        k_scale<<<gm, kT, 0, s>>>(q, z, mi, 1.0 / qn);
        k_spmv<<<g_at, kT, 0, s>>>(at_rp, at_ci, at_v, ni, q, t, nullptr, nullptr);
        k_spmv<<<g_a, kT, 0, s>>>(a_rp, a_ci, a_v, mi, t, z, q, part);
        k_fold<<<1, 32, 0, s>>>(part, g_a, 1, out);
        if ((st = fetch(out, h, 2, s))) return st;
        lambda = h[0];
        zz = h[1];
        const double zn = sqrt(zz);
        k_resid<<<gm, kT, 0, s>>>(q, z, mi, lambda, part);
        k_fold<<<1, 32, 0, s>>>(part, gm, 0, out);
        if ((st = fetch(out, h, 1, s))) return st;
        if (sqrt(h[0]) / (zn + fabs(lambda) + 1e-16) < 1e-4) {
            ++it;
            break;
        }
    }
    NA_CK(cudaGetLastError());
    *lambda_out = (lambda < 0.0 ? 0.0 : lambda) * 1.05;
    if (iterations_out) *iterations_out = it;
    return HPRQP_STATUS_OK;
}

}  // namespace hpr_noalloc

extern "C" HPRQPStatus hprqp_b200_power_lambda_noalloc(int device, size_t m, size_t n, const int *a_row_ptr,
                                                       const int *a_col, const double *a_val, const int *at_row_ptr,
                                                       const int *at_col, const double *at_val, void *stream,
                                                       double *lambda_out, int *iterations_out)
{
    return hpr_noalloc::power_lambda(device, m, n, a_row_ptr, a_col, a_val, at_row_ptr, at_col, at_val, stream,
                                     lambda_out, iterations_out);
}
