// lbm_residual_device: the relative velocity-change residual of erranalysis
// (solution.f90:74-122) on velocity fields that the caller keeps in its own
// device memory, computed without allocating any memory.
//
// Why a separate entry point: lbm_residual works on a handle, and a handle
// owns device buffers it allocated itself. A driver that keeps u, v on the
// GPU on its own (an OpenACC or CUDA Fortran code, as the reference's own
// erranalysis runs on OpenACC device arrays) may be unable to let a library
// allocate: its arrays can take the whole device memory for the largest
// meshes, and cudaMalloc/cudaFree on every call would synchronise the device
// and stall the driver's asynchronous queues. This entry point therefore
// uses one fixed scratch array in device global memory, declared below, and
// no allocation of any kind (device or host).
//
// Scratch: per interior row, the two partial sums (sum of |u - u0|^2, sum of
// |u|^2), a completion counter and the two totals; at most
// LBM_RESIDUAL_MAX_ROWS interior rows (ny - 2), i.e. 256 KiB. Larger ny is
// rejected with LBM_ERR_SIZE before anything is launched.
//
// Set-up: the first call in each CUDA context looks up the scratch's device
// address (cudaGetSymbolAddress) and keeps it for that context. A context is
// the device's primary context that the runtime makes current (one per
// device), or a context the caller created and made current itself, as a
// CUDA Fortran or OpenACC runtime may; each context holds its own copy of the
// scratch at its own address, so the cache is keyed by the context's unique
// ID (cuCtxGetId), which also tells a context re-created after
// cudaDeviceReset from the one it replaces. The first call in a context
// should come before any stream capture in it. Every call then clears the
// completion counter on the caller's stream, launches one kernel and copies
// the two totals back to host memory, so each call waits for its stream.
//
// There is one scratch array per device, shared by every caller: two calls
// whose work overlaps on the GPU (different streams, or different host
// threads on the same device) race on it and may return wrong values. Callers
// must serialise them.
#include <cuda.h>   // CUcontext and CUresult; the two driver calls are looked up at run time
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "lbm_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxContexts = 64;   // contexts whose scratch address is kept
constexpr int kRows = LBM_RESIDUAL_MAX_ROWS;
// layout of the scratch (doubles): [0, 2*kRows) row partials,
// [2*kRows] completion counter (as unsigned), [2*kRows + 2, +4) totals
constexpr int kCounter = 2 * kRows;
constexpr int kTotals = 2 * kRows + 2;
constexpr int kScratchDoubles = 2 * kRows + 4;

static __device__ __align__(256) double lbm_residual_scratch[kScratchDoubles];

std::mutex g_setup_mutex;
struct ScratchAddress {
    unsigned long long ctx_id;   // 0: unused
    double *ptr;
};
ScratchAddress g_scratch[kMaxContexts] = {};
int g_scratch_next = 0;   // entry replaced next when all are in use
using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);
CtxGetCurrentFn g_ctx_current = nullptr;
CtxGetIdFn g_ctx_id = nullptr;

// deterministic sum of one value per thread over the block (fixed tree)
__device__ __forceinline__ void block_sum2(double &a, double &b, double *sh)
{
    for (int off = 16; off; off >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, off);
        b += __shfl_down_sync(0xffffffffu, b, off);
    }
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { sh[2 * wid] = a; sh[2 * wid + 1] = b; }
    __syncthreads();
    if (threadIdx.x == 0) {
        a = b = 0;
        for (int w = 0; w < kThreads / 32; ++w) { a += sh[2 * w]; b += sh[2 * w + 1]; }
    }
}

// one block per interior row j (1..ny-2, 0-based), interior columns 1..nx-2;
// the last block to finish sums the row partials in row order
template <typename C>
__global__ void __launch_bounds__(kThreads) residual_rows(const C *__restrict__ u, const C *__restrict__ v,
                                                          const C *__restrict__ u0, const C *__restrict__ v0,
                                                          int nx, double *scratch)
{
    __shared__ double sh[2 * (kThreads / 32)];
    __shared__ bool last;
    const int r = blockIdx.x;
    const long long base = (long long)(r + 1) * nx;
    double s1 = 0, s2 = 0;
    for (int i = 1 + threadIdx.x; i <= nx - 2; i += kThreads) {
        const double a = (double)u[base + i], b = (double)v[base + i];
        const double da = a - (double)u0[base + i], db = b - (double)v0[base + i];
        s1 += da * da + db * db;
        s2 += a * a + b * b;
    }
    block_sum2(s1, s2, sh);
    unsigned *counter = reinterpret_cast<unsigned *>(scratch + kCounter);
    if (threadIdx.x == 0) {
        scratch[2 * r] = s1;
        scratch[2 * r + 1] = s2;
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t1 = 0, t2 = 0;
    for (int q = threadIdx.x; q < (int)gridDim.x; q += kThreads) {
        t1 += __ldcg(scratch + 2 * q);
        t2 += __ldcg(scratch + 2 * q + 1);
    }
    __syncthreads();   // sh is reused
    block_sum2(t1, t2, sh);
    if (threadIdx.x == 0) {
        scratch[kTotals] = t1;
        scratch[kTotals + 1] = t2;
        *counter = 0u;
    }
}

// unique ID of the CUDA context current on this thread; when none is current
// yet, the current device's primary context is made current first (as the
// runtime's own first call on a thread would). 0 on failure.
unsigned long long current_context_id()
{
    if (!g_ctx_current || !g_ctx_id) {
        void *f1 = nullptr, *f2 = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, nullptr) != cudaSuccess || !f1 ||
            cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, nullptr) != cudaSuccess || !f2)
            return 0;
        g_ctx_current = reinterpret_cast<CtxGetCurrentFn>(f1);
        g_ctx_id = reinterpret_cast<CtxGetIdFn>(f2);
    }
    CUcontext ctx = nullptr;
    if (g_ctx_current(&ctx) != CUDA_SUCCESS) return 0;
    if (!ctx) {
        int dev = -1;
        if (cudaGetDevice(&dev) != cudaSuccess || cudaSetDevice(dev) != cudaSuccess) return 0;
        if (g_ctx_current(&ctx) != CUDA_SUCCESS || !ctx) return 0;
    }
    unsigned long long id = 0;
    if (g_ctx_id(ctx, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// scratch address in the current context, looked up on the first call there
int scratch_for_current_context(double **out)
{
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    const unsigned long long id = current_context_id();
    if (!id) return LBM_ERR_CUDA;
    for (const ScratchAddress &e : g_scratch)
        if (e.ctx_id == id) {
            *out = e.ptr;
            return LBM_OK;
        }
    void *p = nullptr;
    if (cudaGetSymbolAddress(&p, lbm_residual_scratch) != cudaSuccess || !p) return LBM_ERR_CUDA;
    g_scratch[g_scratch_next] = ScratchAddress{id, static_cast<double *>(p)};
    g_scratch_next = (g_scratch_next + 1) % kMaxContexts;
    *out = static_cast<double *>(p);
    return LBM_OK;
}

}  // namespace

extern "C" LBM_API int lbm_residual_device(const void *u, const void *v, const void *u0, const void *v0,
                                           int nx, int ny, int precision, void *stream, double *err)
{
    if (!u || !v || !u0 || !v0 || !err || nx < 3 || ny < 3) return LBM_ERR_ARG;
    if (precision != LBM_PREC_FP32 && precision != LBM_PREC_FP64) return LBM_ERR_ARG;
    if (ny - 2 > LBM_RESIDUAL_MAX_ROWS) return LBM_ERR_SIZE;
    double *scratch = nullptr;
    const int st = scratch_for_current_context(&scratch);
    if (st != LBM_OK) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (cudaMemsetAsync(scratch + kCounter, 0, sizeof(unsigned), s) != cudaSuccess) return LBM_ERR_CUDA;
    const int rows = ny - 2;
    if (precision == LBM_PREC_FP64)
        residual_rows<double><<<rows, kThreads, 0, s>>>((const double *)u, (const double *)v, (const double *)u0,
                                                       (const double *)v0, nx, scratch);
    else
        residual_rows<float><<<rows, kThreads, 0, s>>>((const float *)u, (const float *)v, (const float *)u0,
                                                      (const float *)v0, nx, scratch);
    if (cudaGetLastError() != cudaSuccess) return LBM_ERR_CUDA;
    double tot[2];
    if (cudaMemcpyAsync(tot, scratch + kTotals, sizeof tot, cudaMemcpyDeviceToHost, s) != cudaSuccess)
        return LBM_ERR_CUDA;
    if (cudaStreamSynchronize(s) != cudaSuccess) return LBM_ERR_CUDA;
    *err = std::sqrt(tot[0]) / (std::sqrt(tot[1]) + 1e-30);   // solution.f90:117-121
    return LBM_OK;
}
