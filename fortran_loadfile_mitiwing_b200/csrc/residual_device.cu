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
// Set-up: the first call on each device, with that device current, looks up
// the scratch's device address (cudaGetSymbolAddress) and caches it per
// device. That first call should come before any stream capture on the
// device. Every call then clears the completion counter on the caller's
// stream, launches one kernel and copies the two totals back, synchronising
// that stream.
//
// There is one scratch array per device, shared by every caller: two calls
// whose work overlaps on the GPU (different streams, or different host
// threads on the same device) race on it and may return wrong values. Callers
// must serialise them.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "lbm_b200.h"

namespace {

constexpr int kThreads = 256;
constexpr int kMaxDevices = 64;
constexpr int kRows = LBM_RESIDUAL_MAX_ROWS;
// layout of the scratch (doubles): [0, 2*kRows) row partials,
// [2*kRows] completion counter (as unsigned), [2*kRows + 2, +4) totals
constexpr int kCounter = 2 * kRows;
constexpr int kTotals = 2 * kRows + 2;
constexpr int kScratchDoubles = 2 * kRows + 4;

static __device__ __align__(256) double lbm_residual_scratch[kScratchDoubles];

std::mutex g_setup_mutex;
double *g_scratch[kMaxDevices] = {};

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

// scratch address on the current device, looked up on the first call there
int scratch_for_current_device(double **out)
{
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return LBM_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch[dev]) {
        void *p = nullptr;
        if (cudaGetSymbolAddress(&p, lbm_residual_scratch) != cudaSuccess || !p) return LBM_ERR_CUDA;
        g_scratch[dev] = static_cast<double *>(p);
    }
    *out = g_scratch[dev];
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
    const int st = scratch_for_current_device(&scratch);
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
