// host_xfer.cu -- host<->device copies of the ABI's FP64 host arrays through
// a small pinned staging ring, with the host-side work (copying into and out
// of the caller's pageable arrays, widening FP32 fields to FP64) spread over
// a pool of host threads and overlapped with the DMA of the next chunk.
//
// Why: a cudaMemcpy from or to pageable memory goes through the driver's own
// staging at a fraction of the link's bandwidth, and the FP32 fields of the
// usual storage precision were copied plane by plane and widened on one
// thread. The reference moves its arrays with `!$acc update host/device`
// (main.f90:253, 408, 414), which has the same pageable-copy cost.
//
// The ring (two buffers of kChunk bytes, cudaHostAlloc'd once per process on
// first use and kept until exit) is shared by every handle: transfers take
// it in turn under a mutex.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "lbm_internal.h"

namespace {

// bytes per staging buffer, and per chunk of a device-to-host copy; uploads
// go in chunks of half a buffer: on a B200 host, reading 100 MB back (and
// widening it) took 6.5-7.3 ms in 16 MB chunks against 8.4-9.4 ms in 8 MB
// ones, while uploading 134 MB took 5.2-5.6 ms in 8 MB chunks against
// 6.8-7.8 ms in 16 MB ones (more chunks keep the host copies and the DMA
// overlapped)
constexpr size_t kChunk = 16u << 20;
constexpr size_t kChunkH2D = kChunk / 2;

// A fixed pool of host threads: run(parts, f) calls f(p) for p = 0..parts-1
// on the workers and the calling thread, and returns when all are done. A
// job lives on the caller's stack; run() returns only once no worker holds
// it any more.
class WorkPool {
  public:
    static WorkPool &get()
    {
        static WorkPool *pool = new WorkPool;   // never destroyed: its threads live until exit
        return *pool;
    }
    void run(int parts, const std::function<void(int)> &f)
    {
        if (parts <= 1 || workers_ == 0) {
            for (int p = 0; p < parts; ++p) f(p);
            return;
        }
        std::lock_guard<std::mutex> call(call_mu_);   // one job at a time
        Job job;
        job.f = &f;
        job.parts = parts;
        job.pending = parts;
        {
            std::lock_guard<std::mutex> lk(mu_);
            cur_ = &job;
            ++gen_;
            posted_.store(gen_, std::memory_order_release);
        }
        cv_.notify_all();
        work(job);
        std::unique_lock<std::mutex> lk(mu_);
        done_cv_.wait(lk, [&] { return job.pending == 0 && job.users == 0; });
        cur_ = nullptr;
    }
    int threads() const { return workers_ + 1; }

  private:
    struct Job {
        const std::function<void(int)> *f = nullptr;
        int parts = 0;
        std::atomic<int> next{0};
        int pending = 0;   // parts not finished (under mu_)
        int users = 0;     // workers inside work() on this job (under mu_)
    };
    WorkPool()
    {
        const unsigned hw = std::thread::hardware_concurrency();
        workers_ = (int)std::min(hw > 1 ? hw - 1 : 0u, 15u);
        for (int t = 0; t < workers_; ++t) std::thread([this] { loop(); }).detach();
    }
    void work(Job &j)
    {
        for (;;) {
            const int p = j.next.fetch_add(1);
            if (p >= j.parts) return;
            (*j.f)(p);
            std::lock_guard<std::mutex> lk(mu_);
            if (--j.pending == 0) done_cv_.notify_all();
        }
    }
    void loop()
    {
        long long seen = 0;
        for (;;) {
            Job *j;
            // A transfer posts one job per staging chunk, a fraction of a
            // millisecond apart: a worker that sleeps on the condition
            // variable between them wakes too late to take a part, and the
            // calling thread copies most of the chunk alone (measured: a
            // 67 MB upload 3-4x slower than with workers that stay awake).
            // So a worker first watches for the next job for up to
            // kSpinMicros, then sleeps.
            const auto t0 = std::chrono::steady_clock::now();
            for (int i = 0; posted_.load(std::memory_order_acquire) == seen; ++i) {
                if ((i & 255) == 255 &&
                    std::chrono::steady_clock::now() - t0 > std::chrono::microseconds(kSpinMicros))
                    break;
            }
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return gen_ != seen && cur_ != nullptr; });
                seen = gen_;
                j = cur_;
                ++j->users;
            }
            work(*j);
            std::lock_guard<std::mutex> lk(mu_);
            if (--j->users == 0 && j->pending == 0) done_cv_.notify_all();
        }
    }
    static constexpr int kSpinMicros = 300;
    int workers_ = 0;
    std::atomic<long long> posted_{0};   // gen_ as last posted, read without the lock
    std::mutex call_mu_, mu_;
    std::condition_variable cv_, done_cv_;
    Job *cur_ = nullptr;
    long long gen_ = 0;
};

// the process's pinned staging ring
std::mutex g_ring_mu;
void *g_ring[2] = {nullptr, nullptr};

cudaError_t ring_buffers(void **b)
{
    for (int i = 0; i < 2; ++i) {
        if (!g_ring[i]) {
            const cudaError_t e = cudaHostAlloc(&g_ring[i], kChunk, cudaHostAllocPortable);
            if (e != cudaSuccess) {
                g_ring[i] = nullptr;
                return e;
            }
        }
        b[i] = g_ring[i];
    }
    return cudaSuccess;
}

// dst[0..n) = src[0..n) as 8-byte words: a plain loop, which the compiler
// vectorises (in the thread pool on a B200 host it staged 67 MB in 2.1 ms,
// where the C library's memcpy in the same place took 6.3 ms)
inline void copy_words(uint64_t *__restrict__ dst, const uint64_t *__restrict__ src, size_t n)
{
    for (size_t i = 0; i < n; ++i) dst[i] = src[i];
}

// the element range [0, n) in `parts` nearly equal slices
inline void slice(size_t n, int parts, int p, size_t &a, size_t &b)
{
    a = n * (size_t)p / (size_t)parts;
    b = n * (size_t)(p + 1) / (size_t)parts;
}

struct Events {
    cudaEvent_t e[2] = {nullptr, nullptr};
    cudaError_t make()
    {
        for (auto &x : e) {
            const cudaError_t r = cudaEventCreateWithFlags(&x, cudaEventDisableTiming);
            if (r != cudaSuccess) return r;
        }
        return cudaSuccess;
    }
    ~Events()
    {
        for (auto &x : e)
            if (x) cudaEventDestroy(x);
    }
};

// Device -> host through the ring: chunk c of `src_bytes_total` bytes lands in
// ring buffer c & 1, and `consume(buf, first_byte, bytes)` moves it on from
// there on the host while the next chunk is in flight.
cudaError_t d2h_staged(const void *src, size_t total, size_t unit, cudaStream_t st,
                       const std::function<void(const void *, size_t, size_t)> &consume)
{
    if (total == 0) return cudaSuccess;
    std::lock_guard<std::mutex> lock(g_ring_mu);
    void *buf[2];
    cudaError_t e = ring_buffers(buf);
    if (e != cudaSuccess) return e;
    Events ev;
    if ((e = ev.make()) != cudaSuccess) return e;
    const size_t chunk = kChunk / unit * unit;
    const size_t n = (total + chunk - 1) / chunk;
    auto issue = [&](size_t c) -> cudaError_t {
        const size_t off = c * chunk, len = std::min(chunk, total - off);
        cudaError_t r = cudaMemcpyAsync(buf[c & 1], (const char *)src + off, len, cudaMemcpyDeviceToHost, st);
        if (r == cudaSuccess) r = cudaEventRecord(ev.e[c & 1], st);
        return r;
    };
    if ((e = issue(0)) != cudaSuccess) return e;
    for (size_t c = 0; c < n; ++c) {
        // the buffer of chunk c + 1 held chunk c - 1, consumed in the last pass
        if (c + 1 < n && (e = issue(c + 1)) != cudaSuccess) return e;
        if ((e = cudaEventSynchronize(ev.e[c & 1])) != cudaSuccess) return e;
        consume(buf[c & 1], c * chunk, std::min(chunk, total - c * chunk));
    }
    return cudaSuccess;
}

}  // namespace

// FP32 device array -> FP64 host array (n values)
cudaError_t xfer_d2h_widen(double *dst, const float *src, size_t n, cudaStream_t st)
{
    WorkPool &pool = WorkPool::get();
    return d2h_staged(src, n * sizeof(float), sizeof(float), st, [&](const void *b, size_t off, size_t len) {
        const float *s = (const float *)b;
        double *d = dst + off / sizeof(float);
        const size_t m = len / sizeof(float);
        const int parts = pool.threads();
        pool.run(parts, [&](int p) {
            size_t a, z;
            slice(m, parts, p, a, z);
            for (size_t i = a; i < z; ++i) d[i] = (double)s[i];
        });
    });
}

// device -> host copy of `bytes` bytes
cudaError_t xfer_d2h(void *dst, const void *src, size_t bytes, cudaStream_t st)
{
    WorkPool &pool = WorkPool::get();
    return d2h_staged(src, bytes, 8, st, [&](const void *b, size_t off, size_t len) {
        const int parts = pool.threads();
        pool.run(parts, [&](int p) {
            size_t a, z;
            slice(len / 8, parts, p, a, z);
            copy_words((uint64_t *)((char *)dst + off) + a, (const uint64_t *)b + a, z - a);
            if (p == parts - 1 && len % 8) memcpy((char *)dst + off + len / 8 * 8, (const char *)b + len / 8 * 8, len % 8);
        });
    });
}

// host -> device copy of `bytes` bytes; returns once the copies are queued
// and the ring is free again (its last DMAs done)
cudaError_t xfer_h2d(void *dst, const void *src, size_t bytes, cudaStream_t st)
{
    if (bytes == 0) return cudaSuccess;
    WorkPool &pool = WorkPool::get();
    std::lock_guard<std::mutex> lock(g_ring_mu);
    void *buf[2];
    cudaError_t e = ring_buffers(buf);
    if (e != cudaSuccess) return e;
    Events ev;
    if ((e = ev.make()) != cudaSuccess) return e;
    const size_t n = (bytes + kChunkH2D - 1) / kChunkH2D;
    for (size_t c = 0; c < n; ++c) {
        const size_t off = c * kChunkH2D, len = std::min(kChunkH2D, bytes - off);
        if (c >= 2 && (e = cudaEventSynchronize(ev.e[c & 1])) != cudaSuccess) return e;   // its last DMA
        char *b = (char *)buf[c & 1];
        const int parts = pool.threads();
        pool.run(parts, [&](int p) {
            size_t a, z;
            slice(len / 8, parts, p, a, z);
            copy_words((uint64_t *)b + a, (const uint64_t *)((const char *)src + off) + a, z - a);
            if (p == parts - 1 && len % 8) memcpy(b + len / 8 * 8, (const char *)src + off + len / 8 * 8, len % 8);
        });
        if ((e = cudaMemcpyAsync((char *)dst + off, b, len, cudaMemcpyHostToDevice, st)) != cudaSuccess) return e;
        if ((e = cudaEventRecord(ev.e[c & 1], st)) != cudaSuccess) return e;
    }
    for (size_t c = n > 2 ? n - 2 : 0; c < n; ++c)
        if ((e = cudaEventSynchronize(ev.e[c & 1])) != cudaSuccess) return e;
    return cudaSuccess;
}
