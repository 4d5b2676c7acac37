// lbm_capi.cu -- the extern "C" boundary (include/lbm_b200.h): handle
// lifetime, device memory, initial state, and the per-step launch sequence.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "lbm_internal.h"

namespace {

const double kWref[9] = {4.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0, 1.0 / 9.0,
                         1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0, 1.0 / 36.0};
const int kEx[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
const int kEy[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
const int kRing = 2048;   // force rows kept on the device between host copies


int set_err(lbm_handle *h, int code, const char *msg)
{
    if (h) h->err = msg;
    return code;
}

int cuda_err(lbm_handle *h, cudaError_t e, const char *where)
{
    char buf[256];
    snprintf(buf, sizeof buf, "%s: %s", where, cudaGetErrorString(e));
    return set_err(h, LBM_ERR_CUDA, buf);
}

#define CK(call, where)                                   \
    do {                                                  \
        cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) return cuda_err(h, e_, where); \
    } while (0)

size_t compute_size(int prec) { return prec == LBM_PREC_FP64 ? sizeof(double) : sizeof(float); }

size_t storage_size(int prec)
{
    switch (prec) {
    case LBM_PREC_FP64: return 8;
    case LBM_PREC_FP32: return 4;
    default: return 2;
    }
}

// single-precision lattice weights of D2Q9model (D2Q9model.f90:24-32)
double wsingle(int k) { return k == 0 ? (double)(4.0f / 9.0f) : (k < 5 ? (double)(1.0f / 9.0f) : (double)(1.0f / 36.0f)); }

// D2Q9feq (D2Q9model.f90:35-46), host FP64
double feq(double rh, double u1, double v1, int k)
{
    const double eu = (double)kEx[k] * u1 + (double)kEy[k] * v1;
    const double utwo = u1 * u1 + v1 * v1;
    return wsingle(k) * rh * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * utwo);
}

// device allocations of the handles, owner and size (lbm_device_bytes)
std::mutex g_alloc_mu;
std::unordered_map<void *, std::pair<lbm_handle *, size_t>> g_allocs;

// The handles' device memory comes from one stream-ordered memory pool per
// device, owned by the library, that keeps what freed handles return
// (release threshold: never) for the next allocations: a handle created
// after another was destroyed, as a sweep or a serving loop does many times,
// reuses memory that is already mapped instead of mapping it again, and a
// free does not synchronise the device as cudaFree does. The pool holds the
// process's peak of live handle memory until the process exits.
cudaMemPool_t handle_pool(int dev)
{
    static std::mutex mu;
    static std::unordered_map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    auto it = pools.find(dev);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        pool = nullptr;   // plain cudaMalloc / cudaFree then
    } else {
        unsigned long long keep = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    pools[dev] = pool;
    return pool;
}

// allocations from the pool, by address (freed back to it)
std::unordered_map<void *, bool> g_pooled;

// Every allocation is zero-filled on the handle's stream, ahead of all work
// that uses it (the other streams are ordered after the main stream's
// position by events or a synchronisation), so that no kernel can see data a
// freed allocation of an earlier handle left in the same memory.
template <typename P> cudaError_t dmalloc(lbm_handle *h, P **p, size_t bytes)
{
    void *q = nullptr;
    cudaMemPool_t pool = h->stream ? handle_pool(h->dev) : nullptr;
    cudaError_t e = cudaErrorMemoryAllocation;
    if (pool && (e = cudaMallocFromPoolAsync(&q, bytes, pool, h->stream)) != cudaSuccess) {
        // a pool unusable here (a context other than the one it was made in,
        // or one reset since): a plain allocation
        cudaGetLastError();
        pool = nullptr;
    }
    if (!pool) e = cudaMalloc(&q, bytes);
    if (e != cudaSuccess) return e;
    e = h->stream ? cudaMemsetAsync(q, 0, bytes, h->stream) : cudaMemset(q, 0, bytes);
    if (e != cudaSuccess) {
        if (pool)
            cudaFreeAsync(q, h->stream);
        else
            cudaFree(q);
        return e;
    }
    if (pool) {
        std::lock_guard<std::mutex> lock(g_alloc_mu);
        g_pooled[q] = true;
    }
    *p = (P *)q;
    std::lock_guard<std::mutex> lock(g_alloc_mu);
    g_allocs[q] = {h, bytes};
    h->dev_bytes += (long long)bytes;
    return e;
}

// Callers first synchronise the streams of the handle that owns p (no queued
// work may still use it); a pooled allocation goes back to the pool on the
// owner's main stream, idle by then.
void free_dev(void *&p)
{
    if (p) {
        bool pooled = false;
        cudaStream_t st = nullptr;
        {
            std::lock_guard<std::mutex> lock(g_alloc_mu);
            auto it = g_allocs.find(p);
            if (it != g_allocs.end()) {
                it->second.first->dev_bytes -= (long long)it->second.second;
                st = it->second.first->stream;
                g_allocs.erase(it);
            }
            auto jt = g_pooled.find(p);
            if (jt != g_pooled.end()) {
                pooled = true;
                g_pooled.erase(jt);
            }
        }
        if (pooled)
            cudaFreeAsync(p, st);
        else
            cudaFree(p);
    }
    p = nullptr;
}
template <typename P> void free_devp(P *&p)
{
    void *q = (void *)p;
    free_dev(q);
    p = nullptr;
}

// waits for all of the handle's queued work (lattice, immersed-boundary,
// check and factorization streams): before its device buffers are rewritten
// or freed
void quiesce(lbm_handle *h)
{
    if (h->fstream) cudaStreamSynchronize(h->fstream);
    if (h->side) cudaStreamSynchronize(h->side);
    if (h->cstream) cudaStreamSynchronize(h->cstream);
    if (h->stream) cudaStreamSynchronize(h->stream);
}

// rows of the motion step table (mode.f90:176-269), host FP64
void lookup_row(const std::vector<double> &tab, int rows, int cols, double t, int &idx, double *row)
{
    auto T = [&](int r, int c) { return tab[(size_t)c * rows + r]; };
    if (t <= T(0, 0)) {
        idx = 0;
        for (int c = 0; c < cols; ++c) row[c] = T(0, c);
        row[0] = t;
        return;
    }
    if (t >= T(rows - 1, 0)) {
        idx = std::max(rows - 2, 0);
        for (int c = 0; c < cols; ++c) row[c] = T(rows - 1, c);
        row[0] = t;
        return;
    }
    int mi = std::max(0, std::min(idx, rows - 2));
    while (mi > 0 && t < T(mi, 0)) mi--;
    while (mi < rows - 2 && t > T(mi + 1, 0)) mi++;
    idx = mi;
    if (fabs(t - T(mi, 0)) <= 1.0e-12) {
        for (int c = 0; c < cols; ++c) row[c] = T(mi, c);
        row[0] = t;
        return;
    }
    if (fabs(t - T(mi + 1, 0)) <= 1.0e-12) {
        for (int c = 0; c < cols; ++c) row[c] = T(mi + 1, c);
        row[0] = t;
        return;
    }
    const double t1 = T(mi, 0), t2 = T(mi + 1, 0);
    if (fabs(t2 - t1) <= 1.0e-14) {
        for (int c = 0; c < cols; ++c) row[c] = T(mi, c);
        row[0] = t;
        return;
    }
    const double weight = (t - t1) / (t2 - t1);
    for (int c = 0; c < cols; ++c) row[c] = (1.0 - weight) * T(mi, c) + weight * T(mi + 1, c);
    row[0] = t;
}

// releases the immersed-boundary scratch (sizes depend on geometry and motion)
void free_ib(lbm_handle *h)
{
    if (h->fstream) cudaStreamSynchronize(h->fstream);
    if (h->side) cudaStreamSynchronize(h->side);
    if (h->cstream) cudaStreamSynchronize(h->cstream);
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->ib_ready = 0;
    h->batch_in_half[0] = h->batch_in_half[1] = -1;
    free_devp(h->d_mk); free_devp(h->d_rhs); free_devp(h->d_B); free_devp(h->d_y); free_devp(h->d_partial);
    free_devp(h->d_bD); free_devp(h->d_bL); free_devp(h->d_gf); free_devp(h->d_fmode); free_devp(h->d_fstatus); free_devp(h->d_tiles); free_devp(h->d_nsup); free_devp(h->d_ctile);
    free_devp(h->d_perm); free_devp(h->d_key); free_devp(h->d_reach); free_devp(h->d_wmax);
}

// Allocates the immersed-boundary scratch once geometry and motion are known:
// the correction patch is sized by the largest per-step rectangle of the
// bodies' bounding discs over the whole motion table.
int ensure_ib(lbm_handle *h)
{
    if (h->ib_ready) return LBM_OK;
    int wmax = 0, hmax = 0;
    double gx0 = 1e300, gx1 = -1e300, gy0 = 1e300, gy1 = -1e300;   // motion envelope (lattice units)
    if (h->nseg > 0) {
        std::vector<double> R(h->nwing, 0.0);
        for (int w = 0; w < h->nwing; ++w)
            for (int p = 0; p < h->ppw; ++p) {
                const double x = h->hx0[w * h->ppw + p], y = h->hy0[w * h->ppw + p];
                R[w] = std::max(R[w], sqrt(x * x + y * y));
            }
        for (int s = 0; s < h->msteps; ++s) {
            double xlo = 1e300, xhi = -1e300, ylo = 1e300, yhi = -1e300;
            for (int w = 0; w < h->nwing; ++w) {
                const double sa = h->mstep_host[(size_t)s * h->mcols + 4 + 9 * w];
                const double sb = h->mstep_host[(size_t)s * h->mcols + 7 + 9 * w];
                const double cx = (sa + h->p.xc - h->p.ox) / h->p.scale, cy = (sb + h->p.yc - h->p.oy) / h->p.scale;
                const double r = R[w] / h->p.scale + 4.0;
                xlo = std::min(xlo, cx - r); xhi = std::max(xhi, cx + r);
                ylo = std::min(ylo, cy - r); yhi = std::max(yhi, cy + r);
            }
            wmax = std::max(wmax, (int)ceil(xhi - xlo) + 2);
            hmax = std::max(hmax, (int)ceil(yhi - ylo) + 2);
            gx0 = std::min(gx0, xlo); gx1 = std::max(gx1, xhi);
            gy0 = std::min(gy0, ylo); gy1 = std::max(gy1, yhi);
        }
        wmax = std::min(wmax, h->nx);
        hmax = std::min(hmax, h->ny);
    }
    h->patch_wmax = wmax;
    h->patch_hmax = hmax;
    // split rectangle: every support node of every step lies inside it (the
    // disc of radius R+4 lu around each pivot covers the marker boxes); x
    // bounds rounded out to multiples of 4, clipped to the interior
    h->env_x0 = h->env_y0 = h->env_w = h->env_h = 0;
    if (h->nseg > 0) {
        int x0 = std::max(4, ((int)floor(gx0) - 1) / 4 * 4), x1 = std::min(h->nx - 4, ((int)ceil(gx1) + 2 + 3) / 4 * 4);
        int y0 = std::max(1, (int)floor(gy0) - 1), y1 = std::min(h->ny - 1, (int)ceil(gy1) + 2);
        if (x1 > x0 && y1 > y0) { h->env_x0 = x0; h->env_y0 = y0; h->env_w = x1 - x0; h->env_h = y1 - y0; }
    }
    const int ns = std::max(1, h->nseg);
    const size_t S = (size_t)h->nslots, K = (size_t)h->fbatch;
    CK(dmalloc(h, &h->d_mk, S * sizeof(Marker) * ns), "alloc markers");
    // right-hand sides and solution: one pair per step parity
    CK(dmalloc(h, &h->d_rhs, sizeof(double) * 2 * 2 * ns), "alloc rhs");
    CK(dmalloc(h, &h->d_y, sizeof(double) * 2 * 2 * ns), "alloc y");
    CK(dmalloc(h, &h->d_B, S * sizeof(double) * (size_t)ns * ns), "alloc B");
    ib_factor_scratch(ns, &h->work_blocks, &h->gf_slot);
    CK(dmalloc(h, &h->d_bD, K * sizeof(double) * h->work_blocks), "alloc block D");
    CK(dmalloc(h, &h->d_bL, K * sizeof(double) * h->work_blocks), "alloc block L");
    CK(dmalloc(h, &h->d_gf, S * sizeof(double) * h->gf_slot), "alloc factor blocks");
    CK(dmalloc(h, &h->d_fmode, S * 2 * sizeof(int)), "alloc factor mode");
    CK(dmalloc(h, &h->d_fstatus, S * sizeof(unsigned)), "alloc factor status");
    CK(cudaMemsetAsync(h->d_fmode, 0, S * 2 * sizeof(int), h->stream), "clear factor mode");
    CK(cudaMemsetAsync(h->d_fstatus, 0, S * sizeof(unsigned), h->stream), "clear factor status");
    const int nblk = h->patch_gx() * h->patch_gy();
    // partials of the spread (per patch tile) and of the residual check (per 8 markers)
    // (one set per step parity)
    const size_t npart = std::max((size_t)ib_partials_per_block() * nblk, 2 * (size_t)((ns + 7) / 8));
    h->part_stride = npart;
    CK(dmalloc(h, &h->d_partial, sizeof(double) * 2 * npart), "alloc partials");
    h->tiles_slot = (size_t)ib_tile_ints() * nblk;
    CK(dmalloc(h, &h->d_tiles, S * sizeof(int) * h->tiles_slot), "alloc tile lists");
    CK(cudaMemsetAsync(h->d_tiles, 0, S * sizeof(int) * h->tiles_slot, h->stream), "clear tile lists");
    CK(dmalloc(h, &h->d_nsup, S * sizeof(int)), "alloc tile counts");
    CK(dmalloc(h, &h->d_ctile, S * sizeof(int) * (size_t)nblk), "alloc correction tiles");
    CK(cudaMemsetAsync(h->d_nsup, 0, S * sizeof(int), h->stream), "clear tile counts");
    // solve order of the markers: one rigid body keeps its markers sorted by
    // body-frame chordwise position for the whole run (two markers whose
    // support boxes overlap are less than 5*sqrt(2) lattice units apart in any
    // orientation); several bodies are sorted on the device every step
    CK(dmalloc(h, &h->d_perm, S * sizeof(int) * ns), "alloc perm");
    CK(dmalloc(h, &h->d_key, S * sizeof(double) * ns), "alloc key");
    CK(dmalloc(h, &h->d_reach, sizeof(double)), "alloc reach");
    CK(dmalloc(h, &h->d_wmax, K * sizeof(int)), "alloc wmax");
    CK(cudaMemsetAsync(h->d_wmax, 0, K * sizeof(int), h->stream), "clear wmax");
    h->static_order = h->nwing == 1;
    if (h->static_order) {
        std::vector<int> perm(h->nseg);
        std::vector<double> xk(h->nseg), key(h->nseg);
        for (int k = 0; k < h->nseg; ++k) {
            perm[k] = k;
            xk[k] = 0.5 * (h->hx0[k] + h->hx0[k + 1]);
        }
        std::stable_sort(perm.begin(), perm.end(), [&](int p1, int p2) { return xk[p1] < xk[p2]; });
        for (int q = 0; q < h->nseg; ++q) key[q] = xk[perm[q]];
        const double reach = 7.1 * h->p.scale;
        CK(cudaMemcpyAsync(h->d_perm, perm.data(), sizeof(int) * h->nseg, cudaMemcpyHostToDevice, h->stream), "copy perm");
        CK(cudaMemcpyAsync(h->d_key, key.data(), sizeof(double) * h->nseg, cudaMemcpyHostToDevice, h->stream), "copy key");
        CK(cudaMemcpyAsync(h->d_reach, &reach, sizeof(double), cudaMemcpyHostToDevice, h->stream), "copy reach");
        CK(cudaStreamSynchronize(h->stream), "sync order");
    }
    if (ib_configure(h) != 0) return set_err(h, LBM_ERR_CUDA, "ib_configure failed");
    h->ib_ready = 1;
    return LBM_OK;
}

}  // namespace

// The error code and message of a device status word (the LBM_ST_* bits the
// kernels set); LBM_OK and "" for 0. An index error is reported first: the
// kernel that saw it skipped the access, so the step's results are not valid.
int status_error(unsigned st, std::string &msg)
{
    msg.clear();
    if (!st) return LBM_OK;
    if (st & LBM_ST_INDEX_MASK) {
        static const struct {
            unsigned bit;
            const char *kernel;
        } names[] = {{LBM_ST_INDEX_INTERP, "ib_interp"},     {LBM_ST_INDEX_ASSEMBLE, "ib_assemble"},
                     {LBM_ST_INDEX_FACTOR, "ib_factor"},     {LBM_ST_INDEX_SOLVE, "ib_solve"},
                     {LBM_ST_INDEX_SCATTER, "ib_tile_scatter"}, {LBM_ST_INDEX_SORT, "ib_tile_sort"},
                     {LBM_ST_INDEX_TILE, "ib_tile_update"}, {LBM_ST_INDEX_FORCES, "ib_forces"},
                     {LBM_ST_INDEX_RESIDUAL, "ib_residual"}, {LBM_ST_INDEX_LATTICE, "kf_tma"}};
        msg = "device index out of range, access skipped in:";
        for (const auto &n : names)
            if (st & n.bit) msg += std::string(" ") + n.kernel;
        return LBM_ERR_INDEX;
    }
    if (st & LBM_ST_TIMEOUT) {
        msg = "a bounded wait for a shared-memory copy gave up";
        return LBM_ERR_CUDA;
    }
    if (st & LBM_ST_RANGE) {
        msg = "move_boundary: a marker support box reaches the three outermost node layers";
        return LBM_ERR_RANGE;
    }
    if (st & LBM_ST_OVERFLOW) {
        msg = "immersed boundary: correction patch overflow";
        return LBM_ERR_RANGE;
    }
    if (st & LBM_ST_SOLVER) {
        msg = "immersed boundary: D D^T not positive definite";
        return LBM_ERR_SOLVER;
    }
    if (st & LBM_ST_NONFINITE) {
        msg = "non-finite flow at the markers or force (the flow diverged)";
        return LBM_ERR_NONFINITE;
    }
    msg = "unknown device status";
    return LBM_ERR_CUDA;
}

namespace {

int check_status(lbm_handle *h)
{
    unsigned st = 0;
    CK(cudaMemcpyAsync(&st, h->d_status, sizeof st, cudaMemcpyDeviceToHost, h->stream), "read status");
    CK(cudaStreamSynchronize(h->stream), "step sync");
    if (!st) return LBM_OK;
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned), h->stream), "clear status");
    std::string msg;
    const int code = status_error(st, msg);
    return set_err(h, code, msg.c_str());
}

// Global mass check: queues the FP64 deviation sum of the current populations
// on stream st and its copy into *dsum (the caller synchronises st), then
// mass_result turns it into the mass and checks that it is finite.
int mass_launch(lbm_handle *h, cudaStream_t st, double *dsum)
{
    if (launch_mass(h, h->fbuf[h->cur], st)) return cuda_err(h, cudaGetLastError(), "launch mass");
    CK(cudaMemcpyAsync(dsum, h->d_mass + (mass_slots() - 1), sizeof(double), cudaMemcpyDeviceToHost, st), "copy mass");
    return LBM_OK;
}

int mass_result(lbm_handle *h, double dsum)
{
    const double m = (double)h->nx * (double)h->ny + dsum;   // sum_k w_k = 1 per node
    h->last_mass = m;
    h->last_mass_step = h->steps_done;
    if (!std::isfinite(m)) return set_err(h, LBM_ERR_NONFINITE, "mass check: non-finite populations (the flow diverged)");
    return LBM_OK;
}

// sums the event intervals of `count` step slots after the streams are idle:
// step time is the span from the first step's start to the last step's end
// (gaps between launches included); the lattice time is the sum of the
// lattice kernels' intervals; the IB time is measured on the stream it ran on
int collect_timing(lbm_handle *h, int count, bool split)
{
    if (count < 1) return LBM_OK;
    for (int s = 0; s < count && h->timing == LBM_TIMING_KERNELS; ++s) {
        float a = 0, b = 0, c = 0;
        CK(cudaEventElapsedTime(&a, h->ev[4 * s], h->ev[4 * s + 1]), "event time");
        CK(cudaEventElapsedTime(&b, h->ev[4 * s + 2], h->ev[4 * s + 3]), "event time");
        if (split) {
            CK(cudaEventElapsedTime(&c, h->ev_side[2 * s], h->ev_side[2 * s + 1]), "event time");
            h->t_kf += a + b;
            h->t_ib += c;
        } else {
            h->t_ib += a;
            h->t_kf += b;
        }
    }
    h->t_steps += count;
    float span = 0;
    CK(cudaEventElapsedTime(&span, h->ev[0], h->ev[4 * (count - 1) + 3]), "event time");
    h->t_step += span;
    return LBM_OK;
}

// The per-step sequence. Without a body, or with the split off: IB chain,
// then the fused lattice update, on the main stream. With the split: the IB
// flow chain runs on the side stream (after the previous step) and its force
// row and residual check on the check stream, while the main stream updates
// every node outside the step's correction tiles; the main stream's step
// ends once the side stream has updated the correction tiles.
int run_steps(lbm_handle *h, int nsteps, double *rows_out, int *done_out, bool fields_every)
{
    // the mass is checked at every copy of force rows of lbm_run (every
    // kRing steps and at the end of the call), and by lbm_step on every
    // kRing-th step
    auto mass_due = [&]() { return !fields_every || (h->n - 1) % kRing == 0; };
    if (!h->inited) return set_err(h, LBM_ERR_STATE, "step: lbm_init not called");
    for (int w = 0; w < h->nwing; ++w)
        if (!h->have_wing[w]) return set_err(h, LBM_ERR_STATE, "step: boundary of a wing not set");
    int rc = ensure_ib(h);
    if (rc) return rc;
    const bool split = h->overlap && h->nseg > 0 && h->env_w > 0 && h->env_h > 0;
    if (split) CK(cudaEventRecord(h->ev_inner, h->stream), "event");
    // Factorization of batch b (steps b*K .. b*K+K-1 that the motion table
    // reaches, into slot half b & 1). With the split it runs on the factor
    // stream once the half's previous user (the batch two back) is done;
    // otherwise in order on the main stream.
    const double dt_time = h->p.scale * h->p.uu;
    const int K = h->fbatch;
    // last step with time <= mend, plus one against rounding (factorizing a
    // step that is never run costs nothing but time)
    const int last_step = (int)std::floor((h->mend + 1.0e-12) / dt_time) + 2;
    auto factor_batch = [&](int b) -> int {
        const int half = b & 1;
        const int s0 = std::max(1, b * K), s1 = std::min(b * K + K - 1, last_step);
        h->batch_in_half[half] = b;
        if (h->nseg == 0 || s1 < s0) return LBM_OK;
        cudaStream_t st = split ? h->fstream : h->stream;
        // the half's previous users: the flow chains and checks of its steps
        // (ev_free) and the lattice kernels of those steps on the main stream,
        // which read the slots' patch rectangles and tile counts (ev_inner:
        // the main stream's last completed step)
        if (split) {
            CK(cudaStreamWaitEvent(h->fstream, h->ev_free[half], 0), "wait");
            CK(cudaStreamWaitEvent(h->fstream, h->ev_inner, 0), "wait");
        }
        if (launch_factor(h, s0, s1 - s0 + 1, st)) return cuda_err(h, cudaGetLastError(), "launch factor");
        if (split) CK(cudaEventRecord(h->ev_batch[half], h->fstream), "event");
        return LBM_OK;
    };
    int done = 0, pending = 0;
    rc = LBM_OK;
    for (int s = 0; s < nsteps; ++s) {
        const double time = (double)(h->n - 1) * dt_time;   // main.f90:352
        if (time > h->mend + 1.0e-12) { rc = LBM_DONE; break; }
        const int slot = pending, b = h->n / K, half = b & 1, q = h->n % h->nslots;
        h->pinfo_slot = q;
        const void *fin = h->fbuf[h->cur];
        void *fout = h->fbuf[h->cur ^ 1];
        void *fields = nullptr;
        const bool want = fields_every || s >= nsteps - 2;
        if (want) {
            const int fs = h->fields_slot ^ 1;
            fields = h->d_fields[fs];
            h->fields_slot = fs;
            h->fields_step[fs] = h->n;
        }
        // per-step events (LBM_TIMING_KERNELS); with LBM_TIMING_SPAN only the
        // first step's start and the last step's end of each chunk of steps
        cudaEvent_t *e = h->timing == LBM_TIMING_KERNELS ? &h->ev[4 * slot] : nullptr;
        if (h->timing == LBM_TIMING_SPAN && slot == 0) CK(cudaEventRecord(h->ev[0], h->stream), "event");
        // the solve-residual check: on the last step of each factorization
        // batch and on the last step of the call
        const bool check_res = (h->n + 1) % K == 0 || s == nsteps - 1;
        if (split) {
            // side stream: the immersed-boundary chain and the correction
            // tiles; main stream: every other node, concurrently
            if (h->batch_in_half[half] != b && (rc = factor_batch(b))) return rc;
            CK(cudaStreamWaitEvent(h->side, h->ev_inner, 0), "wait");
            CK(cudaStreamWaitEvent(h->side, h->ev_batch[half], 0), "wait");
            // this step's buffers of its parity were last read by the check
            // two steps back
            CK(cudaStreamWaitEvent(h->side, h->ev_check[h->n & 1], 0), "wait");
            if (e) CK(cudaEventRecord(h->ev_side[2 * slot], h->side), "event");
            cudaEvent_t ei = h->after_interp ? h->ev_interp : nullptr;
            if (launch_flow(h, fin, fout, fields, h->n, slot, q, h->side, ei)) return cuda_err(h, cudaGetLastError(), "launch ib");
            if (e) CK(cudaEventRecord(h->ev_side[2 * slot + 1], h->side), "event");
            CK(cudaEventRecord(h->ev_ib, h->side), "event");
            // the force row and the residual check on their own stream; the
            // slot half is free for the next factorization after them
            CK(cudaStreamWaitEvent(h->cstream, h->ev_ib, 0), "wait");
            if (launch_check(h, q, slot, check_res, h->cstream)) return cuda_err(h, cudaGetLastError(), "launch check");
            CK(cudaEventRecord(h->ev_check[h->n & 1], h->cstream), "event");
            CK(cudaEventRecord(h->ev_free[half], h->cstream), "event");
            // the next batch's factorization, overlapping this batch's steps
            if ((b + 1) * K <= last_step && h->batch_in_half[half ^ 1] != b + 1 && (rc = factor_batch(b + 1))) return rc;
            CK(cudaStreamWaitEvent(h->stream, h->ev_batch[half], 0), "wait");   // the step's correction tiles
            if (ei) CK(cudaStreamWaitEvent(h->stream, ei, 0), "wait");   // the solve starts first
            if (e) CK(cudaEventRecord(e[0], h->stream), "event");
            if (launch_kf(h, fin, fout, fields, KF_OUTER)) return cuda_err(h, cudaGetLastError(), "launch kf");
            if (e) CK(cudaEventRecord(e[1], h->stream), "event");
            CK(cudaStreamWaitEvent(h->stream, h->ev_ib, 0), "wait");
            if (e) {
                CK(cudaEventRecord(e[2], h->stream), "event");
                CK(cudaEventRecord(e[3], h->stream), "event");
            }
            CK(cudaEventRecord(h->ev_inner, h->stream), "event");   // the step is complete
        } else {
            if (e) CK(cudaEventRecord(e[0], h->stream), "event");
            if (h->batch_in_half[half] != b && (rc = factor_batch(b))) return rc;
            if (launch_flow(h, fin, fout, fields, h->n, slot, q, h->stream)) return cuda_err(h, cudaGetLastError(), "launch ib");
            if (launch_check(h, q, slot, check_res, h->stream)) return cuda_err(h, cudaGetLastError(), "launch check");
            if (e) {
                CK(cudaEventRecord(e[1], h->stream), "event");
                CK(cudaEventRecord(e[2], h->stream), "event");
            }
            if (launch_kf(h, fin, fout, fields, h->nseg > 0 ? KF_OUTER : KF_ALL)) return cuda_err(h, cudaGetLastError(), "launch kf");
            if (e) CK(cudaEventRecord(e[3], h->stream), "event");
        }
        h->cur ^= 1;
        h->n++;
        h->steps_done++;
        done++;
        pending++;
        if (pending == h->ring_cap || s == nsteps - 1) {
            if (split) {   // force rows and residual checks run on the check stream after the update
                CK(cudaEventRecord(h->ev_ib, h->side), "event");
                CK(cudaStreamWaitEvent(h->stream, h->ev_ib, 0), "wait");
                CK(cudaEventRecord(h->ev_cjoin, h->cstream), "event");
                CK(cudaStreamWaitEvent(h->stream, h->ev_cjoin, 0), "wait");
            }
            // the span ends with the chunk's last step; the row copy and the
            // mass check after it are per-call work, not per-step work
            if (h->timing == LBM_TIMING_SPAN) CK(cudaEventRecord(h->ev[4 * (pending - 1) + 3], h->stream), "event");
            if (rows_out)
                CK(cudaMemcpyAsync(rows_out + (size_t)(done - pending) * h->row_len, h->d_ring,
                                   sizeof(double) * h->row_len * pending, cudaMemcpyDeviceToHost, h->stream),
                   "copy force rows");
            double dsum = 0.0;
            const bool mass = mass_due();
            int st = mass ? mass_launch(h, h->stream, &dsum) : LBM_OK;
            if (st) return st;
            st = check_status(h);
            if (st) return st;
            if (mass && (st = mass_result(h, dsum))) return st;
            if (h->timing && (st = collect_timing(h, pending, split))) return st;
            pending = 0;
        }
    }
    if (pending) {
        if (split) {
            CK(cudaEventRecord(h->ev_ib, h->side), "event");
            CK(cudaStreamWaitEvent(h->stream, h->ev_ib, 0), "wait");
            CK(cudaEventRecord(h->ev_cjoin, h->cstream), "event");
            CK(cudaStreamWaitEvent(h->stream, h->ev_cjoin, 0), "wait");
        }
        if (h->timing == LBM_TIMING_SPAN) CK(cudaEventRecord(h->ev[4 * (pending - 1) + 3], h->stream), "event");
        if (rows_out)
            CK(cudaMemcpyAsync(rows_out + (size_t)(done - pending) * h->row_len, h->d_ring,
                               sizeof(double) * h->row_len * pending, cudaMemcpyDeviceToHost, h->stream),
               "copy force rows");
        double dsum = 0.0;
        const bool mass = mass_due();
        int st = mass ? mass_launch(h, h->stream, &dsum) : LBM_OK;
        if (st) return st;
        st = check_status(h);
        if (st) return st;
        if (mass && (st = mass_result(h, dsum))) return st;
        if (h->timing && (st = collect_timing(h, pending, split))) return st;
    }
    if (done_out) *done_out = done;
    return rc;
}

}  // namespace

// an empty kernel, compiled like every other kernel of the library: its
// attributes tell which architecture the library's device code is for
__global__ void arch_probe() {}

// for lbm_batch.cu
int handle_prepare_ib(lbm_handle *h) { return ensure_ib(h); }
int handle_mass_launch(lbm_handle *h, cudaStream_t st, double *dsum) { return mass_launch(h, st, dsum); }
int handle_mass_result(lbm_handle *h, double dsum) { return mass_result(h, dsum); }
int handle_error(lbm_handle *h, int code, const char *msg) { return set_err(h, code, msg); }
int handle_status(lbm_handle *h) { return check_status(h); }

// boundary reference values from the edge f0 (FP64, full f; left column,
// right column, bottom row, top row, 9 per node): the moments
// physical_variables takes on the edge columns (solution.f90:516-520) and the
// corner-column f0 populations the top/bottom extrapolation reads
// (boundary_condition.f90:705, 832)
int handle_set_edges(lbm_handle *h, const double *ef)
{
    const int nx = h->nx, ny = h->ny;
    std::vector<double> ec(6 * (size_t)ny + 36);
    for (int side = 0; side < 2; ++side) {
        for (int j = 0; j < ny; ++j) {
            const double *f = ef + 9 * ((size_t)side * ny + j);
            double temprho = 0.0, tempu = 0.0, tempv = 0.0;
            for (int k = 0; k < 9; ++k) {
                temprho = temprho + f[k];
                tempu = tempu + (double)kEx[k] * f[k];
                tempv = tempv + (double)kEy[k] * f[k];
            }
            double *o = ec.data() + (size_t)side * 3 * ny + 3 * (size_t)j;
            o[0] = temprho - 1.0;
            o[1] = tempu / temprho;
            o[2] = tempv / temprho;
        }
    }
    // (1,2), (1,Ny-1), (Nx,2), (Nx,Ny-1) as deviations from the weights
    const int cside[4] = {0, 0, 1, 1}, cj[4] = {1, ny - 2, 1, ny - 2};
    for (int c = 0; c < 4; ++c) {
        const double *f = ef + 9 * ((size_t)cside[c] * ny + cj[c]);
        for (int k = 0; k < 9; ++k) ec[6 * (size_t)ny + 9 * c + k] = f[k] - kWref[k];
    }
    if (compute_size(h->prec) == sizeof(double)) {
        CK(cudaMemcpyAsync(h->edge_c, ec.data(), sizeof(double) * ec.size(), cudaMemcpyHostToDevice, h->stream), "copy edge");
        CK(cudaStreamSynchronize(h->stream), "sync edge");
    } else {
        std::vector<float> ecf(ec.begin(), ec.end());
        CK(cudaMemcpyAsync(h->edge_c, ecf.data(), sizeof(float) * ecf.size(), cudaMemcpyHostToDevice, h->stream), "copy edge");
        CK(cudaStreamSynchronize(h->stream), "sync edge");
    }
    h->edge_f0.assign(ef, ef + 9 * (2 * (size_t)ny + 2 * (size_t)nx));
    return LBM_OK;
}

// readflowfield (solution.f90:1709-1839) on the device: f is packed into the
// storage precision, the field slot gets u and v with density 1 (init's
// rho0; the file has no density), the boundary values come from the edge f0,
// and the step counter continues after `cycle` (main.f90:321-323: n = cycle1
// + 1). The factorization slots are filled again for the restored step.
int handle_restore(lbm_handle *h, const double *f, const double *u, const double *v, const double *edge_f0, int cycle)
{
    quiesce(h);
    const size_t nn = (size_t)h->nx * h->ny;
    if (!h->d_stage) CK(dmalloc(h, &h->d_stage, sizeof(double) * nn * 9), "alloc stage");
    CK(cudaMemcpyAsync(h->d_stage, f, sizeof(double) * nn * 9, cudaMemcpyHostToDevice, h->stream), "copy f");
    if (launch_pack(h, h->d_stage, h->fbuf[0])) return cuda_err(h, cudaGetLastError(), "pack");
    CK(cudaStreamSynchronize(h->stream), "sync f");
    free_devp(h->d_stage);
    h->cur = 0;
    if (compute_size(h->prec) == sizeof(double)) {
        std::vector<double> fl(3 * nn);
        for (size_t q = 0; q < nn; ++q) {
            fl[q] = 1.0;
            fl[nn + q] = u[q];
            fl[2 * nn + q] = v[q];
        }
        CK(cudaMemcpyAsync(h->d_fields[0], fl.data(), sizeof(double) * fl.size(), cudaMemcpyHostToDevice, h->stream),
           "copy fields");
        CK(cudaStreamSynchronize(h->stream), "sync fields");
    } else {
        std::vector<float> fl(3 * nn);
        for (size_t q = 0; q < nn; ++q) {
            fl[q] = 1.0f;
            fl[nn + q] = (float)u[q];
            fl[2 * nn + q] = (float)v[q];
        }
        CK(cudaMemcpyAsync(h->d_fields[0], fl.data(), sizeof(float) * fl.size(), cudaMemcpyHostToDevice, h->stream),
           "copy fields");
        CK(cudaStreamSynchronize(h->stream), "sync fields");
    }
    const int rc = handle_set_edges(h, edge_f0);
    if (rc) return rc;
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned), h->stream), "clear status");
    CK(cudaMemsetAsync(h->d_pinfo, 0, LBM_NSLOT_MAX * sizeof(PatchInfo), h->stream), "clear pinfo");
    CK(cudaStreamSynchronize(h->stream), "sync restore");
    h->n = cycle + 1;
    h->steps_done = cycle;
    h->fields_slot = 0;
    h->fields_step[0] = cycle;
    h->fields_step[1] = -1;
    h->batch_in_half[0] = h->batch_in_half[1] = -1;
    h->fgroup[0] = h->fgroup[1] = -1;
    return LBM_OK;
}

extern "C" {

int lbm_default_params(lbm_params *p)
{
    if (!p) return LBM_ERR_ARG;
    memset(p, 0, sizeof *p);
    p->nx = 4001;                 // nint(40/0.01)+1 (ini_mesh.f90:22)
    p->ny = 2001;                 // nint(20/0.01)+1 (ini_mesh.f90:23)
    p->wing_count = 2;            // main.f90:18
    p->points_per_wing = 205;     // main.f90:21
    p->delta_kernel = LBM_DELTA_SMOOTH;   // boundary_condition.f90:1530
    p->precision = LBM_PREC_FP32;
    p->scale = 0.01;              // mesh_max_scale (main.f90:32)
    p->ox = -20.0;                // -0.5*width (ini_mesh.f90:36)
    p->oy = -10.0;
    p->uu = 0.01;                 // main.f90:12
    p->re = 500.0;                // main.f90:84
    const double s[9] = {0.0, 1.1, 1.05, 0.0, 1.2, 0.0, 1.2, 0.0, 0.0};   // ini_mesh.f90:59-67
    memcpy(p->s, s, sizeof s);
    p->mesh_max_scale = 0.01;
    return LBM_OK;
}

int lbm_create(const lbm_params *p, lbm_t **out)
{
    if (!p || !out) return LBM_ERR_ARG;
    *out = nullptr;
    if (p->nx < 16 || p->ny < 16 || p->wing_count < 0 || p->wing_count > LBM_MAXW ||
        (p->wing_count > 0 && p->points_per_wing < 3) || !(p->scale > 0) || !(p->uu > 0) || !(p->re > 0) ||
        p->precision < 0 || p->precision > 3 || p->delta_kernel < 0 || p->delta_kernel > 1 || (p->flags & ~LBM_FLAG_DENSE_SOLVE) != 0 ||
        (long long)p->wing_count * (p->points_per_wing - 1) > ib_max_markers())
        return LBM_ERR_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return LBM_ERR_CUDA;
    lbm_handle *h = new lbm_handle();
    h->p = *p;
    cudaGetDevice(&h->dev);
    h->nx = p->nx;
    h->ny = p->ny;
    h->pitch = (p->nx + 63) / 64 * 64;
    h->plane = (long long)h->pitch * p->ny;
    h->nwing = p->wing_count;
    h->ppw = h->nwing > 0 ? p->points_per_wing : 0;
    h->spw = h->ppw > 0 ? h->ppw - 1 : 0;
    h->npts = h->nwing * h->ppw;
    h->nseg = h->nwing * h->spw;
    h->niu = p->uu * (1.0 / p->scale) / p->re;   // ini_mesh.f90:30
    h->tau = 3.0 * h->niu + 0.5;                  // ini_mesh.f90:31
    for (int k = 0; k < 9; ++k) h->s[k] = p->s[k];
    if (p->s[7] <= 0) h->s[7] = 1.0 / h->tau;
    if (p->s[8] <= 0) h->s[8] = 1.0 / h->tau;
    h->prec = p->precision;
    h->elem = storage_size(h->prec);
    // nodes per thread of the lattice kernel; LBM_KF_VEC (1, 2 or 4) overrides
    // the default for tuning
    h->kf_vec = 1;
    if (const char *ev = getenv("LBM_KF_VEC")) {
        const int v = atoi(ev);
        if (v == 1 || v == 2 || v == 4) h->kf_vec = v;
    }
    if (const char *ev = getenv("LBM_KF_TMA")) h->kf_tma = atoi(ev) != 0;

    if (const char *ev = getenv("LBM_KF_ROWS")) {
        const int v = atoi(ev);
        if (v >= 1 && v <= 4096) h->kf_rows = v;
    }
    h->hx0.assign(std::max(1, h->npts), 0.0);
    h->hy0.assign(std::max(1, h->npts), 0.0);
    h->harc.assign(std::max(1, h->nseg), 0.0);
    h->have_wing.assign(LBM_MAXW, 0);
    h->row_len = 1 + 3 * h->nwing + 3 + 9 * h->nwing;
    h->ring_cap = kRing;
    auto fail = [&](cudaError_t e, const char *w) {
        lbm_destroy(h);
        (void)e; (void)w;
        return LBM_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    // the immersed-boundary flow chain is on the step's critical path: its
    // stream has the highest priority, so that its CTAs are placed before
    // queued lattice CTAs as SMs free up
    int prio_low = 0, prio_high = 0;
    if ((e = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high)) != cudaSuccess) return fail(e, "priorities");
    if ((e = cudaStreamCreateWithPriority(&h->side, cudaStreamNonBlocking, prio_high)) != cudaSuccess)
        return fail(e, "side stream");
    if ((e = cudaEventCreateWithFlags(&h->ev_ib, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    if ((e = cudaEventCreateWithFlags(&h->ev_inner, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    if ((e = cudaEventCreateWithFlags(&h->ev_interp, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    if (const char *ev = getenv("LBM_AFTER_INTERP")) h->after_interp = atoi(ev) != 0;
    if ((e = cudaStreamCreateWithFlags(&h->fstream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "factor stream");
    if ((e = cudaStreamCreateWithPriority(&h->cstream, cudaStreamNonBlocking, prio_high)) != cudaSuccess)
        return fail(e, "check stream");
    for (cudaEvent_t *ev : {&h->ev_check[0], &h->ev_check[1], &h->ev_cjoin})
        if ((e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    for (int q = 0; q < 2; ++q) {
        if ((e = cudaEventCreateWithFlags(&h->ev_batch[q], cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
        if ((e = cudaEventCreateWithFlags(&h->ev_free[q], cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    }
    if (const char *ov = getenv("LBM_OVERLAP")) h->overlap = atoi(ov) != 0;
    if (const char *fb = getenv("LBM_IB_BATCH")) {
        const int v = atoi(fb);
        if (v >= 1 && 2 * v <= LBM_NSLOT_MAX) h->fbatch = v;
    }
    h->nslots = 2 * h->fbatch;
    // population buffers carry LBM_FPAD elements of padding before and after
    // the 9 planes, so the bulk row copies of the lattice kernel (which read a
    // 16-byte halo left and right of every row segment) stay in bounds
    const size_t fbytes = h->elem * (9 * (size_t)h->plane + 2 * LBM_FPAD);
    for (int b = 0; b < 2; ++b) {
        if ((e = dmalloc(h, &h->falloc[b], fbytes)) != cudaSuccess) return fail(e, "alloc f");
        h->fbuf[b] = (char *)h->falloc[b] + h->elem * LBM_FPAD;
    }
    const size_t cs = compute_size(h->prec);
    const size_t nn = (size_t)h->nx * h->ny;
    for (int b = 0; b < 2; ++b)
        if ((e = dmalloc(h, &h->d_fields[b], 3 * cs * nn)) != cudaSuccess) return fail(e, "alloc fields");
    if ((e = dmalloc(h, &h->edge_c, cs * (6 * (size_t)h->ny + 36))) != cudaSuccess) return fail(e, "alloc edge");
    if ((e = dmalloc(h, &h->d_status, sizeof(unsigned))) != cudaSuccess) return fail(e, "alloc status");
    if ((e = dmalloc(h, &h->d_counter, sizeof(unsigned))) != cudaSuccess) return fail(e, "alloc counter");
    if ((e = dmalloc(h, &h->d_pinfo, LBM_NSLOT_MAX * sizeof(PatchInfo))) != cudaSuccess) return fail(e, "alloc pinfo");
    if ((e = dmalloc(h, &h->d_red, sizeof(double) * 2 * 296)) != cudaSuccess) return fail(e, "alloc red");
    if ((e = dmalloc(h, &h->d_mass, sizeof(double) * mass_slots())) != cudaSuccess) return fail(e, "alloc mass");
    if ((e = dmalloc(h, &h->d_mcount, sizeof(unsigned))) != cudaSuccess) return fail(e, "alloc mass counter");

    // solve residual and half-bandwidth, per step parity
    if ((e = dmalloc(h, &h->d_solve_res, 2 * 2 * sizeof(double))) != cudaSuccess) return fail(e, "alloc res");
    if ((e = dmalloc(h, &h->d_ring, sizeof(double) * h->row_len * (size_t)h->ring_cap)) != cudaSuccess)
        return fail(e, "alloc ring");
    if (h->npts > 0) {
        if ((e = dmalloc(h, &h->d_xb0, sizeof(double) * h->npts)) != cudaSuccess) return fail(e, "alloc xb0");
        if ((e = dmalloc(h, &h->d_yb0, sizeof(double) * h->npts)) != cudaSuccess) return fail(e, "alloc yb0");
        if ((e = dmalloc(h, &h->d_arc, sizeof(double) * h->nseg)) != cudaSuccess) return fail(e, "alloc arc");
    }
    // the zero-fills queued on the handle's stream are done (later calls
    // order their work after them on the same stream in any case)
    if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return fail(e, "sync");
    *out = h;
    return LBM_OK;
}

int lbm_destroy(lbm_t *h)
{
    if (!h) return LBM_ERR_ARG;
    // no queued work of the handle may still use what is freed below
    if (h->fstream) cudaStreamSynchronize(h->fstream);
    if (h->side) cudaStreamSynchronize(h->side);
    if (h->cstream) cudaStreamSynchronize(h->cstream);
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (int b = 0; b < 2; ++b) { free_dev(h->falloc[b]); h->fbuf[b] = nullptr; free_dev(h->d_fields[b]); }
    free_dev(h->edge_c);
    free_devp(h->d_xb0); free_devp(h->d_yb0); free_devp(h->d_arc); free_devp(h->d_mstep);
    free_ib(h);
    free_devp(h->d_pinfo); free_devp(h->d_counter);
    free_devp(h->d_ring); free_devp(h->d_status); free_devp(h->d_solve_res); free_devp(h->d_red);
    free_devp(h->d_mass); free_devp(h->d_mcount);

    free_devp(h->d_stage);
    if (h->side) cudaStreamSynchronize(h->side);
    if (h->cstream) cudaStreamSynchronize(h->cstream);
    if (h->fstream) cudaStreamSynchronize(h->fstream);
    // the frees above went to the pool on the main stream: once they have
    // completed, an allocation on any other stream may reuse the memory (one
    // made before the driver has seen them complete maps new memory instead)
    if (h->stream) cudaStreamSynchronize(h->stream);
    for (auto &e : h->ev) cudaEventDestroy(e);
    for (auto &e : h->ev_side) cudaEventDestroy(e);
    if (h->ev_ib) cudaEventDestroy(h->ev_ib);
    if (h->ev_inner) cudaEventDestroy(h->ev_inner);
    if (h->ev_interp) cudaEventDestroy(h->ev_interp);
    for (int q = 0; q < 2; ++q) {
        if (h->ev_batch[q]) cudaEventDestroy(h->ev_batch[q]);
        if (h->ev_free[q]) cudaEventDestroy(h->ev_free[q]);
    }
    for (cudaEvent_t ev : {h->ev_check[0], h->ev_check[1], h->ev_cjoin})
        if (ev) cudaEventDestroy(ev);
    if (h->cstream) cudaStreamDestroy(h->cstream);
    if (h->fstream) cudaStreamDestroy(h->fstream);
    if (h->side) cudaStreamDestroy(h->side);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return LBM_OK;
}

int lbm_set_boundary(lbm_t *h, int wing, const double *x, const double *y, int npts)
{
    if (!h) return LBM_ERR_ARG;
    quiesce(h);   // queued work may still read what is rewritten below
    if (wing < 1 || wing > h->nwing || !x || !y || npts != h->ppw)
        return set_err(h, LBM_ERR_ARG, "set_boundary: bad wing index or point count");
    const int ps = (wing - 1) * h->ppw, ss = (wing - 1) * h->spw;
    for (int i = 0; i < npts; ++i) {
        if (!std::isfinite(x[i]) || !std::isfinite(y[i])) return set_err(h, LBM_ERR_ARG, "set_boundary: non-finite point");
        h->hx0[ps + i] = x[i];
        h->hy0[ps + i] = y[i];
    }
    for (int i0 = 0; i0 < h->spw; ++i0) {                 // airfoil.f90:235-238
        const double dx = h->hx0[ps + i0 + 1] - h->hx0[ps + i0];
        const double dy = h->hy0[ps + i0 + 1] - h->hy0[ps + i0];
        h->harc[ss + i0] = sqrt(dx * dx + dy * dy) / h->p.scale;
    }
    for (int i = 0; i < npts; ++i) {                      // airfoil.f90:240-241
        h->hx0[ps + i] = h->hx0[ps + i] + (h->p.xc - h->p.xp);
        h->hy0[ps + i] = h->hy0[ps + i] + (h->p.yc - h->p.yp);
    }
    CK(cudaMemcpyAsync(h->d_xb0 + ps, h->hx0.data() + ps, sizeof(double) * npts, cudaMemcpyHostToDevice, h->stream), "copy xb0");
    CK(cudaMemcpyAsync(h->d_yb0 + ps, h->hy0.data() + ps, sizeof(double) * npts, cudaMemcpyHostToDevice, h->stream), "copy yb0");
    CK(cudaMemcpyAsync(h->d_arc + ss, h->harc.data() + ss, sizeof(double) * h->spw, cudaMemcpyHostToDevice, h->stream), "copy arc");
    CK(cudaStreamSynchronize(h->stream), "sync boundary");
    h->have_wing[wing - 1] = 1;
    free_ib(h);
    return LBM_OK;
}

int lbm_set_motion_table(lbm_t *h, const double *table, int rows, int cols)
{
    if (!h) return LBM_ERR_ARG;
    quiesce(h);   // queued work may still read what is rewritten below
    if (!table) return set_err(h, LBM_ERR_ARG, "motion table: null");
    if (cols != 1 + 9 * h->nwing) return set_err(h, LBM_ERR_IO, "motion table: column count must be 1+9*wing_count");
    if (rows < 1) return set_err(h, LBM_ERR_IO, "motion table: empty");          // mode.f90:101-104
    for (int r = 1; r < rows; ++r)                                                 // mode.f90:130-135
        if (table[r] < table[r - 1]) return set_err(h, LBM_ERR_IO, "motion table: time column must be non-decreasing");
    for (size_t q = 0; q < (size_t)rows * cols; ++q)
        if (!std::isfinite(table[q])) return set_err(h, LBM_ERR_IO, "motion table: non-finite value");
    h->mtab.assign(table, table + (size_t)rows * cols);
    h->mrows = rows;
    h->mcols = cols;
    h->mend = table[rows - 1];                                                     // mode.f90:127
    h->mdt = h->p.scale * h->p.uu;                                                 // main.f90:255
    h->msteps = (int)((h->mend + 1.0e-12) / h->mdt) + 1;                           // mode.f90:258
    h->mstep_host.assign((size_t)h->msteps * cols, 0.0);
    int idx = 0;
    std::vector<double> row(cols);
    for (int i = 1; i <= h->msteps; ++i) {                                         // mode.f90:263-268
        lookup_row(h->mtab, rows, cols, (double)(i - 1) * h->mdt, idx, row.data());
        std::copy(row.begin(), row.end(), h->mstep_host.begin() + (size_t)(i - 1) * cols);
    }
    free_devp(h->d_mstep);
    CK(dmalloc(h, &h->d_mstep, sizeof(double) * h->mstep_host.size()), "alloc step table");
    CK(cudaMemcpyAsync(h->d_mstep, h->mstep_host.data(), sizeof(double) * h->mstep_host.size(),
                       cudaMemcpyHostToDevice, h->stream), "copy step table");
    CK(cudaStreamSynchronize(h->stream), "sync motion");
    free_ib(h);
    return LBM_OK;
}

int lbm_init(lbm_t *h, const double *du, const double *dv)
{
    if (!h) return LBM_ERR_ARG;
    if (h->mstep_host.empty()) return set_err(h, LBM_ERR_STATE, "init: motion table not loaded (mode.f90:275-276)");
    quiesce(h);   // queued work may still read what is rewritten below
    const int nx = h->nx, ny = h->ny;
    const size_t nn = (size_t)nx * ny;
    // initial f = feq(rho=1, u=UU(+du), v=0(+dv)) with single-precision weights
    // (solution.f90:33-59), built on the device from the perturbation
    // (launch_init_lattice); the host builds only the edge constants
    auto uv = [&](size_t q, double &u, double &v) {
        u = h->p.uu;
        v = 0.0;
        if (du) u = u + du[q];
        if (dv) v = v + dv[q];
    };
    // edge f0 = the initial f on the four edges (streaming never rewrites
    // them, solution.f90:440-447) and the boundary values taken from them
    std::vector<double> ef(9 * (2 * (size_t)ny + 2 * (size_t)nx));
    auto edge_node = [&](size_t at, int i, int j) {
        double u, v;
        uv((size_t)j * nx + i, u, v);
        for (int k = 0; k < 9; ++k) ef[9 * at + k] = feq(1.0, u, v, k);
    };
    for (int j = 0; j < ny; ++j) {
        edge_node((size_t)j, 0, j);
        edge_node((size_t)ny + j, nx - 1, j);
    }
    for (int i = 0; i < nx; ++i) {
        edge_node(2 * (size_t)ny + i, i, 0);
        edge_node(2 * (size_t)ny + nx + i, i, ny - 1);
    }
    {
        const int rc = handle_set_edges(h, ef.data());
        if (rc) return rc;
    }
    // populations and the initial fields (rho = 1, u, v) in slot 0: u0 of the
    // first step. The perturbation goes up into the second population buffer,
    // which the first step overwrites before anything reads it: 9 planes of
    // at least nx*ny elements of at least 2 bytes hold the 2*nx*ny doubles,
    // and no allocation is needed.
    double *ddu = nullptr, *ddv = nullptr;
    if (du || dv) {
        double *stage = (double *)h->fbuf[1];
        if (du) CK(xfer_h2d(ddu = stage, du, sizeof(double) * nn, h->stream), "copy du");
        if (dv) CK(xfer_h2d(ddv = stage + nn, dv, sizeof(double) * nn, h->stream), "copy dv");
    }
    if (launch_init_lattice(h, ddu, ddv)) return cuda_err(h, cudaGetLastError(), "init");
    h->cur = 0;
    h->fields_slot = 0;
    h->fields_step[0] = 0;
    h->fields_step[1] = -1;
    CK(cudaMemsetAsync(h->d_status, 0, sizeof(unsigned), h->stream), "clear status");
    CK(cudaMemsetAsync(h->d_pinfo, 0, LBM_NSLOT_MAX * sizeof(PatchInfo), h->stream), "clear pinfo");
    CK(cudaStreamSynchronize(h->stream), "sync init");
    h->n = 1;
    h->steps_done = 0;
    // the patch rectangles were cleared above: the factorization slots are
    // filled again from the first step
    h->batch_in_half[0] = h->batch_in_half[1] = -1;
    h->fgroup[0] = h->fgroup[1] = -1;
    h->inited = 1;
    return LBM_OK;
}

int lbm_step(lbm_t *h, double *force_row)
{
    if (!h) return LBM_ERR_ARG;
    return run_steps(h, 1, force_row, nullptr, true);
}

int lbm_run(lbm_t *h, int nsteps, double *force_rows, int *done_steps)
{
    if (!h) return LBM_ERR_ARG;
    if (done_steps) *done_steps = 0;
    if (nsteps < 0) return set_err(h, LBM_ERR_ARG, "run: negative step count");
    if (nsteps == 0) return LBM_OK;
    return run_steps(h, nsteps, force_rows, done_steps, false);
}

int lbm_force_row_length(const lbm_t *h) { return h ? h->row_len : LBM_ERR_ARG; }

int lbm_get_fields(lbm_t *h, double *rho, double *u, double *v)
{
    if (!h) return LBM_ERR_ARG;
    if (!h->inited) return set_err(h, LBM_ERR_STATE, "get_fields: not initialised");
    const int slot = h->fields_slot;
    if (h->fields_step[slot] != h->steps_done)
        return set_err(h, LBM_ERR_STATE, "get_fields: the last step did not keep its fields");
    const size_t nn = (size_t)h->nx * h->ny;
    double *dst[3] = {rho, u, v};
    for (int c = 0; c < 3; ++c) {
        if (!dst[c]) continue;
        if (h->prec == LBM_PREC_FP64)
            CK(xfer_d2h(dst[c], (const double *)h->d_fields[slot] + c * nn, sizeof(double) * nn, h->stream),
               "copy fields");
        else
            CK(xfer_d2h_widen(dst[c], (const float *)h->d_fields[slot] + c * nn, nn, h->stream), "copy fields");
    }
    return LBM_OK;
}

int lbm_get_populations(lbm_t *h, double *f)
{
    if (!h || !f) return LBM_ERR_ARG;
    if (!h->inited) return set_err(h, LBM_ERR_STATE, "get_populations: not initialised");
    const size_t nn = (size_t)h->nx * h->ny;
    if (!h->d_stage) CK(dmalloc(h, &h->d_stage, sizeof(double) * nn * 9), "alloc stage");
    if (launch_unpack(h, h->fbuf[h->cur], h->d_stage)) return cuda_err(h, cudaGetLastError(), "unpack");
    CK(xfer_d2h(f, h->d_stage, sizeof(double) * nn * 9, h->stream), "copy f");
    free_devp(h->d_stage);
    return LBM_OK;
}

int lbm_set_populations(lbm_t *h, const double *f)
{
    if (!h || !f) return LBM_ERR_ARG;
    quiesce(h);   // queued work may still read what is rewritten below
    if (!h->inited) return set_err(h, LBM_ERR_STATE, "set_populations: not initialised");
    const size_t nn = (size_t)h->nx * h->ny;
    if (!h->d_stage) CK(dmalloc(h, &h->d_stage, sizeof(double) * nn * 9), "alloc stage");
    CK(xfer_h2d(h->d_stage, f, sizeof(double) * nn * 9, h->stream), "copy f");
    if (launch_pack(h, h->d_stage, h->fbuf[h->cur])) return cuda_err(h, cudaGetLastError(), "pack");
    CK(cudaStreamSynchronize(h->stream), "sync f");
    free_devp(h->d_stage);
    h->fields_step[0] = h->fields_step[1] = -1;
    return LBM_OK;
}

int lbm_residual(lbm_t *h, double *err)
{
    if (!h || !err) return LBM_ERR_ARG;
    const int a = h->fields_slot, b = a ^ 1;
    if (h->steps_done < 1 || h->fields_step[a] != h->steps_done || h->fields_step[b] != h->steps_done - 1)
        return set_err(h, LBM_ERR_STATE, "residual: fields of the last two states were not kept");
    double s[2];
    if (launch_residual(h, h->d_fields[a], h->d_fields[b], s)) return cuda_err(h, cudaGetLastError(), "residual");
    *err = sqrt(s[0]) / (sqrt(s[1]) + 1e-30);   // solution.f90:120-122
    return LBM_OK;
}

int lbm_mass(lbm_t *h, double *mass)
{
    if (!h || !mass) return LBM_ERR_ARG;
    if (!h->inited) return set_err(h, LBM_ERR_STATE, "mass: not initialised");
    double dsum = 0.0;
    int rc = mass_launch(h, h->stream, &dsum);
    if (rc) return rc;
    CK(cudaStreamSynchronize(h->stream), "sync mass");
    rc = mass_result(h, dsum);
    *mass = h->last_mass;
    return rc;
}

int lbm_get_markers(lbm_t *h, double *xb2, double *yb2, double *solve_residual, int *half_bandwidth)
{
    if (!h) return LBM_ERR_ARG;
    if (!h->ib_ready || h->nseg == 0) return set_err(h, LBM_ERR_STATE, "get_markers: no immersed boundary step run");
    std::vector<Marker> mk(h->nseg);
    const Marker *last = h->d_mk + (size_t)((h->n - 1) % h->nslots) * h->nseg;   // slot of the last step
    CK(cudaMemcpyAsync(mk.data(), last, sizeof(Marker) * h->nseg, cudaMemcpyDeviceToHost, h->stream), "copy markers");
    double res[2] = {0, 0};
    const double *last_res = h->d_solve_res + 2 * ((h->n - 1) & 1);   // parity of the last step
    CK(cudaMemcpyAsync(res, last_res, 2 * sizeof(double), cudaMemcpyDeviceToHost, h->stream), "copy res");
    CK(cudaStreamSynchronize(h->stream), "sync markers");
    for (int k = 0; k < h->nseg; ++k) {
        if (xb2) xb2[k] = mk[k].xm;
        if (yb2) yb2[k] = mk[k].ym;
    }
    if (solve_residual) *solve_residual = res[0];
    if (half_bandwidth) *half_bandwidth = (int)res[1];
    return LBM_OK;
}

int lbm_set_timing(lbm_t *h, int enable)
{
    if (!h) return LBM_ERR_ARG;
    if (enable && h->ev.empty()) {
        h->ev.resize(4 * (size_t)h->ring_cap);
        h->ev_side.resize(2 * (size_t)h->ring_cap);
        for (auto &e : h->ev) CK(cudaEventCreate(&e), "event create");
        for (auto &e : h->ev_side) CK(cudaEventCreate(&e), "event create");
    }
    h->timing = enable == LBM_TIMING_SPAN ? LBM_TIMING_SPAN : (enable ? LBM_TIMING_KERNELS : 0);
    h->t_step = h->t_ib = h->t_kf = 0;
    h->t_steps = 0;
    return LBM_OK;
}

int lbm_get_timing(lbm_t *h, double *step_ms, double *ib_ms, double *lattice_ms, int *steps)
{
    if (!h) return LBM_ERR_ARG;
    if (step_ms) *step_ms = h->t_step;
    if (ib_ms) *ib_ms = h->t_ib;
    if (lattice_ms) *lattice_ms = h->t_kf;
    if (steps) *steps = h->t_steps;
    return LBM_OK;
}

int lbm_get_launch_count(const lbm_t *h, long long *count)
{
    if (!h || !count) return LBM_ERR_ARG;
    *count = h->launches;
    return LBM_OK;
}

int lbm_step_index(const lbm_t *h) { return h ? h->n : LBM_ERR_ARG; }

int lbm_device_bytes(const lbm_t *h, long long *bytes)
{
    if (!h || !bytes) return LBM_ERR_ARG;
    *bytes = h->dev_bytes;
    return LBM_OK;
}

const char *lbm_last_error(const lbm_t *h) { return h ? h->err.c_str() : "lbm_create failed (bad parameters or no CUDA device)"; }

int lbm_device_check(int *binary_version, int *sm_count)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return LBM_ERR_CUDA;
    cudaFuncAttributes fa{};
    if (cudaFuncGetAttributes(&fa, arch_probe) != cudaSuccess) return LBM_ERR_CUDA;
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return LBM_ERR_CUDA;
    if (binary_version) *binary_version = fa.binaryVersion;
    if (sm_count) *sm_count = sms;
    return LBM_OK;
}

int lbm_describe_status(unsigned int status, char *message, int capacity)
{
    std::string msg;
    const int code = status_error(status, msg);
    if (message && capacity > 0) {
        const size_t n = std::min(msg.size(), (size_t)capacity - 1);
        memcpy(message, msg.data(), n);
        message[n] = 0;
    }
    return code;
}

}  // extern "C"
