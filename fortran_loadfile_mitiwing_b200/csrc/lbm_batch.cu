// lbm_batch.cu -- several cases (handles) stepped together on one GPU.
//
// A batch steps its cases in lockstep, with one launch per kernel for all of
// them: the lattice update of every case is one launch of the staged kernel
// driven by a case table (CTA -> case, strip, row chunk), and each stage of
// the immersed boundary (interpolation, solve, correction tiles, forces and
// residual; and, per batch of steps, the factorization chain) is one launch
// with the case as grid z, the cases' arguments read from device arrays. The
// streams and events are the batch's own, with the same structure as one
// handle's step: factorization one batch of steps ahead, the flow chain on a
// high-priority stream beside the lattice update.
//
// Every kernel computes each case exactly as the single-case launches do, so
// a case's results in a batch are bit-for-bit those of running it alone.
#include <algorithm>
#include <cmath>
#include <vector>

#include "lbm_internal.h"

struct lbm_batch {
    std::vector<lbm_handle *> cases;
    int prec = 0, fbatch = 4, nslots = 8;
    cudaStream_t main = nullptr, side = nullptr, fstream = nullptr;
    cudaEvent_t ev_batch[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
    cudaEvent_t ev_ib = nullptr, ev_done = nullptr;
    int batch_in_half[2] = {-1, -1};
    // device argument arrays: factorization (slot 0 base), flow chain (per
    // step, double-buffered so a step's upload never overwrites arguments a
    // queued launch still reads), lattice, case table
    void *d_fargs[2] = {nullptr, nullptr}, *d_sargs[2] = {nullptr, nullptr}, *d_kargs[2] = {nullptr, nullptr};
    int4 *d_table[2] = {nullptr, nullptr};
    void *h_fargs[2] = {nullptr, nullptr}, *h_sargs[2] = {nullptr, nullptr}, *h_kargs[2] = {nullptr, nullptr};
    int4 *h_table[2] = {nullptr, nullptr};
    cudaEvent_t ev_upload[2] = {nullptr, nullptr}, ev_fupload[2] = {nullptr, nullptr};
    size_t ib_sz = 0, kf_sz = 0;
    int table_cap = 0;
    int rows_per_cta = 0;   // 0: the cases' own setting
    std::string err;
};

namespace {

int berr(lbm_batch *b, int code, const std::string &msg)
{
    b->err = msg;
    return code;
}

#define BCK(call, what)                                                                                  \
    do {                                                                                                 \
        cudaError_t e_ = (call);                                                                         \
        if (e_ != cudaSuccess) return berr(b, LBM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void free_batch(lbm_batch *b)
{
    if (b->main) cudaStreamSynchronize(b->main);
    if (b->side) cudaStreamSynchronize(b->side);
    if (b->fstream) cudaStreamSynchronize(b->fstream);
    for (int q = 0; q < 2; ++q) {
        if (b->d_sargs[q]) cudaFree(b->d_sargs[q]);
        if (b->d_kargs[q]) cudaFree(b->d_kargs[q]);
        if (b->d_table[q]) cudaFree(b->d_table[q]);
        if (b->h_sargs[q]) cudaFreeHost(b->h_sargs[q]);
        if (b->h_kargs[q]) cudaFreeHost(b->h_kargs[q]);
        if (b->h_table[q]) cudaFreeHost(b->h_table[q]);
        if (b->ev_batch[q]) cudaEventDestroy(b->ev_batch[q]);
        if (b->ev_free[q]) cudaEventDestroy(b->ev_free[q]);
        if (b->ev_upload[q]) cudaEventDestroy(b->ev_upload[q]);
        if (b->ev_fupload[q]) cudaEventDestroy(b->ev_fupload[q]);
        if (b->d_fargs[q]) cudaFree(b->d_fargs[q]);
        if (b->h_fargs[q]) cudaFreeHost(b->h_fargs[q]);
    }
    if (b->ev_ib) cudaEventDestroy(b->ev_ib);
    if (b->ev_done) cudaEventDestroy(b->ev_done);
    if (b->main) cudaStreamDestroy(b->main);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->fstream) cudaStreamDestroy(b->fstream);
}

}  // namespace

extern "C" {

int lbm_batch_create(lbm_t *const *cases, int count, lbm_batch_t **out)
{
    if (!out || !cases || count < 1) return LBM_ERR_ARG;
    *out = nullptr;
    for (int c = 0; c < count; ++c)
        if (!cases[c]) return LBM_ERR_ARG;
    lbm_handle *h0 = cases[0];
    for (int c = 0; c < count; ++c) {
        lbm_handle *h = cases[c];
        if (!h->inited) return handle_error(h, LBM_ERR_STATE, "batch: lbm_init not called");
        for (int w = 0; w < h->nwing; ++w)
            if (!h->have_wing[w]) return handle_error(h, LBM_ERR_STATE, "batch: boundary of a wing not set");
        if (h->nseg < 1) return handle_error(h, LBM_ERR_ARG, "batch: a case without markers");
        if (h->prec != h0->prec || h->fbatch != h0->fbatch || h->nslots != h0->nslots || h->n != h0->n ||
            h->dev != h0->dev)
            return handle_error(h, LBM_ERR_ARG,
                           "batch: cases must share storage precision, factorization batch, device and step index");
        for (int d = 0; d < c; ++d)
            if (cases[d] == h) return handle_error(h, LBM_ERR_ARG, "batch: a case appears twice");
        const int rc = handle_prepare_ib(h);
        if (rc) return rc;
    }
    lbm_batch *b = new lbm_batch;
    b->cases.assign(cases, cases + count);
    b->prec = h0->prec;
    b->fbatch = h0->fbatch;
    b->nslots = h0->nslots;
    b->ib_sz = ib_args_size();
    b->kf_sz = kf_args_size(b->prec);
    auto fail = [&](cudaError_t e, const char *what) {
        h0->err = std::string("batch: ") + what + ": " + cudaGetErrorString(e);
        free_batch(b);
        delete b;
        return LBM_ERR_CUDA;
    };
    cudaError_t e;
    int prio_low = 0, prio_high = 0;
    if ((e = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high)) != cudaSuccess) return fail(e, "priorities");
    if ((e = cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    if ((e = cudaStreamCreateWithPriority(&b->side, cudaStreamNonBlocking, prio_high)) != cudaSuccess)
        return fail(e, "stream");
    if ((e = cudaStreamCreateWithFlags(&b->fstream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    for (int q = 0; q < 2; ++q) {
        if ((e = cudaEventCreateWithFlags(&b->ev_batch[q], cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
        if ((e = cudaEventCreateWithFlags(&b->ev_free[q], cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
        if ((e = cudaEventCreateWithFlags(&b->ev_upload[q], cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
        if ((e = cudaEventCreateWithFlags(&b->ev_fupload[q], cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    }
    if ((e = cudaEventCreateWithFlags(&b->ev_ib, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    if ((e = cudaEventCreateWithFlags(&b->ev_done, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    // case table capacity: every case's full grid
    int cap = 0;
    for (lbm_handle *h : b->cases) {
        int gx, gy;
        kf_tma_grid(h, &gx, &gy);
        // the autotuner may use 4 rows per CTA: twice the chunks of 8
        cap += gx * (2 * gy + 2);
    }
    b->table_cap = cap;
    const size_t nc = (size_t)count;
    for (int q = 0; q < 2; ++q) {
        if ((e = cudaMalloc(&b->d_fargs[q], nc * b->ib_sz)) != cudaSuccess) return fail(e, "alloc");
        if ((e = cudaMallocHost(&b->h_fargs[q], nc * b->ib_sz)) != cudaSuccess) return fail(e, "alloc");
        if ((e = cudaMalloc(&b->d_sargs[q], nc * b->ib_sz)) != cudaSuccess) return fail(e, "alloc");
        if ((e = cudaMalloc(&b->d_kargs[q], nc * b->kf_sz)) != cudaSuccess) return fail(e, "alloc");
        if ((e = cudaMalloc(&b->d_table[q], sizeof(int4) * (size_t)cap)) != cudaSuccess) return fail(e, "alloc");
        if ((e = cudaMallocHost(&b->h_sargs[q], nc * b->ib_sz)) != cudaSuccess) return fail(e, "alloc");
        if ((e = cudaMallocHost(&b->h_kargs[q], nc * b->kf_sz)) != cudaSuccess) return fail(e, "alloc");
        if ((e = cudaMallocHost((void **)&b->h_table[q], sizeof(int4) * (size_t)cap)) != cudaSuccess)
            return fail(e, "alloc");
    }
    // every case's queued work on its own streams is done before the batch uses it
    for (lbm_handle *h : b->cases) {
        if (h->fstream) cudaStreamSynchronize(h->fstream);
        if (h->side) cudaStreamSynchronize(h->side);
        if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return fail(e, "sync");
        // the batch keeps its own factorization slots: the cases' own
        // lookahead is stale once the batch has stepped them
        h->batch_in_half[0] = h->batch_in_half[1] = -1;
    }
    *out = b;
    return LBM_OK;
}

int lbm_batch_destroy(lbm_batch_t *b)
{
    if (!b) return LBM_ERR_ARG;
    free_batch(b);
    delete b;
    return LBM_OK;
}

int lbm_batch_set_rows(lbm_batch_t *b, int rows_per_cta)
{
    if (!b || rows_per_cta < 0 || rows_per_cta > 4096) return LBM_ERR_ARG;
    b->rows_per_cta = rows_per_cta;
    return LBM_OK;
}

int lbm_batch_run(lbm_batch_t *b, int nsteps, double *const *force_rows, int *done_steps)
{
    if (!b || nsteps < 0) return LBM_ERR_ARG;
    const int nc = (int)b->cases.size();
    for (int c = 0; c < nc; ++c)
        if (done_steps) done_steps[c] = 0;
    if (nsteps == 0) return LBM_OK;
    const int K = b->fbatch;
    // the lattice kernel's rows per CTA (the autotuner's choice, else the cases')
    std::vector<int> rows_saved(nc);
    for (int c = 0; c < nc; ++c) {
        rows_saved[c] = b->cases[c]->kf_rows;
        if (b->rows_per_cta > 0) b->cases[c]->kf_rows = b->rows_per_cta;
    }
    auto restore = [&]() {
        for (int c = 0; c < nc; ++c) b->cases[c]->kf_rows = rows_saved[c];
    };
    std::vector<int> last_step(nc), done(nc, 0), pending_start(nc, 0);
    for (int c = 0; c < nc; ++c) {
        lbm_handle *h = b->cases[c];
        const double dt = h->p.scale * h->p.uu;
        last_step[c] = (int)std::floor((h->mend + 1.0e-12) / dt) + 1;   // last step with time <= mend
    }
    // every case must be at the same step; the batch's factorization slots
    // are recomputed (a case may have been stepped alone since the last run)
    for (int c = 1; c < nc; ++c)
        if (b->cases[c]->n != b->cases[0]->n) {
            restore();
            return berr(b, LBM_ERR_STATE, "batch: cases are not at the same step");
        }
    b->batch_in_half[0] = b->batch_in_half[1] = -1;
    // the factorization of batch bi for every active case, into slot half bi & 1
    auto factor_batch = [&](int bi, const std::vector<lbm_handle *> &act) -> int {
        const int half = bi & 1;
        b->batch_in_half[half] = bi;
        const int s0 = std::max(1, bi * K);
        BCK(cudaStreamWaitEvent(b->fstream, b->ev_free[half], 0), "wait");
        // arguments of the active cases (slot 0 base with the slot strides)
        BCK(cudaEventSynchronize(b->ev_fupload[half]), "sync upload");
        for (size_t c = 0; c < act.size(); ++c) ib_args_write(act[c], nullptr, 0, (char *)b->h_fargs[half] + c * b->ib_sz);
        BCK(cudaMemcpyAsync(b->d_fargs[half], b->h_fargs[half], act.size() * b->ib_sz, cudaMemcpyHostToDevice,
                            b->fstream),
            "upload");
        BCK(cudaEventRecord(b->ev_fupload[half], b->fstream), "event");
        if (launch_factor_batch(act.data(), (int)act.size(), b->d_fargs[half], s0, K, b->fstream))
            return berr(b, LBM_ERR_CUDA, "batch: launch factor");
        BCK(cudaEventRecord(b->ev_batch[half], b->fstream), "event");
        return LBM_OK;
    };
    BCK(cudaEventRecord(b->ev_done, b->main), "event");
    int rc = LBM_OK, pending = 0, step = 0;
    std::vector<lbm_handle *> act;
    for (; step < nsteps; ++step) {
        act.clear();
        std::vector<int> act_idx;
        for (int c = 0; c < nc; ++c)
            if (b->cases[c]->n <= last_step[c]) {
                act.push_back(b->cases[c]);
                act_idx.push_back(c);
            }
        if (act.empty()) break;
        const int n = act[0]->n;   // lockstep: every active case is at step n
        const int bi = n / K, half = bi & 1, q = n % b->nslots, buf = step & 1;
        const bool fields = step >= nsteps - 2;
        if (b->batch_in_half[half] != bi && (rc = factor_batch(bi, act))) break;
        // this step's arguments (the upload buffers of two steps back are free)
        BCK(cudaEventSynchronize(b->ev_upload[buf]), "sync upload");
        int ntab = 0;
        for (size_t c = 0; c < act.size(); ++c) {
            lbm_handle *h = act[c];
            const void *fin = h->fbuf[h->cur];
            void *fout = h->fbuf[h->cur ^ 1];
            void *fd = nullptr;
            if (fields) {
                const int fs = h->fields_slot ^ 1;
                fd = h->d_fields[fs];
                h->fields_slot = fs;
                h->fields_step[fs] = h->n;
            }
            h->pinfo_slot = q;
            ib_args_write(h, fin, q, (char *)b->h_sargs[buf] + c * b->ib_sz);
            kf_args_write(h, fin, fout, fd, KF_OUTER, (char *)b->h_kargs[buf] + c * b->kf_sz);
            int gx, gy;
            kf_tma_grid(h, &gx, &gy);
            for (int by = 0; by < gy; ++by)
                for (int bx = 0; bx < gx; ++bx) b->h_table[buf][ntab++] = make_int4((int)c, bx, by, gx | (gy << 16));
        }
        if (ntab > b->table_cap) { rc = berr(b, LBM_ERR_STATE, "batch: case table overflow"); break; }
        // the previous step is complete (and with it every reader of this step's upload buffers)
        BCK(cudaStreamWaitEvent(b->side, b->ev_done, 0), "wait");
        BCK(cudaMemcpyAsync(b->d_sargs[buf], b->h_sargs[buf], act.size() * b->ib_sz, cudaMemcpyHostToDevice, b->side),
            "upload");
        BCK(cudaMemcpyAsync(b->d_kargs[buf], b->h_kargs[buf], act.size() * b->kf_sz, cudaMemcpyHostToDevice, b->side),
            "upload");
        BCK(cudaMemcpyAsync(b->d_table[buf], b->h_table[buf], sizeof(int4) * ntab, cudaMemcpyHostToDevice, b->side),
            "upload");
        BCK(cudaEventRecord(b->ev_upload[buf], b->side), "event");
        // side stream: the flow chains of all cases
        BCK(cudaStreamWaitEvent(b->side, b->ev_batch[half], 0), "wait");
        if (launch_flow_batch(act.data(), (int)act.size(), b->d_sargs[buf], b->d_kargs[buf], n, pending, fields,
                              b->side)) {
            rc = berr(b, LBM_ERR_CUDA, "batch: launch flow");
            break;
        }
        BCK(cudaEventRecord(b->ev_ib, b->side), "event");
        if (launch_check_batch(act.data(), (int)act.size(), b->d_sargs[buf], pending, b->side)) {
            rc = berr(b, LBM_ERR_CUDA, "batch: launch check");
            break;
        }
        BCK(cudaEventRecord(b->ev_free[half], b->side), "event");
        // the next factorization batch, overlapping this one's steps
        if (b->batch_in_half[half ^ 1] != bi + 1) {
            bool any = false;
            for (size_t c = 0; c < act.size(); ++c) any = any || (bi + 1) * K <= last_step[act_idx[c]];
            if (any && (rc = factor_batch(bi + 1, act))) break;
        }
        // main stream: every case's lattice nodes but its correction tiles
        BCK(cudaStreamWaitEvent(b->main, b->ev_batch[half], 0), "wait");
        BCK(cudaStreamWaitEvent(b->main, b->ev_upload[buf], 0), "wait");
        if (launch_kf_multi(b->prec, b->d_kargs[buf], b->d_table[buf], ntab, fields, b->main)) {
            rc = berr(b, LBM_ERR_CUDA, "batch: launch lattice");
            break;
        }
        for (lbm_handle *h : act) h->launches += 1;
        BCK(cudaStreamWaitEvent(b->main, b->ev_ib, 0), "wait");
        BCK(cudaEventRecord(b->ev_done, b->main), "event");   // the step is complete
        for (size_t c = 0; c < act.size(); ++c) {
            lbm_handle *h = act[c];
            h->cur ^= 1;
            h->n++;
            h->steps_done++;
            done[act_idx[c]]++;
        }
        pending++;
        // force rows to the host every ring's worth of steps and at the end
        const bool flush = pending == b->cases[0]->ring_cap || step == nsteps - 1;
        if (flush) {
            BCK(cudaEventRecord(b->ev_ib, b->side), "event");
            BCK(cudaStreamWaitEvent(b->main, b->ev_ib, 0), "wait");
            for (int c = 0; c < nc; ++c) {
                lbm_handle *h = b->cases[c];
                const int rows = done[c] - pending_start[c];
                if (force_rows && force_rows[c] && rows > 0)
                    BCK(cudaMemcpyAsync(force_rows[c] + (size_t)pending_start[c] * h->row_len, h->d_ring,
                                        sizeof(double) * h->row_len * rows, cudaMemcpyDeviceToHost, b->main),
                        "copy force rows");
            }
            BCK(cudaStreamSynchronize(b->main), "sync");
            for (int c = 0; c < nc; ++c) {
                pending_start[c] = done[c];
                const int st = handle_status(b->cases[c]);
                if (st && !rc) {
                    rc = st;
                    b->err = std::string("batch: case ") + std::to_string(c) + ": " + b->cases[c]->err;
                }
            }
            pending = 0;
            if (rc) break;
        }
    }
    // leave every stream idle: the cases' own calls follow on their streams
    cudaStreamSynchronize(b->side);
    cudaStreamSynchronize(b->fstream);
    cudaStreamSynchronize(b->main);
    restore();
    if (done_steps)
        for (int c = 0; c < nc; ++c) done_steps[c] = done[c];
    if (rc == LBM_OK && step < nsteps) rc = LBM_DONE;
    return rc;
}

const char *lbm_batch_last_error(const lbm_batch_t *b) { return b ? b->err.c_str() : ""; }

}  // extern "C"
