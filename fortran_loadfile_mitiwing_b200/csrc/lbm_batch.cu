// lbm_batch.cu -- several cases (handles) stepped together on one GPU.
//
// A batch steps its cases with one launch per kernel for all of them: the
// lattice update of every case is one launch of the staged kernel driven by a
// case table (CTA -> case, strip, row chunk), and each stage of the immersed
// boundary (interpolation, solve, correction tiles, forces and residual; and
// the factorization chain of a batch of steps) is one launch with the case as
// grid z, the cases' arguments read from device arrays. The streams are the
// batch's own, with the structure of one handle's step: factorization a batch
// of steps ahead, the flow chain on a high-priority stream beside the lattice
// update. Cases may be at different steps (each carries its own step index,
// slots and factorization state, kept in its handle), and may be added and
// removed between runs: the base of the serving loop.
//
// Every kernel computes each case exactly as the single-case launches do, so
// a case's results in a batch are bit-for-bit those of running it alone.
//
// Steady steps run as CUDA graphs (lbm_batch_set_graphs): a segment of
// kGraphSteps steps in which the active cases, the case table and the force
// ring stay as they are and no fields are written is captured once, with
// every dependency of the per-step stream code as a graph edge and all of its
// arguments in one device buffer uploaded by the graph's first node; later
// segments of the same structure (the cases, and where in the segment each
// factorization launch and wait falls) only rewrite that buffer's host copy
// and relaunch the instantiated graph. The steps around them (the first step
// of a run, the last two, a case's last two) go through the stream code.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <string>
#include <vector>

#include "lbm_internal.h"

namespace {
constexpr int kFactorRing = 8;   // staging buffers of factorization arguments in flight
// events of the latest factorization launches; a case's halves are at most
// 2 factorization batches (2K steps, two launches a step) old when used, and
// a wait on a newer recording of a reused event only waits longer
constexpr int kGroupRing = 64;
// per-step argument buffers in flight: the host prepares a step's arguments
// while up to kArgRing - 1 earlier steps are still queued
constexpr int kArgRing = 8;
// steps per CUDA graph segment (a multiple of the factorization batch, so
// that segments of a run share their structure) and instantiated graphs kept
constexpr int kGraphSteps = 16;
constexpr int kGraphCache = 8;

size_t round256(size_t x) { return (x + 255) & ~(size_t)255; }
}

struct lbm_batch {
    std::vector<lbm_handle *> cases;
    int prec = -1, fbatch = 4, nslots = 8, dev = 0;
    cudaStream_t main = nullptr, side = nullptr, fstream = nullptr;
    // the steps' force rows and residual checks run on their own stream,
    // after the step's correction tiles, so that the next step's flow chains
    // need not wait for them (the cases keep what they read per step parity;
    // ev_bcheck[p] marks the checks of the last step of parity p done). ev_side
    // marks a step's flow chains and checks done.
    cudaStream_t cstream = nullptr;
    cudaEvent_t ev_bcheck[2] = {nullptr, nullptr}, ev_cpre = nullptr;
    cudaEvent_t ev_ib = nullptr, ev_done = nullptr, ev_fready = nullptr, ev_side = nullptr;
    // device time of the last run's steps (lbm_batch_get_timing)
    cudaEvent_t ev_t0 = nullptr, ev_t1 = nullptr;
    // the step's interpolations are done; with after_interp the lattice
    // launch waits for it (the solve CTAs then find whole SMs free)
    cudaEvent_t ev_interp = nullptr;
    int after_interp = 1;
    double last_ms = 0.0;
    int last_steps = 0;
    // argument arrays: flow chain and lattice per step (a ring of kArgRing,
    // so a step's upload never overwrites arguments a queued launch still
    // reads), the case table (two buffers, uploaded again only when the set
    // of active cases changes), and a ring of factorization argument buffers
    int cap = 0;         // cases the arrays hold
    int table_cap = 0;   // case-table entries
    void *d_sargs[kArgRing] = {}, *d_kargs[kArgRing] = {};
    void *h_sargs[kArgRing] = {}, *h_kargs[kArgRing] = {};
    cudaEvent_t ev_upload[kArgRing] = {}, ev_kdone[kArgRing] = {};
    int4 *d_table[2] = {nullptr, nullptr}, *h_table[2] = {nullptr, nullptr};
    cudaEvent_t ev_tup[2] = {nullptr, nullptr}, ev_tuse[2] = {nullptr, nullptr};
    void *d_fargs[kFactorRing] = {}, *h_fargs[kFactorRing] = {};
    cudaEvent_t ev_fup[kFactorRing] = {};
    int fring = 0;
    cudaEvent_t ev_group[kGroupRing] = {};
    long long gseq = 0;   // factorization launches so far
    size_t ib_sz = 0, kf_sz = 0;
    int rows_per_cta = 0;   // 0: the cases' own setting
    int ctas_per_sm = 0;    // lattice CTAs per SM at most (0: as many as fit)
    std::vector<int> status;   // each case's status in the last run (lbm_batch_case_status)
    // CUDA graph segments: two argument buffers (device and pinned host) used
    // by alternate segments, each with the event of the last graph launch
    // that read it; the instantiated graphs by segment structure, each with
    // the kernels it launches per case (lbm_get_launch_count)
    int graphs = 1;
    int gset = 0;
    size_t seg_bytes = 0;
    void *d_seg[2] = {}, *h_seg[2] = {};
    cudaEvent_t ev_gdone[2] = {};
    // events of the captured stream code (never waited on outside a capture):
    // [1] upload done, [2] [3] the main and factor streams' joins, [4] to [8]
    // the step's points (flow ready, correction tiles done, checks done, step
    // done, interpolation done), then one per factorization launch of the
    // segment, then the checks of the two step parities and the check
    // stream's join ([0] is not used)
    cudaEvent_t ev_cap[9 + 2 * kGraphSteps + 3] = {};
    cudaEvent_t ev_gpre = nullptr;   // the factor stream's work before a graph launch
    struct GraphEntry {
        std::vector<long long> sig;
        cudaGraphExec_t exec = nullptr;
        std::vector<long long> launches;
    };
    std::vector<GraphEntry> gcache;
    long long graph_steps = 0, graph_launches = 0, graph_builds = 0;   // lbm_batch_graph_stats
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

void sync_streams(lbm_batch *b)
{
    if (b->main) cudaStreamSynchronize(b->main);
    if (b->side) cudaStreamSynchronize(b->side);
    if (b->fstream) cudaStreamSynchronize(b->fstream);
    if (b->cstream) cudaStreamSynchronize(b->cstream);
}

void free_arrays(lbm_batch *b)
{
    for (int q = 0; q < kArgRing; ++q) {
        if (b->d_sargs[q]) cudaFree(b->d_sargs[q]);
        if (b->d_kargs[q]) cudaFree(b->d_kargs[q]);
        if (b->h_sargs[q]) cudaFreeHost(b->h_sargs[q]);
        if (b->h_kargs[q]) cudaFreeHost(b->h_kargs[q]);
        b->d_sargs[q] = b->d_kargs[q] = b->h_sargs[q] = b->h_kargs[q] = nullptr;
    }
    for (int q = 0; q < 2; ++q) {
        if (b->d_table[q]) cudaFree(b->d_table[q]);
        if (b->h_table[q]) cudaFreeHost(b->h_table[q]);
        b->d_table[q] = b->h_table[q] = nullptr;
    }
    for (int r = 0; r < kFactorRing; ++r) {
        if (b->d_fargs[r]) cudaFree(b->d_fargs[r]);
        if (b->h_fargs[r]) cudaFreeHost(b->h_fargs[r]);
        b->d_fargs[r] = b->h_fargs[r] = nullptr;
    }
    // the graphs name these buffers
    for (auto &g : b->gcache)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    b->gcache.clear();
    for (int q = 0; q < 2; ++q) {
        if (b->d_seg[q]) cudaFree(b->d_seg[q]);
        if (b->h_seg[q]) cudaFreeHost(b->h_seg[q]);
        b->d_seg[q] = b->h_seg[q] = nullptr;
    }
    b->seg_bytes = 0;
    b->cap = b->table_cap = 0;
}

void clear_graphs(lbm_batch *b)
{
    for (auto &g : b->gcache)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    b->gcache.clear();
}

void free_batch(lbm_batch *b)
{
    sync_streams(b);
    free_arrays(b);
    for (int q = 0; q < kArgRing; ++q) {
        if (b->ev_upload[q]) cudaEventDestroy(b->ev_upload[q]);
        if (b->ev_kdone[q]) cudaEventDestroy(b->ev_kdone[q]);
    }
    for (int q = 0; q < 2; ++q) {
        if (b->ev_tup[q]) cudaEventDestroy(b->ev_tup[q]);
        if (b->ev_tuse[q]) cudaEventDestroy(b->ev_tuse[q]);
    }
    for (int r = 0; r < kFactorRing; ++r)
        if (b->ev_fup[r]) cudaEventDestroy(b->ev_fup[r]);
    for (int r = 0; r < kGroupRing; ++r)
        if (b->ev_group[r]) cudaEventDestroy(b->ev_group[r]);
    for (cudaEvent_t e : {b->ev_ib, b->ev_done, b->ev_fready, b->ev_side, b->ev_t0, b->ev_t1, b->ev_interp,
                          b->ev_gdone[0], b->ev_gdone[1], b->ev_gpre, b->ev_bcheck[0], b->ev_bcheck[1], b->ev_cpre})
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : b->ev_cap)
        if (e) cudaEventDestroy(e);
    if (b->main) cudaStreamDestroy(b->main);
    if (b->side) cudaStreamDestroy(b->side);
    if (b->fstream) cudaStreamDestroy(b->fstream);
    if (b->cstream) cudaStreamDestroy(b->cstream);
}

// argument arrays for `ncase` cases and `ntab` case-table entries (grown, never shrunk)
int reserve(lbm_batch *b, int ncase, int ntab)
{
    if (ncase <= b->cap && ntab <= b->table_cap) return LBM_OK;
    sync_streams(b);
    const int nc = std::max(ncase, b->cap), nt = std::max(ntab, b->table_cap);
    free_arrays(b);
    for (int q = 0; q < kArgRing; ++q) {
        BCK(cudaMalloc(&b->d_sargs[q], nc * b->ib_sz), "alloc");
        BCK(cudaMalloc(&b->d_kargs[q], nc * b->kf_sz), "alloc");
        BCK(cudaMallocHost(&b->h_sargs[q], nc * b->ib_sz), "alloc");
        BCK(cudaMallocHost(&b->h_kargs[q], nc * b->kf_sz), "alloc");
    }
    for (int q = 0; q < 2; ++q) {
        BCK(cudaMalloc(&b->d_table[q], sizeof(int4) * (size_t)nt), "alloc");
        BCK(cudaMallocHost((void **)&b->h_table[q], sizeof(int4) * (size_t)nt), "alloc");
    }
    for (int r = 0; r < kFactorRing; ++r) {
        BCK(cudaMalloc(&b->d_fargs[r], nc * b->ib_sz), "alloc");
        BCK(cudaMallocHost(&b->h_fargs[r], nc * b->ib_sz), "alloc");
    }
    // a graph segment's arguments: per step the flow-chain and lattice
    // arguments of every case, and up to two factorization launches per step
    b->seg_bytes = round256((size_t)kGraphSteps * nc * b->ib_sz) + round256((size_t)kGraphSteps * nc * b->kf_sz) +
                   round256((size_t)2 * kGraphSteps * nc * b->ib_sz);
    for (int q = 0; q < 2; ++q) {
        BCK(cudaMalloc(&b->d_seg[q], b->seg_bytes), "alloc");
        BCK(cudaMallocHost(&b->h_seg[q], b->seg_bytes), "alloc");
    }
    b->cap = nc;
    b->table_cap = nt;
    return LBM_OK;
}

// case-table entries the case can need (the autotuner may use 4 rows per CTA)
int table_need(lbm_handle *h)
{
    int gx, gy;
    const int saved = h->kf_rows;
    h->kf_rows = std::min(h->kf_rows, 4);
    kf_tma_grid(h, &gx, &gy);
    h->kf_rows = saved;
    return gx * gy;
}

// a case the batch can take: initialised, with markers, matching the batch
int check_case(lbm_batch *b, lbm_handle *h)
{
    if (!h->inited) return handle_error(h, LBM_ERR_STATE, "batch: lbm_init not called");
    for (int w = 0; w < h->nwing; ++w)
        if (!h->have_wing[w]) return handle_error(h, LBM_ERR_STATE, "batch: boundary of a wing not set");
    if (h->nseg < 1) return handle_error(h, LBM_ERR_ARG, "batch: a case without markers");
    if (h->prec != b->prec || h->fbatch != b->fbatch || h->nslots != b->nslots || h->dev != b->dev)
        return handle_error(h, LBM_ERR_ARG, "batch: cases must share storage precision, factorization batch and device");
    for (lbm_handle *o : b->cases)
        if (o == h) return handle_error(h, LBM_ERR_ARG, "batch: the case is already in the batch");
    int rc = handle_prepare_ib(h);
    if (rc) return rc;
    // the case's own queued work is done before the batch's streams use its buffers
    if (h->fstream) cudaStreamSynchronize(h->fstream);
    if (h->side) cudaStreamSynchronize(h->side);
    if (h->cstream) cudaStreamSynchronize(h->cstream);
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return handle_error(h, LBM_ERR_CUDA, "batch: sync");
    return LBM_OK;
}

int add_case(lbm_batch *b, lbm_handle *h)
{
    if (b->cases.empty() && (b->prec != h->prec || b->fbatch != h->fbatch || b->nslots != h->nslots)) {
        // an empty batch takes the settings of the case that joins it
        if (b->prec >= 0) {
            sync_streams(b);
            free_arrays(b);
        }
        b->prec = h->prec;
        b->fbatch = h->fbatch;
        b->nslots = h->nslots;
        b->kf_sz = kf_args_size(b->prec);
    }
    int rc = check_case(b, h);
    if (rc) return rc;
    int need = table_need(h);
    for (lbm_handle *o : b->cases) need += table_need(o);
    if ((rc = reserve(b, (int)b->cases.size() + 1, need))) return rc;
    b->cases.push_back(h);
    sync_streams(b);
    clear_graphs(b);
    return LBM_OK;
}

}  // namespace

extern "C" {

int lbm_batch_create(lbm_t *const *cases, int count, lbm_batch_t **out)
{
    if (!out || count < 0 || (count > 0 && !cases)) return LBM_ERR_ARG;
    *out = nullptr;
    for (int c = 0; c < count; ++c)
        if (!cases[c]) return LBM_ERR_ARG;
    lbm_batch *b = new lbm_batch;
    if (count > 0)
        b->dev = cases[0]->dev;
    else
        cudaGetDevice(&b->dev);
    b->ib_sz = ib_args_size();
    cudaError_t e;
    int prio_low = 0, prio_high = 0;
    auto fail = [&](cudaError_t err, const char *what) {
        if (count > 0) cases[0]->err = std::string("batch: ") + what + ": " + cudaGetErrorString(err);
        free_batch(b);
        delete b;
        return LBM_ERR_CUDA;
    };
    if ((e = cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high)) != cudaSuccess) return fail(e, "priorities");
    if ((e = cudaStreamCreateWithFlags(&b->main, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    if ((e = cudaStreamCreateWithPriority(&b->side, cudaStreamNonBlocking, prio_high)) != cudaSuccess)
        return fail(e, "stream");
    if ((e = cudaStreamCreateWithFlags(&b->fstream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e, "stream");
    if ((e = cudaStreamCreateWithPriority(&b->cstream, cudaStreamNonBlocking, prio_high)) != cudaSuccess)
        return fail(e, "stream");
    for (cudaEvent_t *ev : {&b->ev_t0, &b->ev_t1})
        if ((e = cudaEventCreate(ev)) != cudaSuccess) return fail(e, "event");
    if (const char *ev = getenv("LBM_AFTER_INTERP")) b->after_interp = atoi(ev) != 0;
    if (const char *ev = getenv("LBM_BATCH_GRAPHS")) b->graphs = atoi(ev) != 0;
    for (cudaEvent_t *ev : {&b->ev_interp, &b->ev_ib, &b->ev_done, &b->ev_fready, &b->ev_side, &b->ev_tup[0], &b->ev_tup[1],
                            &b->ev_tuse[0], &b->ev_tuse[1], &b->ev_gdone[0], &b->ev_gdone[1], &b->ev_gpre,
                            &b->ev_bcheck[0], &b->ev_bcheck[1], &b->ev_cpre})
        if ((e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    for (cudaEvent_t &ev : b->ev_cap)
        if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    for (int q = 0; q < kArgRing; ++q)
        for (cudaEvent_t *ev : {&b->ev_upload[q], &b->ev_kdone[q]})
            if ((e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming)) != cudaSuccess) return fail(e, "event");
    for (int r = 0; r < kFactorRing; ++r)
        if ((e = cudaEventCreateWithFlags(&b->ev_fup[r], cudaEventDisableTiming)) != cudaSuccess)
            return fail(e, "event");
    for (int r = 0; r < kGroupRing; ++r)
        if ((e = cudaEventCreateWithFlags(&b->ev_group[r], cudaEventDisableTiming)) != cudaSuccess)
            return fail(e, "event");
    for (int c = 0; c < count; ++c) {
        const int rc = add_case(b, cases[c]);
        if (rc) {
            free_batch(b);
            delete b;
            return rc;
        }
    }
    *out = b;
    return LBM_OK;
}

int lbm_batch_add(lbm_batch_t *b, lbm_t *h)
{
    if (!b || !h) return LBM_ERR_ARG;
    return add_case(b, h);
}

int lbm_batch_remove(lbm_batch_t *b, lbm_t *h)
{
    if (!b || !h) return LBM_ERR_ARG;
    auto it = std::find(b->cases.begin(), b->cases.end(), h);
    if (it == b->cases.end()) return berr(b, LBM_ERR_ARG, "batch: the case is not in the batch");
    sync_streams(b);
    b->cases.erase(it);
    clear_graphs(b);
    return LBM_OK;
}

int lbm_batch_count(const lbm_batch_t *b) { return b ? (int)b->cases.size() : LBM_ERR_ARG; }

int lbm_batch_case_status(const lbm_batch_t *b, int c)
{
    if (!b || c < 0 || c >= (int)b->status.size()) return LBM_ERR_ARG;
    return b->status[c];
}

int lbm_batch_destroy(lbm_batch_t *b)
{
    if (!b) return LBM_ERR_ARG;
    free_batch(b);
    delete b;
    return LBM_OK;
}

int lbm_batch_get_timing(const lbm_batch_t *b, double *ms, int *steps)
{
    if (!b) return LBM_ERR_ARG;
    if (ms) *ms = b->last_ms;
    if (steps) *steps = b->last_steps;
    return LBM_OK;
}

int lbm_batch_set_occupancy(lbm_batch_t *b, int ctas_per_sm)
{
    if (!b || ctas_per_sm < 0 || ctas_per_sm > 8) return LBM_ERR_ARG;
    b->ctas_per_sm = ctas_per_sm;
    return LBM_OK;
}

int lbm_batch_set_graphs(lbm_batch_t *b, int enable)
{
    if (!b) return LBM_ERR_ARG;
    b->graphs = enable != 0;
    return LBM_OK;
}

int lbm_batch_graph_stats(const lbm_batch_t *b, long long *graph_steps, long long *graph_launches,
                          long long *graph_builds)
{
    if (!b) return LBM_ERR_ARG;
    if (graph_steps) *graph_steps = b->graph_steps;
    if (graph_launches) *graph_launches = b->graph_launches;
    if (graph_builds) *graph_builds = b->graph_builds;
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
    b->status.assign(nc, LBM_OK);
    if (nsteps == 0 || nc == 0) return LBM_OK;
    const int K = b->fbatch;
    std::vector<int> rows_saved(nc), last_step(nc), done(nc, 0), start(nc, 0);
    for (int c = 0; c < nc; ++c) {
        lbm_handle *h = b->cases[c];
        rows_saved[c] = h->kf_rows;
        if (b->rows_per_cta > 0) h->kf_rows = b->rows_per_cta;
        const double dt = h->p.scale * h->p.uu;
        last_step[c] = (int)std::floor((h->mend + 1.0e-12) / dt) + 1;   // last step with time <= mend
    }
    auto restore = [&]() {
        for (int c = 0; c < nc; ++c) b->cases[c]->kf_rows = rows_saved[c];
    };
    // a case may have been stepped alone or re-initialised since the last
    // run: its scratch is (re)made, its own queued work finished, and the
    // case table sized for this run's rows per CTA
    int need = 0;
    for (int c = 0; c < nc; ++c) {
        lbm_handle *h = b->cases[c];
        const int rc0 = h->inited ? handle_prepare_ib(h) : handle_error(h, LBM_ERR_STATE, "batch: lbm_init not called");
        if (rc0) {
            restore();
            return berr(b, rc0, std::string("batch: case ") + std::to_string(c) + ": " + h->err);
        }
        if (h->fstream) cudaStreamSynchronize(h->fstream);
        if (h->side) cudaStreamSynchronize(h->side);
        if (h->cstream) cudaStreamSynchronize(h->cstream);
        cudaStreamSynchronize(h->stream);
        int gx, gy;
        kf_tma_grid(h, &gx, &gy);
        need += gx * gy;
    }
    if (const int rc0 = reserve(b, nc, need)) {
        restore();
        return rc0;
    }
    // One launch chain factorizes, for every case that needs it, the batch of
    // steps bi*K .. bi*K+K-1 of that case (each case its own bi) into the
    // case's slot half bi & 1. It follows the side stream's work so far on
    // the factor stream (which finished every earlier use of those halves);
    // the launch's event in the group ring marks it done, and each case
    // remembers which launch filled each half.
    const long long seq_start = b->gseq;
    auto factor_needed = [&](const std::vector<lbm_handle *> &act, const std::vector<int> &idx, bool next) -> int {
        std::vector<lbm_handle *> grp;
        std::vector<int> grp_bi;
        for (size_t c = 0; c < act.size(); ++c) {
            lbm_handle *h = act[c];
            const int bi = h->n / K + (next ? 1 : 0);
            if (h->batch_in_half[bi & 1] == bi) continue;
            if (next && bi * K > last_step[idx[c]]) continue;
            grp.push_back(h);
            grp_bi.push_back(bi);
        }
        if (grp.empty()) return LBM_OK;
        const int r = b->fring;
        b->fring = (b->fring + 1) % kFactorRing;
        BCK(cudaStreamWaitEvent(b->fstream, b->ev_side, 0), "wait");
        BCK(cudaEventSynchronize(b->ev_fup[r]), "sync upload");   // this staging buffer's previous upload
        for (size_t c = 0; c < grp.size(); ++c) {
            const int s0 = std::max(1, grp_bi[c] * K);   // steps start at 1
            ib_factor_args_write(grp[c], s0, grp_bi[c] * K + K - s0, (char *)b->h_fargs[r] + c * b->ib_sz);
        }
        BCK(cudaMemcpyAsync(b->d_fargs[r], b->h_fargs[r], grp.size() * b->ib_sz, cudaMemcpyHostToDevice, b->fstream),
            "upload");
        BCK(cudaEventRecord(b->ev_fup[r], b->fstream), "event");
        if (launch_factor_batch(grp.data(), (int)grp.size(), b->d_fargs[r], 0, K, b->fstream))
            return berr(b, LBM_ERR_CUDA, "batch: launch factor");
        const long long seq = ++b->gseq;
        BCK(cudaEventRecord(b->ev_group[seq % kGroupRing], b->fstream), "event");
        for (size_t c = 0; c < grp.size(); ++c) {
            const int half = grp_bi[c] & 1;
            grp[c]->batch_in_half[half] = grp_bi[c];
            grp[c]->fgroup[half] = seq;
        }
        return LBM_OK;
    };
    int rc = LBM_OK, pending = 0, step = 0;
    // copies the force rows of the steps since the last flush (ring rows
    // 0 .. rows-1, each case its own count) and reads the cases' status
    auto flush = [&]() -> int {
        BCK(cudaStreamWaitEvent(b->main, b->ev_side, 0), "wait");
        for (int c = 0; c < nc; ++c) {
            lbm_handle *h = b->cases[c];
            const int rows = done[c] - start[c];
            if (force_rows && force_rows[c] && rows > 0)
                BCK(cudaMemcpyAsync(force_rows[c] + (size_t)start[c] * h->row_len, h->d_ring,
                                    sizeof(double) * h->row_len * rows, cudaMemcpyDeviceToHost, b->main),
                    "copy force rows");
        }
        BCK(cudaStreamSynchronize(b->main), "sync");
        pending = 0;
        int st0 = LBM_OK;
        for (int c = 0; c < nc; ++c) {
            start[c] = done[c];
            const int st = handle_status(b->cases[c]);
            if (st) b->status[c] = st;
            if (st && !st0) {
                st0 = st;
                b->err = std::string("batch: case ") + std::to_string(c) + ": " + b->cases[c]->err;
            }
        }
        return st0;
    };
    std::vector<lbm_handle *> act, prev_act;
    std::vector<int> act_idx;
    int tcur = -1, ntab = 0;           // table buffer in use, its entries
    bool cons0 = true;                 // every case's conserved-moment relaxation rates are zero
    for (lbm_handle *h : b->cases) cons0 = cons0 && h->s[0] == 0.0 && h->s[3] == 0.0 && h->s[5] == 0.0;
    // One CUDA graph segment of kGraphSteps steps from `step` (the caller has
    // checked that it may run one: the same active cases and case table as
    // the step before, no fields, room in the force ring). The host plans the
    // segment as the stream code would issue it (factorization groups, the
    // waits on them, every step's arguments), writes the arguments into the
    // host copy of one of the two segment buffers, and launches the graph of
    // that structure, which it captures and instantiates first when new.
    struct GroupPlan {
        std::vector<int> members;   // active-case indices
        long long seq = 0;
        size_t off = 0;             // arguments in the segment buffer
    };
    struct StepPlan {
        int cur = -1, next = -1;    // factorization groups before / after the flow chain
        std::vector<int> waits;     // groups of this segment the flow chain waits for
        bool residual = false;      // some case checks its solve residual
    };
    auto graph_segment = [&]() -> int {
        const int G = kGraphSteps, na = (int)act.size();
        const int sb = b->gset;
        b->gset ^= 1;
        BCK(cudaEventSynchronize(b->ev_gdone[sb]), "sync segment");   // the last graph that read this buffer
        char *hs = (char *)b->h_seg[sb], *ds = (char *)b->d_seg[sb];
        const size_t off_k = round256((size_t)G * na * b->ib_sz);
        const size_t off_f = off_k + round256((size_t)G * na * b->kf_sz);
        std::vector<GroupPlan> groups;
        std::vector<StepPlan> plan(G);
        const long long seq_seg = b->gseq;   // groups numbered above it are the segment's own
        // a factorization group, chosen as factor_needed chooses it
        auto plan_factor = [&](bool next) -> int {
            GroupPlan g;
            for (int c = 0; c < na; ++c) {
                lbm_handle *h = act[c];
                const int bi = h->n / K + (next ? 1 : 0);
                if (h->batch_in_half[bi & 1] == bi) continue;
                if (next && bi * K > last_step[act_idx[c]]) continue;
                g.members.push_back(c);
            }
            if (g.members.empty()) return -1;
            g.off = off_f + groups.size() * (size_t)na * b->ib_sz;   // at most two groups a step
            g.seq = ++b->gseq;
            for (size_t m = 0; m < g.members.size(); ++m) {
                lbm_handle *h = act[g.members[m]];
                const int bi = h->n / K + (next ? 1 : 0);
                const int s0 = std::max(1, bi * K);   // steps start at 1
                ib_factor_args_write(h, s0, bi * K + K - s0, hs + g.off + m * b->ib_sz);
                h->batch_in_half[bi & 1] = bi;
                h->fgroup[bi & 1] = g.seq;
            }
            groups.push_back(std::move(g));
            return (int)groups.size() - 1;
        };
        for (int t = 0; t < G; ++t) {
            StepPlan &p = plan[t];
            p.cur = plan_factor(false);
            // groups from before the segment are complete when the graph starts
            for (int c = 0; c < na; ++c) {
                const long long g = act[c]->fgroup[(act[c]->n / K) & 1];
                const int gi = (int)(g - seq_seg - 1);
                if (g > seq_seg && std::find(p.waits.begin(), p.waits.end(), gi) == p.waits.end()) p.waits.push_back(gi);
            }
            for (int c = 0; c < na; ++c) {
                lbm_handle *h = act[c];
                const int q = h->n % b->nslots;
                h->pinfo_slot = q;
                IBArgs *ia = (IBArgs *)(hs + ((size_t)t * na + c) * b->ib_sz);
                ib_args_write(h, h->fbuf[h->cur], q, ia);
                // a segment holds neither the call's nor a case's last step
                ia->check_res = (h->n + 1) % K == 0;
                p.residual = p.residual || ia->check_res;
                ia->ring_row = pending + t;
                kf_args_write(h, h->fbuf[h->cur], h->fbuf[h->cur ^ 1], nullptr, KF_OUTER,
                              hs + off_k + ((size_t)t * na + c) * b->kf_sz);
            }
            p.next = plan_factor(true);
            for (int c = 0; c < na; ++c) {
                lbm_handle *h = act[c];
                h->cur ^= 1;
                h->n++;
                h->steps_done++;
                done[act_idx[c]]++;
            }
        }
        const size_t used = off_f + groups.size() * (size_t)na * b->ib_sz;
        // the structure: what sets grid sizes, kernel variants, buffer
        // addresses and the graph's edges
        std::vector<long long> sig = {sb, G, na, b->prec, cons0, b->after_interp, tcur, ntab, K, (long long)used,
                                      b->ctas_per_sm};
        for (lbm_handle *h : act)
            sig.insert(sig.end(), {(long long)(uintptr_t)h, h->nseg, h->patch_gx(), h->patch_gy(), h->static_order});
        for (const StepPlan &p : plan) {
            sig.insert(sig.end(), {p.cur, p.next, (long long)p.residual, (long long)p.waits.size()});
            sig.insert(sig.end(), p.waits.begin(), p.waits.end());
        }
        for (const GroupPlan &g : groups) {
            sig.push_back((long long)g.members.size());
            sig.insert(sig.end(), g.members.begin(), g.members.end());
        }
        // the segment's stream code: the per-step sequence of the stream path
        // below, with every dependency inside the segment
        auto emit = [&]() -> int {
            cudaEvent_t *E = b->ev_cap;
            // the checks of steps t (parity t & 1) and the check stream's join
            cudaEvent_t *EC = b->ev_cap + 9 + 2 * kGraphSteps;
            BCK(cudaMemcpyAsync(ds, hs, used, cudaMemcpyHostToDevice, b->side), "upload");
            BCK(cudaEventRecord(E[1], b->side), "event");
            BCK(cudaStreamWaitEvent(b->main, E[1], 0), "wait");
            BCK(cudaStreamWaitEvent(b->fstream, E[1], 0), "wait");
            BCK(cudaStreamWaitEvent(b->cstream, E[1], 0), "wait");
            cudaEvent_t ei = b->after_interp ? E[8] : nullptr;
            std::vector<lbm_handle *> grp;
            auto factor = [&](int gi, bool after_side) -> int {
                grp.clear();
                for (int m : groups[gi].members) grp.push_back(act[m]);
                if (after_side) BCK(cudaStreamWaitEvent(b->fstream, E[6], 0), "wait");
                if (launch_factor_batch(grp.data(), (int)grp.size(), ds + groups[gi].off, 0, K, b->fstream))
                    return berr(b, LBM_ERR_CUDA, "batch: launch factor");
                BCK(cudaEventRecord(E[9 + gi], b->fstream), "event");
                return LBM_OK;
            };
            int erc = LBM_OK;
            for (int t = 0; t < G; ++t) {
                const StepPlan &p = plan[t];
                if (p.cur >= 0 && (erc = factor(p.cur, t > 0))) return erc;
                if (t > 0) BCK(cudaStreamWaitEvent(b->side, E[7], 0), "wait");
                for (int gi : p.waits) BCK(cudaStreamWaitEvent(b->side, E[9 + gi], 0), "wait");
                BCK(cudaEventRecord(E[4], b->side), "event");
                // the checks two steps back (those before the segment are done
                // when it starts)
                if (t >= 2) BCK(cudaStreamWaitEvent(b->side, EC[t & 1], 0), "wait");
                const char *sa = ds + (size_t)t * na * b->ib_sz;
                const char *ka = ds + off_k + (size_t)t * na * b->kf_sz;
                if (launch_flow_batch(act.data(), na, sa, ka, 0, 0, false, b->side, ei))
                    return berr(b, LBM_ERR_CUDA, "batch: launch flow");
                BCK(cudaEventRecord(E[5], b->side), "event");
                BCK(cudaStreamWaitEvent(b->cstream, E[5], 0), "wait");
                if (launch_check_batch(act.data(), na, sa, 0, p.residual, b->cstream))
                    return berr(b, LBM_ERR_CUDA, "batch: launch check");
                BCK(cudaEventRecord(EC[t & 1], b->cstream), "event");
                BCK(cudaEventRecord(E[6], b->cstream), "event");   // flow chains and checks of step t
                if (p.next >= 0 && (erc = factor(p.next, true))) return erc;
                BCK(cudaStreamWaitEvent(b->main, E[4], 0), "wait");
                if (ei) BCK(cudaStreamWaitEvent(b->main, ei, 0), "wait");   // the solves start first
                if (launch_kf_multi(b->prec, ka, b->d_table[tcur], ntab, false, cons0, b->ctas_per_sm, b->main))
                    return berr(b, LBM_ERR_CUDA, "batch: launch lattice");
                for (lbm_handle *h : act) h->launches += 1;
                BCK(cudaStreamWaitEvent(b->main, E[5], 0), "wait");
                BCK(cudaEventRecord(E[7], b->main), "event");   // the step is complete
            }
            BCK(cudaEventRecord(E[2], b->main), "event");
            BCK(cudaEventRecord(E[3], b->fstream), "event");
            BCK(cudaEventRecord(EC[2], b->cstream), "event");
            BCK(cudaStreamWaitEvent(b->side, E[2], 0), "wait");
            BCK(cudaStreamWaitEvent(b->side, E[3], 0), "wait");
            BCK(cudaStreamWaitEvent(b->side, EC[2], 0), "wait");
            return LBM_OK;
        };
        // the graph starts after every stream's earlier work
        BCK(cudaEventRecord(b->ev_gpre, b->fstream), "event");
        BCK(cudaEventRecord(b->ev_cpre, b->cstream), "event");
        BCK(cudaStreamWaitEvent(b->side, b->ev_done, 0), "wait");
        BCK(cudaStreamWaitEvent(b->side, b->ev_gpre, 0), "wait");
        BCK(cudaStreamWaitEvent(b->side, b->ev_cpre, 0), "wait");
        lbm_batch::GraphEntry *ge = nullptr;
        for (auto &e : b->gcache)
            if (e.sig == sig) {
                ge = &e;
                break;
            }
        if (!ge) {
            lbm_batch::GraphEntry e;
            e.sig = std::move(sig);
            std::vector<long long> l0(na);
            for (int c = 0; c < na; ++c) l0[c] = act[c]->launches;
            cudaGraph_t graph = nullptr;
            BCK(cudaStreamBeginCapture(b->side, cudaStreamCaptureModeThreadLocal), "graph capture");
            // the capture ends whatever emit returns, so that the streams
            // are usable again
            const int erc = emit();
            const cudaError_t ce = cudaStreamEndCapture(b->side, &graph);
            if (erc == LBM_OK && ce == cudaSuccess) {
                const cudaError_t ie = cudaGraphInstantiate(&e.exec, graph, 0);
                cudaGraphDestroy(graph);
                if (ie != cudaSuccess) return berr(b, LBM_ERR_CUDA, std::string("batch: graph instantiate: ") + cudaGetErrorString(ie));
            } else {
                if (graph) cudaGraphDestroy(graph);
                cudaGetLastError();
                return erc ? erc : berr(b, LBM_ERR_CUDA, std::string("batch: graph capture: ") + cudaGetErrorString(ce));
            }
            e.launches.resize(na);
            for (int c = 0; c < na; ++c) {
                e.launches[c] = act[c]->launches - l0[c];
                act[c]->launches = l0[c];
            }
            if ((int)b->gcache.size() >= kGraphCache) {
                cudaGraphExecDestroy(b->gcache.front().exec);
                b->gcache.erase(b->gcache.begin());
            }
            b->gcache.push_back(std::move(e));
            ge = &b->gcache.back();
            b->graph_builds++;
        }
        BCK(cudaGraphLaunch(ge->exec, b->side), "graph launch");
        for (int c = 0; c < na; ++c) act[c]->launches += ge->launches[c];
        b->graph_launches++;
        b->graph_steps += G;
        // the stream code after the graph sees it as its previous step
        BCK(cudaEventRecord(b->ev_gdone[sb], b->side), "event");
        BCK(cudaEventRecord(b->ev_done, b->side), "event");
        BCK(cudaEventRecord(b->ev_side, b->side), "event");
        BCK(cudaEventRecord(b->ev_tuse[tcur], b->side), "event");
        BCK(cudaEventRecord(b->ev_bcheck[0], b->side), "event");
        BCK(cudaEventRecord(b->ev_bcheck[1], b->side), "event");
        for (const GroupPlan &g : groups) BCK(cudaEventRecord(b->ev_group[g.seq % kGroupRing], b->side), "event");
        BCK(cudaStreamWaitEvent(b->main, b->ev_done, 0), "wait");
        BCK(cudaStreamWaitEvent(b->fstream, b->ev_side, 0), "wait");
        BCK(cudaStreamWaitEvent(b->cstream, b->ev_side, 0), "wait");
        return LBM_OK;
    };
    BCK(cudaEventRecord(b->ev_done, b->main), "event");
    BCK(cudaEventRecord(b->ev_side, b->side), "event");
    BCK(cudaEventRecord(b->ev_t0, b->main), "event");
    b->last_ms = 0.0;
    b->last_steps = 0;
    std::vector<long long> waited;
    std::vector<int> tkey, tkey_now;   // grids of the active cases the current table was built for
    const int ring_cap = b->cases[0]->ring_cap;
    for (; step < nsteps; ++step) {
        prev_act.swap(act);
        act.clear();
        act_idx.clear();
        for (int c = 0; c < nc; ++c)
            if (b->cases[c]->n <= last_step[c]) {
                act.push_back(b->cases[c]);
                act_idx.push_back(c);
            }
        if (act.empty()) break;
        // a graph segment where the next kGraphSteps steps allow one
        if (b->graphs && tcur >= 0 && act == prev_act && step + kGraphSteps <= nsteps - 2 &&
            pending + kGraphSteps <= ring_cap) {
            bool ok = true;
            for (size_t c = 0; c < act.size() && ok; ++c) ok = act[c]->n + kGraphSteps < last_step[act_idx[c]];
            if (ok) {
                if ((rc = graph_segment())) break;
                step += kGraphSteps - 1;
                pending += kGraphSteps;
                if (pending == ring_cap && (rc = flush())) break;
                continue;
            }
        }
        const int buf = step % kArgRing;
        // fields (rho, u, v) for the last two steps of the call and of every
        // case that ends within them (all active cases keep them then)
        bool fields = step >= nsteps - 2;
        for (size_t c = 0; c < act.size() && !fields; ++c) fields = act[c]->n >= last_step[act_idx[c]] - 1;
        if ((rc = factor_needed(act, act_idx, false))) break;
        // this step's arguments (the staging buffer's previous upload, kArgRing
        // steps back, is done)
        BCK(cudaEventSynchronize(b->ev_upload[buf]), "sync upload");
        tkey_now.clear();
        bool any_check = false;   // some case checks its solve residual this step
        for (size_t c = 0; c < act.size(); ++c) {
            lbm_handle *h = act[c];
            const int q = h->n % b->nslots;
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
            IBArgs *ia = (IBArgs *)((char *)b->h_sargs[buf] + c * b->ib_sz);
            ib_args_write(h, fin, q, ia);
            // the solve-residual check: last step of the case's factorization
            // batch, of the call, or of the case's motion
            ia->check_res = (h->n + 1) % K == 0 || step == nsteps - 1 || h->n >= last_step[act_idx[c]];
            any_check = any_check || ia->check_res;
            ia->ring_row = pending;
            kf_args_write(h, fin, fout, fd, KF_OUTER, (char *)b->h_kargs[buf] + c * b->kf_sz);
            int gx, gy;
            kf_tma_grid(h, &gx, &gy);
            tkey_now.push_back(gx | (gy << 16));
        }
        // the case table, built again only when the active cases change; the
        // other of its two buffers is reused once its last reader is done
        if (tcur < 0 || tkey_now != tkey) {
            const int k = tcur < 0 ? 0 : tcur ^ 1;
            BCK(cudaEventSynchronize(b->ev_tup[k]), "sync upload");
            ntab = 0;
            for (size_t c = 0; c < act.size(); ++c) {
                const int gx = tkey_now[c] & 0xffff, gy = tkey_now[c] >> 16;
                if (ntab + gx * gy > b->table_cap) {
                    rc = berr(b, LBM_ERR_STATE, "batch: case table overflow");
                    break;
                }
                for (int by = 0; by < gy; ++by)
                    for (int bx = 0; bx < gx; ++bx) b->h_table[k][ntab++] = make_int4((int)c, bx, by, tkey_now[c]);
            }
            if (rc) break;
            BCK(cudaStreamWaitEvent(b->side, b->ev_tuse[k], 0), "wait");
            BCK(cudaMemcpyAsync(b->d_table[k], b->h_table[k], sizeof(int4) * ntab, cudaMemcpyHostToDevice, b->side),
                "upload");
            BCK(cudaEventRecord(b->ev_tup[k], b->side), "event");
            tcur = k;
            tkey = tkey_now;
        }
        // side stream: the uploads (once the lattice launch that last read this
        // buffer is done), then, after the previous step, the flow chains
        BCK(cudaStreamWaitEvent(b->side, b->ev_kdone[buf], 0), "wait");
        BCK(cudaMemcpyAsync(b->d_sargs[buf], b->h_sargs[buf], act.size() * b->ib_sz, cudaMemcpyHostToDevice, b->side),
            "upload");
        BCK(cudaMemcpyAsync(b->d_kargs[buf], b->h_kargs[buf], act.size() * b->kf_sz, cudaMemcpyHostToDevice, b->side),
            "upload");
        BCK(cudaEventRecord(b->ev_upload[buf], b->side), "event");
        BCK(cudaStreamWaitEvent(b->side, b->ev_done, 0), "wait");
        // the factorization launches of this step's halves (those of earlier
        // runs are complete: every run ends with its streams idle)
        waited.clear();
        for (lbm_handle *h : act) {
            const long long g = h->fgroup[(h->n / K) & 1];
            if (g > seq_start && std::find(waited.begin(), waited.end(), g) == waited.end()) {
                BCK(cudaStreamWaitEvent(b->side, b->ev_group[g % kGroupRing], 0), "wait");
                waited.push_back(g);
            }
        }
        BCK(cudaEventRecord(b->ev_fready, b->side), "event");   // uploads done, factorizations ready
        // the cases' buffers of this step's parity were last read by the
        // checks two steps back
        BCK(cudaStreamWaitEvent(b->side, b->ev_bcheck[step & 1], 0), "wait");
        cudaEvent_t ei = b->after_interp ? b->ev_interp : nullptr;
        if (launch_flow_batch(act.data(), (int)act.size(), b->d_sargs[buf], b->d_kargs[buf], 0, pending, fields,
                              b->side, ei)) {
            rc = berr(b, LBM_ERR_CUDA, "batch: launch flow");
            break;
        }
        BCK(cudaEventRecord(b->ev_ib, b->side), "event");
        BCK(cudaStreamWaitEvent(b->cstream, b->ev_ib, 0), "wait");
        if (launch_check_batch(act.data(), (int)act.size(), b->d_sargs[buf], pending, any_check, b->cstream)) {
            rc = berr(b, LBM_ERR_CUDA, "batch: launch check");
            break;
        }
        BCK(cudaEventRecord(b->ev_bcheck[step & 1], b->cstream), "event");
        BCK(cudaEventRecord(b->ev_side, b->cstream), "event");
        // the next factorization batches, overlapping these steps
        if ((rc = factor_needed(act, act_idx, true))) break;
        // main stream: every case's lattice nodes but its correction tiles
        BCK(cudaStreamWaitEvent(b->main, b->ev_fready, 0), "wait");
        if (ei) BCK(cudaStreamWaitEvent(b->main, ei, 0), "wait");   // the solves start first
        if (launch_kf_multi(b->prec, b->d_kargs[buf], b->d_table[tcur], ntab, fields, cons0, b->ctas_per_sm,
                            b->main)) {
            rc = berr(b, LBM_ERR_CUDA, "batch: launch lattice");
            break;
        }
        BCK(cudaEventRecord(b->ev_kdone[buf], b->main), "event");
        BCK(cudaEventRecord(b->ev_tuse[tcur], b->main), "event");
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
        // force rows to the host every ring's worth of steps
        if (pending == ring_cap) {
            if ((rc = flush())) break;
        }
    }
    // device time of the steps: from before the first step's launches to the
    // end of the last step's side-stream work
    if (step > 0 && rc == LBM_OK) {
        BCK(cudaStreamWaitEvent(b->main, b->ev_side, 0), "wait");
        BCK(cudaEventRecord(b->ev_t1, b->main), "event");
    }
    // the rows of the last steps (also when every case ended before nsteps)
    if (pending > 0 && rc == LBM_OK) rc = flush();
    // the global mass of every case that ran, at the end of the run (FP64 on
    // the device; a non-finite mass fails that case)
    if (rc == LBM_OK) {
        std::vector<double> dsum(nc, 0.0);
        for (int c = 0; c < nc && rc == LBM_OK; ++c)
            if (done[c] > 0) rc = handle_mass_launch(b->cases[c], b->main, &dsum[c]);
        if (rc == LBM_OK) {
            BCK(cudaStreamSynchronize(b->main), "sync mass");
            for (int c = 0; c < nc; ++c) {
                const int st = done[c] > 0 ? handle_mass_result(b->cases[c], dsum[c]) : LBM_OK;
                if (st) {
                    b->status[c] = st;
                    if (rc == LBM_OK) {
                        rc = st;
                        b->err = std::string("batch: case ") + std::to_string(c) + ": " + b->cases[c]->err;
                    }
                }
            }
        } else {
            b->err = std::string("batch: mass check: ") + b->cases[0]->err;
        }
    }
    // leave every stream idle: the cases' own calls follow on their streams
    sync_streams(b);
    if (step > 0 && rc == LBM_OK) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, b->ev_t0, b->ev_t1) == cudaSuccess) {
            b->last_ms = ms;
            b->last_steps = step;
        }
    }
    restore();
    if (done_steps)
        for (int c = 0; c < nc; ++c) done_steps[c] = done[c];
    for (int c = 0; c < nc && rc == LBM_OK; ++c)
        if (done[c] < nsteps) rc = LBM_DONE;
    return rc;
}

const char *lbm_batch_last_error(const lbm_batch_t *b) { return b ? b->err.c_str() : ""; }

}  // extern "C"
