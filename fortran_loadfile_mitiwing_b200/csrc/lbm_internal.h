// lbm_internal.h -- handle layout and kernel launchers (not part of the ABI).
#pragma once
#include <cuda_runtime.h>
#include <string>
#include <vector>

#include "../../include/lbm_b200.h"
#include "lbm_common.cuh"

// constants of the left/right columns that never change after init: the
// moments of the edge f0 that streaming never rewrites (solution.f90:440-447,
// 516-520), and the edge f0 populations the top/bottom extrapolation reads at
// the corner columns (boundary_condition.f90:705, 832).
struct EdgeConst {
    double *col_l;   // [3*ny]: drho, u, v of column 1 (1-based)
    double *col_r;   // [3*ny]: column Nx
    double *corner;  // [4*9] deviation f0 at (1,2), (1,Ny-1), (Nx,2), (Nx,Ny-1)
};

// arguments of the fused stream+collide+boundary kernel
template <typename C>
struct KFArgs {
    const void *fin;
    void *fout;
    int nx, ny, pitch;
    long long plane;
    C s[9];
    C sc[9];   // s[k] times row k of the inverse transform's scale, signed for the paired update
    C cs;
    const C *col_l, *col_r, *corner;   // edge constants in compute precision
    const PatchInfo *pinfo;            // the step's patch rectangle (KF_OUTER)
    const int *tiles;                  // the step's tile lists: count per 16 x 16 tile (KF_OUTER)
    int tiles_x, tile_stride;          // tiles per rectangle row; ints per tile
    int tiles_n;                       // tiles of the grid (bound of the tile index)
    C *rho_out, *u_out, *v_out;        // fields, when requested (else null)
    int mode;                          // KF_ALL, or KF_OUTER (all but the correction tiles)
    int rows_per_cta;                  // row sweep length of the staged kernel
    unsigned *status;                  // device status word (bounded-wait timeouts)
};

#define LBM_NSLOT_MAX 16   // largest slot count of the factorization batches
#define LBM_FPAD 64   // elements of padding before and after the population planes

#define KF_ALL 0
#define KF_OUTER 1


// arguments of the immersed-boundary kernels
struct IBArgs {
    const void *fin;    // populations the step streams from
    int prec;           // LBM_PREC_*
    int nx, ny, pitch;
    long long plane;
    int nwing, ppw, spw, nseg;
    int smooth;
    int force_dense;    // LBM_FLAG_DENSE_SOLVE
    double scale, ox, oy, uu, xc, yc, mesh_max_scale;
    const double *xb0, *yb0, *arc;
    const double *mstep;  // step table, row-major [msteps][mcols]
    int msteps, mcols;
    double mdt;
    // buffers of one slot (the step whose factorization they hold)
    Marker *mk;         // [nseg] marker geometry
    int *perm;          // solve order: sorted position -> marker
    double *key;        // sort key of each sorted position
    double *gf;         // factor blocks [D^-1 | F_L | F_U] of the cyclic reduction
    double *B;          // [nseg*nseg] dense Cholesky factor (fallback), row-major
    int *fmode;         // [2]: 1 if the dense factor is used, half-bandwidth
    unsigned *fstatus;  // errors of the factorization chain of the slot's step
    // per step
    double *rhs;        // [2*nseg]
    double *y;          // [2*nseg]
    double *bD, *bL;    // working diagonal and coupling blocks of the reduction
    double *reach;      // key distance beyond which boxes cannot overlap
    int *wmax;          // half-bandwidth found by the assembly
    // slot and working-set strides of the batched factorization (elements)
    int nslots;
    int static_order;   // one rigid body: fixed solve order (ib_order leaves it)
    int cur_step;       // step index of the flow chain (batched launches: per case)
    int fstep0, fcount; // steps of the factorization chain (batched launches: per case)
    int check_res;      // batched launches: run the solve-residual check for this case's step
    long long st_mk, st_perm, st_B, wk_blocks, wk_gf;
    PatchInfo *pinfo;
    int *tiles;         // per patch tile: marker count, then the listed markers (slot)
    int tiles_x;        // tiles per patch row
    long long st_tiles; // ints per slot of the tile lists
    int patch_wmax, patch_hmax;  // largest patch rectangle (the tile grid covers it)
    int *nsup;          // number of correction tiles (tiles listing a marker) of the slot's step
    int *ctile;         // their tile indices, in no particular order
    double *partial;    // per-block force partials
    unsigned *counter;  // last-block counter
    double *force_ring; // [ring_cap][row_len]
    int row_len;
    // batched launches: the force-ring row of this case's step (the rows
    // held: ring_rows); single-case launches take the row as a parameter
    int ring_row, ring_rows;
    unsigned *status;
    double *solve_res;  // relative residual of the last solve
};

struct lbm_handle {
    lbm_params p;
    int nx = 0, ny = 0, pitch = 0;
    long long plane = 0;
    int nwing = 0, ppw = 0, spw = 0, npts = 0, nseg = 0;
    double niu = 0, tau = 0, s[9] = {0};
    int prec = 0;
    size_t elem = 4;
    int kf_vec = 1;   // nodes per thread of the register-loading lattice kernel (1, 2 or 4)
    int kf_tma = 1;   // bulk-copy staged lattice kernel (the default)
    int kf_rows = 8;  // rows swept by one CTA of the staged kernel
    int dev = 0;
    cudaStream_t stream = nullptr;
    void *fbuf[2] = {nullptr, nullptr};     // first element of plane 0
    void *falloc[2] = {nullptr, nullptr};   // allocations (fbuf - LBM_FPAD elements)
    int cur = 0;
    // edge constants (FP64 master + compute-precision copy)
    EdgeConst edge{};
    void *edge_c = nullptr;  // compute precision: col_l, col_r, corner packed
    // the edge f0 populations they come from (FP64, full f, 9 per node): left
    // column j = 1..Ny, right column j = 1..Ny, bottom row i = 1..Nx, top row
    // i = 1..Nx (the edge part of the reference's restart file)
    std::vector<double> edge_f0;
    // geometry and motion
    std::vector<double> hx0, hy0, harc;
    std::vector<int> have_wing;
    double *d_xb0 = nullptr, *d_yb0 = nullptr, *d_arc = nullptr;
    std::vector<double> mtab;  // column-major rows x cols, as given
    int mrows = 0, mcols = 0;
    double mend = 0, mdt = 0;
    int msteps = 0;
    std::vector<double> mstep_host;  // step table, row-major [msteps][mcols]
    double *d_mstep = nullptr;
    // immersed boundary scratch. The factorization of a step depends on its
    // index only (prescribed motion). Steps are factorized in batches of
    // fbatch consecutive steps (batch b: steps b*fbatch .. b*fbatch+fbatch-1),
    // each step into slot step % nslots (nslots = 2 fbatch): the next batch
    // is factorized while the steps of the current one run.
    int fbatch = 4, nslots = 8;
    int batch_in_half[2] = {-1, -1};                // batch index held by each half of the slots
    Marker *d_mk = nullptr;                         // nslots x nseg
    double *d_B = nullptr;                          // nslots x nseg*nseg
    int *d_fmode = nullptr;                         // nslots x 2
    unsigned *d_fstatus = nullptr;                  // nslots
    double *d_gf = nullptr;                         // nslots x gf_slot doubles
    size_t gf_slot = 0, work_blocks = 0;
    double *d_rhs = nullptr, *d_y = nullptr;
    double *d_bD = nullptr, *d_bL = nullptr;        // fbatch working sets of work_blocks doubles
    int *d_perm = nullptr, *d_wmax = nullptr;       // perm/key: nslots unless static_order; wmax: fbatch
    double *d_key = nullptr, *d_reach = nullptr;
    int static_order = 0;   // one rigid body: fixed body-frame marker order
    PatchInfo *d_pinfo = nullptr;   // LBM_NSLOT_MAX slots (patch rectangle of the slot's step)
    int *d_tiles = nullptr;         // nslots x tile lists of the patch grid
    size_t tiles_slot = 0;          // ints per slot of d_tiles
    int *d_nsup = nullptr;          // nslots: correction tiles of the slot's step
    int *d_ctile = nullptr;         // nslots x tiles: the correction tiles' indices
    int pinfo_slot = 0;             // slot the next lattice launch reads
    int patch_wmax = 0, patch_hmax = 0;
    int patch_gx() const { return patch_wmax > 0 ? (patch_wmax + 15) / 16 : 1; }
    int patch_gy() const { return patch_hmax > 0 ? (patch_hmax + 15) / 16 : 1; }
    int ib_ready = 0;
    // split of the lattice update around the bodies' motion envelope: the
    // outer part runs concurrently with the immersed-boundary kernels on the
    // side stream, the inner part after them (0-based rectangle, x origin and
    // width multiples of 4)
    int overlap = 1;
    int env_x0 = 0, env_y0 = 0, env_w = 0, env_h = 0;
    cudaStream_t side = nullptr;
    cudaEvent_t ev_ib = nullptr, ev_inner = nullptr;
    // the step's interpolation is done (side stream); with after_interp the
    // lattice kernel waits for it, so that the one-CTA solve that follows
    // finds a whole SM free instead of waiting for lattice CTAs to drain out
    cudaEvent_t ev_interp = nullptr;
    int after_interp = 1;
    // factorization batches (with the split): their own stream; ev_batch[h]
    // marks the batch of slot half h factorized, ev_free[h] the last use of
    // that half by a step's flow chain
    cudaStream_t fstream = nullptr;
    cudaEvent_t ev_batch[2] = {nullptr, nullptr}, ev_free[2] = {nullptr, nullptr};
    // the step's force row and solve-residual check (with the split): their
    // own stream, after the step's correction tiles, so that the next step's
    // flow chain need not wait for them. What they read is kept per step
    // parity (right-hand sides, solution, tile partials, residual slots), and
    // ev_check[p] marks the check of the last step of parity p done.
    cudaStream_t cstream = nullptr;
    cudaEvent_t ev_check[2] = {nullptr, nullptr}, ev_cjoin = nullptr;
    size_t part_stride = 0;   // doubles of one parity's tile partials
    double *d_partial = nullptr;
    unsigned *d_counter = nullptr;
    double *d_ring = nullptr;
    int ring_cap = 0;
    int row_len = 0;
    unsigned *d_status = nullptr;
    double *d_solve_res = nullptr;
    // fields of the last field-writing steps (compute precision), two slots
    void *d_fields[2] = {nullptr, nullptr};
    int fields_slot = 0;           // slot written by the last field step
    int fields_step[2] = {-1, -1}; // step index written into each slot
    double *d_red = nullptr;       // residual reduction scratch
    // global mass check: CTA partials, then the deviation sum (mass_slots()
    // doubles), its last-CTA counter, and the last mass found (host)
    double *d_mass = nullptr;
    unsigned *d_mcount = nullptr;
    double last_mass = 0.0;
    int last_mass_step = -1;
    double *d_stage = nullptr;     // FP64 (nx,ny,9) staging for get/set of populations
    // device timing (lbm_set_timing): per step slot of the ring, four events on
    // the main stream (start, lattice part 1 done, lattice part 2 start, end)
    // and two on the side stream (IB start, IB end)
    int timing = 0;
    std::vector<cudaEvent_t> ev, ev_side;
    double t_step = 0, t_ib = 0, t_kf = 0;
    int t_steps = 0;
    long long launches = 0;   // kernels launched by this handle (lbm_get_launch_count)
    long long dev_bytes = 0;  // device memory the handle holds (lbm_device_bytes)
    long long fgroup[2] = {-1, -1};   // batch factorization launch that filled each slot half
    // driver state
    int n = 1;
    int inited = 0;
    int steps_done = 0;
    std::string err;
};

// kernel launchers (kf_kernel.cu, ib_kernels.cu)
int ib_configure(lbm_handle *h);
int ib_max_markers();
int ib_partials_per_block();
void ib_factor_scratch(int nseg, size_t *work_blocks, size_t *factor_slot);
int launch_kf(lbm_handle *h, const void *fin, void *fout, void *fields, int mode = KF_ALL, cudaStream_t st = nullptr);
int launch_factor(lbm_handle *h, int step0, int count, cudaStream_t st);
// after_interp (nullable): recorded on st once the interpolation is done
int launch_flow(lbm_handle *h, const void *fin, void *fout, void *fields, int step_index, int ring_slot, int slot,
                cudaStream_t st, cudaEvent_t after_interp = nullptr);
int launch_check(lbm_handle *h, int slot, int ring_slot, bool residual, cudaStream_t st);
// batches of cases stepped together (lbm_batch.cu)
int handle_prepare_ib(lbm_handle *h);                    // immersed-boundary buffers (once per geometry)
int handle_error(lbm_handle *h, int code, const char *msg);
int handle_status(lbm_handle *h);                        // reads and clears the device status
// global mass check of a case: queue the sum on st into *dsum, then (after st
// is synchronised) check it
int handle_mass_launch(lbm_handle *h, cudaStream_t st, double *dsum);
int handle_mass_result(lbm_handle *h, double dsum);
// boundary reference values from the edge f0 populations (layout of edge_f0)
int handle_set_edges(lbm_handle *h, const double *edge_f0);
// state of a restart file in the reference's layout: populations f(nx,ny,9),
// velocity fields (density 1, as init leaves it), edge f0; next step cycle+1
int handle_restore(lbm_handle *h, const double *f, const double *u, const double *v, const double *edge_f0,
                   int cycle);
size_t kf_args_size(int prec);
void kf_args_write(lbm_handle *h, const void *fin, void *fout, void *fields, int mode, void *dst);
void kf_tma_grid(const lbm_handle *h, int *gx, int *gy);
// cons0: every case's conserved-moment relaxation rates are zero;
// ctas_per_sm: at most that many CTAs on an SM (0: as many as fit)
int launch_kf_multi(int prec, const void *cases, const int4 *table, int nentries, bool fields, bool cons0,
                    int ctas_per_sm, cudaStream_t st);
size_t ib_args_size();
void ib_args_write(lbm_handle *h, const void *fin, int slot, void *dst);
void ib_factor_args_write(lbm_handle *h, int step0, int count, void *dst);
int launch_factor_batch(lbm_handle *const *hs, int ncase, const void *dargs, int step0, int count, cudaStream_t st);
int launch_flow_batch(lbm_handle *const *hs, int ncase, const void *dargs, const void *dkf, int step_index,
                      int ring_slot, bool fields, cudaStream_t st, cudaEvent_t after_interp = nullptr);
// residual: some case runs its solve-residual check this step (IBArgs::check_res)
int launch_check_batch(lbm_handle *const *hs, int ncase, const void *dargs, int ring_slot, bool residual,
                       cudaStream_t st);
int ib_tile_ints();   // ints per patch tile of the tile lists
int launch_residual(lbm_handle *h, const void *fa, const void *fb, double *out2);
int launch_unpack(lbm_handle *h, const void *fsrc, double *dst);   // deviation -> f (FP64)
int launch_pack(lbm_handle *h, const double *src, void *fdst);     // f (FP64) -> deviation
// initial populations and fields (slot 0) of lbm_init from the device copies
// of the perturbation (nullable)
int launch_init_lattice(lbm_handle *h, const double *du, const double *dv);
int launch_fields_to_double(lbm_handle *h, const void *fields, double *rho, double *u, double *v);
// global mass check (FP64, deterministic) of the populations in fsrc
int launch_mass(lbm_handle *h, const void *fsrc, cudaStream_t st);
int mass_slots();
// error code and message of a device status word
int status_error(unsigned st, std::string &msg);
// host <-> device copies of host arrays through the pinned staging ring
// (host_xfer.cu); the d2h calls return with the data on the host, xfer_h2d
// with the copies queued on st
cudaError_t xfer_d2h_widen(double *dst, const float *src, size_t n, cudaStream_t st);
cudaError_t xfer_d2h(void *dst, const void *src, size_t bytes, cudaStream_t st);
cudaError_t xfer_h2d(void *dst, const void *src, size_t bytes, cudaStream_t st);
