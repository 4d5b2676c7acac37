// ib_kernels.cu -- immersed boundary of one time step (FP64), ahead of the
// lattice update of the correction patch.
//
// Reference: move_boundary (airfoil.f90:244-338) and immersed_boundary_Wu
// (boundary_condition.f90:1512-1736). The reference builds dense X1 (nseg x
// nadj) and X2 = X1^T W (W = diag(arc_l)), forms A = X1 X2 with cublasDgemm,
// solves A x = U_b - X1 u* by LU (cusolverDnDgetrf/getrs) and spreads
// du = X2 x. With D = X1, A = (D D^T) W, so y = W x solves the symmetric
// positive definite system (D D^T) y = U_b - D u* and du = D^T y: the same
// correction, with arc_l dropping out.
//
// The marker positions follow the prescribed motion, so D D^T and its
// factorization depend on the step index only, not on the flow. The
// launches are therefore two chains. The factorization chain of a step
// (which the host runs one step ahead, concurrently with the previous step,
// into one of two buffer slots):
//   ib_geometry one thread per marker: position, boundary velocity, support
//               box and one-axis kernel values (move_boundary, :1540-1606);
//   ib_order    (several bodies only) one CTA sorts the markers along the
//               longer axis of the marker cloud. A single rigid body keeps one
//               order for the whole run: its markers sorted by body-frame
//               chordwise position, computed once on the host;
//   ib_assemble one CTA per 16-marker block of that order: D D^T is banded in
//               it (delta supports overlap only for markers less than 5 lu
//               apart per axis), so the CTA builds its diagonal block and the
//               block coupling it to the previous one, and checks that no
//               coupling reaches further;
//   ib_tile_scatter, ib_tile_sort  per 16 x 16 tile of the patch
//               rectangle, the markers whose support box meets it (each
//               marker appends itself; each tile sorts its list);
//   ib_factor   one CTA: correction-patch rectangle, then block cyclic
//               reduction of the block tridiagonal matrix (log2 of the block
//               count levels of Gauss-Jordan block inverses and block
//               products, FP64), keeping per eliminated block D^-1 and the two
//               coupling factors; a dense Cholesky replaces it when a coupling
//               reaches past the neighbouring block.
// The flow chain of the step:
//   ib_interp   one warp per marker: b = D u* over the support box and
//               rhs = U_b - b (:1609-1629);
//   ib_solve    one CTA: the forward and backward sweeps of the reduction
//               over the two right-hand sides, each level's factor blocks
//               staged in shared memory by bulk copies (or the two triangular
//               solves of the dense factor), and the force row's header;
//   ib_tile_update  one CTA per correction tile (a 16 x 16 tile of the
//               patch rectangle that lists a marker): du = D^T y per node,
//               gathered in marker order (no atomics), the lattice update of
//               the tile's nodes with that correction, and the force and
//               moment sums (:1645-1675, solution.f90:327-336) in FP64 with a
//               deterministic two-level reduction. The lattice kernel skips
//               these nodes and updates all others;
//   ib_forces   the force row from the tiles' partials, and
//   ib_residual the solve's residual, both after the step's update.

#include <math.h>

#include "lbm_internal.h"
#include "lbm_node.cuh"

namespace {

constexpr int BS = 16;                 // block size of the cyclic reduction
constexpr int NMARK_MAX = 2048;        // largest marker count
#ifndef LBM_FACTOR_THREADS
#define LBM_FACTOR_THREADS 512
#endif
#ifndef LBM_SOLVE_THREADS
#define LBM_SOLVE_THREADS 1024
#endif
#ifndef LBM_SOLVE_SMEM
#define LBM_SOLVE_SMEM 232192
#endif
constexpr int FACTOR_THREADS = LBM_FACTOR_THREADS;
constexpr int BOPS_WARPS = FACTOR_THREADS / 32;   // warps running block operations
constexpr int SOLVE_THREADS = LBM_SOLVE_THREADS;
constexpr int STAGE_BLOCKS = 32;       // factor blocks of one level staged in shared memory by ib_solve
constexpr int FL = 2 * BS;             // columns of a coupling panel [L_o | L_q^T]
constexpr int GW = 3 * BS;             // row width of a stored factor block [D^-1 | F_L | F_U]
constexpr int GP = BS + 1;             // padded row stride of square blocks in shared memory
constexpr int SOLVE_SMEM_BUDGET = LBM_SOLVE_SMEM;   // dynamic shared memory of ib_solve (bytes)

// factor blocks ib_solve can stage next to the right-hand sides of nb blocks
__host__ __device__ constexpr int stage_cap(int nb)
{
    return (SOLVE_SMEM_BUDGET - 16 - 2 * nb * BS * (int)sizeof(double)) / (BS * GW * (int)sizeof(double)) < STAGE_BLOCKS
               ? (SOLVE_SMEM_BUDGET - 16 - 2 * nb * BS * (int)sizeof(double)) / (BS * GW * (int)sizeof(double))
               : STAGE_BLOCKS;
}
// factor blocks a solve of nb blocks stages at once: level 1's odd blocks or
// those of all the levels above it together, whichever is more (the first
// and the second staging of the resident form), within stage_cap
__host__ __device__ constexpr int stage_blocks(int nb)
{
    int upper = 0;
    for (int st = 2; st < nb; st <<= 1) upper += (nb + st - 1) / (2 * st);
    const int need = nb / 2 > upper ? nb / 2 : upper;
    return need < stage_cap(nb) ? need : stage_cap(nb);
}
constexpr int WS = BS * GP + BS * FL + BS * GP;   // workspace per warp (doubles)
constexpr int NPART = 3 * LBM_MAXW + 3;           // per-CTA partials of ib_tile_update
constexpr int TILE = 16;                          // correction-patch tile (nodes per side)
constexpr int TILE_CAP = 256;                     // markers listed per tile

// one-axis kernel value (boundary_condition.f90:1563-1600), disr = |r|
__device__ __forceinline__ double delta1(double disr, int smooth)
{
    const double pai = 3.1415926535897932384626433832795;
    if (smooth == 0) {
        if (fabs(disr) < 1.0)
            return 0.125 * (3.0 - 2.0 * fabs(disr) + sqrt(1.0 + 4.0 * fabs(disr) - 4.0 * disr * disr));
        else if ((fabs(disr) < 2.0) && (fabs(disr) >= 1.0))
            return 0.125 * (5.0 - 2.0 * fabs(disr) - sqrt(-7.0 + 12.0 * fabs(disr) - 4.0 * disr * disr));
        return 0.0;
    }
    if (fabs(disr) <= 0.5)
        return 0.375 + 0.03125 * pai - 0.25 * disr * disr;
    else if ((fabs(disr) <= 1.5) && (fabs(disr) >= 0.5))
        return 0.25 + 0.125 * (1.0 - disr) * sqrt(-2.0 + 8.0 * disr - 4.0 * disr * disr) -
               0.125 * asin(sqrt(2.0) * (disr - 1.0));
    else if ((fabs(disr) <= 2.5) && (fabs(disr) >= 1.5))
        return 1.0625 - 0.015625 * pai - 0.75 * disr + 0.125 * disr * disr +
               0.0625 * (disr - 2.0) * sqrt(-14.0 + 16.0 * disr - 4.0 * disr * disr) +
               0.0625 * asin(sqrt(2.0) * (disr - 2.0));
    return 0.0;
}


// FP64 moments of the streamed populations at an interior node
template <typename T>
__device__ __forceinline__ void node_moments(const IBArgs &a, int i, int j, double &rho, double &u, double &v)
{
    const T *fin = (const T *)a.fin;
    double g[9];
#pragma unroll
    for (int k = 0; k < 9; ++k)
        g[k] = (double)Store<T>::ld(fin + (long long)k * a.plane + (long long)(j - lbm_ey(k)) * a.pitch +
                                    (i - lbm_ex(k)));
    const double drho = ((g[0] + g[1]) + (g[2] + g[3])) + ((g[4] + g[5]) + (g[6] + g[7])) + g[8];
    const double jx = (g[1] - g[3]) + (g[5] - g[6]) + (g[8] - g[7]);
    const double jy = (g[2] - g[4]) + (g[5] + g[6]) - (g[7] + g[8]);
    rho = 1.0 + drho;
    u = jx / rho;
    v = jy / rho;
}

__device__ __forceinline__ const double *motion_row(const IBArgs &a, int step_index, double *time_out)
{
    const double time = (double)(step_index - 1) * (a.scale * a.uu);   // solution.f90:289
    int idx = (int)llround(time / a.mdt) + 1;                             // mode.f90:280-281
    idx = idx < 1 ? 1 : (idx > a.msteps ? a.msteps : idx);
    if (time_out) *time_out = time;
    return a.mstep + (long long)(idx - 1) * a.mcols;
}

// Step of this CTA's member of a factorization launch: step0 + blockIdx.y,
// or per case in batched launches (the case's own start and count; -1 for
// the members past its count).
template <bool BATCH> __device__ __forceinline__ int factor_step(const IBArgs &base, int step0)
{
    if (!BATCH) return step0 + (int)blockIdx.y;
    return (int)blockIdx.y < base.fcount ? base.fstep0 + (int)blockIdx.y : -1;
}

// Arguments of one member of a batched factorization launch: the step
// step0 + blockIdx.y, its buffer slot (step modulo the slot count) and the
// member's working set.
__device__ __forceinline__ IBArgs member_args(IBArgs a, int step)
{
    const int slot = step % a.nslots, mem = blockIdx.y;
    a.mk += slot * a.st_mk;
    a.perm += slot * a.st_perm;
    a.key += slot * a.st_perm;
    a.B += slot * a.st_B;
    a.gf += slot * a.wk_gf;
    a.pinfo += slot;
    a.tiles += slot * a.st_tiles;
    a.ctile += slot * (a.st_tiles / (TILE_CAP + 1));
    a.nsup += slot;
    a.fmode += 2 * slot;
    a.fstatus += slot;
    a.status = a.fstatus;   // errors of the chain are reported by the step that uses it
    a.bD += mem * a.wk_blocks;
    a.bL += mem * a.wk_blocks;
    a.wmax += mem;
    return a;
}

// marker geometry of segment k (airfoil.f90:255-335, boundary_condition.f90:1540-1606)
__device__ Marker make_marker(const IBArgs &a, const double *row, int k)
{
    const double scale = a.scale, ox = a.ox, oy = a.oy;
    const int w = k / a.spw;
    const int p0 = w * a.ppw + (k - w * a.spw);
    const double angle = row[1 + 9 * w], omega = row[2 + 9 * w];
    const double sa = row[4 + 9 * w], sau = row[5 + 9 * w];
    const double sb = row[7 + 9 * w], sbv = row[8 + 9 * w];
    const double ca = cos(angle), sn = sin(angle);
    // airfoil.f90:261-263 (body_extra_s and movenum are zero: no dynamics)
    const double xa = ca * a.xb0[p0] + sn * a.yb0[p0] + sa + a.xc;
    const double xb = ca * a.xb0[p0 + 1] + sn * a.yb0[p0 + 1] + sa + a.xc;
    const double ya = -sn * a.xb0[p0] + ca * a.yb0[p0] + sb + a.yc;
    const double yb = -sn * a.xb0[p0 + 1] + ca * a.yb0[p0 + 1] + sb + a.yc;
    Marker m;
    m.xm = 0.5 * (xb + xa);                                           // :267-270
    m.ym = 0.5 * (yb + ya);
    // boundary_condition.f90:1547-1550 (body_extra_v is zero)
    m.ub = a.uu * (-omega * sn * 0.5 * (a.xb0[p0 + 1] + a.xb0[p0]) +
                   omega * ca * 0.5 * (a.yb0[p0 + 1] + a.yb0[p0]) + sau);
    m.vb = a.uu * (-omega * ca * 0.5 * (a.xb0[p0 + 1] + a.xb0[p0]) -
                   omega * sn * 0.5 * (a.yb0[p0 + 1] + a.yb0[p0]) + sbv);
    m.wing = w;
    m.pad = 0;
    for (int t = 0; t < LBM_BOX; ++t) m.phx[t] = m.phy[t] = 0.0;
    m.i1 = 3; m.i2 = 2; m.j1 = 3; m.j2 = 2;   // empty box unless set below
    // a marker off the lattice (or not finite) is a range error before any scan
    const double fx = (m.xm - ox) / scale + 1.0, fy = (m.ym - oy) / scale + 1.0;
    if (!(fx > 3.0 && fx < (double)(a.nx - 2) && fy > 3.0 && fy < (double)(a.ny - 2))) {
        atomicOr(a.status, LBM_ST_RANGE);
        return m;
    }
    // support box, 1-based scans of airfoil.f90:290-321
    int i1 = (int)((m.xm - ox) / scale + 1.0);
    for (int i = i1; i >= 1; --i)
        if (fabs((ox + (double)(i - 1) * scale - m.xm) / scale) > 2.5) { i1 = i + 1; break; }
    int i2 = (int)((m.xm - ox) / scale + 1.0);
    for (int i = i2; i <= a.nx; ++i)
        if (fabs((ox + (double)(i - 1) * scale - m.xm) / scale) > 2.5) { i2 = i - 1; break; }
    int j2 = (int)((m.ym - oy) / scale + 1.0);
    for (int i = j2; i <= a.ny; ++i)
        if (fabs((oy + (double)(i - 1) * scale - m.ym) / scale) > 2.5) { j2 = i - 1; break; }
    int j1 = (int)((m.ym - oy) / scale + 1.0);
    for (int i = j1; i >= 1; --i)
        if (fabs((oy + (double)(i - 1) * scale - m.ym) / scale) > 2.5) { j1 = i + 1; break; }
    if (i1 < 4 || j1 < 4 || i2 > a.nx - 3 || j2 > a.ny - 3 || i2 - i1 >= LBM_BOX || j2 - j1 >= LBM_BOX) {
        atomicOr(a.status, LBM_ST_RANGE);
        return m;
    }
    for (int t = 0; t < LBM_BOX; ++t) {
        const int ii = i1 + t, jj = j1 + t;
        m.phx[t] = ii <= i2 ? delta1(fabs((ox + scale * (double)(ii - 1) - m.xm) / scale), a.smooth) : 0.0;
        m.phy[t] = jj <= j2 ? delta1(fabs((oy + scale * (double)(jj - 1) - m.ym) / scale), a.smooth) : 0.0;
    }
    m.i1 = i1 - 1; m.i2 = i2 - 1; m.j1 = j1 - 1; m.j2 = j2 - 1;
    return m;
}


// one thread per marker: geometry of this step (errors go to the slot's status)
template <bool BATCH>
__global__ void __launch_bounds__(128) ib_geometry(const IBArgs base0, const IBArgs *batch, int step0)
{
    const IBArgs &base = BATCH ? batch[blockIdx.z] : base0;
    const int step_index = factor_step<BATCH>(base, step0);
    if (step_index < 0) return;
    const IBArgs a = member_args(base, step_index);
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.nseg) return;
    const double *row = motion_row(a, step_index, nullptr);
    a.mk[k] = make_marker(a, row, k);
}

// one warp per marker: b = D u* over the support box, rhs = U_b - b
template <typename T, bool BATCH>
__global__ void __launch_bounds__(256) ib_interp(const IBArgs a0, const IBArgs *batch)
{
    const IBArgs &a = BATCH ? batch[blockIdx.z] : a0;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // bring the slot's factor blocks, which the lattice kernels have evicted
    // since the factorization wrote them, back into L2 for ib_solve: one
    // 128-byte line per thread
    {
        const long long nlines = (a.wk_gf * (long long)sizeof(double) + 127) / 128;
        const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
        for (long long l = t; l < nlines; l += (long long)gridDim.x * blockDim.x)
            asm volatile("prefetch.global.L2 [%0];" ::"l"(reinterpret_cast<const char *>(a.gf) + 128 * l));
    }
    const int k = blockIdx.x * 8 + warp;
    if (k >= a.nseg) return;
    // the marker's box and kernel values are read where they lie (a local
    // copy of the struct, indexed by node, would live on the stack)
    const Marker *mp = a.mk + k;
    const int i1 = mp->i1, i2 = mp->i2, j1 = mp->j1, j2 = mp->j2;
    const bool ok = box_in_bounds(i1, i2, j1, j2, a.nx, a.ny);
    if (!ok && lane == 0) atomicOr(a.status, LBM_ST_INDEX_INTERP);
    const int nbx = ok ? i2 - i1 + 1 : 0, nby = ok ? j2 - j1 + 1 : 0;
    const int nn = nbx > 0 && nby > 0 ? nbx * nby : 0;
    double su = 0.0, sv = 0.0;
    if (nn > 0) {
        // at most LBM_BOX^2 = 36 nodes: lane t takes nodes t and t + 32, and
        // both nodes' populations are loaded before either is summed (a lane
        // without a second node loads its first again and weighs it 0); the
        // sums are the loop's, node t then node t + 32, each a fused
        // multiply-add onto the running sum
        const bool h0 = lane < nn, h1 = lane + 32 < nn;
        const int t0 = h0 ? lane : 0, t1 = h1 ? lane + 32 : t0;
        const int ii0 = t0 % nbx, jj0 = t0 / nbx, ii1 = t1 % nbx, jj1 = t1 / nbx;
        double rho0, u0, v0, rho1, u1, v1;
        node_moments<T>(a, i1 + ii0, j1 + jj0, rho0, u0, v0);
        node_moments<T>(a, i1 + ii1, j1 + jj1, rho1, u1, v1);
        const double w0 = mp->phx[ii0] * mp->phy[jj0];   // X1(k,i) = kernel1*kernel2 (:1602)
        const double w1 = mp->phx[ii1] * mp->phy[jj1];
        if (h0) {
            su = fma(w0, u0, su);
            sv = fma(w0, v0, sv);
        }
        if (h1) {
            su = fma(w1, u1, su);
            sv = fma(w1, v1, sv);
        }
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        su += __shfl_down_sync(0xffffffffu, su, off);
        sv += __shfl_down_sync(0xffffffffu, sv, off);
    }
    if (lane == 0) {
        a.rhs[k] = mp->ub - su;                 // comj (:1624-1629)
        a.rhs[a.nseg + k] = mp->vb - sv;
    }
}

// (D D^T)(k,l): the delta is separable, so the node sum over the box overlap
// is (sum_i phx_k phx_l)(sum_j phy_k phy_l)
__device__ __forceinline__ double bval(const Marker &mk, const Marker &ml)
{
    const int ia = max(mk.i1, ml.i1), ib = min(mk.i2, ml.i2);
    const int ja = max(mk.j1, ml.j1), jb = min(mk.j2, ml.j2);
    if (ia > ib || ja > jb) return 0.0;
    double sx = 0.0, sy = 0.0;
    for (int i = ia; i <= ib; ++i) sx += mk.phx[i - mk.i1] * ml.phx[i - ml.i1];
    for (int j = ja; j <= jb; ++j) sy += mk.phy[j - mk.j1] * ml.phy[j - ml.j1];
    return sx * sy;
}

__device__ __forceinline__ bool box_overlap(int4 p, int4 q)
{
    return max(p.x, q.x) <= min(p.y, q.y) && max(p.z, q.z) <= min(p.w, q.w);
}

__device__ __forceinline__ int4 mbox(const Marker &m) { return make_int4(m.i1, m.i2, m.j1, m.j2); }

// a marker as make_marker leaves it: support box within bounds (an empty
// box included) and a wing index of the case
__device__ __forceinline__ bool marker_ok(const IBArgs &a, const Marker &m)
{
    return box_in_bounds(m.i1, m.i2, m.j1, m.j2, a.nx, a.ny) && m.wing >= 0 && m.wing < a.nwing;
}

// the marker at position srt of the solve order, or null (and the kernel's
// status bit set) when the order holds an index outside the markers or the
// marker is not as make_marker leaves it
__device__ __forceinline__ const Marker *sorted_marker(const IBArgs &a, int srt, unsigned bit)
{
    const int k = a.perm[srt];
    if (k < 0 || k >= a.nseg || !marker_ok(a, a.mk[k])) {
        atomicOr(a.status, bit);
        return nullptr;
    }
    return a.mk + k;
}

// marker at position s of the solve order, or -1 (and the kernel's status
// bit set) when the order holds an index outside the markers
__device__ __forceinline__ int order_at(const IBArgs &a, int s, unsigned bit)
{
    const int k = a.perm[s];
    if (k < 0 || k >= a.nseg) {
        atomicOr(a.status, bit);
        return -1;
    }
    return k;
}

// tiles of the patch grid (the tile lists of one slot)
__device__ __forceinline__ int patch_tiles(const IBArgs &a) { return (int)(a.st_tiles / (TILE_CAP + 1)); }

// time and motion columns of this step's force.dat row (solution.f90:350-375)
__device__ void write_header(const IBArgs &a, const double *row, double time, int ring_slot)
{
    double *fr = a.force_ring + (long long)ring_slot * a.row_len;
    fr[0] = time;
    const int mc = 1 + 3 * a.nwing + 3;
    for (int w = 0; w < a.nwing; ++w) {
        const double *r = row + 1 + 9 * w;   // angle omega omgac sa sau saac sb sbv sbac
        double *o = fr + mc + 9 * w;         // solution.f90:363-374 order
        o[0] = r[3]; o[1] = r[4]; o[2] = r[5]; o[3] = r[6]; o[4] = r[7]; o[5] = r[8];
        o[6] = r[0]; o[7] = r[1]; o[8] = r[2];
    }
}


// Several bodies: sort the markers along the longer axis of the marker cloud
// (stable, ties by index) into perm/key, with reach = 6 lattice units along
// that axis. One CTA; dynamic shared memory key[ns] (double) + idx[ns] (int).
template <bool BATCH>
__global__ void __launch_bounds__(1024) ib_order(const IBArgs base0, const IBArgs *batch, int step0)
{
    const IBArgs &base = BATCH ? batch[blockIdx.z] : base0;
    const int step_index = factor_step<BATCH>(base, step0);
    if (step_index < 0) return;
    const IBArgs a = member_args(base, step_index);
    if (a.static_order) return;   // one rigid body: fixed order (batched launches reach it)
    extern __shared__ double osm[];
    const int n = a.nseg, tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
    int ns = 1;
    while (ns < n) ns <<= 1;
    double *key = osm;
    int *idx = (int *)(key + ns);
    __shared__ double wext[32][4];
    __shared__ bool by_x;
    double lx0 = 1e300, lx1 = -1e300, ly0 = 1e300, ly1 = -1e300;
    for (int k = tid; k < n; k += nt) {
        const double xm = a.mk[k].xm, ym = a.mk[k].ym;
        lx0 = fmin(lx0, xm); lx1 = fmax(lx1, xm); ly0 = fmin(ly0, ym); ly1 = fmax(ly1, ym);
    }
    for (int off = 16; off; off >>= 1) {
        lx0 = fmin(lx0, __shfl_xor_sync(0xffffffffu, lx0, off));
        lx1 = fmax(lx1, __shfl_xor_sync(0xffffffffu, lx1, off));
        ly0 = fmin(ly0, __shfl_xor_sync(0xffffffffu, ly0, off));
        ly1 = fmax(ly1, __shfl_xor_sync(0xffffffffu, ly1, off));
    }
    if (lane == 0) { wext[warp][0] = lx0; wext[warp][1] = lx1; wext[warp][2] = ly0; wext[warp][3] = ly1; }
    __syncthreads();
    if (tid == 0) {
        double e0 = 1e300, e1 = -1e300, e2 = 1e300, e3 = -1e300;
        for (int w = 0; w < (nt >> 5); ++w) {
            e0 = fmin(e0, wext[w][0]); e1 = fmax(e1, wext[w][1]);
            e2 = fmin(e2, wext[w][2]); e3 = fmax(e3, wext[w][3]);
        }
        by_x = (e1 - e0) >= (e3 - e2);
        *a.reach = 6.0 * a.scale;
    }
    __syncthreads();
    for (int s2 = tid; s2 < ns; s2 += nt) {
        key[s2] = s2 < n ? (by_x ? a.mk[s2].xm : a.mk[s2].ym) : 1e300;
        idx[s2] = s2;
    }
    __syncthreads();
    for (int size = 2; size <= ns; size <<= 1)
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int s2 = tid; s2 < ns; s2 += nt) {
                const int t = s2 ^ stride;
                if (t > s2) {
                    const bool up = (s2 & size) == 0;
                    const bool gt = key[s2] > key[t] || (key[s2] == key[t] && idx[s2] > idx[t]);
                    if (gt == up) {
                        const double kk = key[s2]; key[s2] = key[t]; key[t] = kk;
                        const int ii = idx[s2]; idx[s2] = idx[t]; idx[t] = ii;
                    }
                }
            }
            __syncthreads();
        }
    for (int s2 = tid; s2 < n; s2 += nt) {
        a.perm[s2] = idx[s2];
        a.key[s2] = key[s2];
    }
}


// One CTA per block of BS markers in the solve order: the diagonal block D_b,
// the coupling L_b to block b-1, and the longest coupling in the order
// (half-bandwidth).
template <bool BATCH>
__global__ void __launch_bounds__(256) ib_assemble(const IBArgs base0, const IBArgs *batch, int step0)
{
    const IBArgs &base = BATCH ? batch[blockIdx.z] : base0;
    const int step_index = factor_step<BATCH>(base, step0);
    if (step_index < 0) return;
    const IBArgs a = member_args(base, step_index);
    const int n = a.nseg, blk = blockIdx.x, tid = threadIdx.x;
    if (blk >= (n + BS - 1) / BS) return;   // batched launches size the grid for the largest case
    __shared__ double ph[2 * BS][12];
    __shared__ int4 bx[2 * BS];
    __shared__ int wl;
    if (tid == 0) wl = 0;
    for (int q = tid; q < 2 * BS * 12; q += blockDim.x) {
        const int m = q / 12, c = q % 12, srt = (blk - 1) * BS + m;
        double v = 0.0;
        if (srt >= 0 && srt < n) {
            const Marker *mm = sorted_marker(a, srt, LBM_ST_INDEX_ASSEMBLE);
            if (mm) v = c < 6 ? mm->phx[c] : mm->phy[c - 6];
        }
        ph[m][c] = v;
    }
    for (int m = tid; m < 2 * BS; m += blockDim.x) {
        const int srt = (blk - 1) * BS + m;
        const Marker *mm = (srt >= 0 && srt < n) ? sorted_marker(a, srt, LBM_ST_INDEX_ASSEMBLE) : nullptr;
        bx[m] = mm ? mbox(*mm) : make_int4(1, 0, 1, 0);
    }
    __syncthreads();
    for (int q = tid; q < 2 * BS * BS; q += blockDim.x) {
        const bool lower = q >= BS * BS;
        const int r = (q % (BS * BS)) / BS, c = q % BS;
        const int mr = BS + r, mc = lower ? c : BS + c, sr = blk * BS + r;
        double v = 0.0;
        if (sr >= n) {
            v = (!lower && r == c) ? 1.0 : 0.0;
        } else if ((!lower && blk * BS + c < n) || (lower && blk > 0)) {
            const int4 p = bx[mr], o = bx[mc];
            const int ia = max(p.x, o.x), ib = min(p.y, o.y), ja = max(p.z, o.z), jb = min(p.w, o.w);
            if (ia <= ib && ja <= jb) {
                double sx = 0.0, sy = 0.0;
                for (int i = ia; i <= ib; ++i) sx += ph[mr][i - p.x] * ph[mc][i - o.x];
                for (int j = ja; j <= jb; ++j) sy += ph[mr][6 + j - p.z] * ph[mc][6 + j - o.z];
                v = sx * sy;
            }
        }
        const long long g = (long long)blk * BS * BS + r * BS + c;
        if (lower) a.bL[g] = v;
        else a.bD[g] = v;
    }
    // half-bandwidth: boxes (<= 6 nodes wide) overlap only for markers closer
    // than `reach` along the order's key (ascending in the solve order, so
    // the markers within reach are a run after srt). 16 threads per marker
    // of the block scan that run, thread l the markers srt + 1 + l + 16 i.
    {
        static_assert(BS * 16 == 256, "16 threads per marker of a block");
        const int m = tid >> 4, l = tid & 15, srt = blk * BS + m;
        if (srt < n) {
            const double reach = *a.reach;
            const int4 p = bx[BS + m];
            const double ks = a.key[srt];
            int w = 0;
            for (int t = srt + 1 + l; t < n && a.key[t] - ks <= reach; t += 16) {
                const Marker *mt = sorted_marker(a, t, LBM_ST_INDEX_ASSEMBLE);
                if (mt && box_overlap(p, mbox(*mt))) w = t - srt;
            }
            if (w) atomicMax(&wl, w);
        }
    }
    __syncthreads();
    if (tid == 0 && wl) atomicMax(a.wmax, wl);
}

// In-place inverse of one symmetric positive definite BS x BS block by one
// warp (Gauss-Jordan without pivoting, stable for SPD), row stride GP in
// shared memory. The block is held in registers during the BS elimination
// steps: lane (j, h) owns column j of rows 2e+h; the pivot row and column are
// broadcast by warp shuffles. Returns false if a pivot is not positive.
__device__ bool warp_inv(double *G)
{
    const int lane = threadIdx.x & 31;
    const int j = lane % BS, ih = lane / BS;
    double g[BS / 2];
#pragma unroll
    for (int e = 0; e < BS / 2; ++e) g[e] = G[(2 * e + ih) * GP + j];
    bool ok = true;
#pragma unroll
    for (int k = 0; k < BS; ++k) {
        const int kh = k & 1, ke = k >> 1;            // owner half and register of row k
        const double p = __shfl_sync(0xffffffffu, g[ke], kh * BS + k);
        const bool good = p > 0.0 && isfinite(p);
        ok = ok && good;
        const double piv = good ? 1.0 / p : 1.0;
        const double rowk = __shfl_sync(0xffffffffu, g[ke], kh * BS + j) * piv;   // scaled G[k][j]
        double cik[BS / 2];
#pragma unroll
        for (int e = 0; e < BS / 2; ++e) cik[e] = __shfl_sync(0xffffffffu, g[e], ih * BS + k);   // G[2e+ih][k]
#pragma unroll
        for (int e = 0; e < BS / 2; ++e) {
            const int i = 2 * e + ih;
            if (i == k) g[e] = (j == k) ? piv : rowk;         // row k
            else if (j == k) g[e] = -cik[e] * piv;            // column k
            else g[e] = g[e] - cik[e] * rowk;                 // rank-1 update
        }
    }
#pragma unroll
    for (int e = 0; e < BS / 2; ++e) G[(2 * e + ih) * GP + j] = g[e];
    __syncwarp();
    return ok;
}

// n doubles (a multiple of 32) from global to shared memory, all loads in flight
template <int N>
__device__ __forceinline__ void stage(double *dst, const double *__restrict__ src)
{
    const int lane = threadIdx.x & 31;
    double v[N / 32];
#pragma unroll
    for (int it = 0; it < N / 32; ++it) v[it] = src[lane + 32 * it];
#pragma unroll
    for (int it = 0; it < N / 32; ++it) dst[lane + 32 * it] = v[it];
}

// BS x BS row-major block from global memory into the padded (GP) layout
__device__ __forceinline__ void stage_sq(double *dst, const double *__restrict__ src)
{
    const int lane = threadIdx.x & 31;
    double v[BS * BS / 32];
#pragma unroll
    for (int it = 0; it < BS * BS / 32; ++it) v[it] = src[lane + 32 * it];
#pragma unroll
    for (int it = 0; it < BS * BS / 32; ++it) {
        const int e = lane + 32 * it;
        dst[(e / BS) * GP + e % BS] = v[it];
    }
}


// Block products of the cyclic reduction. Lane 2r+h of a warp owns output
// row r (0..BS-1) and half h of the columns; B rows are read as 16-byte pairs
// that the two lanes of a row share, so a product costs BS x (1 + NH/2)
// shared loads per lane instead of two per multiply-add.
// acc[c] = sum_t A(r,t) B[t*ldb + h*NH + c], c < NH; A(r,t) is A[r][t] in the
// padded (GP) layout, or A[t][r] when TA.
template <int NH, bool TA>
__device__ __forceinline__ void rowmm(const double *A, const double *B, int ldb, double acc[NH])
{
    const int lane = threadIdx.x & 31, r = lane >> 1, h = lane & 1;
#pragma unroll
    for (int c = 0; c < NH; ++c) acc[c] = 0.0;
#pragma unroll
    for (int t = 0; t < BS; ++t) {
        const double a = TA ? A[t * GP + r] : A[r * GP + t];
        const double2 *b = reinterpret_cast<const double2 *>(B + t * ldb + h * NH);
#pragma unroll
        for (int c = 0; c < NH / 2; ++c) {
            const double2 bb = b[c];
            acc[2 * c] += a * bb.x;
            acc[2 * c + 1] += a * bb.y;
        }
    }
}

// dense fallback, factor: Cholesky L L^T of the full D D^T in the solve order
// (row-major, lower triangle, in place), whole CTA
__device__ void dense_factor(const IBArgs &a, int *bad)
{
    const int n = a.nseg, tid = threadIdx.x, nt = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
    double *L = a.B;
    for (long long q = tid; q < (long long)n * n; q += nt) {
        const int k = (int)(q / n), l = (int)(q % n);
        const Marker *mk = sorted_marker(a, k, LBM_ST_INDEX_FACTOR), *ml = sorted_marker(a, l, LBM_ST_INDEX_FACTOR);
        L[q] = mk && ml ? bval(*mk, *ml) : (k == l ? 1.0 : 0.0);
    }
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (tid == 0) {
            const double d = L[(long long)k * n + k];
            double dk = 1.0;
            if (!(d > 0.0) || !isfinite(d)) *bad = 1;
            else dk = sqrt(d);
            L[(long long)k * n + k] = dk;
        }
        __syncthreads();
        const double dk = L[(long long)k * n + k];
        for (int i = k + 1 + tid; i < n; i += nt) L[(long long)i * n + k] /= dk;
        __syncthreads();
        for (int i = k + 1 + warp; i < n; i += nw) {
            const double lik = L[(long long)i * n + k];
            for (int j = k + 1 + lane; j <= i; j += 32) L[(long long)i * n + j] -= lik * L[(long long)j * n + k];
        }
        __syncthreads();
    }
}

// dense fallback, solve: L z = r, then L^T y = z, for the two right-hand
// sides yv[0..n) and yv[n..2n) (shared memory), whole CTA
__device__ void dense_tri(const IBArgs &a, double *yv)
{
    const int n = a.nseg, tid = threadIdx.x, nt = blockDim.x;
    const double *L = a.B;
    for (int k = 0; k < n; ++k) {
        const double dk = L[(long long)k * n + k];
        const double z0 = yv[k] / dk, z1 = yv[n + k] / dk;
        __syncthreads();
        if (tid == 0) { yv[k] = z0; yv[n + k] = z1; }
        for (int i = k + 1 + tid; i < n; i += nt) {
            const double lik = L[(long long)i * n + k];
            yv[i] -= lik * z0;
            yv[n + i] -= lik * z1;
        }
        __syncthreads();
    }
    for (int j = n - 1; j >= 0; --j) {
        if (tid < 2) yv[tid * n + j] /= L[(long long)j * n + j];
        __syncthreads();
        for (int q = tid; q < 2 * j; q += nt) {
            const int c = q / j, i = q % j;
            yv[c * n + i] -= L[(long long)j * n + i] * yv[c * n + j];
        }
        __syncthreads();
    }
}


// Factorization of one step's D D^T, one CTA of FACTOR_THREADS threads;
// dynamic shared memory: one block-operation workspace of WS doubles per warp.
// Block cyclic reduction: at stride st the active blocks are the multiples
// of st, and the odd multiples o are eliminated into their even neighbours.
// For each eliminated block the factor buffer keeps, row by row, BS x GW
// values [D_o^-1 | F_L | F_U] with F_L = D_o^-1 L_o (coupling to o - st) and
// F_U = D_o^-1 L_q^T (coupling to q = o + st); block 0, the last one left,
// keeps D_0^-1. The even neighbours are updated as
//   D_e -= L_q^T F_L(q) + L_e F_U(p),   L_e <- -L_e F_L(p)   (p = e - st, q = e + st).
template <bool BATCH>
__global__ void __launch_bounds__(FACTOR_THREADS, 65536 / (FACTOR_THREADS * 128)) ib_factor(const IBArgs base0, const IBArgs *batch, int step0)
{
    const IBArgs &base = BATCH ? batch[blockIdx.z] : base0;
    const int step_index = factor_step<BATCH>(base, step0);
    if (step_index < 0) return;
    const IBArgs a = member_args(base, step_index);
    extern __shared__ __align__(16) double Wbase[];
    const int n = a.nseg, tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    __shared__ int bad, dense;
    __shared__ int bb[4];
    if (tid == 0) { bb[0] = 1 << 30; bb[1] = 1 << 30; bb[2] = -1; bb[3] = -1; }
    __syncthreads();
    // patch rectangle of the step: bounding box of all support boxes
    {
        int b0 = 1 << 30, b1 = 1 << 30, b2 = -1, b3 = -1;
        for (int k = tid; k < n; k += blockDim.x) {
            const int4 q = mbox(a.mk[k]);
            if (!box_in_bounds(q.x, q.y, q.z, q.w, a.nx, a.ny)) {
                atomicOr(a.status, LBM_ST_INDEX_FACTOR);
                continue;
            }
            if (q.y >= q.x && q.w >= q.z) { b0 = min(b0, q.x); b1 = min(b1, q.z); b2 = max(b2, q.y); b3 = max(b3, q.w); }
        }
        for (int off = 16; off; off >>= 1) {
            b0 = min(b0, __shfl_xor_sync(0xffffffffu, b0, off));
            b1 = min(b1, __shfl_xor_sync(0xffffffffu, b1, off));
            b2 = max(b2, __shfl_xor_sync(0xffffffffu, b2, off));
            b3 = max(b3, __shfl_xor_sync(0xffffffffu, b3, off));
        }
        if (lane == 0) { atomicMin(&bb[0], b0); atomicMin(&bb[1], b1); atomicMax(&bb[2], b2); atomicMax(&bb[3], b3); }
    }
    for (long long t = tid; t < a.st_tiles / (TILE_CAP + 1); t += blockDim.x)
        a.tiles[t * (TILE_CAP + 1)] = 0;   // tile counts, for ib_tile_scatter
    __syncthreads();
    if (tid == 0) {
        PatchInfo pi{0, 0, 0, 0};
        if (bb[2] >= bb[0]) {
            pi.i0 = bb[0]; pi.j0 = bb[1]; pi.w = bb[2] - bb[0] + 1; pi.h = bb[3] - bb[1] + 1;
            if (pi.w > a.patch_wmax || pi.h > a.patch_hmax) {
                atomicOr(a.status, LBM_ST_OVERFLOW);
                pi = PatchInfo{0, 0, 0, 0};
            }
        }
        *a.pinfo = pi;
        *a.nsup = 0;   // counted by ib_tile_scatter
        const int w = *a.wmax;
        bad = 0;
        dense = (w > BS || a.force_dense) ? 1 : 0;
        a.fmode[0] = dense;
        a.fmode[1] = w;
        *a.wmax = 0;   // for the next assembly
    }
    __syncthreads();
    if (n == 0) return;
    if (dense) {
        dense_factor(a, &bad);
        __syncthreads();
        if (tid == 0 && bad) atomicOr(a.status, LBM_ST_SOLVER);
        return;
    }
    const int nb = (n + BS - 1) / BS;
    double *Db = a.bD, *Lb = a.bL, *Gf = a.gf;
    double *W = Wbase + (long long)warp * WS;
    const int pr = lane >> 1, ph = lane & 1;   // product lane layout: row, column half
    for (int st = 1; st < nb; st <<= 1) {
        const int nodd = (nb - st + 2 * st - 1) / (2 * st);
        for (int m = warp; m < nodd; m += BOPS_WARPS) {
            const int o = st * (2 * m + 1), q2 = o + st;
            double *Gs = W, *Rs = W + BS * GP;   // D_o, then [L_o | L_q^T]
            stage_sq(Gs, Db + (long long)o * BS * BS);
            {
                double lv[BS * BS / 32], lq[BS * BS / 32];
#pragma unroll
                for (int it = 0; it < BS * BS / 32; ++it) {
                    lv[it] = Lb[(long long)o * BS * BS + lane + 32 * it];
                    lq[it] = q2 < nb ? Lb[(long long)q2 * BS * BS + lane + 32 * it] : 0.0;
                }
#pragma unroll
                for (int it = 0; it < BS * BS / 32; ++it) {
                    const int e = lane + 32 * it, r = e / BS, c = e % BS;
                    Rs[r * FL + c] = lv[it];
                    Rs[c * FL + BS + r] = lq[it];
                }
            }
            __syncwarp();
            if (!warp_inv(Gs) && lane == 0) bad = 1;
            double *Go = Gf + (long long)o * BS * GW + pr * GW;
#pragma unroll
            for (int c = 0; c < BS / 2; ++c) Go[ph * (BS / 2) + c] = Gs[pr * GP + ph * (BS / 2) + c];
            double acc[BS];
            rowmm<BS, false>(Gs, Rs, FL, acc);
            double2 *F2 = reinterpret_cast<double2 *>(Go + BS + ph * BS);
#pragma unroll
            for (int c = 0; c < BS / 2; ++c) F2[c] = make_double2(acc[2 * c], acc[2 * c + 1]);
            __syncwarp();
        }
        __syncthreads();
        const int neven = (nb + 2 * st - 1) / (2 * st);
        for (int m = warp; m < neven; m += BOPS_WARPS) {
            const int e = 2 * st * m, o1 = e - st, o2 = e + st;
            double *As = W, *Fs = W + BS * GP, *Ds = Fs + BS * FL;
            double *De = Db + (long long)e * BS * BS, *Le = Lb + (long long)e * BS * BS;
            stage_sq(Ds, De);
            if (o2 < nb) {   // D_e -= L_q^T F_L(q)
                stage_sq(As, Lb + (long long)o2 * BS * BS);
                const double *G = Gf + (long long)o2 * BS * GW + BS;
                double v[BS * BS / 32];
#pragma unroll
                for (int it = 0; it < BS * BS / 32; ++it) {
                    const int q = lane + 32 * it;
                    v[it] = G[(q / BS) * GW + q % BS];
                }
#pragma unroll
                for (int it = 0; it < BS * BS / 32; ++it) {
                    const int q = lane + 32 * it;
                    Fs[(q / BS) * FL + q % BS] = v[it];
                }
                __syncwarp();
                double acc[BS / 2];
                rowmm<BS / 2, true>(As, Fs, FL, acc);
#pragma unroll
                for (int c = 0; c < BS / 2; ++c) Ds[pr * GP + ph * (BS / 2) + c] -= acc[c];
                __syncwarp();
            }
            if (m > 0) {   // D_e -= L_e F_U(p), L_e <- -L_e F_L(p); lanes h = 0 hold the new L_e row
                stage_sq(As, Le);
                const double *G = Gf + (long long)o1 * BS * GW + BS;
                double v[BS * FL / 32];
#pragma unroll
                for (int it = 0; it < BS * FL / 32; ++it) {
                    const int q = lane + 32 * it;
                    v[it] = G[(q / FL) * GW + q % FL];
                }
#pragma unroll
                for (int it = 0; it < BS * FL / 32; ++it) Fs[lane + 32 * it] = v[it];
                __syncwarp();
                double acc[BS];
                rowmm<BS, false>(As, Fs, FL, acc);
                if (ph == 0) {
                    double2 *L2 = reinterpret_cast<double2 *>(Le + pr * BS);
#pragma unroll
                    for (int c = 0; c < BS / 2; ++c) L2[c] = make_double2(-acc[2 * c], -acc[2 * c + 1]);
                } else {
#pragma unroll
                    for (int c = 0; c < BS; ++c) Ds[pr * GP + c] -= acc[c];
                }
                __syncwarp();
            }
#pragma unroll
            for (int it = 0; it < BS * BS / 32; ++it) {
                const int q = lane + 32 * it;
                De[q] = Ds[(q / BS) * GP + q % BS];
            }
            __syncwarp();
        }
        __syncthreads();
    }
    // block 0: inverted by every warp on its own copy, stored by warp 0 (a
    // lone warp working while the others wait at the barrier was measured
    // several times slower)
    {
        double *Gs = W;
        stage_sq(Gs, Db);
        __syncwarp();
        const bool ok = warp_inv(Gs);
        if (warp == 0) {
            double *Go = Gf + pr * GW;
#pragma unroll
            for (int c = 0; c < BS / 2; ++c) Go[ph * (BS / 2) + c] = Gs[pr * GP + ph * (BS / 2) + c];
            if (!ok && lane == 0) bad = 1;
        }
    }
    __syncthreads();
    if (tid == 0 && bad) atomicOr(a.status, LBM_ST_SOLVER);
}

// The flow-dependent solve of one step, one CTA (solve_threads: up to
// SOLVE_THREADS threads),
// with the cyclic-reduction factors of the step's slot:
//   forward, st = 1, 2, 4, ...:  r_e -= F_L(q)^T r_q + F_U(p)^T r_p  (even e)
//   block 0:                     x_0 = D_0^-1 r_0
//   backward, st = ..., 2, 1:    x_o = D_o^-1 r_o - F_L(o) x_p - F_U(o) x_q  (odd o)
// (F_L(q)^T = L_q^T D_q^-1 and F_U(p)^T = L_e D_p^-1 since D is symmetric.)
// Each level reads the factor blocks of that level's odd blocks; when they
// fit (at most stage_cap), the lanes of warp 0 bring them into shared memory
// with bulk copies (one 6-KB block each, completion on an mbarrier) before
// the level's arithmetic, so that the level costs one memory round trip
// instead of one per dependent load. The levels above the first usually fit
// together (31 blocks for 1024 markers): they then come in one round trip and
// serve both sweeps, so that the whole solve stages three times (level 1,
// the levels above it, level 1 again) instead of twice per level. Rows of a block are GW = 96 words apart,
// all on one bank: the backward sweep, which reads one row per lane pair,
// walks the columns in a rotated order (lane row i starts at column i) so
// that the 16 rows read in one step fall on distinct banks. Also writes the force row's header and reports the
// errors of the factorization chain. Dynamic shared memory: the staged
// blocks, then the right-hand sides in the solve order (two per marker,
// padded to whole blocks), then the mbarrier.
template <bool BATCH>
__global__ void __launch_bounds__(SOLVE_THREADS, 1024 / SOLVE_THREADS) ib_solve(const IBArgs a0, const IBArgs *batch, int step_index,
                                                          int ring_slot)
{
    const IBArgs &a = BATCH ? batch[blockIdx.z] : a0;
    extern __shared__ __align__(128) double smem[];
    const int n = a.nseg, tid = threadIdx.x, nt = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
    const int nb = (n + BS - 1) / BS;
    double *stage_buf = smem;
    // the staged blocks the launch made room for (solve_smem: stage_blocks(nb)),
    // read back from the dynamic shared-memory size rather than recomputed
    uint32_t dsm;
    asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dsm));
    const int scap = ((int)dsm - 16 - 2 * nb * BS * (int)sizeof(double)) / (BS * GW * (int)sizeof(double));
    double *X = smem + scap * BS * GW;
    uint64_t *bar = reinterpret_cast<uint64_t *>(X + 2 * nb * BS);
    __shared__ int timed_out;
    if (tid == 0) {
        double time;
        const double *row = motion_row(a, BATCH ? a.cur_step : step_index, &time);
        // batched launches take the row from the case's arguments (a CUDA
        // graph replays one launch for many steps)
        const int rr = BATCH ? a.ring_row : ring_slot;
        if (rr >= 0 && rr < a.ring_rows)
            write_header(a, row, time, rr);
        else
            atomicOr(a.status, LBM_ST_INDEX_SOLVE);
        const unsigned fs = *a.fstatus;
        if (fs) { atomicOr(a.status, fs); *a.fstatus = 0u; }
        a.solve_res[1] = (double)a.fmode[1];
        timed_out = 0;
        mbar_init(bar, 1);
        mbar_init_fence();
    }
    __syncthreads();
    if (n == 0) return;
    if (a.fmode[0]) {   // dense factor
        for (int s = tid; s < n; s += nt) {
            const int k = order_at(a, s, LBM_ST_INDEX_SOLVE);
            X[s] = k >= 0 ? a.rhs[k] : 0.0;
            X[n + s] = k >= 0 ? a.rhs[n + k] : 0.0;
        }
        __syncthreads();
        dense_tri(a, X);
        for (int s = tid; s < n; s += nt) {
            const int k = order_at(a, s, LBM_ST_INDEX_SOLVE);
            if (k < 0) continue;
            a.y[k] = X[s];
            a.y[n + k] = X[n + s];
        }
        return;
    }
    for (int s = tid; s < nb * BS; s += nt) {
        const int k = s < n ? order_at(a, s, LBM_ST_INDEX_SOLVE) : -1;
        X[2 * s] = k >= 0 ? a.rhs[k] : 0.0;
        X[2 * s + 1] = k >= 0 ? a.rhs[n + k] : 0.0;
    }
    const double *Gf = a.gf;
    uint32_t parity = 0;
    constexpr uint32_t kBlockBytes = sizeof(double) * BS * GW;
    auto nodd_of = [&](int st) { return (nb - st + 2 * st - 1) / (2 * st); };
    // bounded wait for the staged copies: copies that never land are
    // reported, not waited on forever
    auto stage_wait = [&]() {
        int spins = 0;
        while (!mbar_try_wait(bar, parity)) {
            if (++spins > (1 << 22)) { timed_out = 1; break; }
        }
        parity ^= 1u;
        __syncthreads();   // every thread sees the same timed_out
    };
    // factor blocks of the odd blocks of level st: staged (returns the base
    // of block o at index (o/st - 1)/2), or read from global memory
    auto stage_level = [&](int st) -> bool {
        const int nodd = nodd_of(st);
        if (nodd > scap) return false;
        __syncthreads();   // previous readers of the stage buffer are done
        if (warp == 0) {
            if (lane == 0) mbar_expect_tx(bar, kBlockBytes * (uint32_t)nodd);
            __syncwarp();
            fence_proxy_async();
            for (int m = lane; m < nodd; m += 32)
                bulk_g2s(stage_buf + m * BS * GW, Gf + (long long)st * (2 * m + 1) * BS * GW, kBlockBytes, bar);
        }
        stage_wait();
        return true;
    };
    // When the odd blocks of every level above the first fit in the stage
    // buffer together, they are staged once, in one round trip, when the
    // forward sweep reaches level 2, each level at its own base (upper_base),
    // and stay there for the rest of the forward sweep and for the backward
    // sweep down to level 2; only level 1 is staged twice (first and last).
    int upper = 0;
    for (int st = 2; st < nb; st <<= 1) upper += nodd_of(st);
    const bool resident = nodd_of(1) <= scap && upper <= scap;
    auto upper_base = [&](int st) {
        int b = 0;
        for (int s2 = 2; s2 < st; s2 <<= 1) b += nodd_of(s2);
        return b;
    };
    auto stage_upper = [&]() {
        __syncthreads();   // the first level's readers are done
        if (warp == 0) {
            if (lane == 0) mbar_expect_tx(bar, kBlockBytes * (uint32_t)upper);
            __syncwarp();
            fence_proxy_async();
            int b = 0;
            for (int st = 2; st < nb; st <<= 1) {
                const int nodd = nodd_of(st);
                for (int m = lane; m < nodd; m += 32)
                    bulk_g2s(stage_buf + (b + m) * BS * GW, Gf + (long long)st * (2 * m + 1) * BS * GW, kBlockBytes,
                             bar);
                b += nodd;
            }
        }
        stage_wait();
    };
    // the stage-buffer base (in blocks) of level st's odd blocks, staging
    // them first where needed; -1: read them from global memory
    auto level_base = [&](int st, bool forward) -> int {
        if (resident && st >= 2) {
            if (forward && st == 2) stage_upper();
            return upper_base(st);
        }
        return stage_level(st) ? 0 : -1;
    };
    __syncthreads();
    const int i = lane >> 1, c = lane & 1;   // row of the block, right-hand side
    int levels = 0;
    for (int st = 1; st < nb; st <<= 1, ++levels) {
        const int sbase = level_base(st, true);
        const bool staged = sbase >= 0;
        if (timed_out) break;
        const int neven = (nb + 2 * st - 1) / (2 * st);
        // one even block e per warp: F_L(q) and F_U(p) from block bases that
        // are either staged (shared memory, row stride GW) or global (GW);
        // the two forms are separate so that staged reads stay shared loads
        auto fwd = [&](const double *Fq, const double *Fp, int ld, int e, bool has_q, bool has_p) {
            double acc = 0.0;
            if (has_q) {
                const double *F = Fq + BS + i;       // F_L(q)[t][i]
                const double *r = X + 2 * (e + st) * BS + c;
#pragma unroll
                for (int t = 0; t < BS; ++t) acc += F[t * ld] * r[2 * t];
            }
            if (has_p) {
                const double *F = Fp + 2 * BS + i;   // F_U(p)[t][i]
                const double *r = X + 2 * (e - st) * BS + c;
#pragma unroll
                for (int t = 0; t < BS; ++t) acc += F[t * ld] * r[2 * t];
            }
            X[2 * (e * BS + i) + c] -= acc;
        };
        for (int m = warp; m < neven; m += nw) {
            const int e = 2 * st * m, o1 = e - st, o2 = e + st;
            const bool has_q = o2 < nb, has_p = m > 0;
            if (staged)   // odd block st(2k+1) is staged at index sbase + k
                fwd(stage_buf + (sbase + m) * BS * GW, stage_buf + (sbase + m - 1) * BS * GW, GW, e, has_q, has_p);
            else
                fwd(Gf + (long long)o2 * BS * GW, Gf + (long long)o1 * BS * GW, GW, e, has_q, has_p);
        }
        __syncthreads();
    }
    if (!timed_out) {
        if (warp == 0) {
            const double *G = Gf + i * GW;
            double x = 0.0;
#pragma unroll
            for (int t = 0; t < BS; ++t) x += G[t] * X[2 * t + c];
            __syncwarp();
            X[lane] = x;
        }
        __syncthreads();
        for (int lv = levels - 1; lv >= 0; --lv) {
            const int st = 1 << lv;
            const int sbase = level_base(st, false);
            const bool staged = sbase >= 0;
            if (timed_out) break;
            const int nodd = (nb - st + 2 * st - 1) / (2 * st);
            auto bwd = [&](const double *G, int o) {
                const int p = o - st, q2 = o + st;
                double s1 = 0.0, s2 = 0.0, s3 = 0.0;
#pragma unroll
                for (int t0 = 0; t0 < BS; ++t0) {
                    const int t = (t0 + i) & (BS - 1);   // rotated column order
                    s1 += G[t] * X[2 * (o * BS + t) + c];
                    s2 += G[BS + t] * X[2 * (p * BS + t) + c];
                }
                if (q2 < nb) {
#pragma unroll
                    for (int t0 = 0; t0 < BS; ++t0) {
                        const int t = (t0 + i) & (BS - 1);
                        s3 += G[2 * BS + t] * X[2 * (q2 * BS + t) + c];
                    }
                }
                __syncwarp();
                X[2 * (o * BS + i) + c] = s1 - s2 - s3;
            };
            for (int m = warp; m < nodd; m += nw) {
                const int o = st * (2 * m + 1);
                if (staged)
                    bwd(stage_buf + ((sbase + m) * BS + i) * GW, o);
                else
                    bwd(Gf + ((long long)o * BS + i) * GW, o);
            }
            __syncthreads();
        }
    }
    if (timed_out) {
        // wait (bounded) for copies still in flight before the CTA's shared
        // memory is released, and report
        if (tid == 0) atomicOr(a.status, LBM_ST_TIMEOUT);
        int spins = 0;
        while (!mbar_try_wait(bar, parity ^ 1u) && ++spins < (1 << 22)) {
        }
        return;
    }
    for (int s = tid; s < n; s += nt) {
        const int k = order_at(a, s, LBM_ST_INDEX_SOLVE);
        if (k < 0) continue;
        a.y[k] = X[2 * s];
        a.y[n + k] = X[2 * s + 1];
    }
}

// Markers whose support box meets each 16 x 16 tile of the step's patch
// rectangle. Layout per tile: count, then up to TILE_CAP marker indices in
// increasing order (the order of the tile update's sums); a larger count
// tells the tile update to scan all markers for that tile. Geometry only, so
// part of the factorization chain, in two passes: each marker appends itself
// to the (at most 2 x 2) tiles its box meets, then each tile sorts its list.
// ib_factor has cleared the counts.
template <bool BATCH>
__global__ void __launch_bounds__(256) ib_tile_scatter(const IBArgs base0, const IBArgs *batch, int step0)
{
    const IBArgs &base = BATCH ? batch[blockIdx.z] : base0;
    const int step_index = factor_step<BATCH>(base, step0);
    if (step_index < 0) return;
    const IBArgs a = member_args(base, step_index);
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.nseg) return;
    const PatchInfo pi = *a.pinfo;
    const int4 q = mbox(a.mk[k]);
    if (!box_in_bounds(q.x, q.y, q.z, q.w, a.nx, a.ny)) {
        atomicOr(a.status, LBM_ST_INDEX_SCATTER);
        return;
    }
    if (q.y < q.x || q.w < q.z || pi.w <= 0) return;
    // the box lies in the patch rectangle (its bounding box), which the tile
    // grid covers; a box or rectangle that says otherwise is not indexed
    if (q.x < pi.i0 || q.z < pi.j0 || q.y >= pi.i0 + a.tiles_x * TILE ||
        (long long)((q.w - pi.j0) / TILE + 1) * a.tiles_x > patch_tiles(a)) {
        atomicOr(a.status, LBM_ST_INDEX_SCATTER);
        return;
    }
    const int tx0 = (q.x - pi.i0) / TILE, tx1 = (q.y - pi.i0) / TILE;
    const int ty0 = (q.z - pi.j0) / TILE, ty1 = (q.w - pi.j0) / TILE;
    for (int ty = ty0; ty <= ty1; ++ty)
        for (int tx = tx0; tx <= tx1; ++tx) {
            const int tile = ty * a.tiles_x + tx;
            int *list = a.tiles + (long long)tile * (TILE_CAP + 1);
            const int pos = atomicAdd(list, 1);
            if (pos < TILE_CAP) list[1 + pos] = k;
        }
}

// The step's correction tiles (those listing a marker) in ascending tile
// order, by a block scan of the tile counts: one CTA per member. The order
// fixes the order of the force sum, so the force rows do not depend on the
// order the scatter's atomics happened to run in.
template <bool BATCH>
__global__ void __launch_bounds__(256) ib_tile_compact(const IBArgs base0, const IBArgs *batch, int step0)
{
    const IBArgs &base = BATCH ? batch[blockIdx.z] : base0;
    const int step_index = factor_step<BATCH>(base, step0);
    if (step_index < 0) return;
    const IBArgs a = member_args(base, step_index);
    __shared__ int wsum[8];
    const int nt = (int)(a.st_tiles / (TILE_CAP + 1));
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int per = (nt + 255) / 256, b0 = min(nt, t * per), b1 = min(nt, b0 + per);
    int cnt = 0;
    for (int b = b0; b < b1; ++b) cnt += a.tiles[(long long)b * (TILE_CAP + 1)] > 0;
    int x = cnt;   // inclusive scan within the warp
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    int before = 0;
    for (int w = 0; w < warp; ++w) before += wsum[w];
    int pos = before + x - cnt;
    for (int b = b0; b < b1; ++b)
        if (a.tiles[(long long)b * (TILE_CAP + 1)] > 0) a.ctile[pos++] = b;
    if (t == 255) *a.nsup = before + x;
}

// One warp per correction tile (8 per CTA): most tiles list a few dozen
// markers, which a warp sorts as fast as a CTA while holding an eighth of the
// SM slots the lattice update runs in.
constexpr int SORT_WARPS = 8;
// CTAs per step: 256 warps, about the correction tiles of a 1024-marker
// contour; larger contours loop
constexpr int SORT_CTAS = 32;
template <bool BATCH>
__global__ void __launch_bounds__(32 * SORT_WARPS) ib_tile_sort(const IBArgs base0, const IBArgs *batch, int step0)
{
    const IBArgs &base = BATCH ? batch[blockIdx.z] : base0;
    const int step_index = factor_step<BATCH>(base, step0);
    if (step_index < 0) return;
    const IBArgs a = member_args(base, step_index);
    __shared__ int keys[SORT_WARPS][TILE_CAP];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    int *key = keys[warp];
    const int nt = patch_tiles(a);
    int ntile = *a.nsup;
    if (ntile < 0 || ntile > nt) {
        if (lane == 0) atomicOr(a.status, LBM_ST_INDEX_SORT);
        ntile = 0;
    }
    for (int c = blockIdx.x * SORT_WARPS + warp; c < ntile; c += gridDim.x * SORT_WARPS) {
        const int tile = a.ctile[c];
        if (tile < 0 || tile >= nt) {
            if (lane == 0) atomicOr(a.status, LBM_ST_INDEX_SORT);
            continue;
        }
        int *list = a.tiles + (long long)tile * (TILE_CAP + 1);
        const int m = min(list[0], TILE_CAP);
        int np = 2;   // keys sorted: the power of two at or above the count
        while (np < m) np <<= 1;
        for (int t = lane; t < np; t += 32) key[t] = t < m ? list[1 + t] : 0x7fffffff;
        __syncwarp();
        // bitonic sort of np keys, ascending (the padding keys stay at the
        // end); the pairs (t, t ^ stride) of a stage are disjoint
        for (int size = 2; size <= np; size <<= 1)
            for (int stride = size >> 1; stride > 0; stride >>= 1) {
                for (int t = lane; t < np; t += 32) {
                    const int u = t ^ stride;
                    if (u > t) {
                        const bool up = (t & size) == 0;
                        const int x = key[t], y = key[u];
                        if ((x > y) == up) { key[t] = y; key[u] = x; }
                    }
                }
                __syncwarp();
            }
        for (int t = lane; t < m; t += 32) list[1 + t] = key[t];
        __syncwarp();
    }
}

// The step's force row from the correction tiles' partials, summed over the
// compact tile list in ascending tile order (deterministic), one CTA; no
// correction tile gives zero forces (solution.f90:327-330 normalisation).
// Needed by no kernel of the step, so it runs after the step's update.
template <bool BATCH>
__global__ void __launch_bounds__(256) ib_forces(const IBArgs a0, const IBArgs *batch, int ring_slot)
{
    const IBArgs &a = BATCH ? batch[blockIdx.z] : a0;
    __shared__ double red[8][NPART];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nt = patch_tiles(a);
    int ntile = a.nseg > 0 ? *a.nsup : 0;
    if (ntile < 0 || ntile > nt) {
        if (threadIdx.x == 0) atomicOr(a.status, LBM_ST_INDEX_FORCES);
        ntile = 0;
    }
    for (int w = 0; w < a.nwing; ++w) {
        double s0 = 0, s1 = 0, s2 = 0;
        for (int c = threadIdx.x; c < ntile; c += blockDim.x) {
            const int tile = a.ctile[c];
            if (tile < 0 || tile >= nt) {
                atomicOr(a.status, LBM_ST_INDEX_FORCES);
                continue;
            }
            const double *p = a.partial + (long long)tile * NPART + 3 * w;
            s0 += p[0]; s1 += p[1]; s2 += p[2];
        }
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            s0 += __shfl_down_sync(0xffffffffu, s0, off);
            s1 += __shfl_down_sync(0xffffffffu, s1, off);
            s2 += __shfl_down_sync(0xffffffffu, s2, off);
        }
        if (lane == 0) { red[warp][3 * w] = s0; red[warp][3 * w + 1] = s1; red[warp][3 * w + 2] = s2; }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        const int rr = BATCH ? a.ring_row : ring_slot;
        if (rr < 0 || rr >= a.ring_rows) {
            atomicOr(a.status, LBM_ST_INDEX_FORCES);
            return;
        }
        double *fr = a.force_ring + (long long)rr * a.row_len;
        double tot[3] = {0, 0, 0};
        const double uu = a.uu, scale = a.scale;
        for (int w = 0; w < a.nwing; ++w) {
            double s0 = 0, s1 = 0, s2 = 0;
            for (int w8 = 0; w8 < 8; ++w8) { s0 += red[w8][3 * w]; s1 += red[w8][3 * w + 1]; s2 += red[w8][3 * w + 2]; }
            const double cx = 2.0 * s0 / (uu * uu * (1.0 / scale));
            const double cy = 2.0 * s1 / (uu * uu * (1.0 / scale));
            const double cm = -2.0 * s2 / (uu * uu * (1.0 / (scale * scale)));
            fr[1 + 3 * w] = cx; fr[2 + 3 * w] = cy; fr[3 + 3 * w] = cm;
            tot[0] += cx; tot[1] += cy; tot[2] += cm;
            if (!isfinite(cx) || !isfinite(cy) || !isfinite(cm)) atomicOr(a.status, LBM_ST_NONFINITE);
        }
        fr[1 + 3 * a.nwing] = tot[0];
        fr[2 + 3 * a.nwing] = tot[1];
        fr[3 + 3 * a.nwing] = tot[2];
    }
}

// Residual of the step's solve, ||B y - rhs|| / ||rhs|| with B = D D^T
// recomputed from the marker geometry (independent of the factorization):
// one warp per row of the solve order, lanes over the couplings within the
// half-bandwidth; deterministic two-level sum (CTA partials, last CTA).
// Flags LBM_ST_SOLVER unless it is below 1e-6, or LBM_ST_NONFINITE when the
// right-hand side itself is not finite (the flow at the markers diverged).
template <bool BATCH>
__global__ void __launch_bounds__(256) ib_residual(const IBArgs a0, const IBArgs *batch)
{
    const IBArgs &a = BATCH ? batch[blockIdx.z] : a0;
    if (BATCH && !a.check_res) return;   // this case's step is not checked
    __shared__ double red[8][2];
    __shared__ bool amlast;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = a.nseg, s = blockIdx.x * 8 + warp;
    const int nblk = (n + 7) / 8;
    if ((int)blockIdx.x >= nblk) return;    // batched launches size the grid for the largest case
    const int hw = min(max((int)a.solve_res[1], 0), n);
    double rnum = 0.0, rden = 0.0;
    const int ks = s < n ? order_at(a, s, LBM_ST_INDEX_RESIDUAL) : -1;
    if (ks >= 0) {
        const Marker &ms = a.mk[ks];
        const bool ok_s = marker_ok(a, ms);
        if (!ok_s && lane == 0) atomicOr(a.status, LBM_ST_INDEX_RESIDUAL);
        double b0 = 0.0, b1 = 0.0;
        for (int t = s - hw + lane; t <= s + hw && ok_s; t += 32) {
            if (t < 0 || t >= n) continue;
            const Marker *ml = sorted_marker(a, t, LBM_ST_INDEX_RESIDUAL);
            if (!ml) continue;
            const int l = (int)(ml - a.mk);
            const double b = bval(ms, *ml);
            b0 += b * a.y[l];
            b1 += b * a.y[n + l];
        }
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            b0 += __shfl_xor_sync(0xffffffffu, b0, off);
            b1 += __shfl_xor_sync(0xffffffffu, b1, off);
        }
        const double q0 = a.rhs[ks], q1 = a.rhs[n + ks];
        rnum = (b0 - q0) * (b0 - q0) + (b1 - q1) * (b1 - q1);
        rden = q0 * q0 + q1 * q1;
    }
    if (lane == 0) { red[warp][0] = rnum; red[warp][1] = rden; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t0 = 0, t1 = 0;
        for (int w = 0; w < 8; ++w) { t0 += red[w][0]; t1 += red[w][1]; }
        a.partial[2 * blockIdx.x] = t0;
        a.partial[2 * blockIdx.x + 1] = t1;
        __threadfence();
        amlast = atomicAdd(a.counter, 1u) == (unsigned)(nblk - 1);
    }
    __syncthreads();
    if (!amlast) return;
    __threadfence();
    double s0 = 0.0, s1 = 0.0;
    for (int b = threadIdx.x; b < nblk; b += blockDim.x) {
        s0 += __ldcg(a.partial + 2 * b);
        s1 += __ldcg(a.partial + 2 * b + 1);
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        s0 += __shfl_down_sync(0xffffffffu, s0, off);
        s1 += __shfl_down_sync(0xffffffffu, s1, off);
    }
    __syncthreads();
    if (lane == 0) { red[warp][0] = s0; red[warp][1] = s1; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sn = 0, sd = 0;
        for (int w = 0; w < 8; ++w) { sn += red[w][0]; sd += red[w][1]; }
        const double res = sqrt(sn) / (sqrt(sd) + 1e-300);
        a.solve_res[0] = res;
        if (!isfinite(sd))
            atomicOr(a.status, LBM_ST_NONFINITE);
        else if (!(res < 1e-6))
            atomicOr(a.status, LBM_ST_SOLVER);
        *a.counter = 0u;
    }
}

// The correction tiles of the step (the 16 x 16 tiles of the patch
// rectangle that list a marker), one CTA per tile: du = D^T y per node,
// gathered in marker order over the markers whose box covers the node (no
// atomics); then the lattice update of the tile's nodes with that velocity
// correction (the node path of the lattice kernels); and each node's FP64
// force and moment (boundary_condition.f90:1645-1675, solution.f90:327-336).
// The last CTA sums the per-tile partials in tile order into the step's force
// row. The lattice kernel updates every other node.
template <typename T, typename C, bool FIELDS, bool BATCH>
__global__ void __launch_bounds__(256) ib_tile_update(const IBArgs a0, const IBArgs *batch, const KFArgs<C> kf0,
                                                      const KFArgs<C> *kbatch, int step_index, int ring_slot)
{
    const IBArgs &a = BATCH ? batch[blockIdx.z] : a0;
    const KFArgs<C> &kf = BATCH ? kbatch[blockIdx.z] : kf0;
    __shared__ int wsum[8];
    __shared__ int nlist;
    __shared__ double red[8][NPART];
    // markers whose support box meets the current tile, staged in marker order
    __shared__ int4 sbox[256];
    __shared__ double sph[256][12];
    __shared__ double sy[256][2];
    __shared__ int swing[256];
    const int nt = patch_tiles(a);
    const int ntile = *a.nsup;
    if (ntile == 0) return;   // no correction tile
    if (ntile < 0 || ntile > nt) {
        if (threadIdx.x == 0) atomicOr(a.status, LBM_ST_INDEX_TILE);
        return;
    }
    const PatchInfo pi = *a.pinfo;
    const T *__restrict__ fin = (const T *)kf.fin;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // the correction tiles, strided over the CTAs (the compact list is in no
    // particular order; each tile's result depends on the tile only)
    for (int c = blockIdx.x; c < ntile; c += gridDim.x) {
        const int tile = a.ctile[c];
        if (tile < 0 || tile >= nt) {   // the same for every thread of the CTA
            if (threadIdx.x == 0) atomicOr(a.status, LBM_ST_INDEX_TILE);
            continue;
        }
        const int ti0 = (tile % a.tiles_x) * TILE, tj0 = (tile / a.tiles_x) * TILE;
        const int *tlist = a.tiles + (long long)tile * (TILE_CAP + 1);
        const int listed = tlist[0];
        const int li = ti0 + tx, lj = tj0 + ty;                    // patch-relative
        const int gi = pi.i0 + li, gj = pi.j0 + lj;                // 0-based node
        bool active = li < pi.w && lj < pi.h;
        // the patch rectangle is the bounding box of the support boxes, all
        // interior nodes; a node outside the interior is not updated here
        if (active && (gi < 1 || gi > kf.nx - 2 || gj < 1 || gj > kf.ny - 2)) {
            atomicOr(a.status, LBM_ST_INDEX_TILE);
            active = false;
        }
        const int ta = pi.i0 + ti0, tb = ta + TILE - 1, sa_ = pi.j0 + tj0, sb_ = sa_ + TILE - 1;
        // the node's streamed populations first: their loads overlap the
        // staging of the markers
        C g[9];
        if (active) lbm_node::pull<T, C>(fin, kf.plane, kf.pitch, gi, gj, g);
        double du = 0.0, dv = 0.0;
        int wing = 1 << 20;
        if (listed <= TILE_CAP) {
            // markers listed for this tile by the factorization chain
            if (threadIdx.x == 0) nlist = listed;
            if ((int)threadIdx.x < listed) {
                const int k = tlist[1 + threadIdx.x];
                if (k >= 0 && k < a.nseg && marker_ok(a, a.mk[k])) {
                    const Marker &m = a.mk[k];
                    sbox[threadIdx.x] = mbox(m);
#pragma unroll
                    for (int q = 0; q < 6; ++q) { sph[threadIdx.x][q] = m.phx[q]; sph[threadIdx.x][6 + q] = m.phy[q]; }
                    sy[threadIdx.x][0] = a.y[k];
                    sy[threadIdx.x][1] = a.y[a.nseg + k];
                    swing[threadIdx.x] = m.wing;
                } else {   // not staged: an empty box meets no node
                    atomicOr(a.status, LBM_ST_INDEX_TILE);
                    sbox[threadIdx.x] = make_int4(1, 0, 1, 0);
                    sy[threadIdx.x][0] = sy[threadIdx.x][1] = 0.0;
                    swing[threadIdx.x] = 0;
                }
            }
            __syncthreads();
            if (active) {
                for (int t = 0; t < nlist; ++t) {
                    const int4 b = sbox[t];
                    if (gi >= b.x && gi <= b.y && gj >= b.z && gj <= b.w) {
                        const double wgt = sph[t][gi - b.x] * sph[t][6 + gj - b.z];
                        du += wgt * sy[t][0];
                        dv += wgt * sy[t][1];
                        wing = min(wing, swing[t]);
                    }
                }
            }
        } else {
            // more markers than a list holds: scan all of them, in order
            for (int c0 = 0; c0 < a.nseg; c0 += 256) {
                const int k = c0 + threadIdx.x;
                bool hit = false;
                int4 q = make_int4(1, 0, 1, 0);
                if (k < a.nseg) {
                    if (marker_ok(a, a.mk[k])) {
                        q = mbox(a.mk[k]);
                        hit = q.x <= tb && q.y >= ta && q.z <= sb_ && q.w >= sa_ && q.y >= q.x;
                    } else {
                        atomicOr(a.status, LBM_ST_INDEX_TILE);
                    }
                }
                const unsigned bal = __ballot_sync(0xffffffffu, hit);
                if (lane == 0) wsum[warp] = __popc(bal);
                __syncthreads();
                if (threadIdx.x == 0) {
                    int acc = 0;
                    for (int w = 0; w < 8; ++w) { const int t = wsum[w]; wsum[w] = acc; acc += t; }
                    nlist = acc;
                }
                __syncthreads();
                if (hit) {
                    const int slot = wsum[warp] + __popc(bal & ((1u << lane) - 1u));
                    const Marker &m = a.mk[k];
                    sbox[slot] = q;
#pragma unroll
                    for (int r = 0; r < 6; ++r) { sph[slot][r] = m.phx[r]; sph[slot][6 + r] = m.phy[r]; }
                    sy[slot][0] = a.y[k];
                    sy[slot][1] = a.y[a.nseg + k];
                    swing[slot] = m.wing;
                }
                __syncthreads();
                if (active) {
                    for (int t = 0; t < nlist; ++t) {
                        const int4 b = sbox[t];
                        if (gi >= b.x && gi <= b.y && gj >= b.z && gj <= b.w) {
                            const double wgt = sph[t][gi - b.x] * sph[t][6 + gj - b.z];
                            du += wgt * sy[t][0];
                            dv += wgt * sy[t][1];
                            wing = min(wing, swing[t]);
                        }
                    }
                }
                __syncthreads();
            }
        }
        // lattice update of the node with the correction, and its force and moment
        double fx = 0, fy = 0, mz = 0;
        const bool in_support = active && wing < (1 << 20);
        if (active) {
            C gout[9], frho, fu, fv;
            lbm_node::collide_interior<C>(kf, g, true, (C)du, (C)dv, gout, frho, fu, fv);
            lbm_node::store_node<T, C, FIELDS>(kf, (T *)kf.fout, gi, gj, gout, frho, fu, fv);
            if (in_support) {
                // FP64 density of the same streamed populations
                const double drho = (((double)g[0] + (double)g[1]) + ((double)g[2] + (double)g[3])) +
                                    (((double)g[4] + (double)g[5]) + ((double)g[6] + (double)g[7])) + (double)g[8];
                const double rho = 1.0 + drho;
                const double *row = motion_row(a, BATCH ? a.cur_step : step_index, nullptr);
                const double temp1 = 2.0 * rho * du, temp2 = 2.0 * rho * dv;
                const double sa = row[4 + 9 * wing], sb = row[7 + 9 * wing];
                fx = -temp1;
                fy = -temp2;
                const double x0 = (a.ox + a.scale * (double)gi - (a.xc + sa)) / a.scale;
                const double y0 = (a.oy + a.scale * (double)gj - (a.yc + sb)) / a.scale;
                mz = -x0 * temp2 + y0 * temp1;
            }
        }
        // deterministic tile reduction per wing, into the tile's partials
        for (int w = 0; w < a.nwing; ++w) {
            double v0 = (in_support && wing == w) ? fx : 0.0;
            double v1 = (in_support && wing == w) ? fy : 0.0;
            double v2 = (in_support && wing == w) ? mz : 0.0;
#pragma unroll
            for (int off = 16; off; off >>= 1) {
                v0 += __shfl_down_sync(0xffffffffu, v0, off);
                v1 += __shfl_down_sync(0xffffffffu, v1, off);
                v2 += __shfl_down_sync(0xffffffffu, v2, off);
            }
            if (lane == 0) { red[warp][3 * w] = v0; red[warp][3 * w + 1] = v1; red[warp][3 * w + 2] = v2; }
        }
        __syncthreads();
        if (threadIdx.x < 3 * a.nwing) {
            double sum = 0.0;
            for (int w8 = 0; w8 < 8; ++w8) sum += red[w8][threadIdx.x];
            a.partial[(long long)tile * NPART + threadIdx.x] = sum;
        }
        __syncthreads();   // shared arrays are reused by the next tile
    }
}


size_t order_smem(int n)
{
    int ns = 1;
    while (ns < n) ns <<= 1;
    return (sizeof(double) + sizeof(int)) * ns;
}

constexpr size_t kFactorSmem = sizeof(double) * BOPS_WARPS * WS;
constexpr size_t kSolveSmemMax = SOLVE_SMEM_BUDGET;
size_t solve_smem(int nseg)
{
    const int nb = (nseg + BS - 1) / BS;
    return sizeof(double) * ((size_t)stage_blocks(nb) * BS * GW + 2 * (size_t)nb * BS) + 16;
}

// threads of the solve's CTA: one warp per even block of the first level
// (the widest), from 4 to SOLVE_THREADS / 32 warps. A solve of a few hundred
// markers then holds a fraction of an SM beside the lattice kernel instead
// of a whole one; each block's arithmetic is one warp's whatever the count,
// so the results do not depend on it.
int solve_threads(int nseg)
{
    const int nb = (nseg + BS - 1) / BS;
    return 32 * std::min(SOLVE_THREADS / 32, std::max(4, (nb + 1) / 2));
}

// arguments of the flow chain of the step held in buffer slot `slot`; for
// the batched factorization kernels, the arguments of slot 0 and member 0
// with the strides that member_args applies
IBArgs make_args(lbm_handle *h, const void *fin, int slot)
{
    const size_t ns = (size_t)(h->nseg > 0 ? h->nseg : 1);
    IBArgs a;
    a.fin = fin;
    a.prec = h->prec;
    a.nx = h->nx; a.ny = h->ny; a.pitch = h->pitch; a.plane = h->plane;
    a.nwing = h->nwing; a.ppw = h->ppw; a.spw = h->spw; a.nseg = h->nseg;
    a.smooth = h->p.delta_kernel;
    a.force_dense = (h->p.flags & LBM_FLAG_DENSE_SOLVE) != 0;
    a.scale = h->p.scale; a.ox = h->p.ox; a.oy = h->p.oy; a.uu = h->p.uu;
    a.xc = h->p.xc; a.yc = h->p.yc; a.mesh_max_scale = h->p.mesh_max_scale;
    a.xb0 = h->d_xb0; a.yb0 = h->d_yb0; a.arc = h->d_arc;
    a.mstep = h->d_mstep; a.msteps = h->msteps; a.mcols = h->mcols; a.mdt = h->mdt;
    a.nslots = h->nslots;
    a.static_order = h->static_order;
    a.st_mk = (long long)ns;
    a.st_perm = h->static_order ? 0 : (long long)ns;
    a.st_B = (long long)(ns * ns);
    a.wk_blocks = (long long)h->work_blocks;
    a.wk_gf = (long long)h->gf_slot;
    a.mk = h->d_mk + slot * ns;
    a.perm = h->d_perm + slot * a.st_perm;
    a.key = h->d_key + slot * a.st_perm;
    a.B = h->d_B + slot * ns * ns;
    a.fmode = h->d_fmode + 2 * slot;
    a.fstatus = h->d_fstatus + slot;
    a.pinfo = h->d_pinfo + slot;
    a.tiles_x = h->patch_gx();
    a.st_tiles = (long long)h->patch_gx() * h->patch_gy() * (TILE_CAP + 1);
    a.tiles = h->d_tiles + slot * a.st_tiles;
    a.gf = h->d_gf + slot * h->gf_slot;
    // the step's own right-hand sides, solution, tile partials and residual
    // slots: one set per step parity, so that the check of a step may run
    // while the next step's flow chain fills the other set
    const int par = h->n & 1;
    const long long ns2 = 2ll * (h->nseg > 0 ? h->nseg : 1);
    a.rhs = h->d_rhs + par * ns2; a.y = h->d_y + par * ns2;
    a.bD = h->d_bD; a.bL = h->d_bL;
    a.reach = h->d_reach; a.wmax = h->d_wmax;
    a.nsup = h->d_nsup + slot;
    a.ctile = h->d_ctile + slot * (a.st_tiles / (TILE_CAP + 1));
    a.patch_wmax = h->patch_wmax; a.patch_hmax = h->patch_hmax;
    a.partial = h->d_partial + par * (long long)h->part_stride; a.counter = h->d_counter;
    a.force_ring = h->d_ring; a.row_len = h->row_len;
    a.ring_row = 0; a.ring_rows = h->ring_cap;
    a.status = h->d_status; a.solve_res = h->d_solve_res + 2 * par;
    a.cur_step = h->n;
    a.fstep0 = 0; a.fcount = 0;
    a.check_res = 1;
    return a;
}

template <typename T, typename C>
int launch_flow_t(lbm_handle *h, const void *fin, void *fout, void *fields, int step_index, int ring_slot, int slot,
                  cudaStream_t st, cudaEvent_t after_interp)
{
    IBArgs a = make_args(h, fin, slot);
    if (h->nseg > 0) {
        ib_interp<T, false><<<(h->nseg + 7) / 8, 256, 0, st>>>(a, nullptr);
        h->launches += 1;
    }
    if (after_interp && cudaEventRecord(after_interp, st) != cudaSuccess) return -1;
    ib_solve<false><<<1, solve_threads(h->nseg), solve_smem(h->nseg), st>>>(a, nullptr, step_index, ring_slot);
    const int grid = std::min(h->patch_gx() * h->patch_gy(), 2 * 148);   // strided over the correction tiles
    const KFArgs<C> kf = make_kf_args<C>(h, fin, fout, fields, KF_OUTER);
    if (fields)
        ib_tile_update<T, C, true, false><<<grid, 256, 0, st>>>(a, nullptr, kf, nullptr, step_index, ring_slot);
    else
        ib_tile_update<T, C, false, false><<<grid, 256, 0, st>>>(a, nullptr, kf, nullptr, step_index, ring_slot);
    h->launches += 2;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// the residual check of the step's solve (needed by no later kernel of the step)
template <typename T, typename C>
int launch_check_t(lbm_handle *h, int slot, int ring_slot, bool residual, cudaStream_t st)
{
    IBArgs a = make_args(h, nullptr, slot);
    ib_forces<false><<<1, 256, 0, st>>>(a, nullptr, ring_slot);
    h->launches += 1;
    if (h->nseg == 0 || !residual) return cudaGetLastError() == cudaSuccess ? 0 : -1;
    ib_residual<false><<<(h->nseg + 7) / 8, 256, 0, st>>>(a, nullptr);
    h->launches += 1;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace

// per-CTA partials of ib_tile_update (doubles)
int ib_partials_per_block() { return NPART; }

// ints per patch tile of the tile lists (count + TILE_CAP indices)
int ib_tile_ints() { return TILE_CAP + 1; }

// scratch of the block cyclic reduction (doubles): working diagonal and
// coupling blocks (one set), and the factor buffer of one slot
void ib_factor_scratch(int nseg, size_t *work_blocks, size_t *factor_slot)
{
    const size_t nb = (size_t)(nseg + BS - 1) / BS;
    *work_blocks = nb * BS * BS;
    *factor_slot = nb * BS * GW;
}

int ib_max_markers() { return NMARK_MAX; }

template <bool BATCH>
int ib_configure_t()
{
    if (cudaFuncSetAttribute(ib_factor<BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kFactorSmem) !=
        cudaSuccess)
        return -1;
    if (cudaFuncSetAttribute(ib_solve<BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSolveSmemMax) !=
        cudaSuccess)
        return -1;
    if (cudaFuncSetAttribute(ib_order<BATCH>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)order_smem(NMARK_MAX)) != cudaSuccess)
        return -1;
    return 0;
}

int ib_configure(lbm_handle *h)
{
    (void)h;
    return ib_configure_t<false>() || ib_configure_t<true>() ? -1 : 0;
}

// factorization chains of the `count` steps step0, step0+1, ... (each into
// its slot), one launch per kernel with the steps along grid y
int launch_factor(lbm_handle *h, int step0, int count, cudaStream_t st)
{
    if (h->nseg == 0 || count <= 0) return 0;
    const IBArgs a = make_args(h, nullptr, 0);
    const int nb = (h->nseg + BS - 1) / BS;
    ib_geometry<false><<<dim3((h->nseg + 127) / 128, count), 128, 0, st>>>(a, nullptr, step0);
    if (!h->static_order) ib_order<false><<<dim3(1, count), 1024, order_smem(h->nseg), st>>>(a, nullptr, step0);
    ib_assemble<false><<<dim3(nb, count), 256, 0, st>>>(a, nullptr, step0);
    ib_factor<false><<<dim3(1, count), FACTOR_THREADS, kFactorSmem, st>>>(a, nullptr, step0);
    ib_tile_scatter<false><<<dim3((h->nseg + 255) / 256, count), 256, 0, st>>>(a, nullptr, step0);
    ib_tile_compact<false><<<dim3(1, count), 256, 0, st>>>(a, nullptr, step0);
    const int sort_ctas = std::min((h->patch_gx() * h->patch_gy() + SORT_WARPS - 1) / SORT_WARPS, SORT_CTAS);
    ib_tile_sort<false><<<dim3(sort_ctas, count), 32 * SORT_WARPS, 0, st>>>(a, nullptr, step0);
    h->launches += h->static_order ? 6 : 7;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// force row and residual check of the step held in `slot`, after its flow chain
int launch_check(lbm_handle *h, int slot, int ring_slot, bool residual, cudaStream_t st)
{
    return launch_check_t<float, float>(h, slot, ring_slot, residual, st ? st : h->stream);
}

// flow chain of step `step_index`: interpolation, solve with the factor of
// `slot`, spread and forces
int launch_flow(lbm_handle *h, const void *fin, void *fout, void *fields, int step_index, int ring_slot, int slot,
                cudaStream_t st, cudaEvent_t after_interp)
{
    if (!st) st = h->stream;
    switch (h->prec) {
    case LBM_PREC_FP32:
        return launch_flow_t<float, float>(h, fin, fout, fields, step_index, ring_slot, slot, st, after_interp);
    case LBM_PREC_FP64:
        return launch_flow_t<double, double>(h, fin, fout, fields, step_index, ring_slot, slot, st, after_interp);
    case LBM_PREC_FP16:
        return launch_flow_t<__half, float>(h, fin, fout, fields, step_index, ring_slot, slot, st, after_interp);
    case LBM_PREC_BF16:
        return launch_flow_t<__nv_bfloat16, float>(h, fin, fout, fields, step_index, ring_slot, slot, st, after_interp);
    }
    return -1;
}

// ---- batches of cases (lbm_batch.cu): arguments from device arrays, one
// launch per kernel for all cases (grid z = case), grids sized for the
// largest case

size_t ib_args_size() { return sizeof(IBArgs); }

void ib_args_write(lbm_handle *h, const void *fin, int slot, void *dst) { *(IBArgs *)dst = make_args(h, fin, slot); }

void ib_factor_args_write(lbm_handle *h, int step0, int count, void *dst)
{
    IBArgs a = make_args(h, nullptr, 0);
    a.fstep0 = step0;
    a.fcount = count;
    *(IBArgs *)dst = a;
}

namespace {

int max_seg(lbm_handle *const *hs, int n)
{
    int m = 0;
    for (int c = 0; c < n; ++c) m = std::max(m, hs[c]->nseg);
    return m;
}

constexpr int kBatchTileCtas = 64;

template <typename T, typename C>
int launch_flow_batch_t(lbm_handle *const *hs, int ncase, const IBArgs *dargs, const void *dkf, int step_index,
                        int ring_slot, bool fields, cudaStream_t st, cudaEvent_t after_interp)
{
    const int ns = max_seg(hs, ncase);
    ib_interp<T, true><<<dim3((ns + 7) / 8, 1, ncase), 256, 0, st>>>(IBArgs{}, dargs);
    if (after_interp && cudaEventRecord(after_interp, st) != cudaSuccess) return -1;
    ib_solve<true><<<dim3(1, 1, ncase), solve_threads(ns), solve_smem(ns), st>>>(IBArgs{}, dargs, step_index,
                                                                                ring_slot);
    // CTAs per case, strided over the case's correction tiles: the patch
    // grids bound the tiles several times over (a sweep case of chord 256
    // has some 60 correction tiles in a grid of hundreds), and CTAs past a
    // case's tiles still take lattice slots at the flow chain's priority, so
    // a batch launches at most kBatchTileCtas per case
    int tiles = 1;
    for (int c = 0; c < ncase; ++c) tiles = std::max(tiles, hs[c]->patch_gx() * hs[c]->patch_gy());
    const dim3 grid(std::min(tiles, kBatchTileCtas), 1, ncase);
    const KFArgs<C> *kf = (const KFArgs<C> *)dkf;
    if (fields)
        ib_tile_update<T, C, true, true><<<grid, 256, 0, st>>>(IBArgs{}, dargs, KFArgs<C>{}, kf, step_index, ring_slot);
    else
        ib_tile_update<T, C, false, true><<<grid, 256, 0, st>>>(IBArgs{}, dargs, KFArgs<C>{}, kf, step_index, ring_slot);
    for (int c = 0; c < ncase; ++c) hs[c]->launches += 3;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace

// factorization chains of the steps step0 .. step0+count-1 of every case
int launch_factor_batch(lbm_handle *const *hs, int ncase, const void *dargs, int step0, int count, cudaStream_t st)
{
    if (ncase <= 0 || count <= 0) return 0;
    const IBArgs *d = (const IBArgs *)dargs;
    const int ns = max_seg(hs, ncase), nb = (ns + BS - 1) / BS;
    bool any_order = false;
    int tiles = 1;
    for (int c = 0; c < ncase; ++c) {
        any_order = any_order || !hs[c]->static_order;
        tiles = std::max(tiles, hs[c]->patch_gx() * hs[c]->patch_gy());
    }
    ib_geometry<true><<<dim3((ns + 127) / 128, count, ncase), 128, 0, st>>>(IBArgs{}, d, step0);
    if (any_order) ib_order<true><<<dim3(1, count, ncase), 1024, order_smem(ns), st>>>(IBArgs{}, d, step0);
    ib_assemble<true><<<dim3(nb, count, ncase), 256, 0, st>>>(IBArgs{}, d, step0);
    ib_factor<true><<<dim3(1, count, ncase), FACTOR_THREADS, kFactorSmem, st>>>(IBArgs{}, d, step0);
    ib_tile_scatter<true><<<dim3((ns + 255) / 256, count, ncase), 256, 0, st>>>(IBArgs{}, d, step0);
    ib_tile_compact<true><<<dim3(1, count, ncase), 256, 0, st>>>(IBArgs{}, d, step0);
    ib_tile_sort<true><<<dim3(std::min((tiles + SORT_WARPS - 1) / SORT_WARPS, SORT_CTAS), count, ncase),
                         32 * SORT_WARPS, 0, st>>>(IBArgs{}, d, step0);
    for (int c = 0; c < ncase; ++c) hs[c]->launches += any_order ? 7 : 6;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// flow chains of one step of every case (dargs: the cases' arguments of the
// step's slot; dkf: their lattice arguments)
int launch_flow_batch(lbm_handle *const *hs, int ncase, const void *dargs, const void *dkf, int step_index,
                      int ring_slot, bool fields, cudaStream_t st, cudaEvent_t after_interp)
{
    if (ncase <= 0) return 0;
    const IBArgs *d = (const IBArgs *)dargs;
    switch (hs[0]->prec) {
    case LBM_PREC_FP32:
        return launch_flow_batch_t<float, float>(hs, ncase, d, dkf, step_index, ring_slot, fields, st, after_interp);
    case LBM_PREC_FP64:
        return launch_flow_batch_t<double, double>(hs, ncase, d, dkf, step_index, ring_slot, fields, st, after_interp);
    case LBM_PREC_FP16:
        return launch_flow_batch_t<__half, float>(hs, ncase, d, dkf, step_index, ring_slot, fields, st, after_interp);
    case LBM_PREC_BF16:
        return launch_flow_batch_t<__nv_bfloat16, float>(hs, ncase, d, dkf, step_index, ring_slot, fields, st,
                                                         after_interp);
    }
    return -1;
}

// force rows and residual checks of one step of every case
int launch_check_batch(lbm_handle *const *hs, int ncase, const void *dargs, int ring_slot, bool residual,
                       cudaStream_t st)
{
    if (ncase <= 0) return 0;
    const IBArgs *d = (const IBArgs *)dargs;
    const int ns = max_seg(hs, ncase);
    ib_forces<true><<<dim3(1, 1, ncase), 256, 0, st>>>(IBArgs{}, d, ring_slot);
    for (int c = 0; c < ncase; ++c) hs[c]->launches += 1;
    if (!residual) return cudaGetLastError() == cudaSuccess ? 0 : -1;   // no case checks this step
    ib_residual<true><<<dim3((ns + 7) / 8, 1, ncase), 256, 0, st>>>(IBArgs{}, d);
    for (int c = 0; c < ncase; ++c) hs[c]->launches += 1;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}
