// ib_kernels.cu -- immersed boundary of one time step (FP64), ahead of the
// fused lattice update.
//
// Reference: move_boundary (airfoil.f90:244-338) and immersed_boundary_Wu
// (boundary_condition.f90:1512-1736). The reference builds dense X1 (nseg x
// nadj) and X2 = X1^T W (W = diag(arc_l)), forms A = X1 X2 with cublasDgemm,
// solves A x = U_b - X1 u* by LU (cusolverDnDgetrf/getrs) and spreads
// du = X2 x. With D = X1, A = (D D^T) W, so y = W x solves the symmetric
// positive definite system (D D^T) y = U_b - D u* and du = D^T y: the same
// correction, with arc_l dropping out. The kernels below
//   ib_prepare  marker positions, velocities, support boxes, one-axis kernel
//               values, the bounding rectangle of all boxes (one CTA);
//   ib_interp   b = D u*, one warp per marker, warp-shuffle sum over its box;
//   ib_assemble B = D D^T; the delta is separable, so each entry is
//               (sum_i phx_k phx_l)(sum_j phy_k phy_l) over the box overlap;
//   ib_solve    Cholesky of B and two triangular solves (one CTA);
//   ib_spread   du = D^T y per node, gathered in marker order over the
//               markers whose box covers the node (no atomics), written to the
//               correction patch the lattice kernel reads; force and moment
//               sums in FP64 with a deterministic two-level reduction.
#include <math.h>

#include "lbm_internal.h"

namespace {

const size_t kSolveSmem = 220 * 1024;   // dynamic shared memory cap of ib_solve

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

__global__ void __launch_bounds__(1024) ib_prepare(const IBArgs a, int step_index, int ring_slot)
{
    __shared__ int bb[4];
    if (threadIdx.x == 0) { bb[0] = 1 << 30; bb[1] = 1 << 30; bb[2] = -1; bb[3] = -1; }
    __syncthreads();
    double time;
    const double *row = motion_row(a, step_index, &time);
    const double scale = a.scale, ox = a.ox, oy = a.oy;
    for (int k = threadIdx.x; k < a.nseg; k += blockDim.x) {
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
        // support box, 1-based scans of airfoil.f90:290-321; a marker off the
        // lattice (or not finite) is a range error before any scan runs
        const double fx = (m.xm - ox) / scale + 1.0, fy = (m.ym - oy) / scale + 1.0;
        if (!(fx > 3.0 && fx < (double)(a.nx - 2) && fy > 3.0 && fy < (double)(a.ny - 2))) {
            atomicOr(a.status, LBM_ST_RANGE);
            for (int t = 0; t < LBM_BOX; ++t) m.phx[t] = m.phy[t] = 0.0;
            m.i1 = 3; m.i2 = 2; m.j1 = 3; m.j2 = 2;   // empty box
            m.wing = w;
            m.pad = 0;
            a.mk[k] = m;
            continue;
        }
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
            i1 = 4; i2 = 3; j1 = 4; j2 = 3;   // empty box
        }
        for (int t = 0; t < LBM_BOX; ++t) {
            const int ii = i1 + t, jj = j1 + t;
            m.phx[t] = ii <= i2 ? delta1(fabs((ox + scale * (double)(ii - 1) - m.xm) / scale), a.smooth) : 0.0;
            m.phy[t] = jj <= j2 ? delta1(fabs((oy + scale * (double)(jj - 1) - m.ym) / scale), a.smooth) : 0.0;
        }
        m.i1 = i1 - 1; m.i2 = i2 - 1; m.j1 = j1 - 1; m.j2 = j2 - 1;
        m.wing = w;
        m.pad = 0;
        a.mk[k] = m;
        if (i2 >= i1 && j2 >= j1) {
            atomicMin(&bb[0], i1 - 1); atomicMin(&bb[1], j1 - 1);
            atomicMax(&bb[2], i2 - 1); atomicMax(&bb[3], j2 - 1);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        PatchInfo pi{0, 0, 0, 0};
        if (bb[2] >= bb[0]) {
            pi.i0 = bb[0]; pi.j0 = bb[1]; pi.w = bb[2] - bb[0] + 1; pi.h = bb[3] - bb[1] + 1;
            if ((long long)pi.w * pi.h > a.patch_cap || pi.w > a.patch_wmax || pi.h > a.patch_hmax) { atomicOr(a.status, LBM_ST_OVERFLOW); pi = PatchInfo{0, 0, 0, 0}; }
        }
        *a.pinfo = pi;
        // force.dat row: time and the motion columns (solution.f90:350-375)
        double *fr = a.force_ring + (long long)ring_slot * a.row_len;
        fr[0] = time;
        const int mc = 1 + 3 * a.nwing + 3;
        for (int w = 0; w < a.nwing; ++w) {
            const double *r = row + 1 + 9 * w;   // angle omega omgac sa sau saac sb sbv sbac
            double *o = fr + mc + 9 * w;
            o[0] = r[3]; o[1] = r[4]; o[2] = r[5]; o[3] = r[6]; o[4] = r[7]; o[5] = r[8];
            o[6] = r[0]; o[7] = r[1]; o[8] = r[2];
        }
    }
}

template <typename T>
__global__ void __launch_bounds__(256) ib_interp(const IBArgs a)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int k = blockIdx.x * 8 + warp;
    if (k >= a.nseg) return;
    const Marker &m = a.mk[k];
    const int nbx = m.i2 - m.i1 + 1, nby = m.j2 - m.j1 + 1;
    const int nn = nbx > 0 && nby > 0 ? nbx * nby : 0;
    double su = 0.0, sv = 0.0;
    for (int t = lane; t < nn; t += 32) {
        const int ii = t % nbx, jj = t / nbx;
        double rho, u, v;
        node_moments<T>(a, m.i1 + ii, m.j1 + jj, rho, u, v);
        const double wgt = m.phx[ii] * m.phy[jj];   // X1(k,i) = kernel1*kernel2 (:1602)
        su += wgt * u;
        sv += wgt * v;
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        su += __shfl_down_sync(0xffffffffu, su, off);
        sv += __shfl_down_sync(0xffffffffu, sv, off);
    }
    if (lane == 0) {
        a.rhs[k] = m.ub - su;                 // comj (:1624-1629)
        a.rhs[a.nseg + k] = m.vb - sv;
    }
}

__global__ void __launch_bounds__(128) ib_assemble(const IBArgs a)
{
    const int k = blockIdx.x;
    const Marker mk = a.mk[k];
    for (int l = threadIdx.x; l < a.nseg; l += blockDim.x) {
        const Marker &ml = a.mk[l];
        const int ia = max(mk.i1, ml.i1), ib = min(mk.i2, ml.i2);
        const int ja = max(mk.j1, ml.j1), jb = min(mk.j2, ml.j2);
        double b = 0.0;
        if (ia <= ib && ja <= jb) {
            double sx = 0.0, sy = 0.0;
            for (int i = ia; i <= ib; ++i) sx += mk.phx[i - mk.i1] * ml.phx[i - ml.i1];
            for (int j = ja; j <= jb; ++j) sy += mk.phy[j - mk.j1] * ml.phy[j - ml.j1];
            b = sx * sy;
        }
        a.B[(long long)k * a.nseg + l] = b;
    }
}

// Cholesky B = L L^T (lower triangle, in place) with the forward solve fused
// into the factorisation (column k of L is staged in shared memory, so the
// trailing update reads rows contiguously), then the backward solve L^T y = z
// by rows. One CTA. B lives in shared memory when it fits, else in global
// memory (L2). Dynamic shared memory: colk[n], y[2n], then L[n*n] if resident.
__global__ void __launch_bounds__(1024) ib_solve(const IBArgs a, int use_smem)
{
    extern __shared__ double sm[];
    const int n = a.nseg;
    double *colk = sm, *yv = sm + n;
    double *L = use_smem ? sm + 3 * n : a.B;
    const int tid = threadIdx.x, nt = blockDim.x;
    const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
    if (use_smem)
        for (long long q = tid; q < (long long)n * n; q += nt) L[q] = a.B[q];
    for (int q = tid; q < 2 * n; q += nt) yv[q] = a.rhs[q];
    __shared__ int bad;
    if (tid == 0) bad = 0;
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        if (tid == 0) {
            const double d = L[(long long)k * n + k];
            double dk = 1.0;
            if (!(d > 0.0) || !isfinite(d)) bad = 1;
            else dk = sqrt(d);
            L[(long long)k * n + k] = dk;
            colk[k] = dk;
        }
        __syncthreads();
        const double dk = colk[k];
        for (int i = k + 1 + tid; i < n; i += nt) {
            const double v = L[(long long)i * n + k] / dk;
            L[(long long)i * n + k] = v;
            colk[i] = v;
        }
        if (tid < 2) yv[tid * n + k] /= dk;                    // z_k
        __syncthreads();
        for (int i = k + 1 + warp; i < n; i += nw) {
            const double lik = colk[i];
            for (int j = k + 1 + lane; j <= i; j += 32) L[(long long)i * n + j] -= lik * colk[j];
        }
        const double z0 = yv[k], z1 = yv[n + k];
        for (int i = k + 1 + tid; i < n; i += nt) {
            yv[i] -= colk[i] * z0;
            yv[n + i] -= colk[i] * z1;
        }
        __syncthreads();
    }
    // backward: L^T y = z; row j of L is column j of L^T
    for (int j = n - 1; j >= 0; --j) {
        if (tid < 2) yv[tid * n + j] /= L[(long long)j * n + j];
        __syncthreads();
        for (int q = tid; q < 2 * j; q += nt) {
            const int c = q / j, i = q % j;
            yv[c * n + i] -= L[(long long)j * n + i] * yv[c * n + j];
        }
        __syncthreads();
    }
    for (int q = tid; q < 2 * n; q += nt) a.y[q] = yv[q];
    if (tid == 0 && bad) atomicOr(a.status, LBM_ST_SOLVER);
}

// du = D^T y over the current patch, 16x16 nodes per CTA, plus FP64 force and
// moment partials (boundary_condition.f90:1645-1675)
template <typename T, typename C>
__global__ void __launch_bounds__(256) ib_spread(const IBArgs a, int step_index, int ring_slot)
{
    __shared__ int list[256];
    __shared__ int wsum[8];
    __shared__ int nlist;
    __shared__ double red[8][3 * LBM_MAXW];
    __shared__ bool amlast;
    const PatchInfo pi = *a.pinfo;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int ti0 = blockIdx.x * 16, tj0 = blockIdx.y * 16;
    const int li = ti0 + tx, lj = tj0 + ty;                    // patch-relative
    const int gi = pi.i0 + li, gj = pi.j0 + lj;                // 0-based node
    const bool active = li < pi.w && lj < pi.h;
    const bool tile_active = ti0 < pi.w && tj0 < pi.h;
    const int ta = pi.i0 + ti0, tb = pi.i0 + ti0 + 15, sa_ = pi.j0 + tj0, sb_ = pi.j0 + tj0 + 15;
    double du = 0.0, dv = 0.0;
    int wing = 1 << 20;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (tile_active) {
        for (int c0 = 0; c0 < a.nseg; c0 += 256) {
            const int k = c0 + threadIdx.x;
            bool hit = false;
            if (k < a.nseg) {
                const Marker &m = a.mk[k];
                hit = m.i1 <= tb && m.i2 >= ta && m.j1 <= sb_ && m.j2 >= sa_ && m.i2 >= m.i1;
            }
            const unsigned bal = __ballot_sync(0xffffffffu, hit);
            if (lane == 0) wsum[warp] = __popc(bal);
            __syncthreads();
            if (threadIdx.x == 0) {
                int s = 0;
                for (int w = 0; w < 8; ++w) { const int t = wsum[w]; wsum[w] = s; s += t; }
                nlist = s;
            }
            __syncthreads();
            if (hit) list[wsum[warp] + __popc(bal & ((1u << lane) - 1u))] = k;
            __syncthreads();
            if (active) {
                for (int q = 0; q < nlist; ++q) {
                    const Marker &m = a.mk[list[q]];
                    if (gi >= m.i1 && gi <= m.i2 && gj >= m.j1 && gj <= m.j2) {
                        const double wgt = m.phx[gi - m.i1] * m.phy[gj - m.j1];
                        const int kk = list[q];
                        du += wgt * a.y[kk];
                        dv += wgt * a.y[a.nseg + kk];
                        wing = min(wing, m.wing);
                    }
                }
            }
            __syncthreads();
        }
    }
    if (active) {
        C *patch = (C *)a.patch;
        const long long pq = 2ll * ((long long)lj * pi.w + li);
        patch[pq] = (C)du;
        patch[pq + 1] = (C)dv;
    }
    // force and moment of this node
    double fx = 0, fy = 0, mz = 0;
    const bool in_support = active && wing < (1 << 20);
    double time;
    const double *row = motion_row(a, step_index, &time);
    if (in_support) {
        double rho, u, v;
        node_moments<T>(a, gi, gj, rho, u, v);
        const double temp1 = 2.0 * rho * du, temp2 = 2.0 * rho * dv;
        const double sa = row[4 + 9 * wing], sb = row[7 + 9 * wing];
        fx = -temp1;
        fy = -temp2;
        const double x0 = (a.ox + a.scale * (double)gi - (a.xc + sa)) / a.scale;
        const double y0 = (a.oy + a.scale * (double)gj - (a.yc + sb)) / a.scale;
        mz = -x0 * temp2 + y0 * temp1;
    }
    // deterministic block reduction per wing
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
    const int nblk = gridDim.x * gridDim.y, bid = blockIdx.y * gridDim.x + blockIdx.x;
    if (threadIdx.x < 3 * a.nwing) {
        double s = 0.0;
        for (int w8 = 0; w8 < 8; ++w8) s += red[w8][threadIdx.x];
        a.partial[(long long)bid * 3 * LBM_MAXW + threadIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) amlast = atomicAdd(a.counter, 1u) == (unsigned)(nblk - 1);
    __syncthreads();
    if (!amlast) return;
    __threadfence();
    if (threadIdx.x == 0) {
        double *fr = a.force_ring + (long long)ring_slot * a.row_len;
        double tot[3] = {0, 0, 0};
        const double uu = a.uu, scale = a.scale;
        for (int w = 0; w < a.nwing; ++w) {
            double s0 = 0, s1 = 0, s2 = 0;
            for (int b = 0; b < nblk; ++b) {
                const double *p = a.partial + (long long)b * 3 * LBM_MAXW + 3 * w;
                s0 += __ldcg(p); s1 += __ldcg(p + 1); s2 += __ldcg(p + 2);
            }
            // solution.f90:327-330
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
        *a.counter = 0u;
    }
}

IBArgs make_args(lbm_handle *h, const void *fin)
{
    IBArgs a;
    a.fin = fin;
    a.prec = h->prec;
    a.nx = h->nx; a.ny = h->ny; a.pitch = h->pitch; a.plane = h->plane;
    a.nwing = h->nwing; a.ppw = h->ppw; a.spw = h->spw; a.nseg = h->nseg;
    a.smooth = h->p.delta_kernel;
    a.scale = h->p.scale; a.ox = h->p.ox; a.oy = h->p.oy; a.uu = h->p.uu;
    a.xc = h->p.xc; a.yc = h->p.yc; a.mesh_max_scale = h->p.mesh_max_scale;
    a.xb0 = h->d_xb0; a.yb0 = h->d_yb0; a.arc = h->d_arc;
    a.mstep = h->d_mstep; a.msteps = h->msteps; a.mcols = h->mcols; a.mdt = h->mdt;
    a.mk = h->d_mk; a.rhs = h->d_rhs; a.B = h->d_B; a.y = h->d_y;
    a.pinfo = h->d_pinfo; a.patch = h->d_patch; a.patch_cap = h->patch_cap;
    a.patch_wmax = h->patch_wmax; a.patch_hmax = h->patch_hmax;
    a.partial = h->d_partial; a.counter = h->d_counter;
    a.force_ring = h->d_ring; a.row_len = h->row_len;
    a.status = h->d_status; a.solve_res = h->d_solve_res;
    return a;
}

template <typename T, typename C>
int launch_ib_t(lbm_handle *h, const void *fin, int step_index, int ring_slot)
{
    IBArgs a = make_args(h, fin);
    cudaStream_t st = h->stream;
    ib_prepare<<<1, 1024, 0, st>>>(a, step_index, ring_slot);
    if (h->nseg > 0) {
        ib_interp<T><<<(h->nseg + 7) / 8, 256, 0, st>>>(a);
        ib_assemble<<<h->nseg, 128, 0, st>>>(a);
        const size_t base = sizeof(double) * 3 * (size_t)h->nseg;
        const size_t full = base + sizeof(double) * (size_t)h->nseg * h->nseg;
        const int use_smem = full <= kSolveSmem;
        if (base > kSolveSmem) return -1;
        ib_solve<<<1, 1024, use_smem ? full : base, st>>>(a, use_smem);
    }
    dim3 grid(h->patch_gx(), h->patch_gy());
    ib_spread<T, C><<<grid, 256, 0, st>>>(a, step_index, ring_slot);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

}  // namespace

int ib_configure(lbm_handle *h)
{
    // ib_solve may need up to kSolveSmem of dynamic shared memory
    if (cudaFuncSetAttribute(ib_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSolveSmem) != cudaSuccess)
        return -1;
    return 0;
}

int launch_ib(lbm_handle *h, const void *fin, int step_index, int ring_slot)
{
    switch (h->prec) {
    case LBM_PREC_FP32: return launch_ib_t<float, float>(h, fin, step_index, ring_slot);
    case LBM_PREC_FP64: return launch_ib_t<double, double>(h, fin, step_index, ring_slot);
    case LBM_PREC_FP16: return launch_ib_t<__half, float>(h, fin, step_index, ring_slot);
    case LBM_PREC_BF16: return launch_ib_t<__nv_bfloat16, float>(h, fin, step_index, ring_slot);
    }
    return -1;
}
