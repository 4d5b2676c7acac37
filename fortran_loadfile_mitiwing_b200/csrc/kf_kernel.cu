// kf_kernel.cu -- the fused lattice update: pull streaming, moments, immersed
// boundary correction, MRT collision with forcing, and the outer boundary
// condition, in one pass over the lattice.
//
// Reference path folded into this kernel (one time step):
//   streaming           solution.f90:428-454   f0(i,j,k) = f(i-ex, j-ey, k)
//   physical_variables  solution.f90:471-542   rho, u, v of f0
//   IB velocity/force   boundary_condition.f90:1645-1659 (u = u* + du, g = 2 rho du)
//   colission           solution.f90:573-643   MRT relaxation with forcing
//   boundary_condition1 boundary_condition.f90:288-858 (left/right
//                       characteristic + extrapolation, top/bottom rows)
// Interior nodes read 9 populations and write 9: 72 B per update in FP32.
// Edge nodes recompute the moments of the one or two interior neighbours
// their formula needs (O(perimeter) extra reads) so that no second launch and
// no side buffer is needed for the boundary condition.
#include "lbm_internal.h"

namespace {

template <typename T, typename C>
__device__ __forceinline__ void pull(const T *__restrict__ fin, long long plane, int pitch, int i, int j, C g[9])
{
#pragma unroll
    for (int k = 0; k < 9; ++k)
        g[k] = (C)Store<T>::ld(fin + (long long)k * plane + (long long)(j - lbm_ey(k)) * pitch + (i - lbm_ex(k)));
}

template <typename C>
__device__ __forceinline__ void moments(const C g[9], C &drho, C &u, C &v)
{
    drho = ((g[0] + g[1]) + (g[2] + g[3])) + ((g[4] + g[5]) + (g[6] + g[7])) + g[8];
    const C jx = (g[1] - g[3]) + (g[5] - g[6]) + (g[8] - g[7]);
    const C jy = (g[2] - g[4]) + (g[5] + g[6]) - (g[7] + g[8]);
    const C rho = C(1) + drho;
    u = jx / rho;
    v = jy / rho;
}

// characteristic update of a left (side=0) or right (side=1) column node
// (boundary_condition.f90:418-438 and :500-520). Returns the updated
// (drho, u, v) at the edge node and the streamed populations + moments of its
// first interior neighbour.
template <typename T, typename C>
__device__ __forceinline__ void side_bc(const KFArgs<C> &a, const T *__restrict__ fin, int side, int j, C &dr1,
                                        C &u1, C &v1, C g0n[9], C &drn, C &un, C &vn)
{
    const C *col = side == 0 ? a.col_l : a.col_r;
    const C drs = col[3 * j], us = col[3 * j + 1], vs = col[3 * j + 2];
    const int in1 = side == 0 ? 1 : a.nx - 2, in2 = side == 0 ? 2 : a.nx - 3;
    C g2[9], dr2, u2, v2;
    pull<T, C>(fin, a.plane, a.pitch, in1, j, g0n);
    moments(g0n, drn, un, vn);
    pull<T, C>(fin, a.plane, a.pitch, in2, j, g2);
    moments(g2, dr2, u2, v2);
    const C cs = a.cs, rhos = C(1) + drs;
    if (side == 0) {
        const C rhox = (C(-3) * drs + C(4) * drn - dr2) * C(0.5);
        const C ux = (C(-3) * us + C(4) * un - u2) * C(0.5);
        const C vx = (C(-3) * vs + C(4) * vn - v2) * C(0.5);
        const C lx1 = (us - cs) * (cs * cs * rhox - cs * rhos * ux);
        const C lx2 = us < C(0) ? us * vx : C(0);
        dr1 = drs - lx1 * C(1.5);
        u1 = us + lx1 / (C(2) * cs * (C(1) + dr1));
        v1 = vs - lx2;
    } else {
        const C rhox = (C(3) * drs - C(4) * drn + dr2) * C(0.5);
        const C ux = (C(3) * us - C(4) * un + u2) * C(0.5);
        const C vx = (C(3) * vs - C(4) * vn + v2) * C(0.5);
        const C lx2 = us >= C(0) ? us * vx : C(0);
        const C lx3 = (us + cs) * (cs * cs * rhox + cs * rhos * ux);
        dr1 = drs - lx3 * C(1.5);
        u1 = us + (C(0) - lx3) / (C(2) * cs * (C(1) + dr1));
        v1 = vs - lx2;
    }
}

// interior node: moments of the streamed populations g, immersed-boundary
// correction from the patch, MRT collision with forcing
template <typename C>
__device__ __forceinline__ void collide_interior(const KFArgs<C> &a, const PatchInfo &pi, const C g[9], int i, int j,
                                                 C gout[9], C &frho, C &fu, C &fv)
{
    C drho, u, v;
    moments(g, drho, u, v);
    const C rho = C(1) + drho;
    C gx = C(0), gy = C(0);
    const unsigned pii = (unsigned)(i - pi.i0), pjj = (unsigned)(j - pi.j0);
    if (pii < (unsigned)pi.w && pjj < (unsigned)pi.h) {
        const int pq = 2 * ((int)pjj * pi.w + (int)pii);
        const C du = a.patch[pq], dv = a.patch[pq + 1];
        u = u + du;                       // boundary_condition.f90:1650-1651
        v = v + dv;
        gx = C(2) * rho * du;             // :1652-1656
        gy = C(2) * rho * dv;
    }
    C m[9];
    mrt_forward(g, m);
    const C jx = rho * u, jy = rho * v;
    const C jj = jx * jx + jy * jy;
    C e[9];
    e[0] = C(-1);                          // temp(1)=0 minus (M w)_1
    e[1] = C(-2) * drho + C(3) * jj;       // solution.f90:605 minus (M w)_2
    e[2] = drho - C(3) * jj;               // :606
    e[3] = C(0);
    e[4] = -jx;
    e[5] = C(0);
    e[6] = -jy;
    e[7] = jx * jx - jy * jy;
    e[8] = jx * jy;
    // m' = m + s(meq - m) + fp (solution.f90:632-634); the new populations
    // are taken as g + M^-1 (m' - m), which equals M^-1 m' exactly but
    // rounds relative to the small non-equilibrium update, not to g
    C d[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) d[k] = (e[k] - m[k]) * a.s[k];
    if (gx != C(0) || gy != C(0)) {        // :614-626
        const C ug = u * gx + v * gy;
        d[1] += C(6) * (C(1) - C(0.5) * a.s[1]) * ug;
        d[2] += C(-6) * (C(1) - C(0.5) * a.s[2]) * ug;
        d[3] += gx;
        d[4] += -(C(1) - C(0.5) * a.s[4]) * gx;
        d[5] += gy;
        d[6] += -(C(1) - C(0.5) * a.s[6]) * gy;
        d[7] += C(2) * (C(1) - C(0.5) * a.s[7]) * (u * gx - v * gy);
        d[8] += (C(1) - C(0.5) * a.s[8]) * (u * gy + v * gx);
    }
    mrt_inverse(d, gout);
#pragma unroll
    for (int k = 0; k < 9; ++k) gout[k] += g[k];
    frho = rho; fu = u; fv = v;
}

// edge node: boundary_condition1 (boundary_condition.f90:413-853)
template <typename T, typename C>
__device__ __forceinline__ void edge_update(const KFArgs<C> &a, const T *__restrict__ fin, int i, int j, C gout[9],
                                            C &frho, C &fu, C &fv)
{
    C g0n[9], drn, un, vn;
    if (j == 0 || j == a.ny - 1) {
        // top/bottom row: rho from the adjacent row, u = v = 0
        // (boundary_condition.f90:658-716, 785-843)
        const int jn = j == 0 ? 1 : a.ny - 2;
        if (i == 0 || i == a.nx - 1) {
            const int side = i == 0 ? 0 : 1;
            C d2[9], dr2, u2, v2;
            side_bc<T, C>(a, fin, side, jn, drn, un, vn, d2, dr2, u2, v2);
            const C *c = a.corner + 9 * (2 * side + (j == 0 ? 0 : 1));
#pragma unroll
            for (int k = 0; k < 9; ++k) g0n[k] = c[k];   // edge f0, never rewritten
        } else {
            pull<T, C>(fin, a.plane, a.pitch, i, jn, g0n);
            moments(g0n, drn, un, vn);
        }
        extrapolate_dev<C>(a.s, drn, C(0), C(0), drn, un, vn, g0n, gout);
        frho = C(1) + drn; fu = C(0); fv = C(0);
    } else {
        // left/right column (boundary_condition.f90:413-483, 495-567)
        const int side = i == 0 ? 0 : 1;
        C dr1, u1, v1;
        side_bc<T, C>(a, fin, side, j, dr1, u1, v1, g0n, drn, un, vn);
        extrapolate_dev<C>(a.s, dr1, u1, v1, drn, un, vn, g0n, gout);
        frho = C(1) + dr1; fu = u1; fv = v1;
    }
}

// any node with scalar loads
template <typename T, typename C>
__device__ __forceinline__ void node_update(const KFArgs<C> &a, const PatchInfo &pi, const T *__restrict__ fin, int i,
                                            int j, C gout[9], C &frho, C &fu, C &fv)
{
    if (i == 0 || i == a.nx - 1 || j == 0 || j == a.ny - 1) {
        edge_update<T, C>(a, fin, i, j, gout, frho, fu, fv);
    } else {
        C g[9];
        pull<T, C>(fin, a.plane, a.pitch, i, j, g);
        collide_interior<C>(a, pi, g, i, j, gout, frho, fu, fv);
    }
}

template <typename T, typename C, bool FIELDS>
__device__ __forceinline__ void store_node(const KFArgs<C> &a, T *__restrict__ fout, int i, int j, const C gout[9],
                                           C frho, C fu, C fv)
{
    const long long o = (long long)j * a.pitch + i;
#pragma unroll
    for (int k = 0; k < 9; ++k) Store<T>::st(fout + (long long)k * a.plane + o, gout[k]);
    if (FIELDS) {
        const long long q = (long long)j * a.nx + i;
        a.rho_out[q] = frho;
        a.u_out[q] = fu;
        a.v_out[q] = fv;
    }
}

// one node per thread, scalar loads (any lattice size)
template <typename T, typename C, bool FIELDS>
__global__ void __launch_bounds__(256) kf_kernel(const KFArgs<C> a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y;
    if (a.mode != KF_ALL) {   // split around the step's correction patch
        const PatchInfo r = *a.pinfo;
        if (a.mode == KF_INNER) {
            if (i >= r.w || j >= r.h) return;
            i += r.i0;
            j += r.j0;
        } else if ((unsigned)(i - r.i0) < (unsigned)r.w && (unsigned)(j - r.j0) < (unsigned)r.h) {
            return;
        }
    }
    if (i >= a.nx) return;
    const T *__restrict__ fin = (const T *)a.fin;
    T *__restrict__ fout = (T *)a.fout;
    // the outer part runs while the IB kernels rewrite the patch: it reads
    // neither (no outer node lies in any patch)
    const PatchInfo pi = a.mode == KF_OUTER ? PatchInfo{0, 0, 0, 0} : *a.pinfo;
    C gout[9], frho, fu, fv;
    node_update<T, C>(a, pi, fin, i, j, gout, frho, fu, fv);
    store_node<T, C, FIELDS>(a, fout, i, j, gout, frho, fu, fv);
}

template <typename T, int VEC> struct alignas(sizeof(T) * VEC) VecT {
    T v[VEC];
};

// VEC consecutive nodes of one row per thread: the 9 planes are read with
// aligned VEC-wide loads at rows j - e_y; the x-shifted planes take their
// missing neighbour element from the adjacent lane (warp shuffle), or from
// memory at the warp's ends. 32-bit offsets (9 planes < 2^31 elements).
template <typename T, typename C, bool FIELDS, int VEC>
__global__ void __launch_bounds__(128) kf_vec(const KFArgs<C> a)
{
    const int lane = threadIdx.x & 31;
    int i0 = (blockIdx.x * blockDim.x + threadIdx.x) * VEC;
    int j = blockIdx.y;
    const int iend = a.nx;                     // whole lattice only (KF_ALL)
    const T *__restrict__ fin = (const T *)a.fin;
    T *__restrict__ fout = (T *)a.fout;
    const int pitch = a.pitch, plane = (int)a.plane;
    // the outer part runs while the IB kernels rewrite the patch: it reads
    // neither (no outer node lies in any patch)
    const PatchInfo pi = a.mode == KF_OUTER ? PatchInfo{0, 0, 0, 0} : *a.pinfo;
    if (j == 0 || j == a.ny - 1) {             // warp-uniform: edge rows
        for (int e = 0; e < VEC; ++e) {
            const int i = i0 + e;
            if (i >= a.nx) break;
            C gout[9], frho, fu, fv;
            edge_update<T, C>(a, fin, i, j, gout, frho, fu, fv);
            store_node<T, C, FIELDS>(a, fout, i, j, gout, frho, fu, fv);
        }
        return;
    }
    const bool inrow = i0 < pitch;
    T v[9][VEC];
    T xl[9], xr[9];
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const T *p = fin + k * plane + (j - lbm_ey(k)) * pitch + i0;
        if (inrow) {
            const VecT<T, VEC> w = *reinterpret_cast<const VecT<T, VEC> *>(p);
#pragma unroll
            for (int e = 0; e < VEC; ++e) v[k][e] = w.v[e];
        } else {
#pragma unroll
            for (int e = 0; e < VEC; ++e) v[k][e] = T(0.0f);
        }
        if (lbm_ex(k) == 1) {
            xl[k] = __shfl_up_sync(0xffffffffu, v[k][VEC - 1], 1);
            if (lane == 0) xl[k] = (i0 >= 1 && i0 - 1 < pitch) ? p[-1] : T(0.0f);
        } else if (lbm_ex(k) == -1) {
            xr[k] = __shfl_down_sync(0xffffffffu, v[k][0], 1);
            if (lane == 31) xr[k] = (i0 + VEC < a.nx) ? p[VEC] : T(0.0f);
        }
    }
    if (i0 >= iend) return;
    if (i0 >= 1 && i0 + VEC - 1 <= a.nx - 2) {
        T out[9][VEC];
#pragma unroll
        for (int e = 0; e < VEC; ++e) {
            C g[9];
#pragma unroll
            for (int k = 0; k < 9; ++k) {
                T t;
                if (lbm_ex(k) == 0) t = v[k][e];
                else if (lbm_ex(k) == 1) t = e == 0 ? xl[k] : v[k][e - 1];
                else t = e == VEC - 1 ? xr[k] : v[k][e + 1];
                g[k] = (C)Store<T>::cvt(t);
            }
            C gout[9], frho, fu, fv;
            collide_interior<C>(a, pi, g, i0 + e, j, gout, frho, fu, fv);
#pragma unroll
            for (int k = 0; k < 9; ++k) out[k][e] = Store<T>::pack(gout[k]);
            if (FIELDS) {
                const int q = j * a.nx + i0 + e;
                a.rho_out[q] = frho;
                a.u_out[q] = fu;
                a.v_out[q] = fv;
            }
        }
#pragma unroll
        for (int k = 0; k < 9; ++k) {
            VecT<T, VEC> w;
#pragma unroll
            for (int e = 0; e < VEC; ++e) w.v[e] = out[k][e];
            *reinterpret_cast<VecT<T, VEC> *>(fout + k * plane + j * pitch + i0) = w;
        }
    } else {
        for (int e = 0; e < VEC; ++e) {
            const int i = i0 + e;
            if (i >= a.nx) break;
            C gout[9], frho, fu, fv;
            node_update<T, C>(a, pi, fin, i, j, gout, frho, fu, fv);
            store_node<T, C, FIELDS>(a, fout, i, j, gout, frho, fu, fv);
        }
    }
}

// ---- bulk-copy staged lattice kernel ----------------------------------
// A CTA owns a strip of TW columns and sweeps rows_per_cta interior rows.
// For every output row j one elected thread issues nine 1-D bulk copies
// (cp.async.bulk, completion on an mbarrier) of the plane rows j - e_y with a
// 16-byte halo on both sides into a KS-stage shared-memory ring; the threads
// then read the shifted populations from shared memory. The copies keep
// KS x 9 row segments in flight per CTA without holding them in registers.
// Rows 0 and ny-1 are handled by one extra CTA row of the grid, and columns
// 0 and nx-1 by the scalar edge path.

constexpr int TW = 256;        // strip width (threads per CTA)
constexpr int KS = 4;          // pipeline stages

// mbarrier and bulk-copy helpers: lbm_common.cuh

template <typename T> __host__ __device__ constexpr int tma_halo() { return 16 / (int)sizeof(T); }
template <typename T> __host__ __device__ constexpr int tma_seg() { return TW + 2 * tma_halo<T>(); }
template <typename T> constexpr size_t tma_smem() { return sizeof(T) * KS * 9 * tma_seg<T>() + 2 * 8 * KS; }

template <typename T, typename C, bool FIELDS>
__global__ void __launch_bounds__(TW) kf_tma(const KFArgs<C> a)
{
    constexpr int H = tma_halo<T>(), SEG = tma_seg<T>(), NWARP = TW / 32;
    extern __shared__ __align__(128) unsigned char smraw[];
    T *buf = reinterpret_cast<T *>(smraw);
    uint64_t *full = reinterpret_cast<uint64_t *>(smraw + sizeof(T) * KS * 9 * SEG);
    uint64_t *empty = full + KS;
    const int tid = threadIdx.x, lane = tid & 31;
    const int x0 = blockIdx.x * TW;
    const int i = x0 + tid;
    const T *__restrict__ fin = (const T *)a.fin;
    T *__restrict__ fout = (T *)a.fout;
    const PatchInfo pi = a.mode == KF_OUTER ? PatchInfo{0, 0, 0, 0} : *a.pinfo;
    const PatchInfo rr = a.mode == KF_OUTER ? *a.pinfo : PatchInfo{0, 0, 0, 0};   // nodes the outer part skips
    if (blockIdx.y == gridDim.y - 1) {
        // the edge nodes: rows 0 and ny-1 of this strip, and a share of the
        // nodes of columns 0 and nx-1 (which the strips' row sweeps skip)
        if (i < a.nx)
            for (int j = 0; j < a.ny; j += a.ny - 1) {
                C gout[9], frho, fu, fv;
                edge_update<T, C>(a, fin, i, j, gout, frho, fu, fv);
                store_node<T, C, FIELDS>(a, fout, i, j, gout, frho, fu, fv);
            }
        for (int q = blockIdx.x * TW + tid; q < 2 * (a.ny - 2); q += gridDim.x * TW) {
            const int j = 1 + q / 2, ie = (q & 1) ? a.nx - 1 : 0;
            C gout[9], frho, fu, fv;
            edge_update<T, C>(a, fin, ie, j, gout, frho, fu, fv);
            store_node<T, C, FIELDS>(a, fout, ie, j, gout, frho, fu, fv);
        }
        return;
    }
    const int j0 = 1 + blockIdx.y * a.rows_per_cta;
    const int nrows = min(a.rows_per_cta, a.ny - 1 - j0);
    if (nrows <= 0) return;
    const int width = min(TW, a.nx - x0);
    const uint32_t bytes = (uint32_t)((((width + 2 * H) * (int)sizeof(T)) + 15) / 16 * 16);
    if (tid == 0) {
        for (int s = 0; s < KS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], NWARP);
        }
        mbar_init_fence();
    }
    __syncthreads();
    auto issue = [&](int r) {
        const int s = r % KS, j = j0 + r;
        mbar_expect_tx(&full[s], 9u * bytes);
#pragma unroll
        for (int k = 0; k < 9; ++k)
            bulk_g2s(buf + (s * 9 + k) * SEG,
                     fin + (long long)k * a.plane + (long long)(j - lbm_ey(k)) * a.pitch + (x0 - H), bytes, &full[s]);
    };
    // bounded wait: a barrier that never completes is reported, not waited on forever
    auto wait = [&](uint64_t *bar, uint32_t parity) -> bool {
        int spins = 0;
        while (!mbar_try_wait(bar, parity))
            if (++spins > (1 << 22)) return false;
        return true;
    };
    if (tid == 0)
        for (int r = 0; r < KS && r < nrows; ++r) issue(r);
    // Stage s holds row r = s (mod KS). A warp waits for the row on full[s],
    // and when done reading it arrives on empty[s]; thread 0 refills the stage
    // with row r + KS once all warps have arrived. Only warp 0 waits for the
    // other warps; they run up to KS - 1 rows ahead.
    bool ok = true;
    for (int r = 0; r < nrows; ++r) {
        const int s = r % KS, j = j0 + r;
        const uint32_t parity = (uint32_t)((r / KS) & 1);
        if (!wait(&full[s], parity)) { ok = false; break; }
        const bool skip = (unsigned)(i - rr.i0) < (unsigned)rr.w && (unsigned)(j - rr.j0) < (unsigned)rr.h;
        if (i > 0 && i < a.nx - 1 && !skip) {
            C gout[9], frho, fu, fv;
            C g[9];
            const T *row = buf + s * 9 * SEG + H + tid;
#pragma unroll
            for (int k = 0; k < 9; ++k) g[k] = (C)Store<T>::cvt(row[k * SEG - lbm_ex(k)]);
            collide_interior<C>(a, pi, g, i, j, gout, frho, fu, fv);
            store_node<T, C, FIELDS>(a, fout, i, j, gout, frho, fu, fv);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (tid == 0 && r + KS < nrows) {
            if (!wait(&empty[s], parity)) { ok = false; break; }
            fence_proxy_async();
            issue(r + KS);
        }
    }
    if (!ok) {
        // report, then wait (bounded) for this CTA's copies still in flight
        atomicOr(a.status, LBM_ST_TIMEOUT);
        for (int s = 0; s < KS; ++s) {
            int spins = 0;
            while (!mbar_try_wait(&full[s], 0) && !mbar_try_wait(&full[s], 1) && ++spins < (1 << 20)) {
            }
        }
    }
}

template <typename T, typename C>
void launch_tma(const KFArgs<C> &a, bool fields, int nx, int ny, cudaStream_t st)
{
    dim3 block(TW, 1), grid((nx + TW - 1) / TW, (ny - 2 + a.rows_per_cta - 1) / a.rows_per_cta + 1);
    const size_t smem = tma_smem<T>();
    if (fields)
        kf_tma<T, C, true><<<grid, block, smem, st>>>(a);
    else
        kf_tma<T, C, false><<<grid, block, smem, st>>>(a);
}

template <typename T, typename C>
int configure_tma()
{
    const int smem = (int)tma_smem<T>();
    if (cudaFuncSetAttribute(kf_tma<T, C, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return -1;
    if (cudaFuncSetAttribute(kf_tma<T, C, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) != cudaSuccess)
        return -1;
    return 0;
}

template <typename T, typename C, int VEC>
void launch_vec(const KFArgs<C> &a, bool fields, int nx, int ny, cudaStream_t st)
{
    const int per_block = 128 * VEC;
    dim3 block(128, 1), grid((nx + per_block - 1) / per_block, ny);
    if (fields)
        kf_vec<T, C, true, VEC><<<grid, block, 0, st>>>(a);
    else
        kf_vec<T, C, false, VEC><<<grid, block, 0, st>>>(a);
}

template <typename T, typename C>
int launch_kf_t(lbm_handle *h, const void *fin, void *fout, void *fields, int mode, cudaStream_t st)
{
    KFArgs<C> a;
    a.mode = mode;
    a.fin = fin;
    a.fout = fout;
    a.nx = h->nx;
    a.ny = h->ny;
    a.pitch = h->pitch;
    a.plane = h->plane;
    for (int k = 0; k < 9; ++k) a.s[k] = (C)h->s[k];
    a.cs = (C)((double)sqrtf(3.0f) / 3.0);   // boundary_condition.f90:304
    const C *ec = (const C *)h->edge_c;
    a.col_l = ec;
    a.col_r = ec + 3 * h->ny;
    a.corner = ec + 6 * h->ny;
    a.pinfo = h->d_pinfo + h->pinfo_slot;
    a.patch = (const C *)h->d_patch;
    if (fields) {
        C *fc = (C *)fields;
        const long long nn = (long long)h->nx * h->ny;
        a.rho_out = fc;
        a.u_out = fc + nn;
        a.v_out = fc + 2 * nn;
    } else {
        a.rho_out = a.u_out = a.v_out = nullptr;
    }
    const bool small_index = 9ll * h->plane < (1ll << 31) && (long long)h->nx * h->ny < (1ll << 31);
    const int vec = small_index ? h->kf_vec : 1;
    a.rows_per_cta = h->kf_rows;
    a.status = h->d_status;
    if (!st) st = h->stream;
    if (h->kf_tma && mode != KF_INNER && h->ny >= 3) {
        static bool configured = false;   // per process; the attribute is per function
        if (!configured) {
            if (configure_tma<T, C>()) return -1;
            configured = true;
        }
        launch_tma<T, C>(a, fields != nullptr, h->nx, h->ny, st);
    } else if (mode == KF_ALL && vec == 4 && h->pitch % 4 == 0) {
        launch_vec<T, C, 4>(a, fields != nullptr, h->nx, h->ny, st);
    } else if (mode == KF_ALL && vec == 2 && h->pitch % 2 == 0) {
        launch_vec<T, C, 2>(a, fields != nullptr, h->nx, h->ny, st);
    } else {
        // the inner part covers the largest patch rectangle; its threads
        // outside the step's rectangle return at once
        const int wx = mode == KF_INNER ? h->patch_wmax : h->nx, wy = mode == KF_INNER ? h->patch_hmax : h->ny;
        dim3 block(256, 1), grid((wx + 255) / 256, wy);
        if (fields)
            kf_kernel<T, C, true><<<grid, block, 0, st>>>(a);
        else
            kf_kernel<T, C, false><<<grid, block, 0, st>>>(a);
    }
    h->launches += 1;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// ---- conversions between the host FP64 f(nx,ny,9) and device storage ----

__device__ __forceinline__ double wref(int k) { return k == 0 ? 4.0 / 9.0 : (k < 5 ? 1.0 / 9.0 : 1.0 / 36.0); }

template <typename T>
__global__ void unpack_kernel(const T *__restrict__ src, double *__restrict__ dst, int nx, int ny, int pitch,
                              long long plane)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= nx) return;
    dst[(long long)k * nx * ny + (long long)j * nx + i] =
        (double)Store<T>::ld(src + k * plane + (long long)j * pitch + i) + wref(k);
}

template <typename T>
__global__ void pack_kernel(const double *__restrict__ src, T *__restrict__ dst, int nx, int ny, int pitch,
                            long long plane)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, k = blockIdx.z;
    if (i >= nx) return;
    const double g = src[(long long)k * nx * ny + (long long)j * nx + i] - wref(k);
    Store<T>::st(dst + k * plane + (long long)j * pitch + i, (typename CType<T>::type)g);
}

// interior sums of erranalysis (solution.f90:102-108), FP64, fields in compute precision
template <typename C>
__global__ void residual_kernel(const C *__restrict__ fa, const C *__restrict__ fb, int nx, int ny,
                                double *__restrict__ out)
{
    const long long nn = (long long)nx * ny;
    double s1 = 0, s2 = 0;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < nn;
         q += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(q % nx), j = (int)(q / nx);
        if (i < 1 || i > nx - 2 || j < 1 || j > ny - 2) continue;
        const double u = (double)fa[nn + q], v = (double)fa[2 * nn + q];
        const double u0 = (double)fb[nn + q], v0 = (double)fb[2 * nn + q];
        s1 += (u - u0) * (u - u0) + (v - v0) * (v - v0);
        s2 += u * u + v * v;
    }
    for (int off = 16; off; off >>= 1) {
        s1 += __shfl_down_sync(0xffffffffu, s1, off);
        s2 += __shfl_down_sync(0xffffffffu, s2, off);
    }
    __shared__ double r1[32], r2[32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) { r1[wid] = s1; r2[wid] = s2; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double t1 = 0, t2 = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) { t1 += r1[w]; t2 += r2[w]; }
        out[2 * blockIdx.x] = t1;
        out[2 * blockIdx.x + 1] = t2;
    }
}

}  // namespace

int launch_kf(lbm_handle *h, const void *fin, void *fout, void *fields, int mode, cudaStream_t st)
{
    switch (h->prec) {
    case LBM_PREC_FP32: return launch_kf_t<float, float>(h, fin, fout, fields, mode, st);
    case LBM_PREC_FP64: return launch_kf_t<double, double>(h, fin, fout, fields, mode, st);
    case LBM_PREC_FP16: return launch_kf_t<__half, float>(h, fin, fout, fields, mode, st);
    case LBM_PREC_BF16: return launch_kf_t<__nv_bfloat16, float>(h, fin, fout, fields, mode, st);
    }
    return -1;
}

int launch_unpack(lbm_handle *h, const void *fsrc, double *dst)
{
    dim3 block(256), grid((h->nx + 255) / 256, h->ny, 9);
    switch (h->prec) {
    case LBM_PREC_FP32: unpack_kernel<float><<<grid, block, 0, h->stream>>>((const float *)fsrc, dst, h->nx, h->ny, h->pitch, h->plane); break;
    case LBM_PREC_FP64: unpack_kernel<double><<<grid, block, 0, h->stream>>>((const double *)fsrc, dst, h->nx, h->ny, h->pitch, h->plane); break;
    case LBM_PREC_FP16: unpack_kernel<__half><<<grid, block, 0, h->stream>>>((const __half *)fsrc, dst, h->nx, h->ny, h->pitch, h->plane); break;
    case LBM_PREC_BF16: unpack_kernel<__nv_bfloat16><<<grid, block, 0, h->stream>>>((const __nv_bfloat16 *)fsrc, dst, h->nx, h->ny, h->pitch, h->plane); break;
    }
    h->launches += 1;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int launch_pack(lbm_handle *h, const double *src, void *fdst)
{
    dim3 block(256), grid((h->nx + 255) / 256, h->ny, 9);
    switch (h->prec) {
    case LBM_PREC_FP32: pack_kernel<float><<<grid, block, 0, h->stream>>>(src, (float *)fdst, h->nx, h->ny, h->pitch, h->plane); break;
    case LBM_PREC_FP64: pack_kernel<double><<<grid, block, 0, h->stream>>>(src, (double *)fdst, h->nx, h->ny, h->pitch, h->plane); break;
    case LBM_PREC_FP16: pack_kernel<__half><<<grid, block, 0, h->stream>>>(src, (__half *)fdst, h->nx, h->ny, h->pitch, h->plane); break;
    case LBM_PREC_BF16: pack_kernel<__nv_bfloat16><<<grid, block, 0, h->stream>>>(src, (__nv_bfloat16 *)fdst, h->nx, h->ny, h->pitch, h->plane); break;
    }
    h->launches += 1;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int launch_residual(lbm_handle *h, const void *fa, const void *fb, double *out2)
{
    const int blocks = 296, threads = 256;
    if (h->prec == LBM_PREC_FP64)
        residual_kernel<double><<<blocks, threads, 0, h->stream>>>((const double *)fa, (const double *)fb, h->nx, h->ny, h->d_red);
    else
        residual_kernel<float><<<blocks, threads, 0, h->stream>>>((const float *)fa, (const float *)fb, h->nx, h->ny, h->d_red);
    h->launches += 1;
    if (cudaGetLastError() != cudaSuccess) return -1;
    std::vector<double> part(2 * blocks);
    if (cudaMemcpyAsync(part.data(), h->d_red, sizeof(double) * 2 * blocks, cudaMemcpyDeviceToHost, h->stream) != cudaSuccess)
        return -1;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return -1;
    double t1 = 0, t2 = 0;
    for (int b = 0; b < blocks; ++b) { t1 += part[2 * b]; t2 += part[2 * b + 1]; }
    out2[0] = t1;
    out2[1] = t2;
    return 0;
}
