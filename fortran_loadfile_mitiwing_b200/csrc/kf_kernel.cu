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
#include <algorithm>
#include <cstring>
#include <type_traits>
#include <vector>

#include "lbm_internal.h"
#include "lbm_node.cuh"

namespace {

using namespace lbm_node;

// a node of the step's correction tiles: inside the patch rectangle r, in a
// 16 x 16 tile that lists at least one marker. Those nodes are updated by
// the immersed-boundary tile kernel; the outer part skips them.
template <typename C>
__device__ __forceinline__ bool corr_tile(const KFArgs<C> &a, const PatchInfo &r, int i, int j)
{
    const unsigned li = (unsigned)(i - r.i0), lj = (unsigned)(j - r.j0);
    if (li >= (unsigned)r.w || lj >= (unsigned)r.h) return false;
    const unsigned tx = li >> 4, t = (lj >> 4) * (unsigned)a.tiles_x + tx;
    if (tx >= (unsigned)a.tiles_x || t >= (unsigned)a.tiles_n) {   // a rectangle larger than the tile grid
        atomicOr(a.status, LBM_ST_INDEX_LATTICE);
        return false;
    }
    return a.tiles[(long long)t * a.tile_stride] > 0;
}

// node-level device functions: lbm_node.cuh

// one node per thread, scalar loads (any lattice size)
template <typename T, typename C, bool FIELDS>
__global__ void __launch_bounds__(256) kf_kernel(const KFArgs<C> a)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y;
    if (a.mode == KF_OUTER && corr_tile(a, *a.pinfo, i, j)) return;
    if (i >= a.nx) return;
    const T *__restrict__ fin = (const T *)a.fin;
    T *__restrict__ fout = (T *)a.fout;
    C gout[9], frho, fu, fv;
    node_update<T, C>(a, fin, i, j, gout, frho, fu, fv);
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
            collide_interior<C>(a, g, false, C(0), C(0), gout, frho, fu, fv);
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
            node_update<T, C>(a, fin, i, j, gout, frho, fu, fv);
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
// 0 and nx-1 by the scalar edge path. With FP32 arithmetic (FP32, FP16 and
// BF16 storage) a thread updates two nodes at once with the paired FP32
// instructions (collide_pair), which halves the arithmetic instructions of
// the collision: with FP32 storage rows j and j+1 of its column, with 2-byte
// storage columns i and i+1 of one row. The 2-byte column pair is one 32-bit
// word in shared and in global memory, so it is read with one load (two for
// the x-shifted planes, joined by a byte permute), converted with one paired
// conversion and written with one store; the CTA's strip is then 512
// columns wide, and each staged row segment is 1 KB, as with FP32 storage.

constexpr int TW = 256;        // threads per CTA (the strip width of 4- and 8-byte storage)
#ifndef LBM_KF_STAGES
#define LBM_KF_STAGES 4
#endif
#ifndef LBM_KF_MINB
#define LBM_KF_MINB 4
#endif
// pipeline stages (a stage holds the 9 plane rows of one output row)
template <typename T> __host__ __device__ constexpr int tma_stages() { return LBM_KF_STAGES; }
// columns of a CTA's strip: two per thread with 2-byte storage
template <typename T> __host__ __device__ constexpr int tma_strip() { return sizeof(T) == 2 ? 2 * TW : TW; }
// Resident CTAs per SM the register budget is sized for (64 registers a
// thread at four). Four keep more rows in flight than three, which leave
// registers free for the immersed-boundary CTAs beside the lattice update
// but measured slower beside them as well (FP32 0.1227 against 0.1183 ms a
// step on 4096x2048).
constexpr int KF_MINB = LBM_KF_MINB;
// CTAs per SM the staged kernel is compiled for: FP64 storage keeps 3 (its
// ring alone, ~75 KB a CTA, allows no more), the others LBM_KF_MINB
template <typename T> constexpr int kf_minb() { return sizeof(T) == 8 ? 3 : KF_MINB; }

// mbarrier and bulk-copy helpers: lbm_common.cuh

template <typename T> __host__ __device__ constexpr int tma_halo() { return 16 / (int)sizeof(T); }
template <typename T> __host__ __device__ constexpr int tma_seg() { return tma_strip<T>() + 2 * tma_halo<T>(); }
template <typename T> constexpr size_t tma_smem() { return sizeof(T) * tma_stages<T>() * 9 * tma_seg<T>() + 2 * 8 * tma_stages<T>(); }

// the updated pair of columns i, i+1 of row j (2-byte storage): one 32-bit
// store per plane when both nodes are written (v0, v1), else the one that is
template <typename T, bool FIELDS>
__device__ __forceinline__ void store_pair2(const KFArgs<float> &a, T *__restrict__ fout, int i, int j, bool v0,
                                            bool v1, const float2 o[9], float2 frho, float2 fu, float2 fv)
{
    const long long base = (long long)j * a.pitch + i;
    if (v0 && v1) {
#pragma unroll
        for (int k = 0; k < 9; ++k)
            *reinterpret_cast<uint32_t *>(fout + (long long)k * a.plane + base) = Pair2<T>::pack(o[k]);
    } else if (v0) {
#pragma unroll
        for (int k = 0; k < 9; ++k) fout[(long long)k * a.plane + base] = Store<T>::pack(o[k].x);
    } else {
#pragma unroll
        for (int k = 0; k < 9; ++k) fout[(long long)k * a.plane + base + 1] = Store<T>::pack(o[k].y);
    }
    if (FIELDS) {
        const long long q = (long long)j * a.nx + i;
        if (v0) {
            a.rho_out[q] = frho.x;
            a.u_out[q] = fu.x;
            a.v_out[q] = fv.x;
        }
        if (v1) {
            a.rho_out[q + 1] = frho.y;
            a.u_out[q + 1] = fu.y;
            a.v_out[q + 1] = fv.y;
        }
    }
}

// One CTA of the staged kernel: strip bx (of gx) and row chunk by (of gy; the
// last chunk is the edge CTA row) of the lattice described by `a`.
template <typename T, typename C, bool FIELDS, bool CONS0>
__device__ __forceinline__ void kf_tma_cta(const KFArgs<C> &a, int bx, int by, int gx, int gy, unsigned char *smraw)
{
    constexpr int H = tma_halo<T>(), SEG = tma_seg<T>(), NWARP = TW / 32, KS = tma_stages<T>();
    constexpr int SW = tma_strip<T>();
    constexpr bool XPAIR = sizeof(T) == 2;   // two columns per thread
    T *buf = reinterpret_cast<T *>(smraw);
    uint64_t *full = reinterpret_cast<uint64_t *>(smraw + sizeof(T) * KS * 9 * SEG);
    uint64_t *empty = full + KS;
    const int tid = threadIdx.x, lane = tid & 31;
    const int x0 = bx * SW;
    const int i = x0 + (XPAIR ? 2 * tid : tid);
    const T *__restrict__ fin = (const T *)a.fin;
    T *__restrict__ fout = (T *)a.fout;
    const PatchInfo rr = a.mode == KF_OUTER ? *a.pinfo : PatchInfo{0, 0, 0, 0};   // step's patch rectangle
    if (by == gy - 1) {
        // the edge nodes: rows 0 and ny-1 of this strip, and a share of the
        // nodes of columns 0 and nx-1 (which the strips' row sweeps skip)
        for (int ie = x0 + tid; ie < min(x0 + SW, a.nx); ie += TW)
            for (int j = 0; j < a.ny; j += a.ny - 1) {
                C gout[9], frho, fu, fv;
                edge_update<T, C>(a, fin, ie, j, gout, frho, fu, fv);
                store_node<T, C, FIELDS>(a, fout, ie, j, gout, frho, fu, fv);
            }
        for (int q = bx * TW + tid; q < 2 * (a.ny - 2); q += gx * TW) {
            const int j = 1 + q / 2, ie = (q & 1) ? a.nx - 1 : 0;
            C gout[9], frho, fu, fv;
            edge_update<T, C>(a, fin, ie, j, gout, frho, fu, fv);
            store_node<T, C, FIELDS>(a, fout, ie, j, gout, frho, fu, fv);
        }
        return;
    }
    const int j0 = 1 + by * a.rows_per_cta;
    const int nrows = min(a.rows_per_cta, a.ny - 1 - j0);
    if (nrows <= 0) return;
    const int width = min(SW, a.nx - x0);
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
    // bounded wait: a barrier that never completes is reported, not waited on
    // forever. The outcome is made the same for the whole warp (full_wait), or
    // broadcast from thread 0 (refill), so that a warp leaves the row loop as
    // a whole and no lane is left waiting in __syncwarp for one that left.
    auto wait = [&](uint64_t *bar, uint32_t parity) -> bool {
        int spins = 0;
        while (!mbar_try_wait(bar, parity))
            if (++spins > (1 << 22)) return false;
        return true;
    };
    auto full_wait = [&](int r) -> bool {
        return __all_sync(0xffffffffu, wait(&full[r % KS], (uint32_t)((r / KS) & 1)));
    };
    // thread 0: refills the stage of row q with row q + KS once every warp is
    // done with it; false (in every lane of warp 0) if that wait gave up
    auto refill = [&](int q) -> bool {
        bool good = true;
        if (tid == 0 && q + KS < nrows) {
            good = wait(&empty[q % KS], (uint32_t)((q / KS) & 1));
            if (good) {
                fence_proxy_async();
                issue(q + KS);
            }
        }
        return __shfl_sync(0xffffffffu, good, 0);
    };
    if (tid == 0)
        for (int r = 0; r < KS && r < nrows; ++r) issue(r);
    // Stage s holds row r = s (mod KS). A warp waits for the row on full[s],
    // and when done reading it arrives on empty[s]; thread 0 refills the stage
    // with row r + KS once all warps have arrived. Only warp 0 waits for the
    // other warps; they run up to KS - 1 rows ahead.
    bool ok = true;
    if constexpr (XPAIR) {
        // 2-byte storage: columns i and i+1 of each row as one pair
        for (int r = 0; r < nrows; ++r) {
            const int s = r % KS, j = j0 + r;
            if (!full_wait(r)) { ok = false; break; }
            const bool v0 = i >= 1 && i <= a.nx - 2 && !(a.mode == KF_OUTER && corr_tile(a, rr, i, j));
            const bool v1 = i + 1 <= a.nx - 2 && !(a.mode == KF_OUTER && corr_tile(a, rr, i + 1, j));
            if (v0 || v1) {
                float2 g[9], o[9], frho, fu, fv;
                // word t of a staged plane row holds the columns x0 + 2t, x0 + 2t + 1
                const uint32_t *w = reinterpret_cast<const uint32_t *>(buf + s * 9 * SEG + H) + tid;
#pragma unroll
                for (int k = 0; k < 9; ++k) {
                    const uint32_t *wk = w + k * (SEG / 2);
                    uint32_t pr;
                    if (lbm_ex(k) == 0) pr = wk[0];
                    else if (lbm_ex(k) == 1) pr = __byte_perm(wk[-1], wk[0], 0x5432);   // columns i-1, i
                    else pr = __byte_perm(wk[0], wk[1], 0x5432);                        // columns i+1, i+2
                    g[k] = Pair2<T>::unpack(pr);
                }
                collide_pair<CONS0, FIELDS>(a, g, o, frho, fu, fv);
                store_pair2<T, FIELDS>(a, fout, i, j, v0, v1, o, frho, fu, fv);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&empty[s]);
            if (!refill(r)) { ok = false; break; }
        }
    } else if constexpr (std::is_same<C, float>::value) {
        // FP32 arithmetic: rows r and r + 1 of a thread's column as one pair
        // of the paired instructions (collide_pair); an odd last row is
        // computed in both halves and stored once
        const bool interior = i > 0 && i < a.nx - 1;
        for (int r = 0; r < nrows; r += 2) {
            const int r1 = min(r + 1, nrows - 1);
            const int s0 = r % KS, s1 = r1 % KS, j = j0 + r;
            if (!full_wait(r) || !full_wait(r1)) {
                ok = false;
                break;
            }
            const bool st0 = interior && !(a.mode == KF_OUTER && corr_tile(a, rr, i, j));
            const bool st1 = interior && r1 != r && !(a.mode == KF_OUTER && corr_tile(a, rr, i, j + 1));
            if (st0 || st1) {
                float2 g[9], o[9], frho, fu, fv;
                const T *row0 = buf + s0 * 9 * SEG + H + tid, *row1 = buf + s1 * 9 * SEG + H + tid;
#pragma unroll
                for (int k = 0; k < 9; ++k)
                    g[k] = make_float2(Store<T>::cvt(row0[k * SEG - lbm_ex(k)]), Store<T>::cvt(row1[k * SEG - lbm_ex(k)]));
                collide_pair<CONS0, FIELDS>(a, g, o, frho, fu, fv);
                if (st0) {
                    C go[9];
#pragma unroll
                    for (int k = 0; k < 9; ++k) go[k] = o[k].x;
                    store_node<T, C, FIELDS>(a, fout, i, j, go, frho.x, fu.x, fv.x);
                }
                if (st1) {
                    C go[9];
#pragma unroll
                    for (int k = 0; k < 9; ++k) go[k] = o[k].y;
                    store_node<T, C, FIELDS>(a, fout, i, j + 1, go, frho.y, fu.y, fv.y);
                }
            }
            __syncwarp();
            if (lane == 0) {
                mbar_arrive(&empty[s0]);
                if (r1 != r) mbar_arrive(&empty[s1]);
            }
            if (!refill(r) || (r1 != r && !refill(r1))) {
                ok = false;
                break;
            }
        }
    } else
    for (int r = 0; r < nrows; ++r) {
        const int s = r % KS, j = j0 + r;
        if (!full_wait(r)) { ok = false; break; }
        const bool skip = a.mode == KF_OUTER && corr_tile(a, rr, i, j);
        if (i > 0 && i < a.nx - 1 && !skip) {
            C gout[9], frho, fu, fv;
            C g[9];
            const T *row = buf + s * 9 * SEG + H + tid;
#pragma unroll
            for (int k = 0; k < 9; ++k) g[k] = (C)Store<T>::cvt(row[k * SEG - lbm_ex(k)]);
            collide_interior<C, CONS0>(a, g, false, C(0), C(0), gout, frho, fu, fv);
            store_node<T, C, FIELDS>(a, fout, i, j, gout, frho, fu, fv);
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
        if (!refill(r)) { ok = false; break; }
    }
    if (!ok) {
        // report, then wait (bounded) for this CTA's copies still in flight
        if (lane == 0) atomicOr(a.status, LBM_ST_TIMEOUT);
        for (int s = 0; s < KS; ++s) {
            int spins = 0;
            while (!mbar_try_wait(&full[s], 0) && !mbar_try_wait(&full[s], 1) && ++spins < (1 << 20)) {
            }
        }
    }
}

// One CTA per (strip, row chunk) of the lattice; the edge row's CTAs
// (chunk gy - 1, whose nodes take longer) are numbered first so that they
// start in the first wave rather than in the tail.
// The arguments are __grid_constant__ kernel parameters, read in place from
// the parameter bank: no global loads of them in the row loop (measured as
// 6.6 loads per node when they were read from a table in global memory,
// which every store may alias) and no registers held for them.
template <typename T, typename C, bool FIELDS, bool CONS0>
__global__ void __launch_bounds__(TW, kf_minb<T>()) kf_tma(const __grid_constant__ KFArgs<C> a)
{
    extern __shared__ __align__(128) unsigned char smraw[];
    const int gy = gridDim.y, by = blockIdx.y == 0 ? gy - 1 : blockIdx.y - 1;
    kf_tma_cta<T, C, FIELDS, CONS0>(a, blockIdx.x, by, gridDim.x, gy, smraw);
}

// Several lattices (a batch of cases) in one launch: CTA b runs entry b of
// the case table, {case, strip, row chunk, strips | row chunks << 16}.
template <typename T, typename C, bool FIELDS, bool CONS0>
__global__ void __launch_bounds__(TW, kf_minb<T>()) kf_tma_multi(const KFArgs<C> *cases, const int4 *table)
{
    extern __shared__ __align__(128) unsigned char smraw[];
    const int4 t = table[blockIdx.x];
    kf_tma_cta<T, C, FIELDS, CONS0>(cases[t.x], t.y, t.z, t.w & 0xffff, t.w >> 16, smraw);
}

// the conserved moments' relaxation rates are zero (the reference's setting)
template <typename C> bool cons0(const KFArgs<C> &a) { return a.s[0] == C(0) && a.s[3] == C(0) && a.s[5] == C(0); }

template <typename T, typename C, bool FIELDS>
void launch_tma_f(const KFArgs<C> &a, dim3 grid, cudaStream_t st)
{
    const size_t smem = tma_smem<T>();
    if (cons0(a))
        kf_tma<T, C, FIELDS, true><<<grid, TW, smem, st>>>(a);
    else
        kf_tma<T, C, FIELDS, false><<<grid, TW, smem, st>>>(a);
}

// one CTA per (strip, row chunk) of the lattice, and the edge CTA row
template <typename T, typename C>
void launch_tma(const lbm_handle *h, const KFArgs<C> &a, bool fields, cudaStream_t st)
{
    const dim3 grid((h->nx + tma_strip<T>() - 1) / tma_strip<T>(), (h->ny - 2 + a.rows_per_cta - 1) / a.rows_per_cta + 1);
    if (fields)
        launch_tma_f<T, C, true>(a, grid, st);
    else
        launch_tma_f<T, C, false>(a, grid, st);
}

// the largest dynamic shared memory a CTA may opt in to on the current device
int smem_optin()
{
    static int v = 0;
    if (!v) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
            v = 0;
    }
    return v;
}

template <typename T, typename C, bool FIELDS, bool CONS0>
int configure_one(int smem)
{
    if (cudaFuncSetAttribute(kf_tma<T, C, FIELDS, CONS0>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
        cudaSuccess)
        return -1;
    // the batched launch may ask for more than it uses, to hold fewer CTAs
    // per SM (multi_smem)
    if (cudaFuncSetAttribute(kf_tma_multi<T, C, FIELDS, CONS0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             std::max(smem, smem_optin())) != cudaSuccess)
        return -1;
    return 0;
}

template <typename T, typename C>
int configure_tma()
{
    const int smem = (int)tma_smem<T>();
    if (configure_one<T, C, true, true>(smem) || configure_one<T, C, true, false>(smem) ||
        configure_one<T, C, false, true>(smem) || configure_one<T, C, false, false>(smem))
        return -1;
    return 0;
}

// case table entry {case, strip, chunk, gx | gy << 16} of the staged kernel's
// grid for one lattice
void tma_grid(int nx, int ny, int rows_per_cta, size_t elem, int *gx, int *gy)
{
    const int sw = elem == 2 ? tma_strip<__half>() : TW;
    *gx = (nx + sw - 1) / sw;
    *gy = (ny - 2 + rows_per_cta - 1) / rows_per_cta + 1;
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
    KFArgs<C> a = make_kf_args<C>(h, fin, fout, fields, mode);
    const bool small_index = 9ll * h->plane < (1ll << 31) && (long long)h->nx * h->ny < (1ll << 31);
    const int vec = small_index ? h->kf_vec : 1;
    if (!st) st = h->stream;
    if (h->kf_tma && h->ny >= 3) {
        static bool configured = false;   // per process; the attribute is per function
        if (!configured) {
            if (configure_tma<T, C>()) return -1;
            configured = true;
        }
        launch_tma<T, C>(h, a, fields != nullptr, st);
    } else if (mode == KF_ALL && vec == 4 && h->pitch % 4 == 0) {
        launch_vec<T, C, 4>(a, fields != nullptr, h->nx, h->ny, st);
    } else if (mode == KF_ALL && vec == 2 && h->pitch % 2 == 0) {
        launch_vec<T, C, 2>(a, fields != nullptr, h->nx, h->ny, st);
    } else {
        dim3 block(256, 1), grid((h->nx + 255) / 256, h->ny);
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

// Initial populations and fields (solution.f90:33-59): f = feq(rho = 1,
// u = UU + du, v = 0 + dv) with the single-precision lattice weights
// (D2Q9model.f90:24-46), stored as deviations from the reference weights,
// and the fields (1, u, v). The operations, their order and their rounding
// are those of the host's FP64 evaluation followed by the pack kernel
// (feq - w, + w, then - w), with round-to-nearest intrinsics so nothing is
// contracted into an FMA: the initial state is the same bit for bit.
template <typename T>
__global__ void init_kernel(const double *__restrict__ du, const double *__restrict__ dv, double uu,
                            T *__restrict__ f, typename CType<T>::type *__restrict__ fields, int nx, int ny,
                            int pitch, long long plane)
{
    using C = typename CType<T>::type;
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y;
    if (i >= nx) return;
    const long long q = (long long)j * nx + i, nn = (long long)nx * ny;
    double u = uu, v = 0.0;
    if (du) u = __dadd_rn(u, du[q]);
    if (dv) v = __dadd_rn(v, dv[q]);
    const double utwo = __dadd_rn(__dmul_rn(u, u), __dmul_rn(v, v));
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const double eu = __dadd_rn(__dmul_rn((double)lbm_ex(k), u), __dmul_rn((double)lbm_ey(k), v));
        const double ws = k == 0 ? (double)(4.0f / 9.0f) : (k < 5 ? (double)(1.0f / 9.0f) : (double)(1.0f / 36.0f));
        const double poly = __dsub_rn(__dadd_rn(__dadd_rn(1.0, __dmul_rn(3.0, eu)), __dmul_rn(__dmul_rn(4.5, eu), eu)),
                                      __dmul_rn(1.5, utwo));
        const double fe = __dmul_rn(__dmul_rn(ws, 1.0), poly);
        const double fk = __dadd_rn(__dsub_rn(fe, wref(k)), wref(k));
        Store<T>::st(f + k * plane + (long long)j * pitch + i, (C)__dsub_rn(fk, wref(k)));
    }
    fields[q] = C(1);
    fields[nn + q] = (C)u;
    fields[2 * nn + q] = (C)v;
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

// Global mass check (FP64): the sum over every node and direction of the
// stored deviations g = f - w, whose total plus nx*ny (the weights sum to 1
// per node) is the mass sum_ij sum_k f_k. Each CTA sums a fixed set of rows
// in a fixed order; the last CTA to finish adds the CTA partials in CTA
// order, so the result does not depend on scheduling. The reference's own
// reduction over the lattice is erranalysis (solution.f90:102-109).
constexpr int MASS_BLOCKS = 296, MASS_THREADS = 256;
template <typename T>
__global__ void __launch_bounds__(MASS_THREADS) mass_kernel(const T *__restrict__ f, int nx, int ny, int pitch,
                                                            long long plane, double *__restrict__ part,
                                                            unsigned *__restrict__ counter)
{
    __shared__ double red[MASS_THREADS / 32];
    __shared__ bool amlast;
    double s = 0.0;
    for (int j = blockIdx.x; j < ny; j += gridDim.x)
        for (int i = threadIdx.x; i < nx; i += blockDim.x) {
            const T *p = f + (long long)j * pitch + i;
            double t = 0.0;
#pragma unroll
            for (int k = 0; k < 9; ++k) t += (double)Store<T>::ld(p + k * plane);
            s += t;
        }
    for (int off = 16; off; off >>= 1) s += __shfl_down_sync(0xffffffffu, s, off);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0) red[wid] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < MASS_THREADS / 32; ++w) t += red[w];
        part[blockIdx.x] = t;
        __threadfence();
        amlast = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!amlast) return;
    __threadfence();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int b = 0; b < (int)gridDim.x; ++b) t += __ldcg(part + b);
        part[MASS_BLOCKS] = t;
        *counter = 0u;
    }
}

}  // namespace

// the deviation sum of the populations in `fsrc` into h->d_mass[MASS_BLOCKS],
// on stream st (the caller copies it back)
int launch_mass(lbm_handle *h, const void *fsrc, cudaStream_t st)
{
    switch (h->prec) {
    case LBM_PREC_FP32:
        mass_kernel<float><<<MASS_BLOCKS, MASS_THREADS, 0, st>>>((const float *)fsrc, h->nx, h->ny, h->pitch, h->plane, h->d_mass, h->d_mcount);
        break;
    case LBM_PREC_FP64:
        mass_kernel<double><<<MASS_BLOCKS, MASS_THREADS, 0, st>>>((const double *)fsrc, h->nx, h->ny, h->pitch, h->plane, h->d_mass, h->d_mcount);
        break;
    case LBM_PREC_FP16:
        mass_kernel<__half><<<MASS_BLOCKS, MASS_THREADS, 0, st>>>((const __half *)fsrc, h->nx, h->ny, h->pitch, h->plane, h->d_mass, h->d_mcount);
        break;
    case LBM_PREC_BF16:
        mass_kernel<__nv_bfloat16><<<MASS_BLOCKS, MASS_THREADS, 0, st>>>((const __nv_bfloat16 *)fsrc, h->nx, h->ny, h->pitch, h->plane, h->d_mass, h->d_mcount);
        break;
    default: return -1;
    }
    h->launches += 1;
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

int mass_slots() { return MASS_BLOCKS + 1; }

// Dynamic shared memory of a batched lattice launch that holds at most
// `ctas_per_sm` CTAs on an SM (0: the kernel's own ring, as many CTAs as the
// registers allow, 4 for 2- and 4-byte storage). The kernel uses only its
// ring; the rest of the request is an occupancy limit for the autotuner.
template <typename T>
size_t multi_smem(int ctas_per_sm)
{
    const size_t base = tma_smem<T>();
    if (ctas_per_sm <= 0) return base;
    static int per_sm = 0, reserved = 0;
    if (!per_sm) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev) != cudaSuccess)
            per_sm = reserved = 0;
    }
    if (per_sm <= 0) return base;
    // ctas_per_sm CTAs of this size fit, one more does not
    size_t s = ((size_t)per_sm / ctas_per_sm - (size_t)reserved) & ~(size_t)127;
    return std::min(std::max(s, base), (size_t)std::max(smem_optin(), (int)base));
}

template <typename T, typename C>
int launch_kf_multi_t(const void *cases, const int4 *table, int nentries, bool fields, bool cons0, int ctas_per_sm,
                      cudaStream_t st)
{
    static bool configured = false;   // per process; the attribute is per function
    if (!configured) {
        if (configure_tma<T, C>()) return -1;
        configured = true;
    }
    const size_t smem = multi_smem<T>(ctas_per_sm);
    const KFArgs<C> *c = (const KFArgs<C> *)cases;
    if (fields && cons0)
        kf_tma_multi<T, C, true, true><<<nentries, TW, smem, st>>>(c, table);
    else if (fields)
        kf_tma_multi<T, C, true, false><<<nentries, TW, smem, st>>>(c, table);
    else if (cons0)
        kf_tma_multi<T, C, false, true><<<nentries, TW, smem, st>>>(c, table);
    else
        kf_tma_multi<T, C, false, false><<<nentries, TW, smem, st>>>(c, table);
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

// lattice arguments of one case in the storage precision's compute type
size_t kf_args_size(int prec) { return prec == LBM_PREC_FP64 ? sizeof(KFArgs<double>) : sizeof(KFArgs<float>); }

void kf_args_write(lbm_handle *h, const void *fin, void *fout, void *fields, int mode, void *dst)
{
    if (h->prec == LBM_PREC_FP64)
        *(KFArgs<double> *)dst = make_kf_args<double>(h, fin, fout, fields, mode);
    else
        *(KFArgs<float> *)dst = make_kf_args<float>(h, fin, fout, fields, mode);
}

void kf_tma_grid(const lbm_handle *h, int *gx, int *gy) { tma_grid(h->nx, h->ny, h->kf_rows, h->elem, gx, gy); }

// the staged lattice kernel over a batch of cases (device arrays of their
// arguments and of the case table)
int launch_kf_multi(int prec, const void *cases, const int4 *table, int nentries, bool fields, bool cons0,
                    int ctas_per_sm, cudaStream_t st)
{
    switch (prec) {
    case LBM_PREC_FP32: return launch_kf_multi_t<float, float>(cases, table, nentries, fields, cons0, ctas_per_sm, st);
    case LBM_PREC_FP64:
        return launch_kf_multi_t<double, double>(cases, table, nentries, fields, cons0, ctas_per_sm, st);
    case LBM_PREC_FP16:
        return launch_kf_multi_t<__half, float>(cases, table, nentries, fields, cons0, ctas_per_sm, st);
    case LBM_PREC_BF16:
        return launch_kf_multi_t<__nv_bfloat16, float>(cases, table, nentries, fields, cons0, ctas_per_sm, st);
    }
    return -1;
}

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

int launch_init_lattice(lbm_handle *h, const double *du, const double *dv)
{
    dim3 block(256), grid((h->nx + 255) / 256, h->ny);
    const double uu = h->p.uu;
    switch (h->prec) {
    case LBM_PREC_FP32:
        init_kernel<float><<<grid, block, 0, h->stream>>>(du, dv, uu, (float *)h->fbuf[0], (float *)h->d_fields[0],
                                                          h->nx, h->ny, h->pitch, h->plane);
        break;
    case LBM_PREC_FP64:
        init_kernel<double><<<grid, block, 0, h->stream>>>(du, dv, uu, (double *)h->fbuf[0], (double *)h->d_fields[0],
                                                           h->nx, h->ny, h->pitch, h->plane);
        break;
    case LBM_PREC_FP16:
        init_kernel<__half><<<grid, block, 0, h->stream>>>(du, dv, uu, (__half *)h->fbuf[0], (float *)h->d_fields[0],
                                                           h->nx, h->ny, h->pitch, h->plane);
        break;
    case LBM_PREC_BF16:
        init_kernel<__nv_bfloat16><<<grid, block, 0, h->stream>>>(du, dv, uu, (__nv_bfloat16 *)h->fbuf[0],
                                                                  (float *)h->d_fields[0], h->nx, h->ny, h->pitch,
                                                                  h->plane);
        break;
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
