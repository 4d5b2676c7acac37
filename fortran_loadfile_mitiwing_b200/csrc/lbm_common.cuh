// lbm_common.cuh -- data layout and device helpers shared by the kernels.
//
// Populations are stored as deviations g_k = f_k - w_k from the exact D2Q9
// weights (4/9, 1/9, 1/36), structure of arrays: 9 planes of ny rows, each row
// `pitch` elements (pitch a multiple of 64, x fastest). Plane k, node (i,j)
// (0-based) is at k*plane + j*pitch + i. The reference keeps f(Nx,Ny,9) in
// the same x-fastest plane order (main.f90:145), so the shift is storage only:
// every moment below is the moment of f, carried without the large constant
// part so that FP32/FP16/BF16 storage keeps its precision for the part that
// moves.
#pragma once
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <stdint.h>
#include <string.h>

#define LBM_Q 9
#define LBM_MAXW 8
#define LBM_BOX 6  // a support box spans at most 6 nodes per axis (|r| <= 2.5)

// direction order of D2Q9model (D2Q9model.f90:5-22): 0,E,N,W,S,NE,NW,SW,SE
__host__ __device__ constexpr int lbm_ex(int k)
{
    return k == 1 || k == 5 || k == 8 ? 1 : (k == 3 || k == 6 || k == 7 ? -1 : 0);
}
__host__ __device__ constexpr int lbm_ey(int k)
{
    return k == 2 || k == 5 || k == 6 ? 1 : (k == 4 || k == 7 || k == 8 ? -1 : 0);
}

// status bits written by the kernels, read by the host after a step/run
#define LBM_ST_RANGE 1u      // a support box reached the outer node layers
#define LBM_ST_SOLVER 2u     // IB matrix not positive definite
#define LBM_ST_NONFINITE 4u  // NaN/Inf in forces
#define LBM_ST_OVERFLOW 8u   // patch larger than its allocation
#define LBM_ST_TIMEOUT 16u   // a bounded wait on a shared-memory barrier gave up
// An index read from device memory (a solve-order position, a tile-list
// entry, a correction-tile number, a marker's support box or wing) fell
// outside the buffer it indexes. The kernel that saw it sets its own bit and
// skips that access; the host reports the error naming the kernel.
#define LBM_ST_INDEX_INTERP 0x100u      // ib_interp: support box
#define LBM_ST_INDEX_ASSEMBLE 0x200u    // ib_assemble: solve order, support box
#define LBM_ST_INDEX_FACTOR 0x400u      // ib_factor (dense path): solve order, support box
#define LBM_ST_INDEX_SOLVE 0x800u       // ib_solve: solve order, force-ring row
#define LBM_ST_INDEX_SCATTER 0x1000u    // ib_tile_scatter: tile of a support box
#define LBM_ST_INDEX_SORT 0x2000u       // ib_tile_sort: correction tile
#define LBM_ST_INDEX_TILE 0x4000u       // ib_tile_update: correction tile, listed marker, box, wing
#define LBM_ST_INDEX_FORCES 0x8000u     // ib_forces: correction tile, force-ring row
#define LBM_ST_INDEX_RESIDUAL 0x10000u  // ib_residual: solve order, support box
#define LBM_ST_INDEX_LATTICE 0x20000u   // kf_tma: tile of the patch rectangle
#define LBM_ST_INDEX_MASK 0x3ff00u

// current immersed-boundary correction patch (0-based node rectangle)
struct PatchInfo {
    int i0, j0, w, h;
};

// one Lagrangian marker (segment midpoint) of the current step
struct Marker {
    double xm, ym;            // xb2, yb2 (airfoil.f90:267-270)
    double ub, vb;            // boundary velocity (boundary_condition.f90:1547-1550)
    double phx[LBM_BOX];      // one-axis kernel at nodes i1..i1+5
    double phy[LBM_BOX];      // one-axis kernel at nodes j1..j1+5
    int i1, i2, j1, j2;       // support box, 0-based inclusive (airfoil.f90:290-321)
    int wing;                 // 0-based
    int pad;
};

// A support box (0-based, inclusive: x..y columns, z..w rows) as make_marker
// leaves it: empty, or inside columns 1..nx-2 and rows 1..ny-2 and at most
// LBM_BOX nodes per axis, so that every node of it has all eight neighbours
// and its kernel values index phx/phy within bounds.
__host__ __device__ __forceinline__ bool box_in_bounds(int x, int y, int z, int w, int nx, int ny)
{
    if (y < x || w < z) return true;   // empty: no node is visited
    return x >= 1 && y <= nx - 2 && z >= 1 && w <= ny - 2 && y - x < LBM_BOX && w - z < LBM_BOX;
}

// compute precision of a storage type: FP64 storage computes in FP64,
// everything else in FP32
template <typename T> struct CType { using type = float; };
template <> struct CType<double> { using type = double; };

// storage conversions
template <typename T> struct Store;
// ld/st: one element from/to memory in compute precision; cvt/pack: convert
// an element already in registers
template <> struct Store<float> {
    static __device__ __forceinline__ float ld(const float *p) { return __ldg(p); }
    static __device__ __forceinline__ void st(float *p, float x) { *p = x; }
    static __device__ __forceinline__ float cvt(float x) { return x; }
    static __device__ __forceinline__ float pack(float x) { return x; }
};
template <> struct Store<double> {
    static __device__ __forceinline__ double ld(const double *p) { return __ldg(p); }
    static __device__ __forceinline__ void st(double *p, double x) { *p = x; }
    static __device__ __forceinline__ double cvt(double x) { return x; }
    static __device__ __forceinline__ double pack(double x) { return x; }
};
template <> struct Store<__half> {
    static __device__ __forceinline__ float ld(const __half *p) { return __half2float(__ldg(p)); }
    static __device__ __forceinline__ void st(__half *p, float x) { *p = __float2half_rn(x); }
    static __device__ __forceinline__ float cvt(__half x) { return __half2float(x); }
    static __device__ __forceinline__ __half pack(float x) { return __float2half_rn(x); }
};
template <> struct Store<__nv_bfloat16> {
    static __device__ __forceinline__ float ld(const __nv_bfloat16 *p) { return __bfloat162float(__ldg(p)); }
    static __device__ __forceinline__ void st(__nv_bfloat16 *p, float x) { *p = __float2bfloat16_rn(x); }
    static __device__ __forceinline__ float cvt(__nv_bfloat16 x) { return __bfloat162float(x); }
    static __device__ __forceinline__ __nv_bfloat16 pack(float x) { return __float2bfloat16_rn(x); }
};

// two adjacent 2-byte elements as one 32-bit word (low half: the lower
// column) <-> a float2 (x: the lower column); the paired conversions round
// each element to nearest, as the scalar ones above do
template <typename T> struct Pair2;
template <> struct Pair2<__half> {
    static __device__ __forceinline__ float2 unpack(uint32_t w)
    {
        __half2 h;
        memcpy(&h, &w, 4);
        return __half22float2(h);
    }
    static __device__ __forceinline__ uint32_t pack(float2 f)
    {
        const __half2 h = __float22half2_rn(f);
        uint32_t w;
        memcpy(&w, &h, 4);
        return w;
    }
};
template <> struct Pair2<__nv_bfloat16> {
    static __device__ __forceinline__ float2 unpack(uint32_t w)
    {
        __nv_bfloat162 h;
        memcpy(&h, &w, 4);
        return __bfloat1622float2(h);
    }
    static __device__ __forceinline__ uint32_t pack(float2 f)
    {
        const __nv_bfloat162 h = __float22bfloat162_rn(f);
        uint32_t w;
        memcpy(&w, &h, 4);
        return w;
    }
};

// m = M g for the MRT matrix of solution.f90:17-25 (rows: rho, e, eps, jx, qx,
// jy, qy, pxx, pxy), written out for its 0/+-1/+-2/+-4 entries.
template <typename C>
__device__ __forceinline__ void mrt_forward(const C g[9], C m[9])
{
    const C a = g[1] + g[2] + g[3] + g[4];
    const C d = g[5] + g[6] + g[7] + g[8];
    m[0] = g[0] + a + d;
    m[1] = C(-4) * g[0] - a + C(2) * d;
    m[2] = C(4) * g[0] - C(2) * a + d;
    const C dx = g[5] - g[6] - g[7] + g[8];
    const C dy = g[5] + g[6] - g[7] - g[8];
    m[3] = g[1] - g[3] + dx;
    m[4] = C(-2) * (g[1] - g[3]) + dx;
    m[5] = g[2] - g[4] + dy;
    m[6] = C(-2) * (g[2] - g[4]) + dy;
    m[7] = g[1] - g[2] + g[3] - g[4];
    m[8] = g[5] - g[6] + g[7] - g[8];
}

// g = M^-1 m. The rows of M are orthogonal, so M^-1 = M^T diag(1/|row|^2)
// with |row|^2 = 9, 36, 36, 6, 12, 6, 12, 4, 4 (the matrix nizhen inverts,
// solution.f90:27).
template <typename C>
__device__ __forceinline__ void mrt_inverse(const C m[9], C g[9])
{
    const C a1 = m[0] * C(1.0 / 9.0), a2 = m[1] * C(1.0 / 36.0), a3 = m[2] * C(1.0 / 36.0);
    const C a4 = m[3] * C(1.0 / 6.0), a5 = m[4] * C(1.0 / 12.0), a6 = m[5] * C(1.0 / 6.0);
    const C a7 = m[6] * C(1.0 / 12.0), a8 = m[7] * C(0.25), a9 = m[8] * C(0.25);
    g[0] = a1 - C(4) * a2 + C(4) * a3;
    const C ax = a1 - a2 - C(2) * a3;
    g[1] = ax + a4 - C(2) * a5 + a8;
    g[3] = ax - a4 + C(2) * a5 + a8;
    g[2] = ax + a6 - C(2) * a7 - a8;
    g[4] = ax - a6 + C(2) * a7 - a8;
    const C ad = a1 + C(2) * a2 + a3;
    const C px = a4 + a5, py = a6 + a7;
    g[5] = ad + px + py + a9;
    g[6] = ad - px + py - a9;
    g[7] = ad - px - py + a9;
    g[8] = ad + px - py - a9;
}

// meq of the boundary condition minus M w (boundary_condition.f90:444-455):
// (rho, -2rho+3J/rho, rho-3J/rho, jx, -jx, jy, -jy, (jx^2-jy^2)/rho, jxjy/rho)
// - (1,-2,1,0,...) with j = rho u. drho = rho - 1.
template <typename C>
__device__ __forceinline__ void meq_bc_dev(C drho, C u, C v, C e[9])
{
    const C rho = C(1) + drho;
    const C jx = rho * u, jy = rho * v;
    const C jj = (jx * jx + jy * jy) / rho;
    e[0] = drho;
    e[1] = C(-2) * drho + C(3) * jj;
    e[2] = drho - C(3) * jj;
    e[3] = jx;
    e[4] = -jx;
    e[5] = jy;
    e[6] = -jy;
    e[7] = (jx * jx - jy * jy) / rho;
    e[8] = (jx * jy) / rho;
}

// f_b = M^-1 [ meq(b) + (1-s)(M f0(nbr) - meq(nbr)) ] in deviation form
// (boundary_condition.f90:468-474)
template <typename C>
__device__ __forceinline__ void extrapolate_dev(const C s[9], C drb, C ub, C vb, C drn, C un, C vn,
                                                const C g0n[9], C gout[9])
{
    C m[9], eb[9], en[9];
    mrt_forward(g0n, m);
    meq_bc_dev(drb, ub, vb, eb);
    meq_bc_dev(drn, un, vn, en);
#pragma unroll
    for (int k = 0; k < 9; ++k) m[k] = eb[k] + (C(1) - s[k]) * (m[k] - en[k]);
    mrt_inverse(m, gout);
}

// ---- mbarrier and bulk-copy (cp.async.bulk, no multicast) helpers ----
#ifdef __CUDACC__
static __device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

static __device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

static __device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

static __device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

static __device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

static __device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

static __device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

static __device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
#endif
