// lbm_node.cuh -- node-level device functions of the fused lattice update
// (pull streaming, moments, outer boundary condition, MRT collision with the
// immersed-boundary correction, store), shared by the lattice kernels and by
// the immersed-boundary tile update.
//
// Reference path of one node (one time step):
//   streaming           solution.f90:428-454   f0(i,j,k) = f(i-ex, j-ey, k)
//   physical_variables  solution.f90:471-542   rho, u, v of f0
//   IB velocity/force   boundary_condition.f90:1645-1659 (u = u* + du, g = 2 rho du)
//   colission           solution.f90:573-643   MRT relaxation with forcing
//   boundary_condition1 boundary_condition.f90:288-858 (left/right
//                       characteristic + extrapolation, top/bottom rows)
#pragma once
#include "lbm_internal.h"

int ib_tile_ints();

// arguments of the lattice update of one step (fields optional)
template <typename C>
inline KFArgs<C> make_kf_args(lbm_handle *h, const void *fin, void *fout, void *fields, int mode)
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
    // (e_k - m_k) sc_k is the k-th coefficient of the inverse transform
    // (mrt_inverse: 1/9, 1/36, 1/36, 1/6, 1/12, 1/6, 1/12, 1/4, 1/4), with
    // the sign of the equilibrium folded in where e_k - m_k is formed negated
    const double cinv[9] = {-1.0 / 9.0, 1.0 / 36.0, 1.0 / 36.0, -1.0 / 6.0, -1.0 / 12.0, -1.0 / 6.0, -1.0 / 12.0,
                            0.25, 0.25};
    for (int k = 0; k < 9; ++k) a.sc[k] = (C)(h->s[k] * cinv[k]);
    a.cs = (C)((double)sqrtf(3.0f) / 3.0);   // boundary_condition.f90:304
    const C *ec = (const C *)h->edge_c;
    a.col_l = ec;
    a.col_r = ec + 3 * h->ny;
    a.corner = ec + 6 * h->ny;
    a.pinfo = h->d_pinfo + h->pinfo_slot;
    a.tiles = h->d_tiles ? h->d_tiles + (size_t)h->pinfo_slot * h->tiles_slot : nullptr;
    a.tiles_x = h->patch_gx();
    a.tile_stride = ib_tile_ints();
    a.tiles_n = h->patch_gx() * h->patch_gy();
    if (fields) {
        C *fc = (C *)fields;
        const long long nn = (long long)h->nx * h->ny;
        a.rho_out = fc;
        a.u_out = fc + nn;
        a.v_out = fc + 2 * nn;
    } else {
        a.rho_out = a.u_out = a.v_out = nullptr;
    }
    a.rows_per_cta = h->kf_rows;
    a.status = h->d_status;
    return a;
}

namespace lbm_node {

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
// velocity correction (du, dv) when `corr` (a node of a correction tile),
// MRT collision with forcing
// CONS0: the relaxation rates of the conserved moments (s[0], s[3], s[5])
// are zero, as the reference sets them (ini_mesh.f90:59-67); their terms of
// the update are then left out at compile time.
template <typename C, bool CONS0 = false>
__device__ __forceinline__ void collide_interior(const KFArgs<C> &a, const C g[9], bool corr, C du, C dv, C gout[9],
                                                 C &frho, C &fu, C &fv)
{
    // physical_variables (solution.f90:471-542) on the deviations
    const C drho = ((g[0] + g[1]) + (g[2] + g[3])) + ((g[4] + g[5]) + (g[6] + g[7])) + g[8];
    const C jx0 = (g[1] - g[3]) + (g[5] - g[6]) + (g[8] - g[7]);
    const C jy0 = (g[2] - g[4]) + (g[5] + g[6]) - (g[7] + g[8]);
    const C rho = C(1) + drho;
    C u = jx0 / rho, v = jy0 / rho;   // needed only for the fields and the correction
    // j = rho u of the equilibrium: the summed momentum itself when there is
    // no correction (rho (jx/rho) = jx up to one rounding)
    C jx = jx0, jy = jy0;
    C gx = C(0), gy = C(0);
    if (corr) {
        u = u + du;                       // boundary_condition.f90:1650-1651
        v = v + dv;
        jx = rho * u;
        jy = rho * v;
        gx = C(2) * rho * du;             // :1652-1656
        gy = C(2) * rho * dv;
    }
    // m = M g (solution.f90:580-600); rows 0, 3, 5 are the moments above
    C m[9];
    {
        const C as = g[1] + g[2] + g[3] + g[4];
        const C ds = g[5] + g[6] + g[7] + g[8];
        const C dx = g[5] - g[6] - g[7] + g[8];
        const C dy = g[5] + g[6] - g[7] - g[8];
        m[0] = drho;
        m[1] = C(-4) * g[0] - as + C(2) * ds;
        m[2] = C(4) * g[0] - C(2) * as + ds;
        m[3] = jx0;
        m[4] = C(-2) * (g[1] - g[3]) + dx;
        m[5] = jy0;
        m[6] = C(-2) * (g[2] - g[4]) + dy;
        m[7] = g[1] - g[2] + g[3] - g[4];
        m[8] = g[5] - g[6] + g[7] - g[8];
    }
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
    for (int k = 0; k < 9; ++k) d[k] = (CONS0 && (k == 0 || k == 3 || k == 5)) ? C(0) : (e[k] - m[k]) * a.s[k];
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

// Two interior nodes at once (no correction) with the paired FP32
// instructions of sm_100 (FADD2, FMUL2, FFMA2 on a float2: one instruction
// for both nodes). The same update as collide_interior<float> with the
// products regrouped for the pairs: the relaxation rate and the inverse
// transform's scale are one factor (KFArgs::sc), and the inverse transform
// and the return to g are fused; results agree with collide_interior to FP32
// rounding. Fields: (rho, u, v) of both nodes when FIELDS.
__device__ __forceinline__ float2 p2(float x) { return make_float2(x, x); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 psub(float2 a, float2 b) { return __ffma2_rn(b, p2(-1.0f), a); }   // exact: a - b, one rounding
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

template <bool CONS0, bool FIELDS>
__device__ __forceinline__ void collide_pair(const KFArgs<float> &a, const float2 g[9], float2 o[9], float2 &frho,
                                             float2 &fu, float2 &fv)
{
    // moments (physical_variables, solution.f90:471-542, and m = M g,
    // solution.f90:580-600) from shared sums
    const float2 a13 = psub(g[1], g[3]), a24 = psub(g[2], g[4]);
    const float2 p56 = psub(g[5], g[6]), p87 = psub(g[8], g[7]);
    const float2 s56 = padd(g[5], g[6]), s78 = padd(g[7], g[8]);
    const float2 s13 = padd(g[1], g[3]), s24 = padd(g[2], g[4]);
    const float2 dx = padd(p56, p87), dy = psub(s56, s78);
    const float2 jx = padd(a13, dx), jy = padd(a24, dy);
    const float2 as = padd(s13, s24), ds = padd(s56, s78);
    const float2 drho = padd(padd(g[0], as), ds);
    const float2 m1n = pfma(g[0], p2(4.0f), pfma(ds, p2(-2.0f), as));   // -m1
    const float2 m2 = pfma(g[0], p2(4.0f), pfma(as, p2(-2.0f), ds));
    const float2 m4 = pfma(a13, p2(-2.0f), dx), m6 = pfma(a24, p2(-2.0f), dy);
    const float2 m7 = psub(s13, s24), m8n = psub(p87, p56);             // m7, -m8
    const float2 x2 = pmul(jx, jx), y2 = pmul(jy, jy);
    const float2 jj = padd(x2, y2);
    // (meq - m) sc: meq = (-1, -2drho + 3jj, drho - 3jj, 0, -jx, 0, -jy,
    // jx^2 - jy^2, jx jy) in deviation form (solution.f90:603-612)
    const float2 a2 = pmul(pfma(jj, p2(3.0f), pfma(drho, p2(-2.0f), m1n)), p2(a.sc[1]));
    const float2 a3 = pmul(pfma(jj, p2(-3.0f), psub(drho, m2)), p2(a.sc[2]));
    const float2 a5 = pmul(padd(jx, m4), p2(a.sc[4]));
    const float2 a7 = pmul(padd(jy, m6), p2(a.sc[6]));
    const float2 a8 = pmul(psub(x2, padd(y2, m7)), p2(a.sc[7]));
    const float2 a9 = pmul(pfma(jx, jy, m8n), p2(a.sc[8]));
    // mrt_inverse with the populations added back
    if (CONS0) {
        const float2 ax = psub(pmul(a3, p2(-2.0f)), a2);
        const float2 A = padd(ax, a8), B = psub(ax, a8);
        o[0] = pfma(psub(a3, a2), p2(4.0f), g[0]);
        o[1] = pfma(a5, p2(-2.0f), padd(g[1], A));
        o[3] = pfma(a5, p2(2.0f), padd(g[3], A));
        o[2] = pfma(a7, p2(-2.0f), padd(g[2], B));
        o[4] = pfma(a7, p2(2.0f), padd(g[4], B));
        const float2 ad = pfma(a2, p2(2.0f), a3);
        const float2 P = padd(a5, a7), Q = psub(a7, a5);
        const float2 E = padd(ad, a9), F = psub(ad, a9);
        o[5] = padd(g[5], padd(E, P));
        o[6] = padd(g[6], padd(F, Q));
        o[7] = padd(g[7], psub(E, P));
        o[8] = padd(g[8], psub(F, Q));
    } else {
        const float2 a1 = pmul(padd(drho, p2(1.0f)), p2(a.sc[0]));
        const float2 a4 = pmul(jx, p2(a.sc[3])), a6 = pmul(jy, p2(a.sc[5]));
        const float2 ax = pfma(a3, p2(-2.0f), psub(a1, a2));
        const float2 A = padd(ax, a8), B = psub(ax, a8);
        const float2 q = pfma(a5, p2(-2.0f), a4), r = pfma(a7, p2(-2.0f), a6);
        o[0] = padd(g[0], pfma(psub(a3, a2), p2(4.0f), a1));
        o[1] = padd(padd(g[1], A), q);
        o[3] = psub(padd(g[3], A), q);
        o[2] = padd(padd(g[2], B), r);
        o[4] = psub(padd(g[4], B), r);
        const float2 ad = pfma(a2, p2(2.0f), padd(a1, a3));
        const float2 P = padd(padd(a4, a5), padd(a6, a7)), Q = psub(padd(a6, a7), padd(a4, a5));
        const float2 E = padd(ad, a9), F = psub(ad, a9);
        o[5] = padd(g[5], padd(E, P));
        o[6] = padd(g[6], padd(F, Q));
        o[7] = padd(g[7], psub(E, P));
        o[8] = padd(g[8], psub(F, Q));
    }
    if (FIELDS) {
        frho = padd(drho, p2(1.0f));
        fu = make_float2(jx.x / frho.x, jx.y / frho.y);
        fv = make_float2(jy.x / frho.x, jy.y / frho.y);
    }
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
__device__ __forceinline__ void node_update(const KFArgs<C> &a, const T *__restrict__ fin, int i, int j, C gout[9],
                                            C &frho, C &fu, C &fv)
{
    if (i == 0 || i == a.nx - 1 || j == 0 || j == a.ny - 1) {
        edge_update<T, C>(a, fin, i, j, gout, frho, fu, fv);
    } else {
        C g[9];
        pull<T, C>(fin, a.plane, a.pitch, i, j, g);
        collide_interior<C>(a, g, false, C(0), C(0), gout, frho, fu, fv);
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


}  // namespace lbm_node
