/*
 * Tangent volume kernel of the transient physics (phys/getime), FP64 or FP32.
 *
 * With u(s) = m + s h (m = (u0 + u1)/2, h = (u - u0)/2, see igab_math.cuh),
 * the tangent of the truncated average gradient is
 *   D = 1/2 (H_0/2 + H_1/3 + H_2/4),   H(s) = d2W/du2(m + s h) = sum_j H_j s^j,
 * and its derivatives with respect to the history levels (the discrete adjoint
 * of the time stepping) are, through m and h,
 *   d r/d u1 = 1/2 (H_0 + H_1/2 + H_2/3 + H_3/4),
 *   d r/d u0 = 1/2 (H_0/2 + H_1/6 + H_2/12 + H_3/4),
 * all of the form sum_j w_j H_j (w = igab_geom::tw) plus a value-component mass
 * term (inertia / damping coefficients of u, u1, u0; igab_geom::tmass).
 * Writing H(s) = G(s)^T Phi''(s) G(s) + geo(s) with G(s) = G0 + s G1 exactly linear
 * in s, D becomes a rank-24 form plus an effective geometric block:
 *   D = sum_{a,c in {0,1}} G_a^T M_ac G_c + geo_eff,
 *   M_ac = sum_b w_{a+b+c} Phi''_b,
 *   geo_eff = geo built from sum_j w_j (Phi'_v)_j.
 * M_ac is 2x2 per energy variable (4x4 for the coupled (va, vb) pair). The
 * inertia/damping term (rho/dt^2 + c/(2 dt)) N_a N_b joins the geometric block,
 * which is the same for the three displacement components.
 *
 * Per element (src/snesiga_Tangent.c:104-190 with the getime integrand):
 * 256 threads, 8-colour tiles of 2x2x2 elements as the static kernels; each
 * thread owns 13 upper-triangle entries of the 81x81 element matrix and two
 * entries of the 27x27 geometric block, accumulated over batches of 2 Gauss
 * points (X = G N rows and Y = w M X rows in shared memory).
 */
#include <cuda_runtime.h>
#include "igab_device.cuh"

namespace {

#include "igab_warp_tiles8.inc"

#define GQ 2          /* Gauss points per batch */
#define GNV 24        /* rows per Gauss point: 12 variables x (G0, G1) */

/* point data */
#define GP_F0 0
#define GP_G0 9
#define GP_F1 27
#define GP_G1 36
#define GP_MD 54      /* 12 x (m00, m01, m11) for the diagonal variables (1, 2 unused) */
#define GP_M12 90     /* 4 x 4 coupling of (va, vb) x (G0, G1) */
#define GP_SIG 106
#define GP_D1S 109
#define GP_TAU 112
#define GP_W 121
#define GP_MASS 122
#define GP_N 123

#define GXS 100        /* X / Y row stride (doubles): = 4 mod 16, columns 81..99 stay zero */
#define GROWS (GQ * GNV)
#define GGR 16         /* geometric rows per batch: 7 per point (6 + mass), padded */
#define GGS 36         /* U / V row stride: = 4 mod 16, columns 27..35 stay zero */

template <int TE>
struct gt_smem {
    static constexpr int TC = TE + 2;
    static constexpr int NCP = TC * TC * TC;
    double U[3][NCP * 3];
    double tab[3][TE][IGAB_TAB1D];
    double wh[3][TE][IGAB_NQ];
    double xq[3][TE][IGAB_NQ];
    double A[972];
    double C[864];
    double pt[IGAB_NQ3][GP_N];
    double X[GROWS][GXS];          /* X rows (row 24 qb + 2 v + order, column 3 a + k) */
    double Y[GROWS][GXS];          /* Y = w M X */
    double UT[GGR][GGS];           /* U rows of the geometric block (row 7 qb + i, column a) */
    double VT[GGR][GGS];           /* V rows */
    double gam[32 * 32];           /* upper tiles of Gamma */
    long rbase[81];
    int rsx[81], rsy[81];
};

__device__ __forceinline__ void gt_dmma(double &c0, double &c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

/* one batch of K += X^T Y on the warp's upper 8x8 tiles (A fragments from X, B from Y)
 * and Gamma += U^T V on its Gamma tiles */
template <int W>
__device__ __forceinline__ void gt_warp_mma(const double (*X)[GXS], const double (*Y)[GXS],
                                            const double (*UT)[GGS], const double (*VT)[GGS], int lane,
                                            double (&acc)[9][2], double (&gacc)[10][2])
{
    using WT = warp_tiles8<W>;
    const int r4 = lane & 3, c8 = lane >> 2;
#pragma unroll 2
    for (int kb = 0; kb < GROWS / 4; kb++) {
        const int kr = 4 * kb + r4;
        double f[WT::NB], g[WT::NB];
#pragma unroll
        for (int b = 0; b < WT::NB; b++) {
            f[b] = X[kr][8 * WT::blk(b) + c8];
            g[b] = Y[kr][8 * WT::blk(b) + c8];
        }
#pragma unroll
        for (int t = 0; t < WT::NT; t++) gt_dmma(acc[t][0], acc[t][1], f[WT::ti(t)], g[WT::tj(t)]);
    }
    if constexpr (WT::NGT > 0) {
#pragma unroll
        for (int kb = 0; kb < GGR / 4; kb++) {
            const int kr = 4 * kb + r4;
            double fa[WT::NGA], fb[WT::NGB];
#pragma unroll
            for (int b = 0; b < WT::NGA; b++) fa[b] = UT[kr][8 * WT::gablk(b) + c8];
#pragma unroll
            for (int b = 0; b < WT::NGB; b++) fb[b] = VT[kr][8 * WT::gbblk(b) + c8];
#pragma unroll
            for (int t = 0; t < WT::NGT; t++) gt_dmma(gacc[t][0], gacc[t][1], fa[WT::gti(t)], fb[WT::gtj(t)]);
        }
    }
}

/* the warp's Gamma tiles into gam (upper tiles, stride 32) */
template <int W>
__device__ __forceinline__ void gt_warp_gamma(double *gam, int lane, const double (&gacc)[10][2])
{
    using WT = warp_tiles8<W>;
    const int r = lane >> 2, c = 2 * (lane & 3);
#pragma unroll
    for (int t = 0; t < WT::NGT; t++) {
        const int a1 = 8 * WT::gablk(WT::gti(t)) + r, a2 = 8 * WT::gbblk(WT::gtj(t)) + c;
        gam[a1 * 32 + a2] = gacc[t][0];
        gam[a1 * 32 + a2 + 1] = gacc[t][1];
    }
}

/* the warp's tiles plus Gamma on the diagonal component blocks, added into the CSR
 * values; entry (c1, c2) and its mirror (c2, c1) receive the upper value */
template <int W, typename T>
__device__ __forceinline__ void gt_warp_scatter(T *__restrict__ vals, const long *rbase, const int *rsx,
                                                const int *rsy, const double *gam, int lane,
                                                const double (&acc)[9][2])
{
    using WT = warp_tiles8<W>;
    const int r = lane >> 2, c = 2 * (lane & 3);
#pragma unroll
    for (int t = 0; t < WT::NT; t++) {
        const int bi = WT::blk(WT::ti(t)), bj = WT::blk(WT::tj(t));
        double v2[2] = {acc[t][0], acc[t][1]};
        if (bi == bj) {
            /* diagonal tile: entry (r, c + e) below the diagonal takes (c + e, r),
             * held by lane 4 (c + e) + r / 2, element r & 1 */
            const double x0 = __shfl_sync(0xffffffffu, acc[t][0], 4 * c + (r >> 1));
            const double y0 = __shfl_sync(0xffffffffu, acc[t][1], 4 * c + (r >> 1));
            const double x1 = __shfl_sync(0xffffffffu, acc[t][0], 4 * (c + 1) + (r >> 1));
            const double y1 = __shfl_sync(0xffffffffu, acc[t][1], 4 * (c + 1) + (r >> 1));
            if (r > c) v2[0] = (r & 1) ? y0 : x0;
            if (r > c + 1) v2[1] = (r & 1) ? y1 : x1;
        }
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int c1 = 8 * bi + r, c2 = 8 * bj + c + e;
            if (c1 < 81 && c2 < 81) {
                const int a1 = c1 / 3, a2 = c2 / 3;
                double v = v2[e];
                if (c1 % 3 == c2 % 3) v += a1 <= a2 ? gam[a1 * 32 + a2] : gam[a2 * 32 + a1];
                atomicAdd(vals + rbase[c1] + (c2 / 27) * rsx[c1] + ((c2 / 9) % 3) * rsy[c1] + c2 % 9, T(v));
                if (bi != bj)
                    atomicAdd(vals + rbase[c2] + (c1 / 27) * rsx[c2] + ((c1 / 9) % 3) * rsy[c2] + c1 % 9, T(v));
            }
        }
    }
}

#define GT_WARP_SWITCH(CALL)  \
    switch (warp) {           \
    case 0: CALL(0); break;   \
    case 1: CALL(1); break;   \
    case 2: CALL(2); break;   \
    case 3: CALL(3); break;   \
    case 4: CALL(4); break;   \
    case 5: CALL(5); break;   \
    case 6: CALL(6); break;   \
    default: CALL(7); break;  \
    }

/* X and Y rows of one (point, basis function, component): the 12 variables' gradients
 * (phys/ge variables, unrotated) for both Taylor orders a = 0, 1 (F_a, G_a of the
 * point), contracted with the 9 derivatives of the basis function, then
 * Y_{(v,a)} = w sum_c M[(v,a),(v',c)] X_{(v',c)} (2 x 2 per variable, 4 x 4 for (va, vb)) */
template <int HALF>
__device__ __forceinline__ void gt_xy_task(const double *p, const double *bxp, const double *byp,
                                           const double *bzp, int k, double *xc, double *yc)
{
    const double is2 = IGAB_INV_SQRT2, is3 = IGAB_INV_SQRT3, is6 = IGAB_INV_SQRT6;
    const double bx0 = bxp[0], bx1 = bxp[1], bx2 = bxp[2];
    const double by0 = byp[0], by1 = byp[1], by2 = byp[2];
    const double bz0 = bzp[0], bz1 = bzp[1], bz2 = bzp[2];
    const double b00 = bx0 * by0, b10 = bx1 * by0, b01 = bx0 * by1;
    const double dx = b10 * bz0, dy = b01 * bz0, dz = b00 * bz1;
    const double hxx = bx2 * by0 * bz0, hxy = bx1 * by1 * bz0, hxz = b10 * bz1;
    const double hyy = bx0 * by2 * bz0, hyz = b01 * bz1, hzz = b00 * bz2;
    /* x[2 (v - 6 HALF) + a]: the variables of this half (0..5, or 6..11) */
    double x[12];
#pragma unroll
    for (int a = 0; a < 2; a++) {
        const double *F = p + (a ? GP_F1 : GP_F0) + 3 * k;
        const double F0 = F[0], F1 = F[1], F2 = F[2];
        if (HALF == 0) {
            const double e0 = F0 * dx, e1 = F1 * dy, e2 = F2 * dz;
            x[0 + a] = (e0 + e1 + e2) * is3;
            x[2 + a] = (e0 - e1) * is2;
            x[4 + a] = (e0 + e1 - 2.0 * e2) * is6;
            x[6 + a] = 0.5 * (F1 * dx + F0 * dy);
            x[8 + a] = 0.5 * (F2 * dx + F0 * dz);
            x[10 + a] = 0.5 * (F2 * dy + F1 * dz);
        } else {
            const double *G = p + (a ? GP_G1 : GP_G0) + 6 * k;
            const double G0 = G[0], G1 = G[1], G2 = G[2], G3 = G[3], G4 = G[4], G5 = G[5];
            x[0 + a] = (G0 * dx - G1 * dy + F0 * hxx - F1 * hxy) * is2;
            x[2 + a] = (G1 * dx - G3 * dy + F0 * hxy - F1 * hyy) * is2;
            x[4 + a] = (G2 * dx - G4 * dy + F0 * hxz - F1 * hyz) * is2;
            x[6 + a] = (G0 * dx + G1 * dy - 2.0 * G2 * dz + F0 * hxx + F1 * hxy - 2.0 * F2 * hxz) * is6;
            x[8 + a] = (G1 * dx + G3 * dy - 2.0 * G4 * dz + F0 * hxy + F1 * hyy - 2.0 * F2 * hyz) * is6;
            x[10 + a] = (G2 * dx + G4 * dy - 2.0 * G5 * dz + F0 * hxz + F1 * hyz - 2.0 * F2 * hzz) * is6;
        }
    }
    const double w = p[GP_W];
    const int r0 = 12 * HALF;   /* first row of this half */
#pragma unroll
    for (int r = 0; r < 12; r++) xc[(r0 + r) * GXS] = x[r];
#pragma unroll
    for (int j = 0; j < 6; j++) {
        const int v = 6 * HALF + j;
        if (v == 1 || v == 2) continue;
        const double m00 = p[GP_MD + 3 * v], m01 = p[GP_MD + 3 * v + 1], m11 = p[GP_MD + 3 * v + 2];
        yc[(r0 + 2 * j) * GXS] = w * (m00 * x[2 * j] + m01 * x[2 * j + 1]);
        yc[(r0 + 2 * j + 1) * GXS] = w * (m01 * x[2 * j] + m11 * x[2 * j + 1]);
    }
    if (HALF == 0) {
        const double *M = p + GP_M12;
#pragma unroll
        for (int rr = 0; rr < 4; rr++)
            yc[(2 + rr) * GXS] =
                w * (M[4 * rr] * x[2] + M[4 * rr + 1] * x[3] + M[4 * rr + 2] * x[4] + M[4 * rr + 3] * x[5]);
    }
}

/* U / V rows of the geometric block for (point, basis function): U_i = d_i N_a,
 * V_i = w ((S grad N_a)_i + (T H_a)_i), U_{3+I} = w (T H_a)_I, V_{3+I} = d_I N_a
 * (effective S = sig / d1s, T = tau of the point) and the inertia / damping row
 * U_6 = N_a, V_6 = w mass N_a */
__device__ __forceinline__ void gt_uv_task(const double *p, const double *bxp, const double *byp,
                                           const double *bzp, double *ur, double *vr)
{
    const double bx0 = bxp[0], bx1 = bxp[1], bx2 = bxp[2];
    const double by0 = byp[0], by1 = byp[1], by2 = byp[2];
    const double bz0 = bzp[0], bz1 = bzp[1], bz2 = bzp[2];
    const double b00 = bx0 * by0, b10 = bx1 * by0, b01 = bx0 * by1;
    const double dx = b10 * bz0, dy = b01 * bz0, dz = b00 * bz1;
    const double hxx = bx2 * by0 * bz0, hxy = bx1 * by1 * bz0, hxz = b10 * bz1;
    const double hyy = bx0 * by2 * bz0, hyz = b01 * bz1, hzz = b00 * bz2;
    const double w = p[GP_W];
    const double s00 = p[GP_SIG], s11 = p[GP_SIG + 1], s22 = p[GP_SIG + 2];
    const double s01 = 0.5 * p[GP_D1S], s02 = 0.5 * p[GP_D1S + 1], s12 = 0.5 * p[GP_D1S + 2];
    const double *T = p + GP_TAU;
    const double th0 = T[0] * hxx + T[1] * hxy + T[2] * hxz;
    const double th1 = T[3] * hxy + T[4] * hyy + T[5] * hyz;
    const double th2 = T[6] * hxz + T[7] * hyz + T[8] * hzz;
    ur[0 * GGS] = dx;
    ur[1 * GGS] = dy;
    ur[2 * GGS] = dz;
    vr[0 * GGS] = w * (s00 * dx + s01 * dy + s02 * dz + th0);
    vr[1 * GGS] = w * (s01 * dx + s11 * dy + s12 * dz + th1);
    vr[2 * GGS] = w * (s02 * dx + s12 * dy + s22 * dz + th2);
    ur[3 * GGS] = w * th0;
    ur[4 * GGS] = w * th1;
    ur[5 * GGS] = w * th2;
    vr[3 * GGS] = dx;
    vr[4 * GGS] = dy;
    vr[5 * GGS] = dz;
    const double n0 = b00 * bz0;
    ur[6 * GGS] = n0;
    vr[6 * GGS] = w * p[GP_MASS] * n0;
}

template <typename T, int TE>
__global__ void __launch_bounds__(256) k_tan_getime(igab_geom g, const double *__restrict__ U,
                                                    T *__restrict__ vals, int colour)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    gt_smem<TE> &S = *reinterpret_cast<gt_smem<TE> *>(smem_raw);
    constexpr int TC = TE + 2;
    constexpr int NCP = TC * TC * TC;
    constexpr int NEL = TE * TE * TE;
    tile_t Tl;
    if (!decode_tile(g, TE, colour, blockIdx.x, Tl)) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    for (int idx = tid; idx < NCP * 3; idx += 256) {
        int i = idx % 3, cp = idx / 3;
        int lz = cp % TC, ly = (cp / TC) % TC, lx = cp / (TC * TC);
        const bool in = lx < Tl.nv[0] + 2 && ly < Tl.nv[1] + 2 && lz < Tl.nv[2] + 2;
        const long gi = in ? 3 * cp_index(g, Tl.e0[0] + lx, Tl.e0[1] + ly, Tl.e0[2] + lz) + i : 0;
        S.U[0][idx] = in ? U[gi] : 0.0;
        S.U[1][idx] = in ? g.hist1[gi] : 0.0;
        S.U[2][idx] = in ? g.hist0[gi] : 0.0;
    }
    for (int idx = tid; idx < 3 * TE * IGAB_TAB1D; idx += 256) {
        int d = idx / (TE * IGAB_TAB1D), r = idx % (TE * IGAB_TAB1D), le = r / IGAB_TAB1D, o = r % IGAB_TAB1D;
        S.tab[d][le][o] = le < Tl.nv[d] ? g.tab[d][(long)(Tl.e0[d] + le) * IGAB_TAB1D + o] : 0.0;
    }
    for (int idx = tid; idx < 3 * TE * IGAB_NQ; idx += 256) {
        int d = idx / (TE * IGAB_NQ), r = idx % (TE * IGAB_NQ), le = r / IGAB_NQ, q = r % IGAB_NQ;
        bool ok = le < Tl.nv[d];
        S.wh[d][le][q] = ok ? g.wh[d][(long)(Tl.e0[d] + le) * IGAB_NQ + q] : 0.0;
        S.xq[d][le][q] = ok ? g.xq[d][(long)(Tl.e0[d] + le) * IGAB_NQ + q] : 0.0;
    }
    /* the padding columns (81..99) of X and Y, and the padding rows and columns of U / V, stay zero */
    for (int idx = tid; idx < GROWS * (GXS - 81); idx += 256) {
        const int r = idx / (GXS - 81), cc = 81 + idx % (GXS - 81);
        S.X[r][cc] = 0.0;
        S.Y[r][cc] = 0.0;
    }
    for (int idx = tid; idx < GGR * GGS; idx += 256) {
        (&S.UT[0][0])[idx] = 0.0;
        (&S.VT[0][0])[idx] = 0.0;
    }
    __syncthreads();

    for (int le = 0; le < NEL; le++) {
        const int lex = le / (TE * TE), ley = (le / TE) % TE, lez = le % TE;
        if (!(lex < Tl.nv[0] && ley < Tl.nv[1] && lez < Tl.nv[2])) continue;   /* block-uniform */
        const double *Bx = S.tab[0][lex];
        const double *By = S.tab[1][ley];
        const double *Bz = S.tab[2][lez];
        /* ---- fields of the three history levels at the 64 Gauss points */
        double ul[3][30];
#pragma unroll
        for (int l = 0; l < 3; l++) {
            for (int o = tid; o < 972; o += 256) {
                int i = o % 3, kz = (o / 3) % 3, ay = (o / 9) % 3, ax = (o / 27) % 3, q = o / 81;
                const double *u0 = &S.U[l][(((lex + ax) * TC + (ley + ay)) * TC + lez) * 3 + i];
                S.A[o] = Bz[q * 9 + kz] * u0[0] + Bz[q * 9 + 3 + kz] * u0[3] + Bz[q * 9 + 6 + kz] * u0[6];
            }
            __syncthreads();
            for (int o = tid; o < 864; o += 256) {
                int i = o % 3, kk = (o / 3) % 6, ax = (o / 18) % 3, qq = o / 54;
                int qyy = qq & 3, qzz = qq >> 2;
                const double *a0 = &S.A[((qzz * 3 + ax) * 3) * 9 + kk_kz(kk) * 3 + i];
                S.C[o] = By[qyy * 9 + kk_ky(kk)] * a0[0] + By[qyy * 9 + 3 + kk_ky(kk)] * a0[9] +
                         By[qyy * 9 + 6 + kk_ky(kk)] * a0[18];
            }
            __syncthreads();
            if (tid < IGAB_NQ3) {
                const int qx = tid & 3, qy = (tid >> 2) & 3, qz = tid >> 4, qq = qy + 4 * qz;
#pragma unroll
                for (int a = 0; a < 10; a++)
#pragma unroll
                    for (int i = 0; i < 3; i++) {
                        double s = 0.0;
#pragma unroll
                        for (int ax = 0; ax < 3; ax++)
                            s += Bx[qx * 9 + ax * 3 + a_kx(a)] * S.C[((qq * 3 + ax) * 6 + a_kk(a)) * 3 + i];
                        ul[l][10 * i + a] = s;
                    }
                if (g.periodic)
#pragma unroll
                    for (int i = 0; i < 3; i++)
#pragma unroll
                        for (int J = 0; J < 3; J++) ul[l][10 * i + 1 + J] += g.pp[3 * i + J];
            }
            __syncthreads();
        }
        /* ---- point data along u(s) = m + s h */
        if (tid < IGAB_NQ3) {
            const int qx = tid & 3, qy = (tid >> 2) & 3, qz = tid >> 4;
            igab_tay<4> ut[30];
#pragma unroll
            for (int i = 0; i < 30; i++) {
                ut[i].c[0] = 0.5 * (ul[2][i] + ul[1][i]);
                ut[i].c[1] = 0.5 * (ul[0][i] - ul[2][i]);
                ut[i].c[2] = 0.0;
                ut[i].c[3] = 0.0;
            }
            igab_ge_point<igab_tay<4>> P;
            igab_ge_eval(ut, g.coef, P);
            double *pt = S.pt[tid];
            for (int k = 0; k < 3; k++)
                for (int J = 0; J < 3; J++) {
                    pt[GP_F0 + 3 * k + J] = P.F[k][J].c[0];
                    pt[GP_F1 + 3 * k + J] = P.F[k][J].c[1];
                }
            for (int k = 0; k < 3; k++)
                for (int c = 0; c < 6; c++) {
                    pt[GP_G0 + 6 * k + c] = P.G[k][c].c[0];
                    pt[GP_G1 + 6 * k + c] = P.G[k][c].c[1];
                }
            const double *cw = g.tw;
            for (int v = 0; v < 12; v++) {
                const double *f = P.d2[v].c;
                pt[GP_MD + 3 * v + 0] = cw[0] * f[0] + cw[1] * f[1] + cw[2] * f[2] + cw[3] * f[3];
                pt[GP_MD + 3 * v + 1] = cw[1] * f[0] + cw[2] * f[1] + cw[3] * f[2];
                pt[GP_MD + 3 * v + 2] = cw[2] * f[0] + cw[3] * f[1];
            }
            /* (va, vb) x (G0, G1): row r = 2 i + a, i = 0 (va), 1 (vb) */
            for (int r = 0; r < 4; r++)
                for (int c2 = 0; c2 < 4; c2++) {
                    const int i1 = r >> 1, a = r & 1, i2 = c2 >> 1, c = c2 & 1;
                    const double *f = (i1 == i2) ? P.d2[1 + i1].c : P.d2ab.c;
                    double t = 0.0;
                    for (int b = 0; b < 4; b++)
                        if (a + b + c < 4) t += cw[a + b + c] * f[b];
                    pt[GP_M12 + 4 * r + c2] = t;
                }
            for (int I = 0; I < 3; I++) {
                pt[GP_SIG + I] = cw[0] * P.sig[I].c[0] + cw[1] * P.sig[I].c[1] + cw[2] * P.sig[I].c[2] +
                                 cw[3] * P.sig[I].c[3];
                pt[GP_D1S + I] = cw[0] * P.d1[3 + I].c[0] + cw[1] * P.d1[3 + I].c[1] + cw[2] * P.d1[3 + I].c[2] +
                                 cw[3] * P.d1[3 + I].c[3];
                for (int K = 0; K < 3; K++)
                    pt[GP_TAU + 3 * I + K] = cw[0] * P.tau[I][K].c[0] + cw[1] * P.tau[I][K].c[1] +
                                             cw[2] * P.tau[I][K].c[2] + cw[3] * P.tau[I][K].c[3];
            }
            pt[GP_W] = S.wh[0][lex][qx] * S.wh[1][ley][qy] * S.wh[2][lez][qz] *
                       elem_scale(g, Tl.e0[0] + lex, Tl.e0[1] + ley, Tl.e0[2] + lez);
            pt[GP_MASS] = g.tmass;
        }
        __syncthreads();

        double acc[9][2], gacc[10][2];
#pragma unroll
        for (int t = 0; t < 9; t++) acc[t][0] = acc[t][1] = 0.0;
#pragma unroll
        for (int t = 0; t < 10; t++) gacc[t][0] = gacc[t][1] = 0.0;

        for (int q0 = 0; q0 < IGAB_NQ3; q0 += GQ) {
            /* (a) X and Y rows: tasks (point, half of the variables, basis function, component);
             * U / V rows: tasks (point, basis function) */
            for (int t = tid; t < GQ * 162 + GQ * 27; t += 256) {
                if (t < GQ * 162) {
                    const int qb = t / 162, half = (t / 81) & 1, c = t % 81, a = c / 3, k = c % 3;
                    const int q = q0 + qb, qx = q & 3, qy = (q >> 2) & 3, qz = q >> 4;
                    const double *bxp = Bx + qx * 9 + (a / 9) * 3, *byp = By + qy * 9 + ((a / 3) % 3) * 3,
                                 *bzp = Bz + qz * 9 + (a % 3) * 3;
                    if (half == 0)
                        gt_xy_task<0>(S.pt[q], bxp, byp, bzp, k, &S.X[qb * GNV][c], &S.Y[qb * GNV][c]);
                    else
                        gt_xy_task<1>(S.pt[q], bxp, byp, bzp, k, &S.X[qb * GNV][c], &S.Y[qb * GNV][c]);
                } else {
                    const int tg = t - GQ * 162, qb = tg / 27, a = tg % 27;
                    const int q = q0 + qb, qx = q & 3, qy = (q >> 2) & 3, qz = q >> 4;
                    gt_uv_task(S.pt[q], Bx + qx * 9 + (a / 9) * 3, By + qy * 9 + ((a / 3) % 3) * 3,
                               Bz + qz * 9 + (a % 3) * 3, &S.UT[7 * qb][a], &S.VT[7 * qb][a]);
                }
            }
            __syncthreads();
            /* (b) K += X^T Y and Gamma += U^T V on the DMMA tiles */
#define GT_MMA(Wn) gt_warp_mma<Wn>(S.X, S.Y, S.UT, S.VT, lane, acc, gacc)
            GT_WARP_SWITCH(GT_MMA)
#undef GT_MMA
            __syncthreads();
        }
#define GT_GAM(Wn) gt_warp_gamma<Wn>(S.gam, lane, gacc)
        GT_WARP_SWITCH(GT_GAM)
#undef GT_GAM
        if (tid < 81)
            elem_row_base(g, Tl.e0[0] + lex, Tl.e0[1] + ley, Tl.e0[2] + lez, tid, S.rbase[tid], S.rsx[tid],
                          S.rsy[tid]);
        __syncthreads();
#define GT_SCATTER(Wn) gt_warp_scatter<Wn, T>(vals, S.rbase, S.rsx, S.rsy, S.gam, lane, acc)
        GT_WARP_SWITCH(GT_SCATTER)
#undef GT_SCATTER
        __syncthreads();
    }
}

template <typename T>
int launch_t(igab_ctx *c, const double *dU, T *dv, int level)
{
    igab_geom g = c->geom();
    if (level == 1) {          /* d r / d u1 */
        const double w[4] = {0.5, 0.25, 1.0 / 6.0, 0.125};
        for (int j = 0; j < 4; j++) g.tw[j] = w[j];
        g.tmass = -2.0 * g.rho / (g.dt * g.dt);
    } else if (level == 2) {   /* d r / d u0 */
        const double w[4] = {0.25, 1.0 / 12.0, 1.0 / 24.0, 0.125};
        for (int j = 0; j < 4; j++) g.tw[j] = w[j];
        g.tmass = g.rho / (g.dt * g.dt) - g.cii / (2.0 * g.dt);
    }
    size_t sm = sizeof(gt_smem<2>);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_getime<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    for (int k = 0; k < 8; k++) {
        const int colour = igab_colour_at(c->colour_order, k);
        long nblk = tiles_of_colour(g, 2, colour);
        if (nblk == 0) continue;
        k_tan_getime<T, 2><<<(unsigned)nblk, 256, sm, c->stream>>>(g, dU, dv, colour);
        c->last_launches++;
    }
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

} /* namespace */

int igab_launch_tan_getime(igab_ctx *c, const double *dU, void *dv, int prec)
{
    return igab_launch_tan_getime_level(c, dU, dv, prec, 0);
}

int igab_launch_tan_getime_level(igab_ctx *c, const double *dU, void *dv, int prec, int level)
{
    return prec == IGAB_PREC_FP64 ? launch_t<double>(c, dU, (double *)dv, level)
                                  : launch_t<float>(c, dU, (float *)dv, level);
}
