/*
 * FP64 tangent volume kernel on the FP64 tensor path (mma.sync m8n8k4 f64).
 *
 * Per element (src/snesiga_Tangent.c:104-190), with the energy written as
 * W = Phi(v(u)) over 12 variables (igab_math.cuh):
 *   K_e = sum_q w_q X_q^T Phi''_q X_q  +  blockdiag_k(Gamma),
 *   X_q[v][3a+k] = sum_m dv/du_{k,m}(q) N_a^{m}(q),
 *   Gamma(a,b)   = sum_q sum_{m,n} N_a^m(q) (w_q geo_q[m][n]) N_b^n(q).
 * Phi'' is diagonal except for the (va, vb) pair; rotating those two rows by
 * the eigenvectors of that 2x2 block makes it diagonal, so
 *   K_e = X'^T diag(s) X',   s = w_q * eigenvalues.
 * Both products run on DMMA tiles:
 *   - X' (48 rows = 4 Gauss points x 12 variables, 88 padded columns) is built
 *     in shared memory straight from the 1-D basis tables (sum factorisation of
 *     sum_m dv'/du_{k,m} N_a^m over x, y, z; one task per (point, variable,
 *     component, x-function), the variable warp-uniform); a warp loads its A
 *     fragments from it and forms its B fragments by scaling the same
 *     registers with s.  The 66 upper 8x8 tiles of the 88x88 element matrix are
 *     spread over the 4 warps (table in igab_warp_tiles.inc), the lower
 *     triangle follows by symmetry.
 *   - Gamma (27 x 27, identical for the three components) in the rank-6 form
 *     Gamma = sum_q sum_i U_qi V_qi^T with geo = [[S, T], [T^T, 0]]:
 *       U_i = d_i N_a, V_i = w ((S grad N_a)_i + (T H_a)_i)     (i < 3)
 *       U_i = w (T H_a)_I, V_i = d_I N_a                         (i = 3 + I)
 *     on 10 upper 8x8 tiles of the 32-padded block, 6 k-rows per point.
 * 128 threads and ~90 KB of shared memory per block let two blocks share an
 * SM, so one block's scalar work (field, point integrand, X') overlaps the
 * other's tensor work.  Scatter: fire-and-forget reductions into the CSR
 * values, conflict-free within one of the 8 tile colours (igab_kernels.cu).
 */
#include <cuda_runtime.h>
#include "igab_device.cuh"

namespace {

#include "igab_warp_tiles.inc"

#define NTHR 128
#define DQ 4            /* Gauss points per batch */
#define DROWS (DQ * 12) /* k rows of X' per batch */
#define GROWS (DQ * 6)  /* k rows of the geometric product per batch: U / V rows, 6 per point */
#define XS 100          /* X' row stride (doubles): = 4 mod 16 keeps fragment loads conflict-free */
#define GS 36           /* U / V row stride: = 4 mod 16; columns a >= 27 stay zero */

/* point data */
#define PT_F 0
#define PT_G 9
#define PT_LAM 27   /* 12 diagonal values of the rotated Phi'' */
#define PT_CS 39
#define PT_SN 40
#define PT_SIG 41
#define PT_D1S 44
#define PT_TAU 47
#define PT_W 56
#define PT_N 57

/* work buffer: interpolation A[972] C[864] | X'[48][100] + points[64][57] | K[88][88] + Gamma[32][32] */
#define W_A 0
#define W_C 972
#define W_X 0
#define W_PT (DROWS * XS)
#define W_SIZE (DROWS * XS + IGAB_NQ3 * PT_N)
#define W_GAM (88 * 88)
#define W_ALL (W_SIZE > W_GAM + 32 * 32 ? W_SIZE : W_GAM + 32 * 32)

template <int TE>
struct dmma_smem {
    static constexpr int TC = TE + 2;
    static constexpr int NCP = TC * TC * TC;
    double W[W_ALL];
    double UT[GROWS][GS];     /* U rows of the geometric product: row 6 qb + i, column a */
    double VT[GROWS][GS];     /* V rows */
    double sc[DROWS];
    double U[NCP * 3];
    double tab[3][TE][IGAB_TAB1D];
    double wh[3][TE][IGAB_NQ];
    long rbase[81];       /* CSR row bases of the element matrix (elem_row_base) */
    int rsx[81], rsy[81];
};

__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

/* eigen-rotation of [[a, b], [b, c]] (Jacobi / symmetric Schur 2x2): (cs, sn, l1, l2)
 * with [[a,b],[b,c]] = l1 e1 e1^T + l2 e2 e2^T, e1 = (cs, -sn), e2 = (sn, cs) */
__device__ __forceinline__ void sym2_eig(double a, double b, double c, double &cs, double &sn, double &l1, double &l2)
{
    if (b == 0.0) {
        cs = 1.0; sn = 0.0; l1 = a; l2 = c;
        return;
    }
    double zeta = (c - a) / (2.0 * b);
    double t = (zeta >= 0.0 ? 1.0 : -1.0) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
    cs = 1.0 / sqrt(1.0 + t * t);
    sn = t * cs;
    l1 = a - t * b;
    l2 = c + t * b;
}

template <int W>
__device__ __forceinline__ void warp_mma(const double *__restrict__ X, const double *__restrict__ sc,
                                         const double *__restrict__ UT, const double *__restrict__ VT, int lane,
                                         double (&acc)[17][2], double (&gacc)[3][2])
{
    using WT = warp_tiles<W>;
    const int r4 = lane & 3, c8 = lane >> 2;
#pragma unroll 2
    for (int kb = 0; kb < DROWS / 4; kb++) {
        const int kr = 4 * kb + r4;
        const double s = sc[kr];
        const double *row = X + kr * XS + c8;
        double f[WT::NB], g[WT::NB];
#pragma unroll
        for (int b = 0; b < WT::NB; b++) {
            f[b] = row[8 * WT::blk(b)];
            g[b] = f[b] * s;
        }
#pragma unroll
        for (int t = 0; t < WT::NT; t++) dmma(acc[t][0], acc[t][1], f[WT::ti(t)], g[WT::tj(t)]);
    }
#pragma unroll 3
    for (int kb = 0; kb < GROWS / 4; kb++) {
        const int kr = 4 * kb + r4;
        double fa[WT::NGA], fb[WT::NGB];
#pragma unroll
        for (int b = 0; b < WT::NGA; b++) fa[b] = UT[kr * GS + 8 * WT::gablk(b) + c8];
#pragma unroll
        for (int b = 0; b < WT::NGB; b++) fb[b] = VT[kr * GS + 8 * WT::gbblk(b) + c8];
#pragma unroll
        for (int t = 0; t < WT::NGT; t++) dmma(gacc[t][0], gacc[t][1], fa[WT::gti(t)], fb[WT::gtj(t)]);
    }
}

/* accumulator tiles -> shared K[c1][c2] (stride 88) and Gamma[a1][a2] (stride 32) */
template <int W>
__device__ __forceinline__ void warp_dump(double *__restrict__ K, double *__restrict__ Gam, int lane,
                                          const double (&acc)[17][2], const double (&gacc)[3][2])
{
    using WT = warp_tiles<W>;
    const int r = lane >> 2, c = 2 * (lane & 3);
#pragma unroll
    for (int t = 0; t < WT::NT; t++) {
        const int c1 = 8 * WT::blk(WT::ti(t)) + r, c2 = 8 * WT::blk(WT::tj(t)) + c;
        K[c1 * 88 + c2] = acc[t][0];
        K[c1 * 88 + c2 + 1] = acc[t][1];
    }
#pragma unroll
    for (int t = 0; t < WT::NGT; t++) {
        const int a1 = 8 * WT::gablk(WT::gti(t)) + r, a2 = 8 * WT::gbblk(WT::gtj(t)) + c;
        Gam[a1 * 32 + a2] = gacc[t][0];
        Gam[a1 * 32 + a2 + 1] = gacc[t][1];
    }
}

#define WARP_SWITCH(CALL)    \
    switch (warp) {          \
    case 0: CALL(0); break;  \
    case 1: CALL(1); break;  \
    case 2: CALL(2); break;  \
    default: CALL(3); break; \
    }

/* gradient of rotated variable v with respect to the 9 strain components of
 * displacement component k (igab_ge_grad_var, then the (va, vb) rotation) */
__device__ __forceinline__ void dm_grad_var(const double *p, int v, int k, double g[9])
{
#pragma unroll
    for (int m = 0; m < 9; m++) g[m] = 0.0;
    const double is2 = IGAB_INV_SQRT2, is3 = IGAB_INV_SQRT3, is6 = IGAB_INV_SQRT6;
    const double F0 = p[PT_F + 3 * k], F1 = p[PT_F + 3 * k + 1], F2 = p[PT_F + 3 * k + 2];
    const double *G = p + PT_G + 6 * k;
    if (v == 0) {
        g[0] = F0 * is3; g[1] = F1 * is3; g[2] = F2 * is3;
    } else if (v <= 2) {
        const double cs = p[PT_CS], sn = p[PT_SN];
        const double a0 = F0 * is2, a1 = -F1 * is2;                       /* va */
        const double b0 = F0 * is6, b1 = F1 * is6, b2 = -2.0 * F2 * is6;  /* vb */
        if (v == 1) { g[0] = cs * a0 - sn * b0; g[1] = cs * a1 - sn * b1; g[2] = -sn * b2; }
        else        { g[0] = sn * a0 + cs * b0; g[1] = sn * a1 + cs * b1; g[2] = cs * b2; }
    } else if (v == 3) {
        g[0] = 0.5 * F1; g[1] = 0.5 * F0;
    } else if (v == 4) {
        g[0] = 0.5 * F2; g[2] = 0.5 * F0;
    } else if (v == 5) {
        g[1] = 0.5 * F2; g[2] = 0.5 * F1;
    } else if (v == 6) {   /* strain-gradient variables (idx6: xx xy xz yy yz zz) */
        g[0] = G[0] * is2; g[1] = -G[1] * is2; g[3] = F0 * is2; g[4] = -F1 * is2;
    } else if (v == 7) {
        g[0] = G[1] * is2; g[1] = -G[3] * is2; g[4] = F0 * is2; g[6] = -F1 * is2;
    } else if (v == 8) {
        g[0] = G[2] * is2; g[1] = -G[4] * is2; g[5] = F0 * is2; g[7] = -F1 * is2;
    } else if (v == 9) {
        g[0] = G[0] * is6; g[1] = G[1] * is6; g[2] = -2.0 * G[2] * is6;
        g[3] = F0 * is6; g[4] = F1 * is6; g[5] = -2.0 * F2 * is6;
    } else if (v == 10) {
        g[0] = G[1] * is6; g[1] = G[3] * is6; g[2] = -2.0 * G[4] * is6;
        g[4] = F0 * is6; g[6] = F1 * is6; g[7] = -2.0 * F2 * is6;
    } else {
        g[0] = G[2] * is6; g[1] = G[4] * is6; g[2] = -2.0 * G[5] * is6;
        g[5] = F0 * is6; g[7] = F1 * is6; g[8] = -2.0 * F2 * is6;
    }
}

/* one tile: all NTHR threads of the block, uniformly */
template <int TE>
__device__ __forceinline__ void dmma_tile(const igab_geom &g, const tile_t &Tl, const double *__restrict__ U,
                                          double *__restrict__ vals, dmma_smem<TE> &S)
{
    constexpr int TC = TE + 2;
    constexpr int NCP = TC * TC * TC;
    constexpr int NEL = TE * TE * TE;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    double *const Xb = S.W + W_X;
    double *const PTb = S.W + W_PT;

    for (int idx = tid; idx < NCP * 3; idx += NTHR) {
        int i = idx % 3, cp = idx / 3;
        int lz = cp % TC, ly = (cp / TC) % TC, lx = cp / (TC * TC);
        double v = 0.0;
        if (lx < Tl.nv[0] + 2 && ly < Tl.nv[1] + 2 && lz < Tl.nv[2] + 2)
            v = U[3 * cp_index(g, Tl.e0[0] + lx, Tl.e0[1] + ly, Tl.e0[2] + lz) + i];
        S.U[idx] = v;
    }
    for (int idx = tid; idx < 3 * TE * IGAB_TAB1D; idx += NTHR) {
        int d = idx / (TE * IGAB_TAB1D), r = idx % (TE * IGAB_TAB1D), le = r / IGAB_TAB1D, o = r % IGAB_TAB1D;
        S.tab[d][le][o] = le < Tl.nv[d] ? g.tab[d][(long)(Tl.e0[d] + le) * IGAB_TAB1D + o] : 0.0;
    }
    for (int idx = tid; idx < 3 * TE * IGAB_NQ; idx += NTHR) {
        int d = idx / (TE * IGAB_NQ), r = idx % (TE * IGAB_NQ), le = r / IGAB_NQ, q = r % IGAB_NQ;
        S.wh[d][le][q] = le < Tl.nv[d] ? g.wh[d][(long)(Tl.e0[d] + le) * IGAB_NQ + q] : 0.0;
    }
    /* the padding columns (a >= 27) of U / V stay zero */
    for (int idx = tid; idx < GROWS * GS; idx += NTHR) {
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
        double *const A = S.W + W_A;
        double *const C = S.W + W_C;
        /* ---- field at the 64 Gauss points (sum-factorised, as the residual) */
        for (int o = tid; o < 972; o += NTHR) {
            int i = o % 3, kz = (o / 3) % 3, ay = (o / 9) % 3, ax = (o / 27) % 3, q = o / 81;
            const double *u0 = &S.U[(((lex + ax) * TC + (ley + ay)) * TC + lez) * 3 + i];
            A[o] = Bz[q * 9 + kz] * u0[0] + Bz[q * 9 + 3 + kz] * u0[3] + Bz[q * 9 + 6 + kz] * u0[6];
        }
        __syncthreads();
        for (int o = tid; o < 864; o += NTHR) {
            int i = o % 3, kk = (o / 3) % 6, ax = (o / 18) % 3, qq = o / 54;
            int qyy = qq & 3, qzz = qq >> 2;
            const double *a0 = &A[((qzz * 3 + ax) * 3) * 9 + kk_kz(kk) * 3 + i];
            C[o] = By[qyy * 9 + kk_ky(kk)] * a0[0] + By[qyy * 9 + 3 + kk_ky(kk)] * a0[9] +
                   By[qyy * 9 + 6 + kk_ky(kk)] * a0[18];
        }
        __syncthreads();
        /* ---- point integrand data (64 threads), point order q = 16 qz + 4 qy + qx */
        if (tid < IGAB_NQ3) {
            const int qx = tid & 3, qy = (tid >> 2) & 3, qz = tid >> 4, qq = qy + 4 * qz;
            double u[30];
#pragma unroll
            for (int a = 0; a < 10; a++)
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    double s = 0.0;
#pragma unroll
                    for (int ax = 0; ax < 3; ax++)
                        s += Bx[qx * 9 + ax * 3 + a_kx(a)] * C[((qq * 3 + ax) * 6 + a_kk(a)) * 3 + i];
                    u[10 * i + a] = s;
                }
            if (g.periodic) {
#pragma unroll
                for (int i = 0; i < 3; i++)
#pragma unroll
                    for (int J = 0; J < 3; J++) u[10 * i + 1 + J] += g.pp[3 * i + J];
            }
            igab_ge_point<double> P;
            igab_ge_eval(u, g.coef, P);
            double *pt = PTb + tid * PT_N;
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int J = 0; J < 3; J++) pt[PT_F + 3 * k + J] = P.F[k][J];
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int c = 0; c < 6; c++) pt[PT_G + 6 * k + c] = P.G[k][c];
            double cs, sn, l1, l2;
            sym2_eig(P.d2[1], P.d2ab, P.d2[2], cs, sn, l1, l2);
#pragma unroll
            for (int v = 0; v < 12; v++) pt[PT_LAM + v] = v == 1 ? l1 : (v == 2 ? l2 : P.d2[v]);
            pt[PT_CS] = cs;
            pt[PT_SN] = sn;
#pragma unroll
            for (int I = 0; I < 3; I++) pt[PT_SIG + I] = P.sig[I];
#pragma unroll
            for (int I = 0; I < 3; I++) pt[PT_D1S + I] = P.d1[3 + I];
#pragma unroll
            for (int I = 0; I < 3; I++)
#pragma unroll
                for (int K = 0; K < 3; K++) pt[PT_TAU + 3 * I + K] = P.tau[I][K];
            pt[PT_W] = S.wh[0][lex][qx] * S.wh[1][ley][qy] * S.wh[2][lez][qz] *
                       elem_scale(g, Tl.e0[0] + lex, Tl.e0[1] + ley, Tl.e0[2] + lez);
        }
        __syncthreads();

        double acc[17][2], gacc[3][2];
#pragma unroll
        for (int t = 0; t < 17; t++) acc[t][0] = acc[t][1] = 0.0;
#pragma unroll
        for (int t = 0; t < 3; t++) gacc[t][0] = gacc[t][1] = 0.0;

        for (int q0 = 0; q0 < IGAB_NQ3; q0 += DQ) {
            if (q0 == 0)   /* the interpolation / staging data under X' is dead: padding columns back to zero */
                for (int idx = tid; idx < DROWS * (XS - 81); idx += NTHR)
                    Xb[(idx / (XS - 81)) * XS + 81 + idx % (XS - 81)] = 0.0;
            /* (a) X' rows: task (variable v, point qb, component k, x-function ax) -> 9 outputs
             * (ay, az), X'[(qb, v)][3a + k] = sum_m dv'/du_{k,m} Bx By Bz, summed over x, y, z */
            for (int t = tid; t < DQ * 12 * 9; t += NTHR) {
                const int v = t / (DQ * 9), r = t % (DQ * 9);
                const int qb = r / 9, k = (r / 3) % 3, ax = r % 3;
                const int q = q0 + qb, qx = q & 3, qy = (q >> 2) & 3, qz = q >> 4;
                double gv[9];
                dm_grad_var(PTb + q * PT_N, v, k, gv);
                const double *bxp = Bx + qx * 9 + ax * 3;
                const double bx0 = bxp[0], bx1 = bxp[1], bx2 = bxp[2];
                /* coefficients of By[ky] per kz: derivative m -> (kx, ky, kz) as eval_Bspline */
                const double t00 = gv[0] * bx1 + gv[3] * bx2, t01 = gv[1] * bx0 + gv[4] * bx1, t02 = gv[6] * bx0;
                const double t10 = gv[2] * bx0 + gv[5] * bx1, t11 = gv[7] * bx0;
                const double t20 = gv[8] * bx0;
                double *xr = Xb + (qb * 12 + v) * XS + k;
#pragma unroll
                for (int ay = 0; ay < 3; ay++) {
                    const double *byp = By + qy * 9 + ay * 3;
                    const double cy0 = t00 * byp[0] + t01 * byp[1] + t02 * byp[2];
                    const double cy1 = t10 * byp[0] + t11 * byp[1];
                    const double cy2 = t20 * byp[0];
#pragma unroll
                    for (int az = 0; az < 3; az++) {
                        const double *bzp = Bz + qz * 9 + az * 3;
                        xr[3 * (9 * ax + 3 * ay + az)] = cy0 * bzp[0] + cy1 * bzp[1] + cy2 * bzp[2];
                    }
                }
            }
            /* U / V rows of the geometric block: task (row i, point qb, ax, ay) -> 3 outputs (az) */
            for (int t = tid; t < DQ * 6 * 9; t += NTHR) {
                const int i = t / (DQ * 9), r = t % (DQ * 9);
                const int qb = r / 9, ax = (r / 3) % 3, ay = r % 3;
                const int q = q0 + qb, qx = q & 3, qy = (q >> 2) & 3, qz = q >> 4;
                const double *p = PTb + q * PT_N;
                const double w = p[PT_W];
                const double bx0 = Bx[qx * 9 + ax * 3], bx1 = Bx[qx * 9 + ax * 3 + 1], bx2 = Bx[qx * 9 + ax * 3 + 2];
                const double by0 = By[qy * 9 + ay * 3], by1 = By[qy * 9 + ay * 3 + 1], by2 = By[qy * 9 + ay * 3 + 2];
                const int I = i < 3 ? i : i - 3;
                const double s00 = p[PT_SIG], s11 = p[PT_SIG + 1], s22 = p[PT_SIG + 2];
                const double s01 = 0.5 * p[PT_D1S], s02 = 0.5 * p[PT_D1S + 1], s12 = 0.5 * p[PT_D1S + 2];
                const double tI0 = p[PT_TAU + 3 * I], tI1 = p[PT_TAU + 3 * I + 1], tI2 = p[PT_TAU + 3 * I + 2];
#pragma unroll
                for (int az = 0; az < 3; az++) {
                    const double *bzp = Bz + qz * 9 + az * 3;
                    const double bz0 = bzp[0], bz1 = bzp[1], bz2 = bzp[2];
                    const double dx = bx1 * by0 * bz0, dy = bx0 * by1 * bz0, dz = bx0 * by0 * bz1;
                    /* second derivatives H[idx6(I, K)], K = 0..2 */
                    double h0, h1, h2;
                    if (I == 0) { h0 = bx2 * by0 * bz0; h1 = bx1 * by1 * bz0; h2 = bx1 * by0 * bz1; }
                    else if (I == 1) { h0 = bx1 * by1 * bz0; h1 = bx0 * by2 * bz0; h2 = bx0 * by1 * bz1; }
                    else { h0 = bx1 * by0 * bz1; h1 = bx0 * by1 * bz1; h2 = bx0 * by0 * bz2; }
                    const double th = tI0 * h0 + tI1 * h1 + tI2 * h2;   /* (T H_a)_I */
                    const double dI = I == 0 ? dx : (I == 1 ? dy : dz);
                    const int a = 9 * ax + 3 * ay + az, row = qb * 6 + i;
                    if (i < 3) {
                        const double sg = I == 0 ? s00 * dx + s01 * dy + s02 * dz
                                        : (I == 1 ? s01 * dx + s11 * dy + s12 * dz : s02 * dx + s12 * dy + s22 * dz);
                        S.UT[row][a] = dI;
                        S.VT[row][a] = w * (sg + th);
                    } else {
                        S.UT[row][a] = w * th;
                        S.VT[row][a] = dI;
                    }
                }
            }
            if (tid < DROWS) {
                const double *p = PTb + (q0 + tid / 12) * PT_N;
                S.sc[tid] = p[PT_W] * p[PT_LAM + tid % 12];
            }
            __syncthreads();
            /* (b) tensor-core accumulation K += X'^T diag(sc) X', Gamma += U^T V */
#define MMA_CALL(Wn) warp_mma<Wn>(Xb, S.sc, &S.UT[0][0], &S.VT[0][0], lane, acc, gacc)
            WARP_SWITCH(MMA_CALL)
#undef MMA_CALL
            __syncthreads();
        }
        /* ---- stage K and Gamma in shared memory, then scatter the 81 x 81 element matrix */
        double *const K = S.W;
        double *const Gam = S.W + W_GAM;
#define DUMP_CALL(Wn) warp_dump<Wn>(K, Gam, lane, acc, gacc)
        WARP_SWITCH(DUMP_CALL)
#undef DUMP_CALL
        if (tid < 81)
            elem_row_base(g, Tl.e0[0] + lex, Tl.e0[1] + ley, Tl.e0[2] + lez, tid, S.rbase[tid], S.rsx[tid], S.rsy[tid]);
        __syncthreads();
        /* added into the CSR values with fire-and-forget reductions (red.global.add):
         * the tiles of one colour touch disjoint entries and the elements of a tile
         * are separated by a barrier, so every entry receives its additions in a
         * fixed order */
        for (int idx = tid; idx < 81 * 81; idx += NTHR) {
            const int c1 = idx / 81, c2 = idx % 81;
            const int a1 = c1 / 3, k1 = c1 % 3, a2 = c2 / 3, k2 = c2 % 3;
            double v = c1 <= c2 ? K[c1 * 88 + c2] : K[c2 * 88 + c1];
            if (k1 == k2) v += a1 <= a2 ? Gam[a1 * 32 + a2] : Gam[a2 * 32 + a1];
            atomicAdd(&vals[S.rbase[c1] + (c2 / 27) * S.rsx[c1] + ((c2 / 9) % 3) * S.rsy[c1] + c2 % 9], v);
        }
        __syncthreads();
    }
}

template <int TE>
__global__ void __launch_bounds__(NTHR, 2) k_tan_dmma(igab_geom g, const double *__restrict__ U,
                                                      double *__restrict__ vals, int colour)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    dmma_smem<TE> &S = *reinterpret_cast<dmma_smem<TE> *>(smem_raw);
    tile_t Tl;
    if (!decode_tile(g, TE, colour, blockIdx.x, Tl)) return;
    dmma_tile<TE>(g, Tl, U, vals, S);
}

/* persistent FP64 tangent over the tiles of every instance of a batch */
__global__ void __launch_bounds__(NTHR, 2) k_tan_dmma_batch(igab_batch_dev B, const double *__restrict__ U,
                                                            double *__restrict__ vals)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    dmma_smem<2> &S = *reinterpret_cast<dmma_smem<2> *>(smem_raw);
    __shared__ batch_slot sl;
    while (batch_next(B, sl)) {
        tile_t Tl;
        decode_tile(sl.g, 2, sl.colour, sl.tile, Tl);
        dmma_tile<2>(sl.g, Tl, U + B.dof_off[sl.inst], vals + B.nnz_off[sl.inst], S);
        batch_done(B, sl);
    }
}

} /* namespace */

int igab_launch_tan_dmma_batch(const igab_batch_dev &B, int grid, cudaStream_t st, const double *dU, double *dv)
{
    const size_t sm = sizeof(dmma_smem<2>);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_dmma_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_tan_dmma_batch<<<grid, NTHR, sm, st>>>(B, dU, dv);
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int igab_batch_occupancy_dmma(int *per_sm)
{
    const size_t sm = sizeof(dmma_smem<2>);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_dmma_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    IGAB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_tan_dmma_batch, NTHR, sm));
    return 0;
}

int igab_launch_tan_dmma(igab_ctx *c, const double *dU, double *dv)
{
    igab_geom g = c->geom();
    size_t sm = sizeof(dmma_smem<2>);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_dmma<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    for (int colour = 0; colour < 8; colour++) {
        long nblk = tiles_of_colour(g, 2, colour);
        if (nblk == 0) continue;
        k_tan_dmma<2><<<(unsigned)nblk, NTHR, sm, c->stream>>>(g, dU, dv, colour);
        c->last_launches++;
    }
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}
