/*
 * FP64 tangent volume kernel on the FP64 tensor path (mma.sync m8n8k4 f64).
 *
 * Per element (src/snesiga_Tangent.c:104-190), with the energy written as
 * W = Phi(v(u)) over 12 variables (igab_math.cuh):
 *   K_e = sum_q w_q X_q^T Phi''_q X_q  +  blockdiag_k(Gamma),
 *   X_q[v][3a+k] = sum_m dv/du_{k,m}(q) N_a^{m}(q).
 * Phi'' is diagonal except for the (va, vb) pair; rotating those two rows by
 * the eigenvectors of that 2x2 block makes it diagonal, so
 *   K_e = X'^T diag(s) X',   s = w_q * eigenvalues.
 * X' (96 rows = 8 Gauss points x 12 variables, 88 padded columns) sits in
 * shared memory once; a warp loads its A fragments from it and forms the B
 * fragments by scaling the same registers with s.  The 66 upper-triangle 8x8
 * tiles of the 88x88 element matrix are spread over the 8 warps (<= 9 tiles,
 * <= 5 fragment blocks each, table below); the lower triangle is written by
 * symmetry.  The geometric block Gamma (same for the three displacement
 * components) is accumulated on the FP64 pipe by its owning threads.
 * Scatter: read-modify-write into the CSR values, conflict-free within one
 * of the 8 tile colours (see igab_kernels.cu).
 */
#include <cuda_runtime.h>
#include "igab_device.cuh"

namespace {

#include "igab_warp_tiles.inc"

#define DQ 8            /* Gauss points per batch */
#define DROWS (DQ * 12) /* k rows per batch */
#define XS 100          /* row stride of X' in doubles: 100 = 4 (mod 16) keeps fragment loads conflict-free */

#define PT_F 0
#define PT_G 9
#define PT_D2 27
#define PT_D2AB 39
#define PT_SIG 40
#define PT_D1S 43
#define PT_TAU 46
#define PT_W 55
#define PT_ROT 56 /* cs, sn, l1, l2 of the (va, vb) block */
#define PT_N 60

template <int TE>
struct dmma_smem {
    static constexpr int TC = TE + 2;
    static constexpr int NCP = TC * TC * TC;
    double U[NCP * 3];
    double tab[3][TE][IGAB_TAB1D];
    double wh[3][TE][IGAB_NQ];
    double A[972];
    double C[864];
    double pt[IGAB_NQ3][PT_N];
    double N[DQ][27][9];      /* N_a^{m+1} */
    double Gv[DQ][12][27];    /* rotated dv/du_s */
    double GN[DQ][9][27];     /* w * geo * N */
    double geo[DQ][9][9];     /* geometric block per Gauss point */
    double gcoef[12][9];      /* dv/du_{k,m} = gcoef[v][m] * src_k[gsrc[v][m]] */
    int gsrc[12][9];          /* src_k = (F_k0, F_k1, F_k2, G_k0..G_k5), -1 = zero */
    double sc[DROWS];         /* w * eigenvalue per k row */
    double X[DROWS][XS];
    double Gam[27 * 27];
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
__device__ __forceinline__ void warp_mma(const double *__restrict__ X, const double *__restrict__ sc, int lane,
                                         double (&acc)[9][2])
{
    using WT = warp_tiles<W>;
#pragma unroll 2
    for (int kb = 0; kb < DROWS / 4; kb++) {
        const int kr = 4 * kb + (lane & 3);
        const double s = sc[kr];
        const double *row = X + kr * XS + (lane >> 2);
        double f[WT::NB], g[WT::NB];
#pragma unroll
        for (int b = 0; b < WT::NB; b++) {
            f[b] = row[8 * WT::blk(b)];
            g[b] = f[b] * s;
        }
#pragma unroll
        for (int t = 0; t < WT::NT; t++) dmma(acc[t][0], acc[t][1], f[WT::ti(t)], g[WT::tj(t)]);
    }
}

/* accumulator tiles -> shared K[c1][c2] (upper triangle tiles only) */
template <int W>
__device__ __forceinline__ void warp_dump(double *__restrict__ K, int lane, const double (&acc)[9][2])
{
    using WT = warp_tiles<W>;
#pragma unroll
    for (int t = 0; t < WT::NT; t++) {
        const int c1 = 8 * WT::blk(WT::ti(t)) + (lane >> 2);
        const int c2 = 8 * WT::blk(WT::tj(t)) + 2 * (lane & 3);
        K[c1 * 88 + c2] = acc[t][0];
        K[c1 * 88 + c2 + 1] = acc[t][1];
    }
}

#define WARP_SWITCH(CALL)          \
    switch (warp) {                \
    case 0: CALL(0); break;        \
    case 1: CALL(1); break;        \
    case 2: CALL(2); break;        \
    case 3: CALL(3); break;        \
    case 4: CALL(4); break;        \
    case 5: CALL(5); break;        \
    case 6: CALL(6); break;        \
    default: CALL(7); break;       \
    }

template <int TE>
__global__ void __launch_bounds__(256, 1) k_tan_dmma(igab_geom g, const double *__restrict__ U,
                                                     double *__restrict__ vals, int colour)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    dmma_smem<TE> &S = *reinterpret_cast<dmma_smem<TE> *>(smem_raw);
    constexpr int TC = TE + 2;
    constexpr int NCP = TC * TC * TC;
    constexpr int NEL = TE * TE * TE;
    tile_t Tl;
    if (!decode_tile(g, TE, colour, blockIdx.x, Tl)) return;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

    /* owned geometric entries (a1 <= a2), 378 over 256 threads */
    int gown[2];
#pragma unroll
    for (int j = 0; j < 2; j++) {
        int idx = tid + 256 * j;
        int a1 = 0, rem = idx;
        while (a1 < 27 && rem >= 27 - a1) { rem -= 27 - a1; a1++; }
        gown[j] = a1 < 27 ? (a1 << 8) | (a1 + rem) : -1;
    }

    for (int idx = tid; idx < NCP * 3; idx += 256) {
        int i = idx % 3, cp = idx / 3;
        int lz = cp % TC, ly = (cp / TC) % TC, lx = cp / (TC * TC);
        double v = 0.0;
        if (lx < Tl.nv[0] + 2 && ly < Tl.nv[1] + 2 && lz < Tl.nv[2] + 2)
            v = U[3 * cp_index(g, Tl.e0[0] + lx, Tl.e0[1] + ly, Tl.e0[2] + lz) + i];
        S.U[idx] = v;
    }
    for (int idx = tid; idx < 3 * TE * IGAB_TAB1D; idx += 256) {
        int d = idx / (TE * IGAB_TAB1D), r = idx % (TE * IGAB_TAB1D), le = r / IGAB_TAB1D, o = r % IGAB_TAB1D;
        S.tab[d][le][o] = le < Tl.nv[d] ? g.tab[d][(long)(Tl.e0[d] + le) * IGAB_TAB1D + o] : 0.0;
    }
    for (int idx = tid; idx < 3 * TE * IGAB_NQ; idx += 256) {
        int d = idx / (TE * IGAB_NQ), r = idx % (TE * IGAB_NQ), le = r / IGAB_NQ, q = r % IGAB_NQ;
        S.wh[d][le][q] = le < Tl.nv[d] ? g.wh[d][(long)(Tl.e0[d] + le) * IGAB_NQ + q] : 0.0;
    }
    /* sparse structure of dv/du_{k,m}: one source term per (v, m) (igab_ge_grad_var) */
    if (tid < 108) {
        const int v = tid / 9, m = tid % 9;
        int src = -1;
        double cf = 0.0;
        const double is2 = IGAB_INV_SQRT2, is3 = IGAB_INV_SQRT3, is6 = IGAB_INV_SQRT6;
        if (v == 0) { if (m < 3) { src = m; cf = is3; } }
        else if (v == 1) { if (m == 0) { src = 0; cf = is2; } else if (m == 1) { src = 1; cf = -is2; } }
        else if (v == 2) { if (m < 2) { src = m; cf = is6; } else if (m == 2) { src = 2; cf = -2.0 * is6; } }
        else if (v == 3) { if (m == 0) { src = 1; cf = 0.5; } else if (m == 1) { src = 0; cf = 0.5; } }
        else if (v == 4) { if (m == 0) { src = 2; cf = 0.5; } else if (m == 2) { src = 0; cf = 0.5; } }
        else if (v == 5) { if (m == 1) { src = 2; cf = 0.5; } else if (m == 2) { src = 1; cf = 0.5; } }
        else {
            const int K = v < 9 ? v - 6 : v - 9;
            const int q0 = igab_idx6(0, K), q1 = igab_idx6(1, K), q2 = igab_idx6(2, K);
            if (v < 9) {
                if (m == 0) { src = 3 + q0; cf = is2; }
                else if (m == 1) { src = 3 + q1; cf = -is2; }
                else if (m == 3 + q0) { src = 0; cf = is2; }
                else if (m == 3 + q1) { src = 1; cf = -is2; }
            } else {
                if (m == 0) { src = 3 + q0; cf = is6; }
                else if (m == 1) { src = 3 + q1; cf = is6; }
                else if (m == 2) { src = 3 + q2; cf = -2.0 * is6; }
                else if (m == 3 + q0) { src = 0; cf = is6; }
                else if (m == 3 + q1) { src = 1; cf = is6; }
                else if (m == 3 + q2) { src = 2; cf = -2.0 * is6; }
            }
        }
        S.gsrc[v][m] = src;
        S.gcoef[v][m] = cf;
    }
    /* padding columns 81..99 of X' stay zero */
    for (int idx = tid; idx < DROWS * XS; idx += 256) (&S.X[0][0])[idx] = 0.0;
    __syncthreads();

    for (int le = 0; le < NEL; le++) {
        const int lex = le / (TE * TE), ley = (le / TE) % TE, lez = le % TE;
        if (!(lex < Tl.nv[0] && ley < Tl.nv[1] && lez < Tl.nv[2])) continue;   /* block-uniform */
        const double *Bx = S.tab[0][lex];
        const double *By = S.tab[1][ley];
        const double *Bz = S.tab[2][lez];
        /* ---- field at the 64 Gauss points (sum-factorised, as the residual) */
        for (int o = tid; o < 972; o += 256) {
            int i = o % 3, kz = (o / 3) % 3, ay = (o / 9) % 3, ax = (o / 27) % 3, q = o / 81;
            const double *u0 = &S.U[(((lex + ax) * TC + (ley + ay)) * TC + lez) * 3 + i];
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
            double u[30];
#pragma unroll
            for (int a = 0; a < 10; a++)
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    double s = 0.0;
#pragma unroll
                    for (int ax = 0; ax < 3; ax++)
                        s += Bx[qx * 9 + ax * 3 + a_kx(a)] * S.C[((qq * 3 + ax) * 6 + a_kk(a)) * 3 + i];
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
            /* point order q = 16 qz + 4 qy + qx */
            double *pt = S.pt[tid];
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int J = 0; J < 3; J++) pt[PT_F + 3 * k + J] = P.F[k][J];
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int c = 0; c < 6; c++) pt[PT_G + 6 * k + c] = P.G[k][c];
#pragma unroll
            for (int v = 0; v < 12; v++) pt[PT_D2 + v] = P.d2[v];
            pt[PT_D2AB] = P.d2ab;
#pragma unroll
            for (int I = 0; I < 3; I++) pt[PT_SIG + I] = P.sig[I];
#pragma unroll
            for (int I = 0; I < 3; I++) pt[PT_D1S + I] = P.d1[3 + I];
#pragma unroll
            for (int I = 0; I < 3; I++)
#pragma unroll
                for (int K = 0; K < 3; K++) pt[PT_TAU + 3 * I + K] = P.tau[I][K];
            pt[PT_W] = S.wh[0][lex][qx] * S.wh[1][ley][qy] * S.wh[2][lez][qz];
            sym2_eig(P.d2[1], P.d2ab, P.d2[2], pt[PT_ROT], pt[PT_ROT + 1], pt[PT_ROT + 2], pt[PT_ROT + 3]);
        }
        __syncthreads();

        double acc[9][2];
#pragma unroll
        for (int t = 0; t < 9; t++) acc[t][0] = acc[t][1] = 0.0;
        double gacc[2] = {0.0, 0.0};

        for (int q0 = 0; q0 < IGAB_NQ3; q0 += DQ) {
            /* (a) basis products, rotated variable gradients, scales, geometric blocks */
            for (int o = tid; o < DQ * 243; o += 256) {
                int m = o % 9, a = (o / 9) % 27, qb = o / 243;
                int q = q0 + qb, qx = q & 3, qy = (q >> 2) & 3, qz = q >> 4;
                int al = m + 1;
                S.N[qb][a][m] = Bx[qx * 9 + (a / 9) * 3 + a_kx(al)] * By[qy * 9 + ((a / 3) % 3) * 3 + a_ky(al)] *
                                Bz[qz * 9 + (a % 3) * 3 + a_kz(al)];
            }
            for (int o = tid; o < DQ * 12 * 27; o += 256) {
                const int sidx = o % 27, v = (o / 27) % 12, qb = o / 324;
                const int k = sidx / 9, m = sidx % 9;
                const double *pt = S.pt[q0 + qb];
                double val;
                if (v == 1 || v == 2) {
                    const int i1 = S.gsrc[1][m], i2 = S.gsrc[2][m];
                    const double g1 = i1 < 0 ? 0.0 : S.gcoef[1][m] * (i1 < 3 ? pt[PT_F + 3 * k + i1] : pt[PT_G + 6 * k + i1 - 3]);
                    const double g2 = i2 < 0 ? 0.0 : S.gcoef[2][m] * (i2 < 3 ? pt[PT_F + 3 * k + i2] : pt[PT_G + 6 * k + i2 - 3]);
                    const double cs = pt[PT_ROT], sn = pt[PT_ROT + 1];
                    val = v == 1 ? cs * g1 - sn * g2 : sn * g1 + cs * g2;
                    if (sidx == 0) S.sc[qb * 12 + v] = pt[PT_W] * pt[PT_ROT + 1 + v];
                } else {
                    const int i0 = S.gsrc[v][m];
                    val = i0 < 0 ? 0.0 : S.gcoef[v][m] * (i0 < 3 ? pt[PT_F + 3 * k + i0] : pt[PT_G + 6 * k + i0 - 3]);
                    if (sidx == 0) S.sc[qb * 12 + v] = pt[PT_W] * pt[PT_D2 + v];
                }
                S.Gv[qb][v][sidx] = val;
            }
            for (int o = tid; o < DQ * 81; o += 256) {
                const int n = o % 9, m = (o / 9) % 9, qb = o / 81;
                const double *pt = S.pt[q0 + qb];
                const int lo = m < n ? m : n, hi = m < n ? n : m;
                double gv = 0.0;
                if (hi < 3) {
                    gv = lo == hi ? pt[PT_SIG + lo] : 0.5 * pt[PT_D1S + (lo == 0 ? hi - 1 : 2)];
                } else if (lo < 3) {
                    /* slot hi = 3 + idx6(lo, K) for exactly one K, if any */
#pragma unroll
                    for (int K = 0; K < 3; K++)
                        if (3 + igab_idx6(lo, K) == hi) gv = pt[PT_TAU + 3 * lo + K];
                }
                S.geo[qb][m][n] = gv;
            }
            __syncthreads();
            /* (b) X' = Gv' . N (rows of 9 outputs per task) and GN = w geo N */
            for (int o = tid; o < DQ * 12 * 3 * 3; o += 256) {
                const int part = o % 3, k = (o / 3) % 3, v = (o / 9) % 12, qb = o / 108;
                double gr[9];
#pragma unroll
                for (int m = 0; m < 9; m++) gr[m] = S.Gv[qb][v][9 * k + m];
                double *xr = &S.X[qb * 12 + v][0];
                if (v < 6) {
#pragma unroll
                    for (int j = 0; j < 9; j++) {
                        const int a = 9 * part + j;
                        const double *nr = S.N[qb][a];
                        xr[3 * a + k] = gr[0] * nr[0] + gr[1] * nr[1] + gr[2] * nr[2];
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < 9; j++) {
                        const int a = 9 * part + j;
                        const double *nr = S.N[qb][a];
                        double t = 0.0;
#pragma unroll
                        for (int m = 0; m < 9; m++) t += gr[m] * nr[m];
                        xr[3 * a + k] = t;
                    }
                }
            }
            for (int o = tid; o < DQ * 243; o += 256) {
                const int b = o % 27, m = (o / 27) % 9, qb = o / 243;
                const double *gr = S.geo[qb][m];
                const double *nr = S.N[qb][b];
                double t = 0.0;
#pragma unroll
                for (int n = 0; n < 9; n++) t += gr[n] * nr[n];
                S.GN[qb][m][b] = S.pt[q0 + qb][PT_W] * t;
            }
            __syncthreads();
            /* (c) tensor-core accumulation K += X'^T diag(sc) X' */
#define MMA_CALL(Wn) warp_mma<Wn>(&S.X[0][0], S.sc, lane, acc)
            WARP_SWITCH(MMA_CALL)
#undef MMA_CALL
            /* geometric block for the owned entries (FP64 pipe, overlaps the tensor work of other warps) */
#pragma unroll
            for (int j = 0; j < 2; j++) {
                if (gown[j] < 0) continue;
                int a1 = gown[j] >> 8, a2 = gown[j] & 255;
                double t = gacc[j];
                for (int qb = 0; qb < DQ; qb++)
#pragma unroll
                    for (int m = 0; m < 9; m++) t += S.N[qb][a1][m] * S.GN[qb][m][a2];
                gacc[j] = t;
            }
            __syncthreads();
        }
#pragma unroll
        for (int j = 0; j < 2; j++) {
            if (gown[j] < 0) continue;
            int a1 = gown[j] >> 8, a2 = gown[j] & 255;
            S.Gam[a1 * 27 + a2] = gacc[j];
            S.Gam[a2 * 27 + a1] = gacc[j];
        }
        __syncthreads();
#define DUMP_CALL(Wn) warp_dump<Wn>(&S.X[0][0], lane, acc)
        WARP_SWITCH(DUMP_CALL)
#undef DUMP_CALL
        __syncthreads();
        /* ---- scatter the full 81 x 81 element matrix row by row (lower half mirrored) */
        {
            const double *K = &S.X[0][0];
            for (int idx = tid; idx < 81 * 81; idx += 256) {
                const int c1 = idx / 81, c2 = idx % 81;
                const int a1 = c1 / 3, k1 = c1 % 3, a2 = c2 / 3, k2 = c2 % 3;
                double val = c1 <= c2 ? K[c1 * 88 + c2] : K[c2 * 88 + c1];
                if (k1 == k2) val += S.Gam[a1 * 27 + a2];
                const int x1 = Tl.e0[0] + lex + a1 / 9, y1 = Tl.e0[1] + ley + (a1 / 3) % 3, z1 = Tl.e0[2] + lez + a1 % 3;
                const int x2 = Tl.e0[0] + lex + a2 / 9, y2 = Tl.e0[1] + ley + (a2 / 3) % 3, z2 = Tl.e0[2] + lez + a2 % 3;
                const long r1 = 3 * cp_index(g, x1, y1, z1) + k1;
                vals[g.rowptr[r1] + csr_pos(g, x1, y1, z1, x2, y2, z2, k2)] += val;
            }
        }
        __syncthreads();
        /* the staged K overwrote padding columns of X'; they must be zero again */
        for (int idx = tid; idx < DROWS * (XS - 81); idx += 256) S.X[idx / (XS - 81)][81 + idx % (XS - 81)] = 0.0;
        __syncthreads();
    }
}

} /* namespace */

int igab_launch_tan_dmma(igab_ctx *c, const double *dU, double *dv)
{
    igab_geom g = c->geom();
    size_t sm = sizeof(dmma_smem<2>);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_dmma<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    for (int colour = 0; colour < 8; colour++) {
        long nblk = tiles_of_colour(g, 2, colour);
        if (nblk == 0) continue;
        k_tan_dmma<2><<<(unsigned)nblk, 256, sm, c->stream>>>(g, dU, dv, colour);
        c->last_launches++;
    }
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}
