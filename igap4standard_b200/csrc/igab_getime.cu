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

#define GQ 2          /* Gauss points per batch */
#define GNV 24        /* rows per Gauss point: 12 variables x (G0, G1) */
#define GOWN 13       /* owned upper-triangle entries per thread */

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

template <typename T, int TE>
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
    T N[GQ][27][10];          /* N_a^{alpha}, alpha = value, 9 derivatives */
    T Gv[GQ][GNV][27];
    T X[GQ][GNV][81];
    T Y[GQ][GNV][81];
    T GN[GQ][10][27];         /* effective geo x N (+ mass x N on the value row) */
};

/* dv/du_{k,m}: one source term per (v, m) from (F, G) of one Taylor order;
 * with_identity adds the unit diagonal of F (order 0 only) -- F passed already includes it */
template <typename T>
__device__ __forceinline__ void grad_row(const double *F, const double *G, int v, T g[9])
{
    const double is2 = IGAB_INV_SQRT2, is3 = IGAB_INV_SQRT3, is6 = IGAB_INV_SQRT6;
#pragma unroll
    for (int m = 0; m < 9; m++) g[m] = T(0);
    switch (v) {
    case 0: g[0] = T(F[0] * is3); g[1] = T(F[1] * is3); g[2] = T(F[2] * is3); break;
    case 1: g[0] = T(F[0] * is2); g[1] = T(-F[1] * is2); break;
    case 2: g[0] = T(F[0] * is6); g[1] = T(F[1] * is6); g[2] = T(-2.0 * F[2] * is6); break;
    case 3: g[0] = T(0.5 * F[1]); g[1] = T(0.5 * F[0]); break;
    case 4: g[0] = T(0.5 * F[2]); g[2] = T(0.5 * F[0]); break;
    case 5: g[1] = T(0.5 * F[2]); g[2] = T(0.5 * F[1]); break;
    default:
        if (v < 9) {
            const int K = v - 6, q0 = igab_idx6(0, K), q1 = igab_idx6(1, K);
            g[0] = T(G[q0] * is2); g[1] = T(-G[q1] * is2);
            g[3 + q0] = T(F[0] * is2); g[3 + q1] = T(-F[1] * is2);
        } else {
            const int K = v - 9, q0 = igab_idx6(0, K), q1 = igab_idx6(1, K), q2 = igab_idx6(2, K);
            g[0] = T(G[q0] * is6); g[1] = T(G[q1] * is6); g[2] = T(-2.0 * G[q2] * is6);
            g[3 + q0] = T(F[0] * is6); g[3 + q1] = T(F[1] * is6); g[3 + q2] = T(-2.0 * F[2] * is6);
        }
    }
}

template <typename T, int TE>
__global__ void __launch_bounds__(256) k_tan_getime(igab_geom g, const double *__restrict__ U,
                                                    T *__restrict__ vals, int colour)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    gt_smem<T, TE> &S = *reinterpret_cast<gt_smem<T, TE> *>(smem_raw);
    constexpr int TC = TE + 2;
    constexpr int NCP = TC * TC * TC;
    constexpr int NEL = TE * TE * TE;
    tile_t Tl;
    if (!decode_tile(g, TE, colour, blockIdx.x, Tl)) return;
    const int tid = threadIdx.x;

    int own[GOWN];
#pragma unroll
    for (int j = 0; j < GOWN; j++) {
        int idx = tid + 256 * j;
        int c1 = 0, rem = idx;
        while (c1 < 81 && rem >= 81 - c1) { rem -= 81 - c1; c1++; }
        own[j] = c1 < 81 ? (c1 << 8) | (c1 + rem) : -1;
    }
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

        T acc[GOWN];
#pragma unroll
        for (int j = 0; j < GOWN; j++) acc[j] = T(0);
        T gacc[2] = {T(0), T(0)};

        for (int q0 = 0; q0 < IGAB_NQ3; q0 += GQ) {
            /* (a) basis values and gradient rows */
            for (int o = tid; o < GQ * 270; o += 256) {
                int al = o % 10, a = (o / 10) % 27, qb = o / 270;
                int q = q0 + qb, qx = q & 3, qy = (q >> 2) & 3, qz = q >> 4;
                S.N[qb][a][al] = T(Bx[qx * 9 + (a / 9) * 3 + a_kx(al)] * By[qy * 9 + ((a / 3) % 3) * 3 + a_ky(al)] *
                                   Bz[qz * 9 + (a % 3) * 3 + a_kz(al)]);
            }
            for (int o = tid; o < GQ * GNV * 3; o += 256) {
                const int k = o % 3, r = (o / 3) % GNV, qb = o / (3 * GNV);
                const double *pt = S.pt[q0 + qb];
                const int v = r >> 1, a = r & 1;
                T gg[9];
                grad_row<T>(pt + (a ? GP_F1 : GP_F0) + 3 * k, pt + (a ? GP_G1 : GP_G0) + 6 * k, v, gg);
#pragma unroll
                for (int m = 0; m < 9; m++) S.Gv[qb][r][9 * k + m] = gg[m];
            }
            __syncthreads();
            /* (b) X = G N and the effective geometric block x N */
            for (int o = tid; o < GQ * GNV * 81; o += 256) {
                const int c = o % 81, r = (o / 81) % GNV, qb = o / (81 * GNV);
                const int a = c / 3, k = c % 3;
                T s = T(0);
#pragma unroll
                for (int m = 0; m < 9; m++) s += S.Gv[qb][r][9 * k + m] * S.N[qb][a][m + 1];
                S.X[qb][r][c] = s;
            }
            for (int o = tid; o < GQ * 10 * 27; o += 256) {
                const int b = o % 27, m = (o / 27) % 10, qb = o / 270;
                const double *pt = S.pt[q0 + qb];
                const T *Nb = &S.N[qb][b][1];
                T s = T(0);
                if (m == 9) {
                    s = T(pt[GP_MASS]) * S.N[qb][b][0];
                } else if (m < 3) {
                    const double *sig = pt + GP_SIG, *d1s = pt + GP_D1S, *tau = pt + GP_TAU;
                    const int o1 = (m + 1) % 3, o2 = (m + 2) % 3;
                    const int p1 = (m == 0 || o1 == 0) ? ((m + o1 == 1) ? 0 : 1) : 2;
                    const int p2 = (m == 0 || o2 == 0) ? ((m + o2 == 1) ? 0 : 1) : 2;
                    s = T(sig[m]) * Nb[m] + T(0.5 * d1s[p1]) * Nb[o1] + T(0.5 * d1s[p2]) * Nb[o2];
                    for (int K = 0; K < 3; K++) s += T(tau[3 * m + K]) * Nb[3 + igab_idx6(m, K)];
                } else {
                    const double *tau = pt + GP_TAU;
                    const int c = m - 3;
                    for (int I = 0; I < 3; I++)
                        for (int K = 0; K < 3; K++)
                            if (igab_idx6(I, K) == c) s += T(tau[3 * I + K]) * Nb[I];
                }
                S.GN[qb][m][b] = s;
            }
            __syncthreads();
            /* (c) Y = w M X */
            for (int o = tid; o < GQ * GNV * 81; o += 256) {
                const int c = o % 81, r = (o / 81) % GNV, qb = o / (81 * GNV);
                const double *pt = S.pt[q0 + qb];
                const int v = r >> 1, a = r & 1;
                T s;
                if (v == 1 || v == 2) {
                    const int rr = 2 * (v - 1) + a;
                    s = T(pt[GP_M12 + 4 * rr + 0]) * S.X[qb][2][c] + T(pt[GP_M12 + 4 * rr + 1]) * S.X[qb][3][c] +
                        T(pt[GP_M12 + 4 * rr + 2]) * S.X[qb][4][c] + T(pt[GP_M12 + 4 * rr + 3]) * S.X[qb][5][c];
                } else {
                    const double m0 = a == 0 ? pt[GP_MD + 3 * v] : pt[GP_MD + 3 * v + 1];
                    const double m1 = a == 0 ? pt[GP_MD + 3 * v + 1] : pt[GP_MD + 3 * v + 2];
                    s = T(m0) * S.X[qb][2 * v][c] + T(m1) * S.X[qb][2 * v + 1][c];
                }
                S.Y[qb][r][c] = T(pt[GP_W]) * s;
            }
            __syncthreads();
            /* (d) owned entries */
#pragma unroll
            for (int j = 0; j < GOWN; j++) {
                if (own[j] < 0) continue;
                int c1 = own[j] >> 8, c2 = own[j] & 255;
                T s = acc[j];
                for (int qb = 0; qb < GQ; qb++)
#pragma unroll 8
                    for (int r = 0; r < GNV; r++) s += S.X[qb][r][c1] * S.Y[qb][r][c2];
                acc[j] = s;
            }
#pragma unroll
            for (int j = 0; j < 2; j++) {
                if (gown[j] < 0) continue;
                int a1 = gown[j] >> 8, a2 = gown[j] & 255;
                T s = gacc[j];
                for (int qb = 0; qb < GQ; qb++) {
                    T t = S.N[qb][a1][0] * S.GN[qb][9][a2];
#pragma unroll
                    for (int m = 0; m < 9; m++) t += S.N[qb][a1][m + 1] * S.GN[qb][m][a2];
                    s += T(S.pt[q0 + qb][GP_W]) * t;
                }
                gacc[j] = s;
            }
            __syncthreads();
        }
        T *Gam = &S.X[0][0][0];
#pragma unroll
        for (int j = 0; j < 2; j++) {
            if (gown[j] < 0) continue;
            int a1 = gown[j] >> 8, a2 = gown[j] & 255;
            Gam[a1 * 27 + a2] = gacc[j];
            Gam[a2 * 27 + a1] = gacc[j];
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < GOWN; j++) {
            if (own[j] < 0) continue;
            int c1 = own[j] >> 8, c2 = own[j] & 255;
            int a1 = c1 / 3, k1 = c1 % 3, a2 = c2 / 3, k2 = c2 % 3;
            T val = acc[j];
            if (k1 == k2) val += Gam[a1 * 27 + a2];
            int x1 = Tl.e0[0] + lex + a1 / 9, y1 = Tl.e0[1] + ley + (a1 / 3) % 3, z1 = Tl.e0[2] + lez + a1 % 3;
            int x2 = Tl.e0[0] + lex + a2 / 9, y2 = Tl.e0[1] + ley + (a2 / 3) % 3, z2 = Tl.e0[2] + lez + a2 % 3;
            long r1 = 3 * cp_index(g, x1, y1, z1) + k1;
            vals[g.rowptr[r1] + csr_pos(g, x1, y1, z1, x2, y2, z2, k2)] += val;
            if (c1 != c2) {
                long r2 = 3 * cp_index(g, x2, y2, z2) + k2;
                vals[g.rowptr[r2] + csr_pos(g, x2, y2, z2, x1, y1, z1, k1)] += val;
            }
        }
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
    size_t sm = sizeof(gt_smem<T, 2>);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_getime<T, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    for (int colour = 0; colour < 8; colour++) {
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
