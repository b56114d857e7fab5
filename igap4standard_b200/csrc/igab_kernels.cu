/*
 * Element-assembly kernels for sm_100a (FP64 residual; FP64 / FP32 tangent).
 *
 * Schedule (both operators): the mesh is cut into tiles of TE^3 elements
 * (TE >= 2).  Tiles are coloured by the parity of their tile coordinates
 * (8 colours); two tiles of one colour are at least TE elements apart, so
 * the control points they touch are disjoint and one launch per colour can
 * read-modify-write the global residual / CSR values without atomics.  Inside
 * a tile the accumulation order is fixed, so results are bitwise repeatable.
 *
 * Residual (src/snesiga_Residual.c:99-174): per element, 64 threads, one per
 * Gauss point.  The field and its derivatives at the Gauss points come from
 * a sum-factorised interpolation (z, then y in shared memory, then x in
 * registers).  The test-function contraction runs the same factorisation
 * backwards, with the sums over the Gauss points of x, y and z done by warp
 * shuffles (reduce-scatter across the 4 lanes of a direction) and one
 * shared-memory step across the two warps.
 *
 * Tangent (src/snesiga_Tangent.c:99-190): per element, 256 threads.  With
 * the energy written as W = Phi(v(u)) over 12 variables (igab_math.cuh),
 *   K_e = sum_q w_q [ X_q^T Phi''_q X_q + blockdiag(Gamma_q) ],
 * X_q[v][(a,k)] = sum_m dv/du_{k,m} N_a^{m}(q), a rank-12 update per point
 * plus a geometric block shared by the three displacement components.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include "igab_internal.h"

#include "igab_device.cuh"

namespace {

/* ============================================================ residual */

template <int TE, int NL>
struct res_smem {
    static constexpr int TC = TE + 2;
    static constexpr int NCP = TC * TC * TC;
    double U[NL][NCP * 3];   /* history levels: t_{n+1}, t_n, t_{n-1} (transient) */
    double Racc[NCP * 3];
    double tab[3][TE][IGAB_TAB1D];
    double wh[3][TE][IGAB_NQ];
    double xq[3][TE][IGAB_NQ];
    double A[4][972];
    double C[4][864];
    double red[4][81];
    double Re[4][81];
};

/* field and derivatives at this thread's Gauss point from one staged level:
 * z then y contraction in shared memory, x in registers (sum factorisation) */
template <int TE, int NL>
__device__ __forceinline__ void res_interp(res_smem<TE, NL> &S, const double *__restrict__ Ul, int group, int gt,
                                           int lex, int ley, int lez, const double *Bx, const double *By,
                                           const double *Bz, int qx, int qy, int qz, double u[30])
{
    constexpr int TC = TE + 2;
    for (int o = gt; o < 972; o += 64) {
        int i = o % 3, kz = (o / 3) % 3, ay = (o / 9) % 3, ax = (o / 27) % 3, q = o / 81;
        const double *u0 = &Ul[(((lex + ax) * TC + (ley + ay)) * TC + lez) * 3 + i];
        S.A[group][o] = Bz[q * 9 + 0 * 3 + kz] * u0[0] + Bz[q * 9 + 1 * 3 + kz] * u0[3] + Bz[q * 9 + 2 * 3 + kz] * u0[6];
    }
    group_sync(group);
    for (int o = gt; o < 864; o += 64) {
        int i = o % 3, kk = (o / 3) % 6, ax = (o / 18) % 3, qq = o / 54;
        int qyy = qq & 3, qzz = qq >> 2;
        int ky = kk_ky(kk), kz = kk_kz(kk);
        const double *a0 = &S.A[group][((qzz * 3 + ax) * 3) * 9 + kz * 3 + i];
        S.C[group][o] = By[qyy * 9 + 0 * 3 + ky] * a0[0] + By[qyy * 9 + 1 * 3 + ky] * a0[9] + By[qyy * 9 + 2 * 3 + ky] * a0[18];
    }
    group_sync(group);
    const int qq = qy + 4 * qz;
#pragma unroll
    for (int a = 0; a < 10; a++) {
#pragma unroll
        for (int i = 0; i < 3; i++) {
            double s = 0.0;
#pragma unroll
            for (int ax = 0; ax < 3; ax++) s += Bx[qx * 9 + ax * 3 + a_kx(a)] * S.C[group][((qq * 3 + ax) * 6 + a_kk(a)) * 3 + i];
            u[10 * i + a] = s;
        }
    }
    group_sync(group);   /* A and C are reused by the next level */
}

__device__ __forceinline__ void add_periodic(const igab_geom &g, const double X[3], double u[30])
{
#pragma unroll
    for (int i = 0; i < 3; i++) {
        u[10 * i] += g.pp[3 * i] * X[0] + g.pp[3 * i + 1] * X[1] + g.pp[3 * i + 2] * X[2];
#pragma unroll
        for (int J = 0; J < 3; J++) u[10 * i + 1 + J] += g.pp[3 * i + J];
    }
}

/* VJP = false: add the tile's element residuals into R.
 * VJP = true: adjoint mode; nothing is added to R, instead grad[e] = lam_e . R_e
 * for every element of the tile (lam with Dirichlet rows already zeroed), i.e.
 * the vector-Jacobian product lam^T dR/dg_e of the scaled residual. */
template <int TE, bool GT, bool VJP>
__device__ __forceinline__ void res_tile(const igab_geom &g, const tile_t &T, const double *__restrict__ U,
                                         double *__restrict__ R, const double *__restrict__ lam,
                                         double *__restrict__ grad, res_smem<TE, GT ? 3 : 1> &S)
{
    constexpr int NL = GT ? 3 : 1;
    constexpr int TC = TE + 2;
    constexpr int NCP = TC * TC * TC;
    constexpr int NEL = TE * TE * TE;
    const int tid = threadIdx.x;

    /* ---- stage control-point values (all history levels) and 1-D tables of the tile */
    for (int idx = tid; idx < NCP * 3; idx += blockDim.x) {
        int i = idx % 3, cp = idx / 3;
        int lz = cp % TC, ly = (cp / TC) % TC, lx = cp / (TC * TC);
        const bool in = lx < T.nv[0] + 2 && ly < T.nv[1] + 2 && lz < T.nv[2] + 2;
        const long gi = in ? 3 * cp_index(g, T.e0[0] + lx, T.e0[1] + ly, T.e0[2] + lz) + i : 0;
#pragma unroll
        for (int l = 0; l < NL; l++) {
            const double *src = l == 0 ? U : (l == 1 ? g.hist1 : g.hist0);
            S.U[l][idx] = in ? src[gi] : 0.0;
        }
        S.Racc[idx] = VJP ? (in ? lam[gi] : 0.0) : 0.0;   /* adjoint mode keeps lam here */
    }
    for (int idx = tid; idx < 3 * TE * IGAB_TAB1D; idx += blockDim.x) {
        int d = idx / (TE * IGAB_TAB1D), r = idx % (TE * IGAB_TAB1D), le = r / IGAB_TAB1D, o = r % IGAB_TAB1D;
        S.tab[d][le][o] = le < T.nv[d] ? g.tab[d][(long)(T.e0[d] + le) * IGAB_TAB1D + o] : 0.0;
    }
    for (int idx = tid; idx < 3 * TE * IGAB_NQ; idx += blockDim.x) {
        int d = idx / (TE * IGAB_NQ), r = idx % (TE * IGAB_NQ), le = r / IGAB_NQ, q = r % IGAB_NQ;
        bool ok = le < T.nv[d];
        S.wh[d][le][q] = ok ? g.wh[d][(long)(T.e0[d] + le) * IGAB_NQ + q] : 0.0;
        S.xq[d][le][q] = ok ? g.xq[d][(long)(T.e0[d] + le) * IGAB_NQ + q] : 0.0;
    }
    __syncthreads();

    const int group = tid >> 6;
    const int gt = tid & 63;
    const int qx = gt & 3, qy = (gt >> 2) & 3, qz = gt >> 4;

    for (int base = 0; base < NEL; base += 4) {
        const int le = base + group;
        const int lex = le / (TE * TE), ley = (le / TE) % TE, lez = le % TE;
        const bool valid = lex < T.nv[0] && ley < T.nv[1] && lez < T.nv[2];
        if (valid) {
            const double *Bx = S.tab[0][lex];
            const double *By = S.tab[1][ley];
            const double *Bz = S.tab[2][lez];
            double u[30];
            const double X[3] = {S.xq[0][lex][qx], S.xq[1][ley][qy], S.xq[2][lez][qz]};
            res_interp<TE, NL>(S, S.U[0], group, gt, lex, ley, lez, Bx, By, Bz, qx, qy, qz, u);
            if (g.periodic) add_periodic(g, X, u);
            /* integrand */
            double r[30];
            if (GT) {
                double u1[30], u0[30];
                res_interp<TE, NL>(S, S.U[NL > 1 ? 1 : 0], group, gt, lex, ley, lez, Bx, By, Bz, qx, qy, qz, u1);
                res_interp<TE, NL>(S, S.U[NL > 2 ? 2 : 0], group, gt, lex, ley, lez, Bx, By, Bz, qx, qy, qz, u0);
                if (g.periodic) {
                    add_periodic(g, X, u1);
                    add_periodic(g, X, u0);
                }
                igab_getime_residual(u, u1, u0, g.coef, g.rho, g.cii, g.dt, r);
            } else {
                igab_ge_point<double> P;
                igab_ge_eval(u, g.coef, P);
                igab_ge_residual(P, r);
            }
            const double w = S.wh[0][lex][qx] * S.wh[1][ley][qy] * S.wh[2][lez][qz] *
                             elem_scale(g, T.e0[0] + lex, T.e0[1] + ley, T.e0[2] + lez);
#pragma unroll
            for (int k = 0; k < 30; k++) r[k] *= w;

            /* backward step 1: partial sums over x for this point, P1[ax][kk][i] */
            double P1[3][18];
#pragma unroll
            for (int ax = 0; ax < 3; ax++)
#pragma unroll
                for (int s = 0; s < 18; s++) P1[ax][s] = 0.0;
#pragma unroll
            for (int a = 0; a < 10; a++)
#pragma unroll
                for (int ax = 0; ax < 3; ax++) {
                    double b = Bx[qx * 9 + ax * 3 + a_kx(a)];
#pragma unroll
                    for (int i = 0; i < 3; i++) P1[ax][a_kk(a) * 3 + i] += b * r[10 * i + a];
                }
            /* reduce-scatter over the 4 x-lanes: lane qx keeps ax = qx (qx < 3) */
            const int b1 = (qx >> 1) & 1, b0 = qx & 1;
#pragma unroll
            for (int s = 0; s < 18; s++) {
                double x1 = b1 ? P1[0][s] : P1[2][s];
                double y1 = shfl_xor(x1, 2);
                double x2 = b1 ? P1[1][s] : 0.0;
                double y2 = shfl_xor(x2, 2);
                if (b1) P1[2][s] += y1; else { P1[0][s] += y1; P1[1][s] += y2; }
            }
            double Y[18];
#pragma unroll
            for (int s = 0; s < 18; s++) {
                double x = b1 ? P1[2][s] : (b0 ? P1[0][s] : P1[1][s]);
                double y = shfl_xor(x, 1);
                double mine = b1 ? P1[2][s] : (b0 ? P1[1][s] : P1[0][s]);
                Y[s] = mine + y;
            }
            /* backward step 2: contract y for ax = qx; P2[ay][kz][i] */
            double P2[3][9];
#pragma unroll
            for (int ay = 0; ay < 3; ay++)
#pragma unroll
                for (int s = 0; s < 9; s++) P2[ay][s] = 0.0;
#pragma unroll
            for (int kk = 0; kk < 6; kk++)
#pragma unroll
                for (int ay = 0; ay < 3; ay++) {
                    double b = By[qy * 9 + ay * 3 + kk_ky(kk)];
#pragma unroll
                    for (int i = 0; i < 3; i++) P2[ay][kk_kz(kk) * 3 + i] += b * Y[kk * 3 + i];
                }
            /* reduce-scatter over the 4 y-lanes (lane bits 2,3): lane qy keeps ay = qy */
            const int c1 = (qy >> 1) & 1, c0 = qy & 1;
#pragma unroll
            for (int s = 0; s < 9; s++) {
                double x1 = c1 ? P2[0][s] : P2[2][s];
                double y1 = shfl_xor(x1, 8);
                double x2 = c1 ? P2[1][s] : 0.0;
                double y2 = shfl_xor(x2, 8);
                if (c1) P2[2][s] += y1; else { P2[0][s] += y1; P2[1][s] += y2; }
            }
            double Z[9];
#pragma unroll
            for (int s = 0; s < 9; s++) {
                double x = c1 ? P2[2][s] : (c0 ? P2[0][s] : P2[1][s]);
                double y = shfl_xor(x, 4);
                double mine = c1 ? P2[2][s] : (c0 ? P2[1][s] : P2[0][s]);
                Z[s] = mine + y;
            }
            /* backward step 3: contract z for (ax, ay) = (qx, qy); sum over qz */
            double P3[9];
#pragma unroll
            for (int az = 0; az < 3; az++)
#pragma unroll
                for (int i = 0; i < 3; i++) {
                    double s = 0.0;
#pragma unroll
                    for (int kz = 0; kz < 3; kz++) s += Bz[qz * 9 + az * 3 + kz] * Z[kz * 3 + i];
                    P3[az * 3 + i] = s;
                }
#pragma unroll
            for (int s = 0; s < 9; s++) P3[s] += shfl_xor(P3[s], 16);
            const bool owner = qx < 3 && qy < 3 && (qz & 1) == 0;
            if (owner && qz == 2)
#pragma unroll
                for (int s = 0; s < 9; s++) S.red[group][(qx * 3 + qy) * 9 + s] = P3[s];
            group_sync(group);
            if (owner && qz == 0)
#pragma unroll
                for (int s = 0; s < 9; s++) S.Re[group][(qx * 3 + qy) * 9 + s] = P3[s] + S.red[group][(qx * 3 + qy) * 9 + s];
        }
        __syncthreads();
        if (VJP) {
            /* one warp per element: grad_e = sum_k Re[k] lam[k], fixed order */
            const int w = tid >> 5, lane = tid & 31;
            if (w < 4) {
                const int e = base + w;
                const int ex = e / (TE * TE), ey = (e / TE) % TE, ez = e % TE;
                if (e < NEL && ex < T.nv[0] && ey < T.nv[1] && ez < T.nv[2]) {
                    double s = 0.0;
                    for (int k = lane; k < 81; k += 32) {
                        const int i = k % 3, az = (k / 3) % 3, ay = (k / 9) % 3, ax = k / 27;
                        s += S.Re[w][k] * S.Racc[(((ex + ax) * TC + (ey + ay)) * TC + (ez + az)) * 3 + i];
                    }
#pragma unroll
                    for (int m = 16; m >= 1; m >>= 1) s += shfl_xor(s, m);
                    if (lane == 0)
                        grad[((long)(T.e0[0] + ex) * g.ne[1] + (T.e0[1] + ey)) * g.ne[2] + (T.e0[2] + ez)] = s;
                }
            }
            __syncthreads();
            continue;
        }
        /* ---- fixed-order accumulation of the (up to) 4 element vectors into the tile */
        for (int idx = tid; idx < NCP * 3; idx += blockDim.x) {
            int i = idx % 3, cp = idx / 3;
            int lz = cp % TC, ly = (cp / TC) % TC, lx = cp / (TC * TC);
            double acc = S.Racc[idx];
            for (int gg = 0; gg < 4; gg++) {
                int e = base + gg;
                if (e >= NEL) break;
                int ex = e / (TE * TE), ey = (e / TE) % TE, ez = e % TE;
                if (ex >= T.nv[0] || ey >= T.nv[1] || ez >= T.nv[2]) continue;
                int ax = lx - ex, ay = ly - ey, az = lz - ez;
                if (ax < 0 || ax > 2 || ay < 0 || ay > 2 || az < 0 || az > 2) continue;
                acc += S.Re[gg][((ax * 3 + ay) * 3 + az) * 3 + i];
            }
            S.Racc[idx] = acc;
        }
        __syncthreads();
    }
    if (VJP) return;
    /* ---- add the tile into the global residual (no other tile of this colour touches these points) */
    for (int idx = tid; idx < NCP * 3; idx += blockDim.x) {
        int i = idx % 3, cp = idx / 3;
        int lz = cp % TC, ly = (cp / TC) % TC, lx = cp / (TC * TC);
        if (lx < T.nv[0] + 2 && ly < T.nv[1] + 2 && lz < T.nv[2] + 2) {
            long gi = 3 * cp_index(g, T.e0[0] + lx, T.e0[1] + ly, T.e0[2] + lz) + i;
            R[gi] = __ldcg(&R[gi]) + S.Racc[idx];   /* L2 read: another CTA may have written it */
        }
    }
}

template <int TE, bool GT, bool VJP>
__global__ void __launch_bounds__(256) k_res_volume(igab_geom g, const double *__restrict__ U,
                                                    double *__restrict__ R, int colour,
                                                    const double *__restrict__ lam, double *__restrict__ grad)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    res_smem<TE, GT ? 3 : 1> &S = *reinterpret_cast<res_smem<TE, GT ? 3 : 1> *>(smem_raw);
    tile_t T;
    if (!decode_tile(g, TE, colour, blockIdx.x, T)) return;
    res_tile<TE, GT, VJP>(g, T, U, R, lam, grad, S);
}

/* Neumann surface terms (src/snesiga_Residual.c:243-320): one thread per
 * boundary dof, gathering every active (face, order) combo that reaches it. */
__global__ void k_res_neumann(igab_geom g, long nrows, const int *__restrict__ row_dof,
                              const int *__restrict__ ptr, const int4 *__restrict__ ent,
                              const int *__restrict__ cinfo, const double *__restrict__ dnz,
                              const double *__restrict__ hval, double *__restrict__ R)
{
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= nrows) return;
    double acc = 0.0;
    for (int k = ptr[t]; k < ptr[t + 1]; k++) {
        int4 e = ent[k];   /* (combo, layer slot, bx, by) */
        const int *ci = cinfo + 8 * e.x;
        int face = ci[0], order = ci[1], ne0 = ci[3], ne1 = ci[4];
        long off = (long)(unsigned)ci[5] | ((long)ci[6] << 32);
        int d0 = ci[7] & 3, d1 = (ci[7] >> 2) & 3;
        double fz = order ? dnz[face * 2 + e.y] : 1.0;
        int bx = e.z, by = e.w;
        double s = 0.0;
        for (int ex = bx - 2 > 0 ? bx - 2 : 0; ex <= bx && ex < ne0; ex++)
            for (int ey = by - 2 > 0 ? by - 2 : 0; ey <= by && ey < ne1; ey++) {
                const double *t0 = g.tab[d0] + (long)ex * IGAB_TAB1D;
                const double *t1 = g.tab[d1] + (long)ey * IGAB_TAB1D;
                const double *w0 = g.wh[d0] + (long)ex * IGAB_NQ;
                const double *w1 = g.wh[d1] + (long)ey * IGAB_NQ;
                const double *h = hval + off + ((long)ex * ne1 + ey) * 16;
                for (int q0 = 0; q0 < 4; q0++)
                    for (int q1 = 0; q1 < 4; q1++)
                        s += w0[q0] * w1[q1] * t0[q0 * 9 + (bx - ex) * 3] * t1[q1 * 9 + (by - ey) * 3] * h[q0 * 4 + q1];
            }
        acc -= fz * s;
    }
    R[row_dof[t]] += acc;
}

/* Dirichlet rows R = U - g, written after all additions (src/snesiga_Residual.c:326-412) */
__global__ void k_res_dirichlet(long nd, const int *__restrict__ drow, const double *__restrict__ dg,
                                const double *__restrict__ U, double *__restrict__ R)
{
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= nd) return;
    int r = drow[t];
    R[r] = U[r] - dg[t];
}

/* ============================================================ tangent */

#define TAN_Q 4          /* Gauss points per batch */
#define TAN_NPT 56       /* doubles of point data */
#define TAN_NOWN 13      /* upper-triangle entries owned per thread (3321 / 256) */

template <typename T, int TE>
struct tan_smem {
    static constexpr int TC = TE + 2;
    static constexpr int NCP = TC * TC * TC;
    double U[NCP * 3];
    double tab[3][TE][IGAB_TAB1D];
    double wh[3][TE][IGAB_NQ];
    double xq[3][TE][IGAB_NQ];
    double A[972];
    double C[864];
    double pt[IGAB_NQ3][TAN_NPT];   /* F 9, G 18, d2 12, d2ab 1, sig 3, d1[3..5] 3, tau 9, w 1 */
    T N[TAN_Q][27][9];              /* N_a^{m+1} */
    T Gv[TAN_Q][12][27];            /* dv/du_s */
    T X[TAN_Q][12][81];
    T Y[TAN_Q][12][81];
    T GN[TAN_Q][9][27];             /* geo * N */
};

/* point data offsets */
#define PT_F 0
#define PT_G 9
#define PT_D2 27
#define PT_D2AB 39
#define PT_SIG 40
#define PT_D1S 43
#define PT_TAU 46
#define PT_W 55

template <typename T>
__device__ __forceinline__ void load_point(const double *pt, igab_ge_point<T> &P)
{
    for (int k = 0; k < 3; k++)
        for (int J = 0; J < 3; J++) P.F[k][J] = T(pt[PT_F + 3 * k + J]);
    for (int k = 0; k < 3; k++)
        for (int c = 0; c < 6; c++) P.G[k][c] = T(pt[PT_G + 6 * k + c]);
}

template <typename T, int TE>
__global__ void __launch_bounds__(256) k_tan_volume(igab_geom g, const double *__restrict__ U,
                                                    T *__restrict__ vals, int colour)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    tan_smem<T, TE> &S = *reinterpret_cast<tan_smem<T, TE> *>(smem_raw);
    constexpr int TC = TE + 2;
    constexpr int NCP = TC * TC * TC;
    constexpr int NEL = TE * TE * TE;
    tile_t Tl;
    if (!decode_tile(g, TE, colour, blockIdx.x, Tl)) return;
    const int tid = threadIdx.x;

    /* owned upper-triangle entries (c1 <= c2), c = 3a + k */
    int own[TAN_NOWN];
#pragma unroll
    for (int j = 0; j < TAN_NOWN; j++) {
        int idx = tid + 256 * j;
        int c1 = 0, rem = idx;
        while (c1 < 81 && rem >= 81 - c1) { rem -= 81 - c1; c1++; }
        own[j] = c1 < 81 ? (c1 << 8) | (c1 + rem) : -1;
    }
    /* owned geometric entries (a1 <= a2), 378 */
    int gown[2];
#pragma unroll
    for (int j = 0; j < 2; j++) {
        int idx = tid + 256 * j;
        int a1 = 0, rem = idx;
        while (a1 < 27 && rem >= 27 - a1) { rem -= 27 - a1; a1++; }
        gown[j] = a1 < 27 ? (a1 << 8) | (a1 + rem) : -1;
    }

    for (int idx = tid; idx < NCP * 3; idx += blockDim.x) {
        int i = idx % 3, cp = idx / 3;
        int lz = cp % TC, ly = (cp / TC) % TC, lx = cp / (TC * TC);
        double v = 0.0;
        if (lx < Tl.nv[0] + 2 && ly < Tl.nv[1] + 2 && lz < Tl.nv[2] + 2)
            v = U[3 * cp_index(g, Tl.e0[0] + lx, Tl.e0[1] + ly, Tl.e0[2] + lz) + i];
        S.U[idx] = v;
    }
    for (int idx = tid; idx < 3 * TE * IGAB_TAB1D; idx += blockDim.x) {
        int d = idx / (TE * IGAB_TAB1D), r = idx % (TE * IGAB_TAB1D), le = r / IGAB_TAB1D, o = r % IGAB_TAB1D;
        S.tab[d][le][o] = le < Tl.nv[d] ? g.tab[d][(long)(Tl.e0[d] + le) * IGAB_TAB1D + o] : 0.0;
    }
    for (int idx = tid; idx < 3 * TE * IGAB_NQ; idx += blockDim.x) {
        int d = idx / (TE * IGAB_NQ), r = idx % (TE * IGAB_NQ), le = r / IGAB_NQ, q = r % IGAB_NQ;
        bool ok = le < Tl.nv[d];
        S.wh[d][le][q] = ok ? g.wh[d][(long)(Tl.e0[d] + le) * IGAB_NQ + q] : 0.0;
        S.xq[d][le][q] = ok ? g.xq[d][(long)(Tl.e0[d] + le) * IGAB_NQ + q] : 0.0;
    }
    __syncthreads();

    for (int le = 0; le < NEL; le++) {
        const int lex = le / (TE * TE), ley = (le / TE) % TE, lez = le % TE;
        if (!(lex < Tl.nv[0] && ley < Tl.nv[1] && lez < Tl.nv[2])) continue;   /* uniform over the block */
        const double *Bx = S.tab[0][lex];
        const double *By = S.tab[1][ley];
        const double *Bz = S.tab[2][lez];
        /* ---- interpolation (as the residual, all 256 threads for stages A and C) */
        for (int o = tid; o < 972; o += 256) {
            int i = o % 3, kz = (o / 3) % 3, ay = (o / 9) % 3, ax = (o / 27) % 3, q = o / 81;
            const double *u0 = &S.U[(((lex + ax) * TC + (ley + ay)) * TC + lez) * 3 + i];
            S.A[o] = Bz[q * 9 + kz] * u0[0] + Bz[q * 9 + 3 + kz] * u0[3] + Bz[q * 9 + 6 + kz] * u0[6];
        }
        __syncthreads();
        for (int o = tid; o < 864; o += 256) {
            int i = o % 3, kk = (o / 3) % 6, ax = (o / 18) % 3, qq = o / 54;
            int qyy = qq & 3, qzz = qq >> 2;
            int ky = kk_ky(kk), kz = kk_kz(kk);
            const double *a0 = &S.A[((qzz * 3 + ax) * 3) * 9 + kz * 3 + i];
            S.C[o] = By[qyy * 9 + ky] * a0[0] + By[qyy * 9 + 3 + ky] * a0[9] + By[qyy * 9 + 6 + ky] * a0[18];
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
            igab_ge_point<T> P;
            T uT[30];
#pragma unroll
            for (int k = 0; k < 30; k++) uT[k] = T(u[k]);
            igab_ge_eval(uT, g.coef, P);
            double *pt = S.pt[tid];
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int J = 0; J < 3; J++) pt[PT_F + 3 * k + J] = double(P.F[k][J]);
#pragma unroll
            for (int k = 0; k < 3; k++)
#pragma unroll
                for (int c = 0; c < 6; c++) pt[PT_G + 6 * k + c] = double(P.G[k][c]);
#pragma unroll
            for (int v = 0; v < 12; v++) pt[PT_D2 + v] = double(P.d2[v]);
            pt[PT_D2AB] = double(P.d2ab);
#pragma unroll
            for (int I = 0; I < 3; I++) pt[PT_SIG + I] = double(P.sig[I]);
#pragma unroll
            for (int I = 0; I < 3; I++) pt[PT_D1S + I] = double(P.d1[3 + I]);
#pragma unroll
            for (int I = 0; I < 3; I++)
#pragma unroll
                for (int K = 0; K < 3; K++) pt[PT_TAU + 3 * I + K] = double(P.tau[I][K]);
            pt[PT_W] = S.wh[0][lex][qx] * S.wh[1][ley][qy] * S.wh[2][lez][qz] *
                       elem_scale(g, Tl.e0[0] + lex, Tl.e0[1] + ley, Tl.e0[2] + lez);
        }
        __syncthreads();

        T acc[TAN_NOWN];
#pragma unroll
        for (int j = 0; j < TAN_NOWN; j++) acc[j] = T(0);
        T gacc[2] = {T(0), T(0)};

        for (int q0 = 0; q0 < IGAB_NQ3; q0 += TAN_Q) {
            /* (a) basis products and variable gradients for the batch */
            for (int o = tid; o < TAN_Q * 27 * 9; o += 256) {
                int m = o % 9, a = (o / 9) % 27, qb = o / 243;
                int q = q0 + qb, qx = q & 3, qy = (q >> 2) & 3, qz = q >> 4;
                int ax = a / 9, ay = (a / 3) % 3, az = a % 3;
                int al = m + 1;
                double v = Bx[qx * 9 + ax * 3 + a_kx(al)] * By[qy * 9 + ay * 3 + a_ky(al)] * Bz[qz * 9 + az * 3 + a_kz(al)];
                S.N[qb][a][m] = T(v);
            }
            for (int o = tid; o < TAN_Q * 12 * 3; o += 256) {
                int k = o % 3, v = (o / 3) % 12, qb = o / 36;
                igab_ge_point<T> P;
                load_point(S.pt[q0 + qb], P);
                T gg[9];
                igab_ge_grad_var(P, v, k, gg);
#pragma unroll
                for (int m = 0; m < 9; m++) S.Gv[qb][v][9 * k + m] = gg[m];
            }
            /* geometric block times N: GN[m][b] = sum_n geo[m][n] N_b^{n} */
            for (int o = tid; o < TAN_Q * 9 * 27; o += 256) {
                int b = o % 27, m = (o / 27) % 9, qb = o / 243;
                const double *pt = S.pt[q0 + qb];
                T s = T(0);
                if (m < 3) {
                    s = T(pt[PT_SIG + m]) * S.N[qb][b][m];
                    int o1 = (m + 1) % 3, o2 = (m + 2) % 3;
                    /* off-diagonal E terms: (0,1)->d1[3], (0,2)->d1[4], (1,2)->d1[5] */
                    int pr1 = (m == 0 || o1 == 0) ? ((m + o1 == 1) ? 0 : 1) : 2;
                    int pr2 = (m == 0 || o2 == 0) ? ((m + o2 == 1) ? 0 : 1) : 2;
                    s += T(0.5) * T(pt[PT_D1S + pr1]) * S.N[qb][b][o1];
                    s += T(0.5) * T(pt[PT_D1S + pr2]) * S.N[qb][b][o2];
                    for (int K = 0; K < 3; K++) s += T(pt[PT_TAU + 3 * m + K]) * S.N[qb][b][3 + igab_idx6(m, K)];
                } else {
                    int c = m - 3;
                    for (int I = 0; I < 3; I++)
                        for (int K = 0; K < 3; K++)
                            if (igab_idx6(I, K) == c) s += T(pt[PT_TAU + 3 * I + K]) * S.N[qb][b][I];
                }
                S.GN[qb][m][b] = s;
            }
            __syncthreads();
            /* (b) X = Gv . N and Y = w Phi'' X */
            for (int o = tid; o < TAN_Q * 12 * 81; o += 256) {
                int c = o % 81, v = (o / 81) % 12, qb = o / 972;
                int a = c / 3, k = c % 3;
                T s = T(0);
#pragma unroll
                for (int m = 0; m < 9; m++) s += S.Gv[qb][v][9 * k + m] * S.N[qb][a][m];
                S.X[qb][v][c] = s;
            }
            __syncthreads();
            for (int o = tid; o < TAN_Q * 12 * 81; o += 256) {
                int c = o % 81, v = (o / 81) % 12, qb = o / 972;
                const double *pt = S.pt[q0 + qb];
                T w = T(pt[PT_W]);
                T s = T(pt[PT_D2 + v]) * S.X[qb][v][c];
                if (v == 1) s += T(pt[PT_D2AB]) * S.X[qb][2][c];
                if (v == 2) s += T(pt[PT_D2AB]) * S.X[qb][1][c];
                S.Y[qb][v][c] = w * s;
            }
            __syncthreads();
            /* (c) accumulate owned entries */
#pragma unroll
            for (int j = 0; j < TAN_NOWN; j++) {
                if (own[j] < 0) continue;
                int c1 = own[j] >> 8, c2 = own[j] & 255;
                T s = acc[j];
                for (int qb = 0; qb < TAN_Q; qb++)
#pragma unroll
                    for (int v = 0; v < 12; v++) s += S.X[qb][v][c1] * S.Y[qb][v][c2];
                acc[j] = s;
            }
#pragma unroll
            for (int j = 0; j < 2; j++) {
                if (gown[j] < 0) continue;
                int a1 = gown[j] >> 8, a2 = gown[j] & 255;
                T s = gacc[j];
                for (int qb = 0; qb < TAN_Q; qb++) {
                    T w = T(S.pt[q0 + qb][PT_W]);
                    T t = T(0);
#pragma unroll
                    for (int m = 0; m < 9; m++) t += S.N[qb][a1][m] * S.GN[qb][m][a2];
                    s += w * t;
                }
                gacc[j] = s;
            }
            __syncthreads();
        }
        /* geometric block to shared memory (reuse X) */
        T *Gam = &S.X[0][0][0];
#pragma unroll
        for (int j = 0; j < 2; j++) {
            if (gown[j] < 0) continue;
            int a1 = gown[j] >> 8, a2 = gown[j] & 255;
            Gam[a1 * 27 + a2] = gacc[j];
            Gam[a2 * 27 + a1] = gacc[j];
        }
        __syncthreads();
        /* ---- scatter into the CSR values (read-modify-write, conflict-free within a colour) */
#pragma unroll
        for (int j = 0; j < TAN_NOWN; j++) {
            if (own[j] < 0) continue;
            int c1 = own[j] >> 8, c2 = own[j] & 255;
            int a1 = c1 / 3, k1 = c1 % 3, a2 = c2 / 3, k2 = c2 % 3;
            T val = acc[j];
            if (k1 == k2) val += Gam[a1 * 27 + a2];
            int x1 = Tl.e0[0] + lex + a1 / 9, y1 = Tl.e0[1] + ley + (a1 / 3) % 3, z1 = Tl.e0[2] + lez + a1 % 3;
            int x2 = Tl.e0[0] + lex + a2 / 9, y2 = Tl.e0[1] + ley + (a2 / 3) % 3, z2 = Tl.e0[2] + lez + a2 % 3;
            long r1 = 3 * cp_index(g, x1, y1, z1) + k1;
            long o1 = g.rowptr[r1] + csr_pos(g, x1, y1, z1, x2, y2, z2, k2);
            vals[o1] += val;
            if (c1 != c2) {
                long r2 = 3 * cp_index(g, x2, y2, z2) + k2;
                long o2 = g.rowptr[r2] + csr_pos(g, x2, y2, z2, x1, y1, z1, k1);
                vals[o2] += val;
            }
        }
        __syncthreads();
    }
}

/* MatZeroRowsColumns(P, rows, 1.0) on the structured pattern (src/snesiga_Tangent.c:270):
 * one thread per (Dirichlet row, entry of that row); only entries in rows [r0, r1) are
 * written (every write to an entry writes the same value, so the rows may be done in parts). */
template <typename T>
__device__ __forceinline__ void tan_dirichlet_entry(const igab_geom &g, int r, int s, T *__restrict__ vals,
                                                    long r0 = 0, long r1 = 0x7fffffffffffffffL)
{
    int cp = r / 3;
    int z = cp % g.nb[2], y = (cp / g.nb[2]) % g.nb[1], x = cp / (g.nb[2] * g.nb[1]);
    int nc = g.rowptr[r + 1] - g.rowptr[r];
    if (s >= nc) return;
    int x0 = x > 2 ? x - 2 : 0;
    int y0 = y > 2 ? y - 2 : 0, y1 = y + 2 < g.nb[1] - 1 ? y + 2 : g.nb[1] - 1;
    int z0 = z > 2 ? z - 2 : 0, z1 = z + 2 < g.nb[2] - 1 ? z + 2 : g.nb[2] - 1;
    int nyb = y1 - y0 + 1, nzb = z1 - z0 + 1;
    int k2 = s % 3, q = s / 3;
    int cz = z0 + q % nzb, cy = y0 + (q / nzb) % nyb, cx = x0 + q / (nzb * nyb);
    long c = 3 * cp_index(g, cx, cy, cz) + k2;
    if (r >= r0 && r < r1) vals[g.rowptr[r] + s] = (c == r) ? T(1) : T(0);
    if (c != r && c >= r0 && c < r1) vals[g.rowptr[c] + csr_pos(g, cx, cy, cz, x, y, z, r % 3)] = T(0);
}

template <typename T>
__global__ void k_tan_dirichlet(igab_geom g, long nd, const int *__restrict__ drow, T *__restrict__ vals, long r0,
                                long r1)
{
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long j = t / 375;
    int s = (int)(t % 375);
    if (j >= nd) return;
    tan_dirichlet_entry<T>(g, drow[j], s, vals, r0, r1);
}

/* zero the Dirichlet rows of a CSR matrix (no column change, no diagonal): one thread per
 * (row, entry of that row) */
template <typename T>
__global__ void k_zero_csr_rows(igab_geom g, long nd, const int *__restrict__ drow, T *__restrict__ vals)
{
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long j = t / 375;
    int s = (int)(t % 375);
    if (j >= nd) return;
    const int r = drow[j];
    if (s < g.rowptr[r + 1] - g.rowptr[r]) vals[g.rowptr[r] + s] = T(0);
}

/* the same over the Dirichlet rows of all instances of a batch (row j of instance dinst[j]) */
template <typename T>
__global__ void k_tan_dirichlet_batch(igab_batch_dev B, long nd, const int *__restrict__ dinst,
                                      const int *__restrict__ drow, T *__restrict__ vals)
{
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long j = t / 375;
    int s = (int)(t % 375);
    if (j >= nd) return;
    const int inst = dinst[j];
    tan_dirichlet_entry<T>(B.geoms[inst], drow[j], s, vals + B.nnz_off[inst]);
}

/* persistent residual over the tiles of every instance of a batch (TE = 2, phys/ge) */
__global__ void __launch_bounds__(256, 2) k_res_batch(igab_batch_dev B, const double *__restrict__ U,
                                                   double *__restrict__ R)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    res_smem<2, 1> &S = *reinterpret_cast<res_smem<2, 1> *>(smem_raw);
    __shared__ batch_slot sl;
    while (batch_next(B, sl)) {
        tile_t T;
        decode_tile(sl.g, 2, sl.colour, sl.tile, T);
        const long off = B.dof_off[sl.inst];
        res_tile<2, false, false>(sl.g, T, U + off, R + off, nullptr, nullptr, S);
        batch_done(B, sl);
    }
}

/* column indices of the CSR pattern, one thread per row */
__global__ void k_csr_cols(igab_geom g, int *__restrict__ cols)
{
    long r = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (r >= g.ndof) return;
    int cp = (int)(r / 3);
    int z = cp % g.nb[2], y = (cp / g.nb[2]) % g.nb[1], x = cp / (g.nb[2] * g.nb[1]);
    int x0 = x > 2 ? x - 2 : 0, x1 = x + 2 < g.nb[0] - 1 ? x + 2 : g.nb[0] - 1;
    int y0 = y > 2 ? y - 2 : 0, y1 = y + 2 < g.nb[1] - 1 ? y + 2 : g.nb[1] - 1;
    int z0 = z > 2 ? z - 2 : 0, z1 = z + 2 < g.nb[2] - 1 ? z + 2 : g.nb[2] - 1;
    long o = g.rowptr[r];
    for (int cx = x0; cx <= x1; cx++)
        for (int cy = y0; cy <= y1; cy++)
            for (int cz = z0; cz <= z1; cz++)
                for (int k = 0; k < 3; k++) cols[o++] = (int)(3 * cp_index(g, cx, cy, cz) + k);
}

/* y = K^T x on the structured CSR values (vals).  One block per output
 * segment: control points (cx, cy, z) for z in [zlo, zhi], all 3 components.
 * Column (cx,cy,z,k) of K is held by the rows of the 25 neighbouring z-lines
 * (sx, sy); each such row stores its entries for line (cx, cy) as one
 * contiguous run of <= 15 values (5 z x 3 k, columns ascending).  The block
 * stages those runs line by line in shared memory with coalesced loads and
 * every output row sums its column in a fixed order. */
#define KT_ZMAX 32
template <typename T>
__global__ void __launch_bounds__(128) k_tangent_transpose(igab_geom g, const T *__restrict__ vals,
                                                           const double *__restrict__ x, double *__restrict__ y,
                                                           int nchunk)
{
    __shared__ T band[(KT_ZMAX + 4) * 3][15];
    __shared__ double xs[(KT_ZMAX + 4) * 3];
    const int nz = g.nb[2];
    const int chunk = blockIdx.x % nchunk;
    const int line = blockIdx.x / nchunk;
    const int cy = line % g.nb[1], cx = line / g.nb[1];
    const int zlo = (int)(((long)chunk * nz) / nchunk);
    const int zhi = (int)(((long)(chunk + 1) * nz) / nchunk) - 1;
    const int slo = zlo - 2 > 0 ? zlo - 2 : 0, shi = zhi + 2 < nz - 1 ? zhi + 2 : nz - 1;
    const int nsrc = (shi - slo + 1) * 3;
    const int tid = threadIdx.x;
    const int oz = zlo + tid / 3, ok = tid % 3;
    const bool owner = oz <= zhi;
    double acc = 0.0;
    const int sx0 = cx - 2 > 0 ? cx - 2 : 0, sx1 = cx + 2 < g.nb[0] - 1 ? cx + 2 : g.nb[0] - 1;
    const int sy0 = cy - 2 > 0 ? cy - 2 : 0, sy1 = cy + 2 < g.nb[1] - 1 ? cy + 2 : g.nb[1] - 1;
    for (int sx = sx0; sx <= sx1; sx++)
        for (int sy = sy0; sy <= sy1; sy++) {
            for (int idx = tid; idx < nsrc * 15; idx += blockDim.x) {
                const int r = idx / 15, t = idx % 15;
                const int sz = slo + r / 3, sk = r % 3;
                /* columns of this row inside line (cx,cy) and inside [zlo, zhi] */
                const int c0 = sz - 2 > zlo ? sz - 2 : zlo;
                const int c1 = sz + 2 < zhi ? sz + 2 : zhi;
                if (t < (c1 - c0 + 1) * 3) {
                    const long j = 3 * cp_index(g, sx, sy, sz) + sk;
                    band[r][(c0 - sz + 2) * 3 + t] = vals[g.rowptr[j] + csr_pos(g, sx, sy, sz, cx, cy, c0, 0) + t];
                }
            }
            for (int idx = tid; idx < nsrc; idx += blockDim.x)
                xs[idx] = x[3 * cp_index(g, sx, sy, slo + idx / 3) + idx % 3];
            __syncthreads();
            if (owner) {
                const int z0 = oz - 2 > 0 ? oz - 2 : 0, z1 = oz + 2 < nz - 1 ? oz + 2 : nz - 1;
                for (int sz = z0; sz <= z1; sz++)
#pragma unroll
                    for (int sk = 0; sk < 3; sk++) {
                        const int r = (sz - slo) * 3 + sk;
                        acc += double(band[r][(oz - sz + 2) * 3 + ok]) * xs[r];
                    }
            }
            __syncthreads();
        }
    if (owner) y[3 * cp_index(g, cx, cy, oz) + ok] = acc;
}

__global__ void k_exp_scale(const double *__restrict__ gl, double *__restrict__ s, long n)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) s[i] = exp(gl[i]);
}

/* lam with the Dirichlet rows zeroed (those rows of R do not depend on g) */
__global__ void k_zero_rows(long nd, const int *__restrict__ rows, double *__restrict__ v)
{
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t < nd) v[rows[t]] = 0.0;
}

template <typename T>
__global__ void k_check_finite(const T *__restrict__ v, long n, int *__restrict__ flag)
{
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    bool bad = false;
    for (; i < n; i += stride) bad |= !isfinite(v[i]);
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicExch(flag, 1);
}

template <int TE, bool GT, bool VJP = false>
int launch_res_volume_t(igab_ctx *c, const igab_geom &g, const double *dU, double *dR,
                        const double *dlam = nullptr, double *dgrad = nullptr)
{
    size_t sm = sizeof(res_smem<TE, GT ? 3 : 1>);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_res_volume<TE, GT, VJP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    for (int k = 0; k < 8; k++) {
        const int colour = igab_colour_at(c->colour_order, k);
        long nblk = tiles_of_colour(g, TE, colour);
        if (nblk == 0) continue;
        k_res_volume<TE, GT, VJP><<<(unsigned)nblk, 256, sm, c->stream>>>(g, dU, dR, colour, dlam, dgrad);
        c->last_launches++;
    }
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

template <typename T, int TE>
int launch_tan_volume(igab_ctx *c, const igab_geom &g, const double *dU, T *dv)
{
    size_t sm = sizeof(tan_smem<T, TE>);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_volume<T, TE>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    for (int k = 0; k < 8; k++) {
        const int colour = igab_colour_at(c->colour_order, k);
        long nblk = tiles_of_colour(g, TE, colour);
        if (nblk == 0) continue;
        k_tan_volume<T, TE><<<(unsigned)nblk, 256, sm, c->stream>>>(g, dU, dv, colour);
        c->last_launches++;
    }
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

/* the selected tangent volume kernels, over the x tiles [tx0, tx1) (tiles of 2 elements)
 * where the kernel takes a range, else over the whole mesh */
template <typename T>
int launch_tan_volume_x(igab_ctx *c, const igab_geom &g, const double *dU, T *dv, int tx0, int tx1)
{
    if (c->phys == IGAB_PHYS_GETIME)
        return igab_launch_tan_getime(c, dU, dv, sizeof(T) == 8 ? IGAB_PREC_FP64 : IGAB_PREC_FP32);
    if (sizeof(T) == 8 && c->tan_kernel == 1) return igab_launch_tan_dmma(c, dU, (double *)dv, tx0, tx1);
    if (sizeof(T) == 4 && c->tan32_kernel == 1) return igab_launch_tan_tc32(c, dU, (float *)dv, tx0, tx1);
    return launch_tan_volume<T, 2>(c, g, dU, dv);
}

template <typename T>
int launch_tan_dirichlet(igab_ctx *c, const igab_geom &g, T *dv, long r0, long r1)
{
    if (c->nd == 0) return 0;
    long n = c->nd * 375;
    k_tan_dirichlet<T><<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(g, c->nd, c->d_drow, dv, r0, r1);
    c->last_launches++;
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

template <typename T>
int launch_tangent_t(igab_ctx *c, const double *dU, T *dv)
{
    igab_geom g = c->geom();
    IGAB_CUDA_TRY(cudaMemsetAsync(dv, 0, (size_t)c->nnz * sizeof(T), c->stream));
    igab_mark(c, 3);
    int l0 = c->last_launches;
    int e = launch_tan_volume_x<T>(c, g, dU, dv, 0, (c->ne[0] + 1) / 2);
    if (e) return e;
    c->nvol_tan = c->last_launches - l0;
    igab_mark(c, 4);
    if ((e = launch_tan_dirichlet<T>(c, g, dv, 0, c->ndof))) return e;
    igab_mark(c, 5);
    c->ev_tan = c->profiling;
    return 0;
}

/* x-slab boundaries (odd tile coordinates, increasing) of the host-pointer tangent:
 * slabs of 8 tiles, then 4, 2, 2 and 1 (or 2) tiles at the end, so that the rows
 * finished last, whose download cannot overlap any compute, are few.  None below
 * 12 tiles. */
int slab_bounds(int ntx, int *b)
{
    if (ntx < 12) return 0;
    int tmp[IGAB_MAX_SLABS], n = 0;
    int x = (ntx - 1) % 2 == 1 ? ntx - 1 : ntx - 2;
    tmp[n++] = x;
    const int tail[3] = {2, 2, 4};
    for (int i = 0; i < 3; i++) {
        if (x - tail[i] < 8) break;
        x -= tail[i];
        tmp[n++] = x;
    }
    while (x - 8 >= 8 && n < IGAB_MAX_SLABS - 1) {
        x -= 8;
        tmp[n++] = x;
    }
    for (int i = 0; i < n; i++) b[i] = tmp[n - 1 - i];
    return n;
}

template <typename T>
int launch_tangent_slabs_t(igab_ctx *c, const double *dU, T *dv, long *row_end, int *nslab)
{
    igab_geom g = c->geom();
    const int ntx = (c->ne[0] + 1) / 2;
    int b[IGAB_MAX_SLABS];
    const bool ranged = c->phys != IGAB_PHYS_GETIME && (sizeof(T) == 8 ? c->tan_kernel == 1 : c->tan32_kernel == 1);
    const int nb = ranged ? slab_bounds(ntx, b) : 0;
    for (int i = 0; i <= nb; i++)
        if (!c->slab_ev[i]) IGAB_CUDA_TRY(cudaEventCreateWithFlags(&c->slab_ev[i], cudaEventDisableTiming));
    IGAB_CUDA_TRY(cudaMemsetAsync(dv, 0, (size_t)c->nnz * sizeof(T), c->stream));
    igab_mark(c, 3);
    int nvol = 0;
    const long plane = 3L * c->nb[1] * c->nb[2];   /* rows per control-point layer in x */
    long r0 = 0;
    for (int i = 0; i <= nb; i++) {
        const int tx0 = i ? b[i - 1] : 0, tx1 = i < nb ? b[i] : ntx;
        const int lv = c->last_launches;
        int e = launch_tan_volume_x<T>(c, g, dU, dv, tx0, tx1);
        if (e) return e;
        nvol += c->last_launches - lv;
        if (i == nb) igab_mark(c, 4);
        /* control points below x = 2 tx1 are touched by no element of a later slab */
        const long r1 = i < nb ? 2L * tx1 * plane : c->ndof;
        if ((e = launch_tan_dirichlet<T>(c, g, dv, r0, r1))) return e;
        IGAB_CUDA_TRY(cudaEventRecord(c->slab_ev[i], c->stream));
        row_end[i] = r1;
        r0 = r1;
    }
    c->nvol_tan = nvol;
    igab_mark(c, 5);
    c->ev_tan = c->profiling;
    *nslab = nb + 1;
    return 0;
}

} /* namespace */

int igab_launch_residual(igab_ctx *c, const double *dU, double *dR)
{
    c->last_launches = 0;
    igab_geom g = c->geom();
    IGAB_CUDA_TRY(cudaMemsetAsync(dR, 0, (size_t)c->ndof * sizeof(double), c->stream));
    igab_mark(c, 0);
    int e;
    if (c->phys == IGAB_PHYS_GETIME)
        e = c->tile_res == 4 ? launch_res_volume_t<4, true>(c, g, dU, dR) : launch_res_volume_t<2, true>(c, g, dU, dR);
    else
        e = c->tile_res == 4 ? launch_res_volume_t<4, false>(c, g, dU, dR) : launch_res_volume_t<2, false>(c, g, dU, dR);
    if (e) return e;
    c->nvol_res = c->last_launches;
    igab_mark(c, 1);
    if ((c->neumann_nonzero || c->force_neumann) && c->n_neu_rows > 0) {
        k_res_neumann<<<(unsigned)((c->n_neu_rows + 127) / 128), 128, 0, c->stream>>>(
            g, c->n_neu_rows, c->d_neu_row, c->d_neu_ptr, c->d_neu_ent, c->d_combo_info, c->d_dnz, c->d_hval, dR);
        c->last_launches++;
        IGAB_CUDA_TRY(cudaGetLastError());
    }
    if (c->nd > 0) {
        k_res_dirichlet<<<(unsigned)((c->nd + 255) / 256), 256, 0, c->stream>>>(c->nd, c->d_drow, c->d_dg, dU, dR);
        c->last_launches++;
        IGAB_CUDA_TRY(cudaGetLastError());
    }
    igab_mark(c, 2);
    c->ev_res = c->profiling;
    return 0;
}

int igab_launch_tangent(igab_ctx *c, const double *dU, void *dvals, int prec)
{
    c->last_launches = 0;
    if (prec == IGAB_PREC_FP64) return launch_tangent_t<double>(c, dU, (double *)dvals);
    if (prec == IGAB_PREC_FP32) return launch_tangent_t<float>(c, dU, (float *)dvals);
    return IGAB_ERR_ARG;
}

int igab_launch_tangent_slabs(igab_ctx *c, const double *dU, void *dvals, int prec, long *row_end, int *nslab)
{
    c->last_launches = 0;
    if (prec == IGAB_PREC_FP64) return launch_tangent_slabs_t<double>(c, dU, (double *)dvals, row_end, nslab);
    if (prec == IGAB_PREC_FP32) return launch_tangent_slabs_t<float>(c, dU, (float *)dvals, row_end, nslab);
    return IGAB_ERR_ARG;
}

int igab_launch_exp_scale(igab_ctx *c, const double *dg)
{
    k_exp_scale<<<(unsigned)((c->nel + 255) / 256), 256, 0, c->stream>>>(dg, c->d_escale, c->nel);
    c->last_launches++;
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

/* grad_e = lam~^T dR/dg_e with lam~ = lam outside the Dirichlet rows (c->d_lam is scratch) */
int igab_launch_adjoint_dRdg(igab_ctx *c, const double *dU, const double *dlam, double *dgrad)
{
    igab_geom g = c->geom();
    IGAB_CUDA_TRY(cudaMemcpyAsync(c->d_lam, dlam, (size_t)c->ndof * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    if (c->nd > 0) {
        k_zero_rows<<<(unsigned)((c->nd + 255) / 256), 256, 0, c->stream>>>(c->nd, c->d_drow, c->d_lam);
        c->last_launches++;
        IGAB_CUDA_TRY(cudaGetLastError());
    }
    if (c->phys == IGAB_PHYS_GETIME)
        return c->tile_res == 4 ? launch_res_volume_t<4, true, true>(c, g, dU, nullptr, c->d_lam, dgrad)
                                : launch_res_volume_t<2, true, true>(c, g, dU, nullptr, c->d_lam, dgrad);
    return c->tile_res == 4 ? launch_res_volume_t<4, false, true>(c, g, dU, nullptr, c->d_lam, dgrad)
                            : launch_res_volume_t<2, false, true>(c, g, dU, nullptr, c->d_lam, dgrad);
}

int igab_launch_tangent_transpose(igab_ctx *c, const void *dvals, int prec, const double *dx, double *dy)
{
    igab_geom g = c->geom();
    const int nchunk = (c->nb[2] + KT_ZMAX - 1) / KT_ZMAX;
    const long nblk = (long)c->nb[0] * c->nb[1] * nchunk;
    if (prec == IGAB_PREC_FP64)
        k_tangent_transpose<double><<<(unsigned)nblk, 128, 0, c->stream>>>(g, (const double *)dvals, dx, dy, nchunk);
    else
        k_tangent_transpose<float><<<(unsigned)nblk, 128, 0, c->stream>>>(g, (const float *)dvals, dx, dy, nchunk);
    c->last_launches++;
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int igab_launch_res_batch(const igab_batch_dev &B, int grid, cudaStream_t st, const double *dU, double *dR)
{
    const size_t sm = sizeof(res_smem<2, 1>);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_res_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_res_batch<<<grid, 256, sm, st>>>(B, dU, dR);
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int igab_batch_occupancy_res(int *per_sm)
{
    const size_t sm = sizeof(res_smem<2, 1>);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_res_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    IGAB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_res_batch, 256, sm));
    return 0;
}

int igab_launch_res_dirichlet_rows(long nd, const int *drow, const double *dg, const double *dU, double *dR,
                                   cudaStream_t st)
{
    if (nd <= 0) return 0;
    k_res_dirichlet<<<(unsigned)((nd + 255) / 256), 256, 0, st>>>(nd, drow, dg, dU, dR);
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int igab_launch_tan_dirichlet_batch(const igab_batch_dev &B, long nd, const int *dinst, const int *drow, void *dv,
                                    int prec, cudaStream_t st)
{
    if (nd <= 0) return 0;
    const long n = nd * 375;
    if (prec == IGAB_PREC_FP64)
        k_tan_dirichlet_batch<double><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(B, nd, dinst, drow, (double *)dv);
    else
        k_tan_dirichlet_batch<float><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(B, nd, dinst, drow, (float *)dv);
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int igab_launch_zero_csr_rows(igab_ctx *c, void *dv, int prec)
{
    if (c->nd <= 0) return 0;
    const igab_geom g = c->geom();
    const long n = c->nd * 375;
    if (prec == IGAB_PREC_FP64)
        k_zero_csr_rows<double><<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(g, c->nd, c->d_drow, (double *)dv);
    else
        k_zero_csr_rows<float><<<(unsigned)((n + 255) / 256), 256, 0, c->stream>>>(g, c->nd, c->d_drow, (float *)dv);
    c->last_launches++;
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int igab_launch_csr_cols(igab_ctx *c, int *dcols)
{
    igab_geom g = c->geom();
    k_csr_cols<<<(unsigned)((c->ndof + 255) / 256), 256, 0, c->stream>>>(g, dcols);
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int igab_launch_check_finite(igab_ctx *c, const void *dev, long n, int prec, int *all_finite)
{
    int *dflag = nullptr;
    IGAB_CUDA_TRY(cudaMallocAsync((void **)&dflag, sizeof(int), c->stream));
    IGAB_CUDA_TRY(cudaMemsetAsync(dflag, 0, sizeof(int), c->stream));
    unsigned nb = (unsigned)((n + 255) / 256);
    if (nb > 148u * 16u) nb = 148u * 16u;
    if (nb == 0) nb = 1;
    if (prec == IGAB_PREC_FP64)
        k_check_finite<double><<<nb, 256, 0, c->stream>>>((const double *)dev, n, dflag);
    else
        k_check_finite<float><<<nb, 256, 0, c->stream>>>((const float *)dev, n, dflag);
    int h = 0;
    IGAB_CUDA_TRY(cudaMemcpyAsync(&h, dflag, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    IGAB_CUDA_TRY(cudaFreeAsync(dflag, c->stream));
    IGAB_CUDA_TRY(cudaStreamSynchronize(c->stream));
    *all_finite = h == 0;
    return 0;
}

/* ============================================================ set-up kernels */

namespace {
/* 1-D basis tables at the Gauss points of every element of one direction
 * (mesh/nurbs/eval_Bspline.c:64-74 evaluated at src/snesiga_Residual.c:116-121 points) */
__global__ void k_basis_tables(const double *__restrict__ kv, int ne, const double *__restrict__ gx,
                               const double *__restrict__ gw, double *__restrict__ tab,
                               double *__restrict__ wh, double *__restrict__ xq)
{
    int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ne * IGAB_NQ) return;
    int e = t / IGAB_NQ, q = t % IGAB_NQ;
    double X0 = kv[e + 2], X1 = kv[e + 3];
    double xi = gx[q];
    double x = (-xi + 1.0) * X0 + xi * X1;
    double out[3][3];
    double win[6];
    for (int i = 0; i < 6; i++) win[i] = kv[e + i];
    igab_bspline_p2(win, x, out);
    for (int l = 0; l < 3; l++)
        for (int k = 0; k < 3; k++) tab[(long)e * IGAB_TAB1D + q * 9 + l * 3 + k] = out[l][k];
    wh[(long)e * IGAB_NQ + q] = gw[q] * (X1 - X0);
    xq[(long)e * IGAB_NQ + q] = x;
}
} /* namespace */

int igab_launch_basis_tables(igab_ctx *c, int d, const double *dkv, const double *dgx, const double *dgw)
{
    int n = c->ne[d] * IGAB_NQ;
    k_basis_tables<<<(n + 127) / 128, 128, 0, c->stream>>>(dkv, c->ne[d], dgx, dgw, c->d_tab[d], c->d_wh[d], c->d_xq[d]);
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

/* ============================================================ FMA peak probe */
namespace {
template <typename T>
__global__ void __launch_bounds__(256) k_fma_peak(T *out, int iters, T b, T c)
{
    T a0 = T(threadIdx.x), a1 = a0 + T(1), a2 = a0 + T(2), a3 = a0 + T(3);
    T a4 = a0 + T(4), a5 = a0 + T(5), a6 = a0 + T(6), a7 = a0 + T(7);
    for (int i = 0; i < iters; i++) {
        a0 = a0 * b + c; a1 = a1 * b + c; a2 = a2 * b + c; a3 = a3 * b + c;
        a4 = a4 * b + c; a5 = a5 * b + c; a6 = a6 * b + c; a7 = a7 * b + c;
    }
    T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == T(-12345)) out[0] = s;   /* keeps the chains live */
}

template <typename T>
int fma_peak_t(double *tflops)
{
    int dev = 0, nsm = 0;
    IGAB_CUDA_TRY(cudaGetDevice(&dev));
    IGAB_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    T *out = nullptr;
    IGAB_CUDA_TRY(cudaMalloc((void **)&out, sizeof(T)));
    cudaEvent_t e0, e1;
    IGAB_CUDA_TRY(cudaEventCreate(&e0));
    IGAB_CUDA_TRY(cudaEventCreate(&e1));
    const int iters = 1 << 14;
    unsigned nblk = (unsigned)nsm * 8u;
    k_fma_peak<T><<<nblk, 256>>>(out, iters, T(0.999999), T(1e-7));   /* warm-up */
    float best = 1e30f;
    for (int rep = 0; rep < 3; rep++) {
        cudaEventRecord(e0);
        k_fma_peak<T><<<nblk, 256>>>(out, iters, T(0.999999), T(1e-7));
        cudaEventRecord(e1);
        IGAB_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) best = ms;
    }
    IGAB_CUDA_TRY(cudaGetLastError());
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    double flops = 2.0 * 8.0 * iters * (double)nblk * 256.0;
    *tflops = flops / (best * 1e-3) / 1e12;
    return 0;
}
} /* namespace */

int igab_launch_fma_peak(int prec, double *tflops)
{
    return prec == IGAB_PREC_FP64 ? fma_peak_t<double>(tflops) : fma_peak_t<float>(tflops);
}
