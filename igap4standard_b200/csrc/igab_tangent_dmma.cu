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
 * Gamma in the rank-6 form Gamma = sum_q sum_i U_qi V_qi^T, geo = [[S, T], [T^T, 0]]:
 *   U_i = d_i N_a, V_i = w ((S grad N_a)_i + (T H_a)_i)     (i < 3)
 *   U_i = w (T H_a)_I, V_i = d_I N_a                         (i = 3 + I)
 *
 * Warp-specialised, one 512-thread block per SM, persistent over the tiles
 * (2x2x2 elements) of one colour or of a batched work list:
 *   - 8 builder warps compute, per element, the field at the 64 Gauss points
 *     (sum factorisation), the point integrand, and then per batch of 4 points
 *     the 48 rows of X' (one task per (point, basis function, component): the
 *     9 derivatives of the basis function from the 1-D tables, then all 12
 *     variables' entries in straight-line code), the 24 U / V rows (one task
 *     per (point, basis function)) and the scales s, into one of two
 *     shared-memory slots;
 *   - 8 consumer warps run the DMMA products on the slot: the 66 upper 8x8
 *     tiles of the 88x88 element matrix and the 10 upper tiles of the 32x32
 *     Gamma block, split over the warps by igab_warp_tiles8.inc, with the
 *     accumulators in registers for the whole element.  At the end of an
 *     element they add Gamma to the diagonal component blocks and reduce the
 *     81x81 matrix into the CSR values straight from the accumulators
 *     (fire-and-forget red.global.add; the lower triangle mirrors the upper
 *     one exactly).  Tiles of one colour touch disjoint entries and the
 *     elements of a tile are separated by a consumer barrier, so every entry
 *     receives its additions in a fixed order.
 * The slots are handed over with mbarriers (full: 256 builder arrivals, empty:
 * 256 consumer arrivals).  Every wait is bounded; a wait that gives up sets the
 * block's abort flag and the status word, and both roles leave their loops.
 */
#include <cuda_runtime.h>
#include "igab_device.cuh"
#include "igab_tc.cuh"

namespace {

#include "igab_warp_tiles8.inc"

#define NCONS 256       /* consumer threads (warps 0-7): DMMA tiles and scatter */
#define NBLD 256        /* builder threads (warps 8-15): field, integrand, X', U / V */
#define NTHR (NCONS + NBLD)
#define NSLOT 2         /* X' / U / V slots in flight */
#define BAR_CONS 1      /* named barrier of the consumers */
#define BAR_BLD 2       /* named barrier of the builders */
#define DQ 4            /* Gauss points per batch */
#define DROWS (DQ * 12) /* k rows of X' per batch */
#define GROWS (DQ * 6)  /* k rows of the geometric product per batch: U / V rows, 6 per point */
#define XS 100          /* X' row stride (doubles): = 4 mod 16 keeps fragment loads conflict-free */
#define GS 36           /* U / V row stride: = 4 mod 16; columns a >= 27 stay zero */
#define TE 2            /* tile edge (elements) */
#define TCP (TE + 2)    /* control points per tile edge */

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

/* one tile of work as the builders publish it to the consumers */
struct dws_tile {
    igab_geom g;
    const double *U;
    double *vals;
    int tile, colour, inst, pos;   /* tile < 0: no more work; pos: sweep position of a batch item */
};

struct dws_smem {
    double X[NSLOT][DROWS * XS];     /* X' rows (row 12 qb + v, column 3 a + k) */
    double UT[NSLOT][GROWS * GS];    /* U rows of the geometric product (row 6 qb + i, column a) */
    double VT[NSLOT][GROWS * GS];    /* V rows */
    double sc[NSLOT][DROWS];         /* s of the X' rows */
    double pt[IGAB_NQ3 * PT_N];      /* point data of the element being built */
    double AC[972 + 864];            /* interpolation scratch */
    double gam[32 * 32];             /* upper tiles of Gamma at the end of an element */
    double U[TCP * TCP * TCP * 3];   /* displacements of the tile's control points */
    double tab[3][TE][IGAB_TAB1D];
    double wh[3][TE][IGAB_NQ];
    long rbase[81];                  /* CSR row bases of the element matrix (elem_row_base) */
    int rsx[81], rsy[81];
    dws_tile td[2];                  /* tile k in td[k & 1] */
    unsigned long long full[NSLOT], empty[NSLOT];
    int abort_flag;
};

__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                 : "+d"(c0), "+d"(c1)
                 : "d"(a), "d"(b));
}

__device__ __forceinline__ void red_add(double *p, double v)
{
    atomicAdd(p, v);   /* result unused: a fire-and-forget reduction */
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

/* ---------------------------------------------------------------- work sources */

/* the tiles of one colour, dealt round-robin over the persistent blocks */
struct src_colour {
    igab_geom g;
    const double *U;
    double *vals;
    int colour;
    long tile0;    /* first tile id (an x-slab of the colour) */
    long ntiles;
    int *status;
    __device__ void fetch(int k, dws_tile &R) const
    {
        const long t = blockIdx.x + (long)k * gridDim.x;
        R.tile = t < ntiles ? (int)(tile0 + t) : -1;
        if (R.tile < 0) return;
        R.g = g;
        R.U = U;
        R.vals = vals;
        R.colour = colour;
        R.inst = 0;
    }
    __device__ void done(const dws_tile &) const {}
};

/* the batched work list: items (instance, sweep position, tile, colour) in colour-major
 * order; an item starts once every earlier position of its instance is complete */
struct src_batch {
    igab_batch_dev B;
    const double *U;
    double *vals;
    int *status;
    __device__ void fetch(int, dws_tile &R) const
    {
        const int it = atomicAdd(B.counter, 1);
        if (it >= B.nitems) {
            R.tile = -1;
            return;
        }
        const int4 w = B.items[it];
        batch_wait_colours(B, w.x, w.y);
        __threadfence();
        R.g = B.geoms[w.x];
        R.U = U + B.dof_off[w.x];
        R.vals = vals + B.nnz_off[w.x];
        R.tile = w.z;
        R.colour = w.w;
        R.pos = w.y;
        R.inst = w.x;
    }
    /* consumers, after the tile's last reduction: publish the finished tile */
    __device__ void done(const dws_tile &R) const
    {
        __threadfence();
        tc_bar_sync(BAR_CONS, NCONS);
        if (threadIdx.x == 0) atomicAdd(&B.done[8 * R.inst + R.pos], 1);
    }
};

/* ---------------------------------------------------------------- builders */

/* wait until slot (gb % NSLOT) is free again; uniform over the builders */
__device__ __forceinline__ bool bld_acquire(dws_smem &S, int gb)
{
    const int b = gb % NSLOT, u = gb / NSLOT;
    const volatile int *abort = &S.abort_flag;
    bool ok = !*abort;
    /* one builder waits; the named barrier orders the others' slot writes after it */
    if (ok && u > 0 && threadIdx.x == NCONS) ok = tc_mbar_wait_abortable(&S.empty[b], (u - 1) & 1, abort);
    return tc_bar_and(BAR_BLD, NBLD, ok);
}

/* X', U / V and s of the batch of points q0 .. q0 + 3 into slot b.
 * X' task (point qb, basis function a, component k): the 9 derivatives of N_a
 * (dx, dy, dz, xx, xy, xz, yy, yz, zz) from the 1-D tables, then the 12 rows
 *   X'[(qb, v)][3a + k] = sum_m dv'/du_{k,m} N_a^m
 * with dv/du_{k,m} of igab_ge_grad_var written out per variable (F = F[k][.],
 * G = G[k][.]; the (va, vb) pair rotated by (cs, sn)).
 * U / V task (point qb, basis function a): the six rows of the geometric
 * product, U_i = d_i N_a, V_i = w ((S grad N_a)_i + (T H_a)_i), U_{3+I} =
 * w (T H_a)_I, V_{3+I} = d_I N_a, with (T H_a)_I = sum_K T[I][K] N_a^{(I,K)}. */
__device__ __forceinline__ void bld_batch(dws_smem &S, int b, int q0, const double *Bx, const double *By,
                                          const double *Bz, int tb)
{
    double *const Xs = S.X[b];
    double *const UTs = S.UT[b];
    double *const VTs = S.VT[b];
    const double *const PTb = S.pt;
    const double is2 = IGAB_INV_SQRT2, is3 = IGAB_INV_SQRT3, is6 = IGAB_INV_SQRT6;
    for (int t = tb; t < DQ * 81 + DQ * 27; t += NBLD) {
        const bool xtask = t < DQ * 81;
        const int tg = xtask ? t : t - DQ * 81;
        const int qb = xtask ? tg / 81 : tg / 27;
        const int a = xtask ? (tg % 81) / 3 : tg % 27;
        const int q = q0 + qb, qx = q & 3, qy = (q >> 2) & 3, qz = q >> 4;
        const int ax = a / 9, ay = (a / 3) % 3, az = a % 3;
        const double *bxp = Bx + qx * 9 + ax * 3, *byp = By + qy * 9 + ay * 3, *bzp = Bz + qz * 9 + az * 3;
        const double bx0 = bxp[0], bx1 = bxp[1], bx2 = bxp[2];
        const double by0 = byp[0], by1 = byp[1], by2 = byp[2];
        const double bz0 = bzp[0], bz1 = bzp[1], bz2 = bzp[2];
        const double b00 = bx0 * by0, b10 = bx1 * by0, b01 = bx0 * by1;
        const double dx = b10 * bz0, dy = b01 * bz0, dz = b00 * bz1;
        const double hxx = bx2 * by0 * bz0, hxy = bx1 * by1 * bz0, hxz = b10 * bz1;
        const double hyy = bx0 * by2 * bz0, hyz = b01 * bz1, hzz = b00 * bz2;
        const double *p = PTb + q * PT_N;
        if (xtask) {
            const int k = tg % 3;
            const double F0 = p[PT_F + 3 * k], F1 = p[PT_F + 3 * k + 1], F2 = p[PT_F + 3 * k + 2];
            const double *G = p + PT_G + 6 * k;
            const double G0 = G[0], G1 = G[1], G2 = G[2], G3 = G[3], G4 = G[4], G5 = G[5];
            const double cs = p[PT_CS], sn = p[PT_SN];
            const double e0 = F0 * dx, e1 = F1 * dy, e2 = F2 * dz;
            const double va = (e0 - e1) * is2, vb = (e0 + e1 - 2.0 * e2) * is6;
            double *xc = Xs + (qb * 12) * XS + 3 * a + k;
            xc[0 * XS] = (e0 + e1 + e2) * is3;
            xc[1 * XS] = cs * va - sn * vb;
            xc[2 * XS] = sn * va + cs * vb;
            xc[3 * XS] = 0.5 * (F1 * dx + F0 * dy);
            xc[4 * XS] = 0.5 * (F2 * dx + F0 * dz);
            xc[5 * XS] = 0.5 * (F2 * dy + F1 * dz);
            xc[6 * XS] = (G0 * dx - G1 * dy + F0 * hxx - F1 * hxy) * is2;
            xc[7 * XS] = (G1 * dx - G3 * dy + F0 * hxy - F1 * hyy) * is2;
            xc[8 * XS] = (G2 * dx - G4 * dy + F0 * hxz - F1 * hyz) * is2;
            xc[9 * XS] = (G0 * dx + G1 * dy - 2.0 * G2 * dz + F0 * hxx + F1 * hxy - 2.0 * F2 * hxz) * is6;
            xc[10 * XS] = (G1 * dx + G3 * dy - 2.0 * G4 * dz + F0 * hxy + F1 * hyy - 2.0 * F2 * hyz) * is6;
            xc[11 * XS] = (G2 * dx + G4 * dy - 2.0 * G5 * dz + F0 * hxz + F1 * hyz - 2.0 * F2 * hzz) * is6;
        } else {
            const double w = p[PT_W];
            const double s00 = p[PT_SIG], s11 = p[PT_SIG + 1], s22 = p[PT_SIG + 2];
            const double s01 = 0.5 * p[PT_D1S], s02 = 0.5 * p[PT_D1S + 1], s12 = 0.5 * p[PT_D1S + 2];
            const double *T = p + PT_TAU;
            const double th0 = T[0] * hxx + T[1] * hxy + T[2] * hxz;
            const double th1 = T[3] * hxy + T[4] * hyy + T[5] * hyz;
            const double th2 = T[6] * hxz + T[7] * hyz + T[8] * hzz;
            double *ur = UTs + (qb * 6) * GS + a, *vr = VTs + (qb * 6) * GS + a;
            ur[0 * GS] = dx;
            ur[1 * GS] = dy;
            ur[2 * GS] = dz;
            vr[0 * GS] = w * (s00 * dx + s01 * dy + s02 * dz + th0);
            vr[1 * GS] = w * (s01 * dx + s11 * dy + s12 * dz + th1);
            vr[2 * GS] = w * (s02 * dx + s12 * dy + s22 * dz + th2);
            ur[3 * GS] = w * th0;
            ur[4 * GS] = w * th1;
            ur[5 * GS] = w * th2;
            vr[3 * GS] = dx;
            vr[4 * GS] = dy;
            vr[5 * GS] = dz;
        }
    }
    if (tb < DROWS) {
        const double *p = PTb + (q0 + tb / 12) * PT_N;
        S.sc[b][tb] = p[PT_W] * p[PT_LAM + tb % 12];
    }
}

template <class Src>
__device__ void dws_builder(const Src &F, dws_smem &S)
{
    const int tb = threadIdx.x - NCONS;
    int gb = 0;   /* batches published so far */
    bool aborted = false;
    for (int k = 0; !aborted; k++) {
        dws_tile &R = S.td[k & 1];
        if (tb == 0) F.fetch(k, R);
        tc_bar_sync(BAR_BLD, NBLD);
        if (R.tile < 0) {
            /* the end of the work, published through the next slot */
            if (!bld_acquire(S, gb)) aborted = true;
            else tc_mbar_arrive(&S.full[gb % NSLOT]);
            break;
        }
        const igab_geom &g = R.g;
        tile_t Tl;
        decode_tile(g, TE, R.colour, R.tile, Tl);
        for (int idx = tb; idx < TCP * TCP * TCP * 3; idx += NBLD) {
            int i = idx % 3, cp = idx / 3;
            int lz = cp % TCP, ly = (cp / TCP) % TCP, lx = cp / (TCP * TCP);
            double v = 0.0;
            if (lx < Tl.nv[0] + 2 && ly < Tl.nv[1] + 2 && lz < Tl.nv[2] + 2)
                v = R.U[3 * cp_index(g, Tl.e0[0] + lx, Tl.e0[1] + ly, Tl.e0[2] + lz) + i];
            S.U[idx] = v;
        }
        for (int idx = tb; idx < 3 * TE * IGAB_TAB1D; idx += NBLD) {
            int d = idx / (TE * IGAB_TAB1D), r = idx % (TE * IGAB_TAB1D), le = r / IGAB_TAB1D, o = r % IGAB_TAB1D;
            S.tab[d][le][o] = le < Tl.nv[d] ? g.tab[d][(long)(Tl.e0[d] + le) * IGAB_TAB1D + o] : 0.0;
        }
        for (int idx = tb; idx < 3 * TE * IGAB_NQ; idx += NBLD) {
            int d = idx / (TE * IGAB_NQ), r = idx % (TE * IGAB_NQ), le = r / IGAB_NQ, q = r % IGAB_NQ;
            S.wh[d][le][q] = le < Tl.nv[d] ? g.wh[d][(long)(Tl.e0[d] + le) * IGAB_NQ + q] : 0.0;
        }
        tc_bar_sync(BAR_BLD, NBLD);
        for (int le = 0; le < TE * TE * TE && !aborted; le++) {
            const int lex = le / (TE * TE), ley = (le / TE) % TE, lez = le % TE;
            if (!(lex < Tl.nv[0] && ley < Tl.nv[1] && lez < Tl.nv[2])) continue;   /* uniform */
            const double *Bx = S.tab[0][lex];
            const double *By = S.tab[1][ley];
            const double *Bz = S.tab[2][lez];
            double *const A = S.AC;
            double *const C = S.AC + 972;
            /* ---- field at the 64 Gauss points (sum-factorised, as the residual) */
            for (int o = tb; o < 972; o += NBLD) {
                int i = o % 3, kz = (o / 3) % 3, ay = (o / 9) % 3, ax = (o / 27) % 3, q = o / 81;
                const double *u0 = &S.U[(((lex + ax) * TCP + (ley + ay)) * TCP + lez) * 3 + i];
                A[o] = Bz[q * 9 + kz] * u0[0] + Bz[q * 9 + 3 + kz] * u0[3] + Bz[q * 9 + 6 + kz] * u0[6];
            }
            tc_bar_sync(BAR_BLD, NBLD);
            for (int o = tb; o < 864; o += NBLD) {
                int i = o % 3, kk = (o / 3) % 6, ax = (o / 18) % 3, qq = o / 54;
                int qyy = qq & 3, qzz = qq >> 2;
                const double *a0 = &A[((qzz * 3 + ax) * 3) * 9 + kk_kz(kk) * 3 + i];
                C[o] = By[qyy * 9 + kk_ky(kk)] * a0[0] + By[qyy * 9 + 3 + kk_ky(kk)] * a0[9] +
                       By[qyy * 9 + 6 + kk_ky(kk)] * a0[18];
            }
            tc_bar_sync(BAR_BLD, NBLD);
            /* ---- point integrand data (64 threads), point order q = 16 qz + 4 qy + qx */
            if (tb < IGAB_NQ3) {
                const int qx = tb & 3, qy = (tb >> 2) & 3, qz = tb >> 4, qq = qy + 4 * qz;
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
                double *pt = S.pt + tb * PT_N;
#pragma unroll
                for (int k2 = 0; k2 < 3; k2++)
#pragma unroll
                    for (int J = 0; J < 3; J++) pt[PT_F + 3 * k2 + J] = P.F[k2][J];
#pragma unroll
                for (int k2 = 0; k2 < 3; k2++)
#pragma unroll
                    for (int c = 0; c < 6; c++) pt[PT_G + 6 * k2 + c] = P.G[k2][c];
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
            tc_bar_sync(BAR_BLD, NBLD);
            /* ---- the 16 batches of this element */
            for (int q0 = 0; q0 < IGAB_NQ3; q0 += DQ) {
                if (!bld_acquire(S, gb)) {
                    aborted = true;
                    break;
                }
                const int b = gb % NSLOT;
                bld_batch(S, b, q0, Bx, By, Bz, tb);
                tc_mbar_arrive(&S.full[b]);
                gb++;
            }
        }
    }
    if (aborted && tb == 0) {
        S.abort_flag = 1;
        atomicOr(F.status, 1);
    }
}

/* ---------------------------------------------------------------- consumers */

/* wait until slot (gb % NSLOT) holds batch gb; uniform over the consumers */
__device__ __forceinline__ bool cons_acquire(dws_smem &S, int gb)
{
    const int b = gb % NSLOT;
    const volatile int *abort = &S.abort_flag;
    bool ok = !*abort;
    /* one consumer waits; the named barrier orders the others' slot reads after it */
    if (ok && threadIdx.x == 0) ok = tc_mbar_wait_abortable(&S.full[b], (gb / NSLOT) & 1, abort);
    return tc_bar_and(BAR_CONS, NCONS, ok);
}

template <int W>
struct cons_acc {
    using WT = warp_tiles8<W>;
    double k[WT::NT > 0 ? WT::NT : 1][2];
    double g[WT::NGT > 0 ? WT::NGT : 1][2];
};

/* one batch of the DMMA products: K += X'^T diag(sc) X' on the warp's K tiles,
 * Gamma += U^T V on its Gamma tiles */
template <int W>
__device__ __forceinline__ void warp_mma8(const double *__restrict__ X, const double *__restrict__ sc,
                                          const double *__restrict__ UT, const double *__restrict__ VT, int lane,
                                          cons_acc<W> &a)
{
    using WT = warp_tiles8<W>;
    const int r4 = lane & 3, c8 = lane >> 2;
    if constexpr (WT::NT > 0) {
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
            for (int t = 0; t < WT::NT; t++) dmma(a.k[t][0], a.k[t][1], f[WT::ti(t)], g[WT::tj(t)]);
        }
    }
    if constexpr (WT::NGT > 0) {
#pragma unroll 3
        for (int kb = 0; kb < GROWS / 4; kb++) {
            const int kr = 4 * kb + r4;
            double fa[WT::NGA], fb[WT::NGB];
#pragma unroll
            for (int b = 0; b < WT::NGA; b++) fa[b] = UT[kr * GS + 8 * WT::gablk(b) + c8];
#pragma unroll
            for (int b = 0; b < WT::NGB; b++) fb[b] = VT[kr * GS + 8 * WT::gbblk(b) + c8];
#pragma unroll
            for (int t = 0; t < WT::NGT; t++) dmma(a.g[t][0], a.g[t][1], fa[WT::gti(t)], fb[WT::gtj(t)]);
        }
    }
}

__device__ __forceinline__ long csr_at(const dws_smem &S, int c1, int c2)
{
    return S.rbase[c1] + (c2 / 27) * S.rsx[c1] + ((c2 / 9) % 3) * S.rsy[c1] + c2 % 9;
}

/* the warp's K tiles plus Gamma on the diagonal component blocks, reduced into
 * the CSR values; entry (c1, c2) and its mirror (c2, c1) receive the upper value */
template <int W>
__device__ __forceinline__ void warp_scatter8(double *__restrict__ vals, const dws_smem &S, int lane,
                                              const cons_acc<W> &a)
{
    using WT = warp_tiles8<W>;
    const int r = lane >> 2, c = 2 * (lane & 3);
#pragma unroll
    for (int t = 0; t < WT::NT; t++) {
        const int bi = WT::blk(WT::ti(t)), bj = WT::blk(WT::tj(t));
        double v2[2] = {a.k[t][0], a.k[t][1]};
        if (bi == bj) {
            /* diagonal tile: entry (r, c + e) below the diagonal takes (c + e, r),
             * held by lane 4 (c + e) + r / 2, element r & 1 */
            const double x0 = __shfl_sync(0xffffffffu, a.k[t][0], 4 * c + (r >> 1));
            const double y0 = __shfl_sync(0xffffffffu, a.k[t][1], 4 * c + (r >> 1));
            const double x1 = __shfl_sync(0xffffffffu, a.k[t][0], 4 * (c + 1) + (r >> 1));
            const double y1 = __shfl_sync(0xffffffffu, a.k[t][1], 4 * (c + 1) + (r >> 1));
            if (r > c) v2[0] = (r & 1) ? y0 : x0;
            if (r > c + 1) v2[1] = (r & 1) ? y1 : x1;
        }
#pragma unroll
        for (int e = 0; e < 2; e++) {
            const int c1 = 8 * bi + r, c2 = 8 * bj + c + e;
            if (c1 < 81 && c2 < 81) {
                const int a1 = c1 / 3, a2 = c2 / 3;
                double v = v2[e];
                if (c1 % 3 == c2 % 3) v += a1 <= a2 ? S.gam[a1 * 32 + a2] : S.gam[a2 * 32 + a1];
                red_add(vals + csr_at(S, c1, c2), v);
                if (bi != bj) red_add(vals + csr_at(S, c2, c1), v);
            }
        }
    }
}

template <int W, class Src>
__device__ void dws_consumer(const Src &F, dws_smem &S)
{
    using WT = warp_tiles8<W>;
    const int tid = threadIdx.x, lane = tid & 31;
    int gb = 0;   /* batches consumed so far */
    bool aborted = false;
    for (int k = 0;; k++) {
        /* the first batch of tile k (or the end of the work) */
        if (!cons_acquire(S, gb)) {
            aborted = true;
            break;
        }
        const dws_tile &R = S.td[k & 1];
        if (R.tile < 0) break;
        tile_t Tl;
        decode_tile(R.g, TE, R.colour, R.tile, Tl);
        bool have = true;
        for (int le = 0; le < TE * TE * TE && !aborted; le++) {
            const int lex = le / (TE * TE), ley = (le / TE) % TE, lez = le % TE;
            if (!(lex < Tl.nv[0] && ley < Tl.nv[1] && lez < Tl.nv[2])) continue;   /* uniform */
            cons_acc<W> a;
#pragma unroll
            for (int t = 0; t < (WT::NT > 0 ? WT::NT : 1); t++) a.k[t][0] = a.k[t][1] = 0.0;
#pragma unroll
            for (int t = 0; t < (WT::NGT > 0 ? WT::NGT : 1); t++) a.g[t][0] = a.g[t][1] = 0.0;
            for (int q0 = 0; q0 < IGAB_NQ3; q0 += DQ) {
                if (!have && !cons_acquire(S, gb)) {
                    aborted = true;
                    break;
                }
                have = false;
                const int b = gb % NSLOT;
                warp_mma8<W>(S.X[b], S.sc[b], S.UT[b], S.VT[b], lane, a);
                tc_mbar_arrive(&S.empty[b]);
                gb++;
            }
            if (aborted) break;
            /* Gamma (upper tiles) and the CSR row bases of the element */
            if constexpr (WT::NGT > 0) {
                const int r = lane >> 2, c = 2 * (lane & 3);
#pragma unroll
                for (int t = 0; t < WT::NGT; t++) {
                    const int a1 = 8 * WT::gablk(WT::gti(t)) + r, a2 = 8 * WT::gbblk(WT::gtj(t)) + c;
                    S.gam[a1 * 32 + a2] = a.g[t][0];
                    S.gam[a1 * 32 + a2 + 1] = a.g[t][1];
                }
            }
            if (tid < 81)
                elem_row_base(R.g, Tl.e0[0] + lex, Tl.e0[1] + ley, Tl.e0[2] + lez, tid, S.rbase[tid], S.rsx[tid],
                              S.rsy[tid]);
            tc_bar_sync(BAR_CONS, NCONS);
            warp_scatter8<W>(R.vals, S, lane, a);
            tc_bar_sync(BAR_CONS, NCONS);
        }
        if (aborted) break;
        F.done(R);
    }
    if (aborted && tid == 0) {
        S.abort_flag = 1;
        atomicOr(F.status, 1);
    }
}

template <class Src>
__device__ __forceinline__ void dws_run(const Src &F)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    dws_smem &S = *reinterpret_cast<dws_smem *>(smem_raw);
    const int tid = threadIdx.x;
    if (tid == 0) {
        S.abort_flag = 0;
        for (int b = 0; b < NSLOT; b++) {
            tc_mbar_init(&S.full[b], NBLD);
            tc_mbar_init(&S.empty[b], NCONS);
        }
        tc_fence_mbar_init();
    }
    /* the padding columns of X' (a >= 27) and of U / V stay zero */
    for (int idx = tid; idx < NSLOT * DROWS * (XS - 81); idx += NTHR) {
        const int b = idx / (DROWS * (XS - 81)), r = idx % (DROWS * (XS - 81));
        S.X[b][(r / (XS - 81)) * XS + 81 + r % (XS - 81)] = 0.0;
    }
    for (int idx = tid; idx < NSLOT * GROWS * GS; idx += NTHR) {
        (&S.UT[0][0])[idx] = 0.0;
        (&S.VT[0][0])[idx] = 0.0;
    }
    __syncthreads();
    if (tid >= NCONS) {
        dws_builder(F, S);
        return;
    }
    switch (tid >> 5) {
    case 0: dws_consumer<0>(F, S); break;
    case 1: dws_consumer<1>(F, S); break;
    case 2: dws_consumer<2>(F, S); break;
    case 3: dws_consumer<3>(F, S); break;
    case 4: dws_consumer<4>(F, S); break;
    case 5: dws_consumer<5>(F, S); break;
    case 6: dws_consumer<6>(F, S); break;
    default: dws_consumer<7>(F, S); break;
    }
}

__global__ void __launch_bounds__(NTHR, 1) k_tan_dmma(src_colour F)
{
    dws_run(F);
}

/* persistent FP64 tangent over the tiles of every instance of a batch */
__global__ void __launch_bounds__(NTHR, 1) k_tan_dmma_batch(src_batch F)
{
    dws_run(F);
}

int sm_count()
{
    static int n = 0;
    if (n == 0) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
            n = 148;
    }
    return n;
}

} /* namespace */

int igab_launch_tan_dmma_batch(const igab_batch_dev &B, int grid, cudaStream_t st, const double *dU, double *dv)
{
    const size_t sm = sizeof(dws_smem);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_dmma_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    src_batch F;
    F.B = B;
    F.U = dU;
    F.vals = dv;
    F.status = B.status;
    k_tan_dmma_batch<<<grid, NTHR, sm, st>>>(F);
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int igab_batch_occupancy_dmma(int *per_sm)
{
    const size_t sm = sizeof(dws_smem);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_dmma_batch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    IGAB_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k_tan_dmma_batch, NTHR, sm));
    return 0;
}

/* FP64 tensor-pipe issue rate: every warp issues back-to-back mma.sync m8n8k4 f64 on
 * eight independent accumulator pairs (512 flops per warp instruction) */
__global__ void __launch_bounds__(256) k_dmma_peak(int reps, double *sink)
{
    double c[8][2];
#pragma unroll
    for (int i = 0; i < 8; i++) c[i][0] = c[i][1] = 0.0;
    const double a = 1.0 + 1e-9 * threadIdx.x, b = 0.999;
    for (int r = 0; r < reps; r++) {
#pragma unroll
        for (int i = 0; i < 8; i++) dmma(c[i][0], c[i][1], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int i = 0; i < 8; i++) s += c[i][0] + c[i][1];
    if (s == -12345.0) sink[0] = s;   /* keeps the chains live */
}

int igab_launch_dmma_peak(double *tflops)
{
    int dev = 0, nsm = 0;
    IGAB_CUDA_TRY(cudaGetDevice(&dev));
    IGAB_CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    double *sink = nullptr;
    IGAB_CUDA_TRY(cudaMalloc((void **)&sink, sizeof(double)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t err = cudaEventCreate(&e0);
    if (err == cudaSuccess) err = cudaEventCreate(&e1);
    const int reps = 1 << 13;
    const unsigned nblk = (unsigned)nsm * 4u;   /* 32 warps per SM */
    float best = 1e30f;
    if (err == cudaSuccess) {
        k_dmma_peak<<<nblk, 256>>>(reps, sink);   /* warm-up */
        for (int rep = 0; rep < 3 && err == cudaSuccess; rep++) {
            cudaEventRecord(e0);
            k_dmma_peak<<<nblk, 256>>>(reps, sink);
            cudaEventRecord(e1);
            err = cudaEventSynchronize(e1);
            float ms = 0.f;
            if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
            if (err == cudaSuccess && ms < best) best = ms;
        }
        if (err == cudaSuccess) err = cudaGetLastError();
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    cudaFree(sink);
    if (err != cudaSuccess) {
        igab_set_error("igab_dmma_peak: %s", cudaGetErrorString(err));
        return IGAB_ERR_CUDA;
    }
    const double flops = 512.0 * 8.0 * reps * (double)nblk * 8.0;   /* per warp instruction x chains x warps */
    *tflops = flops / (best * 1e-3) / 1e12;
    return 0;
}

int igab_launch_tan_dmma(igab_ctx *c, const double *dU, double *dv, int tx0, int tx1)
{
    igab_geom g = c->geom();
    const size_t sm = sizeof(dws_smem);
    IGAB_CUDA_TRY(cudaFuncSetAttribute(k_tan_dmma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    const int nsm = sm_count();
    for (int k = 0; k < 8; k++) {
        const int colour = igab_colour_at(c->colour_order, k);
        long first = 0;
        const long nt = tiles_of_colour_in(g, TE, colour, tx0, tx1, &first);
        if (nt == 0) continue;
        src_colour F;
        F.g = g;
        F.U = dU;
        F.vals = dv;
        F.colour = colour;
        F.tile0 = first;
        F.ntiles = nt;
        F.status = c->d_status;
        k_tan_dmma<<<(unsigned)(nt < nsm ? nt : nsm), NTHR, sm, c->stream>>>(F);
        c->last_launches++;
    }
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}
