/*
 * Integrated densities (src/iga_intdensity.c:10-293): the volume integral of
 * the physics' point density over all elements minus the Neumann boundary
 * integrals of its boundary density, as ndensity scalars.
 *
 *   phys/ge     (13 densities, phys/ge/density.c:6-76): W, 2 dW/dE_II (I = 0..2
 *               at hh[1], hh[4], hh[6]), 4 e345 E_IJ (I < J at hh[2], hh[3],
 *               hh[5]), and the six volume-fraction indicators of (va, vb, W);
 *               boundary (:79-84): u * traction on the current level.
 *   phys/getime (2 densities, phys/getime/density.c:6-53): the ge energy at the
 *               midpoint of history levels 1 and 2 plus rho/(2 dt^2) |u1 - u0|^2
 *               of the value components, 0; boundary (:57-62):
 *               (u1 + u2)/2 * traction, 1.
 *
 * Kernels:
 *   k_density_volume   persistent; one thread per Gauss point (4 elements per
 *                      256-thread block, element groups dealt round-robin),
 *                      direct interpolation of the 30 field components from the
 *                      27 staged control points and the 1-D basis tables, the
 *                      periodic term of src/iga_intdensity.c:137-141, the density
 *                      times the Gauss weight summed per thread, then per block
 *                      in a fixed order into one partial row per block.
 *   k_density_surface  one thread per surface Gauss point of the Neumann combos
 *                      (the residual's point table and traction values), the
 *                      boundary value u_b (normal derivative for order 1) from
 *                      the 3 x 3 face functions, partial rows per block.
 *   k_density_reduce   one block: HH[i] = sum of volume partials - sum of surface
 *                      partials, in a fixed order (bitwise repeatable).
 */
#include <cuda_runtime.h>
#include "igab_device.cuh"

namespace {

#define DN_MAX 13
#define VOL_THREADS 256
#define SURF_THREADS 128
#define RED_THREADS 256

struct dens_geom {
    igab_geom g;
    const double *lev[3];   /* field levels the density reads (level 0 = U, 1, 2 = history) */
    int nd;                 /* densities */
};

/* block sum of v[0..nd) in a fixed order; thread 0 writes the row */
template <int NT, int ND>
__device__ __forceinline__ void block_rows(const double (&v)[DN_MAX], double *row, double *red)
{
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int i = 0; i < ND; i++) {
        double s = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) red[warp * DN_MAX + i] = s;
    }
    __syncthreads();
    if (tid < ND) {
        double s = 0.0;
        for (int w = 0; w < NT / 32; w++) s += red[w * DN_MAX + tid];
        row[tid] = s;
    }
    __syncthreads();
}

/* the 13 ge densities of one point from the 30 field components */
__device__ __forceinline__ void ge_density13(const double *u, const igab_ge_coef &c, double (&hh)[DN_MAX],
                                             double &W)
{
    igab_ge_point<double> P;
    igab_ge_eval(u, c, P);
    const double vv = P.v[0], va = P.v[1], vb = P.v[2];
    const double s2 = va * va + vb * vb;
    double gs = 0.0;
#pragma unroll
    for (int i = 6; i < 12; i++) gs += P.v[i] * P.v[i];
    W = c.c36 * vb * (vb * vb - 3.0 * va * va) + c.c37 * s2 + c.c38 * s2 * s2 + c.p2 * vv * vv +
        c.p3 * (P.v[3] * P.v[3] + P.v[4] * P.v[4] + P.v[5] * P.v[5]) + c.p4sq * gs;
    hh[0] = W;
    hh[1] = 2.0 * P.sig[0];
    hh[2] = 2.0 * P.d1[3];
    hh[3] = 2.0 * P.d1[4];
    hh[4] = 2.0 * P.sig[1];
    hh[5] = 2.0 * P.d1[5];
    hh[6] = 2.0 * P.sig[2];
    hh[7] = (va > 0.0 && vb > -0.5 * va) ? 1.0 : 0.0;
    hh[8] = (va < 0.0 && vb > 0.5 * va) ? 1.0 : 0.0;
    hh[9] = (vb < 0.5 * va && vb < -0.5 * va) ? 1.0 : 0.0;
    hh[10] = (W < -0.5 && va > 0.0 && vb > 0.0) ? 1.0 : 0.0;
    hh[11] = (W < -0.5 && va < 0.0 && vb > 0.0) ? 1.0 : 0.0;
    hh[12] = (W < -0.5 && vb < 0.0) ? 1.0 : 0.0;
}

template <int ND>
__global__ void __launch_bounds__(VOL_THREADS) k_density_volume(dens_geom D, double *__restrict__ part)
{
    const igab_geom &g = D.g;
    __shared__ double cpU[4][2][27 * 3];   /* per element slot: up to two levels */
    __shared__ double red[(VOL_THREADS / 32) * DN_MAX];
    const int tid = threadIdx.x, slot = tid >> 6, q = tid & 63;
    const int qx = q & 3, qy = (q >> 2) & 3, qz = q >> 4;
    const int nlev = g.phys == IGAB_PHYS_GETIME ? 2 : 1;
    const long nel = (long)g.ne[0] * g.ne[1] * g.ne[2];
    const long ngroups = (nel + 3) / 4;
    double acc[DN_MAX];
#pragma unroll
    for (int i = 0; i < DN_MAX; i++) acc[i] = 0.0;

    for (long grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
        const long e = grp * 4 + slot;
        const bool valid = e < nel;
        int ex = 0, ey = 0, ez = 0;
        if (valid) {
            ez = (int)(e % g.ne[2]);
            ey = (int)((e / g.ne[2]) % g.ne[1]);
            ex = (int)(e / ((long)g.ne[2] * g.ne[1]));
        }
        __syncthreads();   /* the previous group's reads of cpU are done */
        if (valid)
            for (int idx = q; idx < nlev * 81; idx += 64) {
                const int l = idx / 81, r = idx % 81, a = r / 3, k = r % 3;
                const int ax = a / 9, ay = (a / 3) % 3, az = a % 3;
                cpU[slot][l][r] = D.lev[l][3 * cp_index(g, ex + ax, ey + ay, ez + az) + k];
            }
        __syncthreads();
        if (!valid) continue;
        const double *tx = g.tab[0] + (long)ex * IGAB_TAB1D + qx * 9;
        const double *ty = g.tab[1] + (long)ey * IGAB_TAB1D + qy * 9;
        const double *tz = g.tab[2] + (long)ez * IGAB_TAB1D + qz * 9;
        double u[2][30];
#pragma unroll
        for (int l = 0; l < 2; l++)
#pragma unroll
            for (int i = 0; i < 30; i++) u[l][i] = 0.0;
        for (int a = 0; a < 27; a++) {
            const int ax = a / 9, ay = (a / 3) % 3, az = a % 3;
            double bx[3], by[3], bz[3];
#pragma unroll
            for (int k = 0; k < 3; k++) {
                bx[k] = tx[ax * 3 + k];
                by[k] = ty[ay * 3 + k];
                bz[k] = tz[az * 3 + k];
            }
            double N[10];
#pragma unroll
            for (int m = 0; m < 10; m++) N[m] = bx[a_kx(m)] * by[a_ky(m)] * bz[a_kz(m)];
#pragma unroll
            for (int l = 0; l < 2; l++) {
                if (l >= nlev) break;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    const double c = cpU[slot][l][3 * a + k];
#pragma unroll
                    for (int m = 0; m < 10; m++) u[l][10 * k + m] += N[m] * c;
                }
            }
        }
        /* periodic term: value pp . x and gradient pp on every level (src/iga_intdensity.c:137-141) */
        if (g.periodic) {
            const double x0 = g.xq[0][(long)ex * IGAB_NQ + qx], x1 = g.xq[1][(long)ey * IGAB_NQ + qy],
                         x2 = g.xq[2][(long)ez * IGAB_NQ + qz];
#pragma unroll
            for (int l = 0; l < 2; l++)
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    u[l][10 * k] += g.pp[3 * k] * x0 + g.pp[3 * k + 1] * x1 + g.pp[3 * k + 2] * x2;
#pragma unroll
                    for (int J = 0; J < 3; J++) u[l][10 * k + 1 + J] += g.pp[3 * k + J];
                }
        }
        double hh[DN_MAX], W;
        if (g.phys == IGAB_PHYS_GETIME) {
            /* energy at the midpoint of levels 1 and 2, kinetic term of their difference */
            double um[30];
#pragma unroll
            for (int i = 0; i < 30; i++) um[i] = 0.5 * (u[0][i] + u[1][i]);
            ge_density13(um, g.coef, hh, W);
            double kin = 0.0;
#pragma unroll
            for (int k = 0; k < 3; k++) {
                const double d = u[0][10 * k] - u[1][10 * k];
                kin += d * d;
            }
            hh[0] = W + g.rho * kin / (2.0 * g.dt * g.dt);
            hh[1] = 0.0;
        } else {
            ge_density13(u[0], g.coef, hh, W);
        }
        const double w = g.wh[0][(long)ex * IGAB_NQ + qx] * g.wh[1][(long)ey * IGAB_NQ + qy] *
                         g.wh[2][(long)ez * IGAB_NQ + qz];
#pragma unroll
        for (int i = 0; i < DN_MAX; i++) acc[i] += w * hh[i];
    }
    block_rows<VOL_THREADS, ND>(acc, part + (long)blockIdx.x * DN_MAX, red);
}

/* surface Gauss points of the Neumann combos: point p of combo k lies at
 * offset(k) + (ex ne1 + ey) 16 + 4 q0 + q1 */
template <int ND>
__global__ void __launch_bounds__(SURF_THREADS) k_density_surface(dens_geom D, int ncombo,
                                                                  const int *__restrict__ cinfo,
                                                                  const double *__restrict__ dnz,
                                                                  const double *__restrict__ hval, long npoints,
                                                                  double *__restrict__ part)
{
    const igab_geom &g = D.g;
    __shared__ double red[(SURF_THREADS / 32) * DN_MAX];
    double acc[DN_MAX];
#pragma unroll
    for (int i = 0; i < DN_MAX; i++) acc[i] = 0.0;
    const long p = blockIdx.x * (long)SURF_THREADS + threadIdx.x;
    if (p < npoints) {
        int k = 0;
        for (; k + 1 < ncombo; k++) {
            const long next = (long)(unsigned)cinfo[8 * (k + 1) + 5] | ((long)cinfo[8 * (k + 1) + 6] << 32);
            if (p < next) break;
        }
        const int *ci = cinfo + 8 * k;
        const int face = ci[0], order = ci[1], dof = ci[2], ne1 = ci[4];
        const long off = (long)(unsigned)ci[5] | ((long)ci[6] << 32);
        const int d0 = ci[7] & 3, d1 = (ci[7] >> 2) & 3, dn = 3 - d0 - d1;
        const long r = p - off;
        const int q1 = (int)(r & 3), q0 = (int)((r >> 2) & 3);
        const long se = r >> 4;
        const int ey = (int)(se % ne1), ex = (int)(se / ne1);
        const double *t0 = g.tab[d0] + (long)ex * IGAB_TAB1D + q0 * 9;
        const double *t1 = g.tab[d1] + (long)ey * IGAB_TAB1D + q1 * 9;
        const int nslot = order ? 2 : 1;
        const int nlev = g.phys == IGAB_PHYS_GETIME ? 2 : 1;   /* the levels in D.lev the density reads */
        double ub[2] = {0.0, 0.0};
        for (int s = 0; s < nslot; s++) {
            const int layer = (face % 2 == 0) ? s : g.nb[dn] - 1 - s;
            const double fz = order ? dnz[2 * face + s] : 1.0;
            for (int b0 = 0; b0 < 3; b0++)
                for (int b1 = 0; b1 < 3; b1++) {
                    const int i0 = ex + b0, i1 = ey + b1;
                    const int cx = d0 == 0 ? i0 : (d1 == 0 ? i1 : layer);
                    const int cy = d0 == 1 ? i0 : (d1 == 1 ? i1 : layer);
                    const int cz = d0 == 2 ? i0 : (d1 == 2 ? i1 : layer);
                    const double nn = t0[b0 * 3] * t1[b1 * 3] * fz;
                    const long idx = 3 * cp_index(g, cx, cy, cz) + dof;
                    for (int l = 0; l < nlev; l++) ub[l] += nn * D.lev[l][idx];
                }
        }
        const double t = hval[p];
        const double w = g.wh[d0][(long)ex * IGAB_NQ + q0] * g.wh[d1][(long)ey * IGAB_NQ + q1];
        if (g.phys == IGAB_PHYS_GETIME) {
            acc[0] = w * (0.5 * (ub[0] + ub[1]) * t);
            acc[1] = w;
        } else {
            acc[0] = w * (ub[0] * t);
        }
    }
    block_rows<SURF_THREADS, ND>(acc, part + (long)blockIdx.x * DN_MAX, red);
}

template <int ND>
__global__ void __launch_bounds__(RED_THREADS) k_density_reduce(const double *__restrict__ part, long nvol, long nsurf, double *__restrict__ HH)
{
    __shared__ double red[(RED_THREADS / 32) * DN_MAX];
    const int tid = threadIdx.x;   /* RED_THREADS threads */
    double v[DN_MAX], s[DN_MAX];
#pragma unroll
    for (int i = 0; i < DN_MAX; i++) v[i] = s[i] = 0.0;
    for (long b = tid; b < nvol; b += blockDim.x)
#pragma unroll
        for (int i = 0; i < ND; i++) v[i] += part[b * DN_MAX + i];
    for (long b = tid; b < nsurf; b += blockDim.x)
#pragma unroll
        for (int i = 0; i < ND; i++) s[i] += part[(nvol + b) * DN_MAX + i];
    __shared__ double rows[2][DN_MAX];
    block_rows<RED_THREADS, ND>(v, rows[0], red);
    block_rows<RED_THREADS, ND>(s, rows[1], red);
    if (tid < ND) HH[tid] = rows[0][tid] - rows[1][tid];
}

template <int ND>
void launch_density(igab_ctx *c, const dens_geom &D, long nvol, long nsurf, double *dHH)
{
    if (nvol > 0) {
        k_density_volume<ND><<<(unsigned)nvol, VOL_THREADS, 0, c->stream>>>(D, c->d_dens_part);
        c->last_launches++;
    }
    if (nsurf > 0) {
        k_density_surface<ND><<<(unsigned)nsurf, SURF_THREADS, 0, c->stream>>>(
            D, (int)c->combos.size(), c->d_combo_info, c->d_dnz, c->d_hval, c->n_neu_points,
            c->d_dens_part + nvol * DN_MAX);
        c->last_launches++;
    }
    k_density_reduce<ND><<<1, RED_THREADS, 0, c->stream>>>(c->d_dens_part, nvol, nsurf, dHH);
    c->last_launches++;
}

} /* namespace */

int igab_launch_density(igab_ctx *c, const double *dU, double *dHH)
{
    dens_geom D;
    D.g = c->geom();
    D.nd = c->phys == IGAB_PHYS_GETIME ? 2 : 13;
    if (c->phys == IGAB_PHYS_GETIME) {
        D.lev[0] = c->d_hist;              /* level 1 */
        D.lev[1] = c->d_hist + c->ndof;    /* level 2 */
        D.lev[2] = nullptr;
    } else {
        D.lev[0] = dU;
        D.lev[1] = D.lev[2] = nullptr;
    }
    int nsm = 148;
    {
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    }
    const long ngroups = (c->nel + 3) / 4;
    const long nvol = ngroups < (long)nsm * 8 ? ngroups : (long)nsm * 8;
    const long nsurf = (c->n_neu_points + SURF_THREADS - 1) / SURF_THREADS;
    const size_t need = (size_t)(nvol + nsurf) * DN_MAX * sizeof(double);
    if (need > c->dens_part_bytes) {
        cudaFree(c->d_dens_part);
        c->d_dens_part = nullptr;
        c->dens_part_bytes = 0;
        IGAB_CUDA_TRY(cudaMalloc((void **)&c->d_dens_part, need));
        c->dens_part_bytes = need;
    }
    c->last_launches = 0;
    if (D.nd == 13)
        launch_density<13>(c, D, nvol, nsurf, dHH);
    else
        launch_density<2>(c, D, nvol, nsurf, dHH);
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}
