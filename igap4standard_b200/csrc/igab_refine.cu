/*
 * Mesh refinement by knot insertion and the solution file format.
 *
 * igab_knot_insert replaces mesh/nurbs/nurbs_knotinsert.c:7: the control
 * points of a p = 2 B-spline field on nelem / 2^nref elements per direction are
 * refined nref times by inserting the mid-point of every knot span (uniform
 * spans; the 1-D weights of one control point on the refined points 2 i - 2 ..
 * 2 i + 1, periodic or not, are the tables of nurbs_knotinsert.c:36-77).  One
 * GPU thread per refined control point gathers the at most 2 x 2 x 2 coarse
 * points that contribute, in the reference's lexicographic (x, y, z) order and
 * with the same product order, so the sums are taken in the same sequence.
 * The array is refined in place in the caller's host memory (laid out as
 * U_universal[ndof * cp + dof], cp = (x nb1 + y) nb2 + z, nb = nelem + 2, or
 * nelem along a periodic direction): one upload of the coarse points, the
 * periodic wrap, the levels and the unwrap on the device, one download.  The two
 * device buffers are kept per device between calls (grown on demand, freed by
 * igab_knot_release): a cudaMalloc / cudaFree pair per call cost 1.4 ms at best
 * and up to 20 ms after large allocations had been freed, against 0.2 ms of
 * device work for a 32^3 -> 64^3 field.  Calls in one process are serialised.
 *
 * igab_write_solution / igab_read_solution replace src/ioutil.c:89 and :126 on
 * one rank: history levels ihist0 .. ihist1 - 1 of U_hist (ndof each) written
 * as raw doubles in universal dof order, level after level.
 */
#include <cuda_runtime.h>
#include <stdio.h>
#include <mutex>
#include "igab_internal.h"

namespace {

/* per-device scratch of igab_knot_insert: two halves of cap doubles each */
constexpr int KNOT_MAX_DEVICES = 64;
std::mutex knot_mu;
double *knot_buf[KNOT_MAX_DEVICES];
size_t knot_cap[KNOT_MAX_DEVICES];

/* weights of coarse point i on the refined points 2 i - 2 + j, j = 0..3
 * (nurbs_knotinsert.c:36-77); nel = coarse elements along the direction */
__device__ __forceinline__ void ki_weights(int i, int nel, int periodic, double v[4])
{
    if (!periodic) {
        if (i == 0)             { v[0] = 0.0;  v[1] = 0.0;  v[2] = 1.0;  v[3] = 0.5; }
        else if (i == 1)        { v[0] = 0.0;  v[1] = 0.5;  v[2] = 0.75; v[3] = 0.25; }
        else if (i < nel)       { v[0] = 0.25; v[1] = 0.75; v[2] = 0.75; v[3] = 0.25; }
        else if (i == nel)      { v[0] = 0.25; v[1] = 0.75; v[2] = 0.5;  v[3] = 0.0; }
        else                    { v[0] = 0.5;  v[1] = 1.0;  v[2] = 0.0;  v[3] = 0.0; }
    } else {
        if (i == 0)             { v[0] = 0.0;  v[1] = 0.0;  v[2] = 0.75; v[3] = 0.25; }
        else if (i <= nel)      { v[0] = 0.25; v[1] = 0.75; v[2] = 0.75; v[3] = 0.25; }
        else                    { v[0] = 0.25; v[1] = 0.75; v[2] = 0.0;  v[3] = 0.0; }
    }
}

/* one refinement level: old (nel + 2)^3 points -> new (2 nel + 2)^3 points, ndof interleaved */
__global__ void k_knot_refine(const double *__restrict__ Uold, double *__restrict__ Unew, int nex, int ney,
                              int nez, int px, int py, int pz, int ndof)
{
    const int nbo[3] = {nex + 2, ney + 2, nez + 2};
    const int nbn[3] = {2 * nex + 2, 2 * ney + 2, 2 * nez + 2};
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long nnew = (long)nbn[0] * nbn[1] * nbn[2];
    if (t >= nnew) return;
    const int Z = (int)(t % nbn[2]), Y = (int)((t / nbn[2]) % nbn[1]), X = (int)(t / ((long)nbn[2] * nbn[1]));
    for (int d = 0; d < ndof; d++) {
        double acc = 0.0;
        for (int ix = X / 2; ix <= X / 2 + 1; ix++) {
            const int jx = X + 2 - 2 * ix;
            if (ix >= nbo[0] || jx < 0 || jx > 3) continue;
            double vx[4];
            ki_weights(ix, nex, px, vx);
            for (int iy = Y / 2; iy <= Y / 2 + 1; iy++) {
                const int jy = Y + 2 - 2 * iy;
                if (iy >= nbo[1] || jy < 0 || jy > 3) continue;
                double vy[4];
                ki_weights(iy, ney, py, vy);
                for (int iz = Z / 2; iz <= Z / 2 + 1; iz++) {
                    const int jz = Z + 2 - 2 * iz;
                    if (iz >= nbo[2] || jz < 0 || jz > 3) continue;
                    double vz[4];
                    ki_weights(iz, nez, pz, vz);
                    if (vx[jx] * vy[jy] * vz[jz] != 0.0) {
                        const double u = Uold[((long)(ix * nbo[1] + iy) * nbo[2] + iz) * ndof + d];
                        acc += u * vx[jx] * vy[jy] * vz[jz];
                    }
                }
            }
        }
        Unew[t * ndof + d] = acc;
    }
}

/* the stored array (nbs points per direction, periodic directions without the two
 * duplicates) -> the full (n + 2)^3 array with the periodic wrap (nurbs_knotinsert.c:25-29) */
__global__ void k_knot_wrap(const double *__restrict__ Us, double *__restrict__ Uf, int n0, int n1, int n2,
                            int s0, int s1, int s2, int ndof)
{
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long nf = (long)(n0 + 2) * (n1 + 2) * (n2 + 2);
    if (t >= nf) return;
    const int k = (int)(t % (n2 + 2)), j = (int)((t / (n2 + 2)) % (n1 + 2)), i = (int)(t / ((long)(n2 + 2) * (n1 + 2)));
    const long src = ((long)(i % s0) * s1 + (j % s1)) * s2 + (k % s2);
    for (int d = 0; d < ndof; d++) Uf[t * ndof + d] = Us[src * ndof + d];
}

/* the full array -> the stored one (nurbs_knotinsert.c:99-104) */
__global__ void k_knot_unwrap(const double *__restrict__ Uf, double *__restrict__ Us, int n0, int n1, int n2,
                              int s0, int s1, int s2, int ndof)
{
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    const long ns = (long)s0 * s1 * s2;
    if (t >= ns) return;
    const int k = (int)(t % s2), j = (int)((t / s2) % s1), i = (int)(t / ((long)s2 * s1));
    const long src = ((long)i * (n1 + 2) + j) * (n2 + 2) + k;
    for (int d = 0; d < ndof; d++) Us[t * ndof + d] = Uf[src * ndof + d];
}

} /* namespace */

extern "C" int igab_knot_insert(double *U_universal, const int nelem[3], int nref, int porder, int ndof,
                                const int bc_periodic[3], int device)
{
    if (!U_universal || !nelem || !bc_periodic || nref < 0 || ndof < 1) {
        igab_set_error("igab_knot_insert: bad argument");
        return IGAB_ERR_ARG;
    }
    if (porder != 2) {
        igab_set_error("igab_knot_insert: only porder 2 (as the reference)");
        return IGAB_ERR_ARG;
    }
    int ne[3], nbs[3];
    for (int d = 0; d < 3; d++) {
        if (nelem[d] < 1 || (nelem[d] >> nref) << nref != nelem[d] || (nelem[d] >> nref) < 1) {
            igab_set_error("igab_knot_insert: nelem must be a positive multiple of 2^nref");
            return IGAB_ERR_ARG;
        }
        ne[d] = nelem[d] >> nref;
    }
    if (nref == 0) return 0;
    for (int d = 0; d < 3; d++) nbs[d] = ne[d] + (bc_periodic[d] == 0) * 2;
    const long nstored_c = (long)nbs[0] * nbs[1] * nbs[2];
    const long nfine = (long)(nelem[0] + 2) * (nelem[1] + 2) * (nelem[2] + 2);
    if (device < 0 || device >= KNOT_MAX_DEVICES) {
        igab_set_error("igab_knot_insert: device %d out of range", device);
        return IGAB_ERR_ARG;
    }
    IGAB_CUDA_TRY(cudaSetDevice(device));
    std::lock_guard<std::mutex> lock(knot_mu);
    const size_t need = (size_t)nfine * ndof;
    cudaError_t e = cudaSuccess;
    if (knot_cap[device] < need) {
        if (knot_buf[device]) cudaFree(knot_buf[device]);
        knot_buf[device] = nullptr;
        knot_cap[device] = 0;
        e = cudaMalloc((void **)&knot_buf[device], 2 * need * sizeof(double));
        if (e != cudaSuccess) {
            knot_buf[device] = nullptr;
            igab_set_error("igab_knot_insert: %s", cudaGetErrorString(e));
            return IGAB_ERR_CUDA;
        }
        knot_cap[device] = need;
    }
    double *buf[2] = {knot_buf[device], knot_buf[device] + knot_cap[device]};
    /* the stored coarse array in buf[1], wrapped into buf[0] */
    e = cudaMemcpy(buf[1], U_universal, (size_t)nstored_c * ndof * sizeof(double), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const long nw = (long)(ne[0] + 2) * (ne[1] + 2) * (ne[2] + 2);
        k_knot_wrap<<<(unsigned)((nw + 255) / 256), 256>>>(buf[1], buf[0], ne[0], ne[1], ne[2], nbs[0], nbs[1],
                                                           nbs[2], ndof);
        e = cudaGetLastError();
    }
    int cur = 0;
    for (int lev = 0; lev < nref && e == cudaSuccess; lev++) {
        const long nnew = (long)(2 * ne[0] + 2) * (2 * ne[1] + 2) * (2 * ne[2] + 2);
        k_knot_refine<<<(unsigned)((nnew + 255) / 256), 256>>>(buf[cur], buf[1 - cur], ne[0], ne[1], ne[2],
                                                               bc_periodic[0] != 0, bc_periodic[1] != 0,
                                                               bc_periodic[2] != 0, ndof);
        e = cudaGetLastError();
        cur = 1 - cur;
        for (int d = 0; d < 3; d++) ne[d] *= 2;
    }
    /* the refined array without the periodic duplicates, back into the caller's array */
    for (int d = 0; d < 3; d++) nbs[d] = ne[d] + (bc_periodic[d] == 0) * 2;
    const long nstored_f = (long)nbs[0] * nbs[1] * nbs[2];
    if (e == cudaSuccess) {
        k_knot_unwrap<<<(unsigned)((nstored_f + 255) / 256), 256>>>(buf[cur], buf[1 - cur], ne[0], ne[1], ne[2],
                                                                    nbs[0], nbs[1], nbs[2], ndof);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = cudaMemcpy(U_universal, buf[1 - cur], (size_t)nstored_f * ndof * sizeof(double), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        igab_set_error("igab_knot_insert: %s", cudaGetErrorString(e));
        return IGAB_ERR_CUDA;
    }
    return 0;
}

extern "C" int igab_knot_release(int device)
{
    if (device < 0 || device >= KNOT_MAX_DEVICES) {
        igab_set_error("igab_knot_release: device %d out of range", device);
        return IGAB_ERR_ARG;
    }
    std::lock_guard<std::mutex> lock(knot_mu);
    if (!knot_buf[device]) return 0;
    IGAB_CUDA_TRY(cudaSetDevice(device));
    const cudaError_t e = cudaFree(knot_buf[device]);
    knot_buf[device] = nullptr;
    knot_cap[device] = 0;
    if (e != cudaSuccess) {
        igab_set_error("igab_knot_release: %s", cudaGetErrorString(e));
        return IGAB_ERR_CUDA;
    }
    return 0;
}

extern "C" int igab_write_solution(const char *fname, const double *U_hist, long ndof, int ihist0, int ihist1)
{
    if (!fname || !U_hist || ndof < 1 || ihist0 < 0 || ihist1 < ihist0) {
        igab_set_error("igab_write_solution: bad argument");
        return IGAB_ERR_ARG;
    }
    FILE *f = fopen(fname, "wb");
    if (!f) {
        igab_set_error("igab_write_solution: cannot open %s", fname);
        return IGAB_ERR_ARG;
    }
    const size_t n = (size_t)(ihist1 - ihist0) * (size_t)ndof;
    const size_t w = fwrite(U_hist + (size_t)ihist0 * ndof, sizeof(double), n, f);
    const int closed = fclose(f);
    if (w != n || closed != 0) {
        igab_set_error("igab_write_solution: short write to %s", fname);
        return IGAB_ERR_ARG;
    }
    return 0;
}

extern "C" int igab_read_solution(const char *fname, double *U_hist, long ndof, int ihist0, int ihist1)
{
    if (!fname || !U_hist || ndof < 1 || ihist0 < 0 || ihist1 < ihist0) {
        igab_set_error("igab_read_solution: bad argument");
        return IGAB_ERR_ARG;
    }
    FILE *f = fopen(fname, "rb");
    if (!f) {
        igab_set_error("igab_read_solution: cannot open %s", fname);
        return IGAB_ERR_ARG;
    }
    const size_t n = (size_t)(ihist1 - ihist0) * (size_t)ndof;
    /* a short file is an error before anything is read: the caller's array stays as it was */
    long bytes = -1;
    if (fseek(f, 0, SEEK_END) == 0) bytes = ftell(f);
    if (bytes < 0 || (size_t)bytes < n * sizeof(double) || fseek(f, 0, SEEK_SET) != 0) {
        fclose(f);
        igab_set_error("igab_read_solution: %s holds fewer than %zu values", fname, n);
        return IGAB_ERR_ARG;
    }
    const size_t r = fread(U_hist + (size_t)ihist0 * ndof, sizeof(double), n, f);
    fclose(f);
    if (r != n) {
        igab_set_error("igab_read_solution: %s holds fewer than %zu values", fname, n);
        return IGAB_ERR_ARG;
    }
    return 0;
}
