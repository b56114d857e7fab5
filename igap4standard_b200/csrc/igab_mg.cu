/*
 * Geometric multigrid on nested spline spaces, as the preconditioner of a GMRES or
 * conjugate gradient solve with the assembled tangent (no reference counterpart: it
 * stands in for the PETSc KSP of the reference application, src/snes_init.c:24-39,
 * which is outside the assembly path).
 *
 * Why: the phys/ge tangent is a fourth-order operator (the strain-gradient term
 * le^2 |grad grad u|^2), so its condition number grows like h^-4; Jacobi-preconditioned
 * Krylov iterations stall at 32^3 and 64^3.  Multigrid keeps the iteration count flat.
 *
 * Hierarchy.  Level 0 is the caller's mesh.  Level l+1 removes every other interior
 * knot of level l in each direction (n elements -> n / 2), so its spline space is a
 * subspace of level l's: the prolongation is knot insertion of the removed knots
 * (Boehm's algorithm for p = 2, built on the host as three 1-D matrices, applied on
 * the device as their tensor product), the restriction its transpose.  Coarsening stops
 * at about a thousand dofs, or where a direction has an odd element count.  Coarse
 * operators are rediscretised: each coarse level is an igab context with the same
 * material, boundary tables and (averaged) element scales, whose tangent is assembled
 * at the zero state by the library's own kernels (a preconditioner, so the state it is
 * linearised at only affects the convergence rate).  The coarsest level is solved
 * directly (dense LU with partial pivoting on the host).  Dirichlet rows, identity rows
 * of every level's tangent, are masked out of the restricted residuals and of the
 * prolonged corrections, which keeps the V-cycle symmetric.
 *
 * Smoother: Chebyshev polynomial of degree 3 in D^-1 K on [lmax / 10, 1.1 lmax], lmax
 * estimated by power iteration; the same polynomial before and after the coarse
 * correction, so the V-cycle is a symmetric preconditioner and CG applies.
 *
 * Coarsest level: its tangent (symmetric positive definite: the zero-state tangent with
 * unit Dirichlet rows and columns) is inverted on the device by Gauss-Jordan elimination
 * without pivoting, one launch per pivot, and each V-cycle applies the inverse as a dense
 * product with a fixed summation order (no host round trip).  A pivot that is not
 * positive and finite (an unstable material) falls back to a dense LU with partial
 * pivoting on the host.
 *
 * Operators: every level's is the tangent at the zero state (the fine one in FP32, the
 * coarse ones in FP64), symmetric positive definite for a stable material, so the V-cycle
 * does not depend on the Newton iterate.  The hierarchy is rebuilt when the material, the
 * boundary tables' values or the element scales change (the context's parameter
 * version).  Every dot product is a fixed-order reduction: solves are bitwise repeatable.
 * Measured and rejected: the smoothing operators stored in half precision (64^3: 4.58 ->
 * 4.36 ms per GMRES iteration, but one more iteration per solve; no gain per Newton step).
 */
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>
#include <cuda_runtime.h>
#include "igab_internal.h"
#include "igab_reduce.cuh"

namespace {

#define MG_THREADS 256
#define MG_BLOCKS 296
#define MG_MAX_LEVELS 8
#define MG_DEGREE 3            /* Chebyshev degree per smoothing */
#define MG_POWER_ITERS 12      /* power iterations for lmax of D^-1 K */
#define MG_COARSE_DOF 1200     /* the coarsest level is solved directly below this size */

/* 1-D prolongation along one direction: fine coefficient i = sum_a w[i][a] coarse idx[i][a]
 * (kp entries per fine point), restriction coarse j = sum_b rw[j][b] fine ridx[j][b] */
struct mg_dir {
    int nf = 0, nc = 0, kp = 0, kr = 0;
    int *p_idx = nullptr;
    double *p_w = nullptr;
    int *r_idx = nullptr;
    double *r_w = nullptr;
};

struct mg_level {
    igab_ctx *ctx = nullptr;       /* level 0: the caller's; coarser: owned */
    long n = 0;
    const void *vals = nullptr;    /* the level's tangent values */
    int prec = IGAB_PREC_FP64;
    double *own_vals = nullptr;    /* coarse levels: FP64 tangent at the zero state */
    double *dinv = nullptr;
    double lmax = 0.0;
    double *x = nullptr, *b = nullptr, *r = nullptr, *d = nullptr, *t = nullptr;
    mg_dir dir[3];                 /* transfer between this level (coarse) and the one above */
};

__global__ void k_mg_diag_inv(igab_geom g, const void *__restrict__ vals, int prec, double *__restrict__ dinv)
{
    const long r = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (r >= g.ndof) return;
    const long cp = r / 3;
    const int k1 = (int)(r % 3);
    const int z1 = (int)(cp % g.nb[2]), y1 = (int)((cp / g.nb[2]) % g.nb[1]), x1 = (int)(cp / ((long)g.nb[2] * g.nb[1]));
    const int x0 = x1 > 2 ? x1 - 2 : 0, y0 = y1 > 2 ? y1 - 2 : 0, z0 = z1 > 2 ? z1 - 2 : 0;
    const int ye = y1 + 2 < g.nb[1] - 1 ? y1 + 2 : g.nb[1] - 1;
    const int ze = z1 + 2 < g.nb[2] - 1 ? z1 + 2 : g.nb[2] - 1;
    const int nyb = ye - y0 + 1, nzb = ze - z0 + 1;
    const long pos = g.rowptr[r] + (((long)(x1 - x0) * nyb + (y1 - y0)) * nzb + (z1 - z0)) * 3 + k1;
    const double dv = prec == IGAB_PREC_FP64 ? ((const double *)vals)[pos] : (double)((const float *)vals)[pos];
    dinv[r] = dv != 0.0 ? 1.0 / dv : 1.0;
}

#define MG_LOOP(i, n) for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < (n); i += (long)gridDim.x * blockDim.x)

/* d = s * dinv * r */
__global__ void k_mg_jac(long n, const double *__restrict__ dinv, const double *__restrict__ r, double s,
                         double *__restrict__ d)
{
    MG_LOOP(i, n) d[i] = s * dinv[i] * r[i];
}

/* x += d, (x was zero when first) */
__global__ void k_mg_add(long n, const double *__restrict__ d, double *__restrict__ x, int first)
{
    MG_LOOP(i, n) x[i] = first ? d[i] : x[i] + d[i];
}

/* r -= t; d = a d + c dinv r */
__global__ void k_mg_cheb(long n, const double *__restrict__ t, const double *__restrict__ dinv, double a, double c,
                          double *__restrict__ r, double *__restrict__ d, int update_d)
{
    MG_LOOP(i, n)
    {
        const double ri = r[i] - t[i];
        r[i] = ri;
        if (update_d) d[i] = a * d[i] + c * dinv[i] * ri;
    }
}

/* r = b - t */
__global__ void k_mg_sub(long n, const double *__restrict__ b, const double *__restrict__ t, double *__restrict__ r)
{
    MG_LOOP(i, n) r[i] = b[i] - t[i];
}

/* y = a x + b y */
__global__ void k_mg_axpby(long n, double a, const double *__restrict__ x, double b, double *__restrict__ y)
{
    MG_LOOP(i, n) y[i] = a * x[i] + b * y[i];
}

__global__ void k_mg_copy(long n, const double *__restrict__ x, double *__restrict__ y)
{
    MG_LOOP(i, n) y[i] = x[i];
}

__global__ void k_mg_zero_rows(long nd, const int *__restrict__ rows, double *__restrict__ v)
{
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t < nd) v[rows[t]] = 0.0;
}

struct mg_dirs_dev {
    const int *p_idx[3];
    const double *p_w[3];
    const int *r_idx[3];
    const double *r_w[3];
    int kp[3], kr[3];
    int nbf[3], nbc[3];
};

/* xf += P xc (tensor product of the three 1-D prolongations, per displacement component) */
__global__ void k_mg_prolong(mg_dirs_dev D, const double *__restrict__ xc, double *__restrict__ xf)
{
    const long nf = (long)D.nbf[0] * D.nbf[1] * D.nbf[2];
    MG_LOOP(f, nf)
    {
        const int iz = (int)(f % D.nbf[2]), iy = (int)((f / D.nbf[2]) % D.nbf[1]), ix = (int)(f / ((long)D.nbf[2] * D.nbf[1]));
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int a = 0; a < D.kp[0]; a++) {
            const double wa = D.p_w[0][ix * D.kp[0] + a];
            const int ja = D.p_idx[0][ix * D.kp[0] + a];
            for (int b = 0; b < D.kp[1]; b++) {
                const double wab = wa * D.p_w[1][iy * D.kp[1] + b];
                const long jab = ((long)ja * D.nbc[1] + D.p_idx[1][iy * D.kp[1] + b]) * D.nbc[2];
                for (int c = 0; c < D.kp[2]; c++) {
                    const double w = wab * D.p_w[2][iz * D.kp[2] + c];
                    const double *u = xc + 3 * (jab + D.p_idx[2][iz * D.kp[2] + c]);
                    s0 += w * u[0];
                    s1 += w * u[1];
                    s2 += w * u[2];
                }
            }
        }
        xf[3 * f] += s0;
        xf[3 * f + 1] += s1;
        xf[3 * f + 2] += s2;
    }
}

/* rc = P^T rf */
__global__ void k_mg_restrict(mg_dirs_dev D, const double *__restrict__ rf, double *__restrict__ rc)
{
    const long nc = (long)D.nbc[0] * D.nbc[1] * D.nbc[2];
    MG_LOOP(j, nc)
    {
        const int jz = (int)(j % D.nbc[2]), jy = (int)((j / D.nbc[2]) % D.nbc[1]), jx = (int)(j / ((long)D.nbc[2] * D.nbc[1]));
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (int a = 0; a < D.kr[0]; a++) {
            const double wa = D.r_w[0][jx * D.kr[0] + a];
            const int ia = D.r_idx[0][jx * D.kr[0] + a];
            for (int b = 0; b < D.kr[1]; b++) {
                const double wab = wa * D.r_w[1][jy * D.kr[1] + b];
                const long iab = ((long)ia * D.nbf[1] + D.r_idx[1][jy * D.kr[1] + b]) * D.nbf[2];
                for (int c = 0; c < D.kr[2]; c++) {
                    const double w = wab * D.r_w[2][jz * D.kr[2] + c];
                    const double *u = rf + 3 * (iab + D.r_idx[2][jz * D.kr[2] + c]);
                    s0 += w * u[0];
                    s1 += w * u[1];
                    s2 += w * u[2];
                }
            }
        }
        rc[3 * j] = s0;
        rc[3 * j + 1] = s1;
        rc[3 * j + 2] = s2;
    }
}

} /* namespace */

/* 1-D prolongation by knot insertion (Boehm, p = 2): the coarse knot vector kc (open)
 * refined by the knots `ins` (ascending, inside the open interval) into the fine one.
 * P[i][j] (nb_f x nb_c, row-major) maps coarse spline coefficients to fine ones. */
static void igab_mg_knot_prolongation(const std::vector<double> &kc, const std::vector<double> &ins,
                                      std::vector<double> &P, int &nbf, int &nbc)
{
    std::vector<double> kv = kc;
    nbc = (int)kc.size() - 3;
    std::vector<std::vector<double>> M(nbc, std::vector<double>(nbc, 0.0));
    for (int j = 0; j < nbc; j++) M[j][j] = 1.0;
    for (double t : ins) {
        const int nk = (int)kv.size(), nb = nk - 3;
        int k = 2;
        while (k + 1 < nk - 3 && !(kv[k] <= t && t < kv[k + 1])) k++;
        std::vector<std::vector<double>> Q(nb + 1, std::vector<double>(nbc, 0.0));
        for (int i = 0; i <= nb; i++) {
            if (i <= k - 2) Q[i] = M[i];
            else if (i >= k + 1) Q[i] = M[i - 1];
            else {
                const double a = (t - kv[i]) / (kv[i + 2] - kv[i]);
                for (int j = 0; j < nbc; j++) Q[i][j] = a * M[i][j] + (1.0 - a) * M[i - 1][j];
            }
        }
        M.swap(Q);
        kv.insert(kv.begin() + k + 1, t);
    }
    nbf = (int)M.size();
    P.assign((size_t)nbf * nbc, 0.0);
    for (int i = 0; i < nbf; i++)
        for (int j = 0; j < nbc; j++) P[(size_t)i * nbc + j] = M[i][j];
}

struct igab_mg {
    int nlev = 0;
    mg_level L[MG_MAX_LEVELS];
    long version = -1;
    bool direct = false;            /* coarsest level solved directly */
    bool dev_inv = false;           /* by the device inverse (else by the host LU) */
    int nd = 0;                     /* its size */
    std::vector<double> lu;
    std::vector<int> piv;
    double *h_vec = nullptr;        /* pinned nd doubles */
    double *inv = nullptr;          /* nd x nd inverse of the coarsest tangent (row-major) */
    double *gj = nullptr;           /* Gauss-Jordan pivot row and column buffers, 2 x 2 x nd */
    int *gj_flag = nullptr;         /* set by a pivot that is not positive and finite */
    double *part = nullptr, *dots = nullptr, *h_dots = nullptr;
    double *zero = nullptr;         /* zero state (fine size) */
    long zero_n = 0;
    void *fine_vals = nullptr;      /* the caller's tangent at the zero state, FP32 */
    double *kv = nullptr;           /* Krylov vectors of the caller's mesh */
    long kv_n = 0;
    double *mpart = nullptr;        /* multi-dot partial sums [GM_RESTART + 1][RD_BLOCKS] and results */
    double *h_md = nullptr;         /* pinned results of a multi-dot */
    int launches = 0;
};

namespace {

int mg_free_level(mg_level &L, bool own)
{
    if (own && L.ctx) igab_destroy(L.ctx);
    cudaFree(L.own_vals);
    cudaFree(L.dinv);
    cudaFree(L.x);
    for (int d = 0; d < 3; d++) {
        cudaFree(L.dir[d].p_idx);
        cudaFree(L.dir[d].p_w);
        cudaFree(L.dir[d].r_idx);
        cudaFree(L.dir[d].r_w);
    }
    L = mg_level();
    return 0;
}

void mg_free(igab_mg *m)
{
    if (!m) return;
    for (int l = 0; l < m->nlev; l++) mg_free_level(m->L[l], l > 0);
    cudaFree(m->part);
    cudaFree(m->zero);
    cudaFree(m->fine_vals);
    cudaFree(m->kv);
    cudaFree(m->mpart);
    cudaFreeHost(m->h_md);
    cudaFreeHost(m->h_vec);
    cudaFree(m->inv);
    cudaFree(m->gj);
    cudaFree(m->gj_flag);
    cudaFreeHost(m->h_dots);
    delete m;
}

int mg_vectors(mg_level &L)
{
    const size_t bytes = (size_t)L.n * sizeof(double);
    IGAB_CUDA_TRY(cudaMalloc((void **)&L.x, 5 * bytes));
    L.b = L.x + L.n;
    L.r = L.b + L.n;
    L.d = L.r + L.n;
    L.t = L.d + L.n;
    IGAB_CUDA_TRY(cudaMalloc((void **)&L.dinv, bytes));
    return 0;
}

int mg_upload_dir(mg_dir &D, const std::vector<double> &P, int nbf, int nbc)
{
    std::vector<std::vector<std::pair<int, double>>> rows(nbf), cols(nbc);
    for (int i = 0; i < nbf; i++)
        for (int j = 0; j < nbc; j++) {
            const double w = P[(size_t)i * nbc + j];
            if (w != 0.0) {
                rows[i].push_back({j, w});
                cols[j].push_back({i, w});
            }
        }
    int kp = 1, kr = 1;
    for (auto &r : rows) kp = std::max(kp, (int)r.size());
    for (auto &c : cols) kr = std::max(kr, (int)c.size());
    std::vector<int> pi((size_t)nbf * kp, 0), ri((size_t)nbc * kr, 0);
    std::vector<double> pw((size_t)nbf * kp, 0.0), rw((size_t)nbc * kr, 0.0);
    for (int i = 0; i < nbf; i++)
        for (size_t a = 0; a < rows[i].size(); a++) {
            pi[(size_t)i * kp + a] = rows[i][a].first;
            pw[(size_t)i * kp + a] = rows[i][a].second;
        }
    for (int j = 0; j < nbc; j++)
        for (size_t b = 0; b < cols[j].size(); b++) {
            ri[(size_t)j * kr + b] = cols[j][b].first;
            rw[(size_t)j * kr + b] = cols[j][b].second;
        }
    D.nf = nbf;
    D.nc = nbc;
    D.kp = kp;
    D.kr = kr;
    IGAB_CUDA_TRY(cudaMalloc((void **)&D.p_idx, pi.size() * sizeof(int)));
    IGAB_CUDA_TRY(cudaMalloc((void **)&D.p_w, pw.size() * sizeof(double)));
    IGAB_CUDA_TRY(cudaMalloc((void **)&D.r_idx, ri.size() * sizeof(int)));
    IGAB_CUDA_TRY(cudaMalloc((void **)&D.r_w, rw.size() * sizeof(double)));
    IGAB_CUDA_TRY(cudaMemcpy(D.p_idx, pi.data(), pi.size() * sizeof(int), cudaMemcpyHostToDevice));
    IGAB_CUDA_TRY(cudaMemcpy(D.p_w, pw.data(), pw.size() * sizeof(double), cudaMemcpyHostToDevice));
    IGAB_CUDA_TRY(cudaMemcpy(D.r_idx, ri.data(), ri.size() * sizeof(int), cudaMemcpyHostToDevice));
    IGAB_CUDA_TRY(cudaMemcpy(D.r_w, rw.data(), rw.size() * sizeof(double), cudaMemcpyHostToDevice));
    return 0;
}

mg_dirs_dev dirs_view(const mg_level &C)
{
    mg_dirs_dev D;
    for (int d = 0; d < 3; d++) {
        D.p_idx[d] = C.dir[d].p_idx;
        D.p_w[d] = C.dir[d].p_w;
        D.r_idx[d] = C.dir[d].r_idx;
        D.r_w[d] = C.dir[d].r_w;
        D.kp[d] = C.dir[d].kp;
        D.kr[d] = C.dir[d].kr;
        D.nbf[d] = C.dir[d].nf;
        D.nbc[d] = C.dir[d].nc;
    }
    return D;
}

/* dense LU with partial pivoting (column-major n x n in a), in place */
bool lu_factor(int n, std::vector<double> &a, std::vector<int> &piv)
{
    piv.resize(n);
    for (int k = 0; k < n; k++) {
        int p = k;
        double mx = std::fabs(a[(size_t)k * n + k]);
        for (int i = k + 1; i < n; i++)
            if (std::fabs(a[(size_t)k * n + i]) > mx) { mx = std::fabs(a[(size_t)k * n + i]); p = i; }
        if (mx == 0.0) return false;
        piv[k] = p;
        if (p != k)
            for (int j = 0; j < n; j++) std::swap(a[(size_t)j * n + k], a[(size_t)j * n + p]);
        const double inv = 1.0 / a[(size_t)k * n + k];
        for (int i = k + 1; i < n; i++) a[(size_t)k * n + i] *= inv;
        for (int j = k + 1; j < n; j++) {
            const double akj = a[(size_t)j * n + k];
            if (akj != 0.0)
                for (int i = k + 1; i < n; i++) a[(size_t)j * n + i] -= a[(size_t)k * n + i] * akj;
        }
    }
    return true;
}

void lu_solve(int n, const std::vector<double> &a, const std::vector<int> &piv, double *x)
{
    for (int k = 0; k < n; k++) std::swap(x[k], x[piv[k]]);
    for (int j = 0; j < n; j++)
        for (int i = j + 1; i < n; i++) x[i] -= a[(size_t)j * n + i] * x[j];
    for (int j = n - 1; j >= 0; j--) {
        x[j] /= a[(size_t)j * n + j];
        for (int i = 0; i < j; i++) x[i] -= a[(size_t)j * n + i] * x[j];
    }
}

int spmv(igab_mg *m, mg_level &L, const double *x, double *y)
{
    const int rc = igab_launch_spmv(L.ctx, L.vals, L.prec, x, y);
    m->launches++;
    return rc;
}

/* lmax of D^-1 K by power iteration from a fixed start vector */
int estimate_lmax(igab_mg *m, mg_level &L)
{
    cudaStream_t st = L.ctx->stream;
    const long n = L.n;
    std::vector<double> v0((size_t)n);
    unsigned s = 12345u;
    for (long i = 0; i < n; i++) {
        s = s * 1664525u + 1013904223u;
        v0[(size_t)i] = 0.5 + (double)(s >> 8) / (double)(1u << 24);
    }
    IGAB_CUDA_TRY(cudaMemcpyAsync(L.d, v0.data(), (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st));
    double lam = 0.0, dd[2];
    for (int it = 0; it < MG_POWER_ITERS; it++) {
        int rc = spmv(m, L, L.d, L.t);
        if (rc) return rc;
        k_mg_jac<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, L.dinv, L.t, 1.0, L.r);   /* r = D^-1 K d */
        IGAB_CUDA_TRY(rd_dot2(st, n, L.r, L.r, L.d, L.d, m->part, m->dots, m->h_dots, dd));
        const double nr = std::sqrt(dd[0]);
        lam = dd[1] > 0.0 ? nr / std::sqrt(dd[1]) : 0.0;
        if (nr == 0.0) break;
        k_mg_axpby<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, 1.0 / nr, L.r, 0.0, L.d);   /* d = r / ||r|| */
        m->launches += 4;
    }
    L.lmax = lam > 0.0 ? lam : 1.0;
    return 0;
}

/* Chebyshev smoothing of K x = b on level L from the current (x, r = b - K x);
 * first: x is zero (x and r written from scratch: r = b on entry) */
int chebyshev(igab_mg *m, mg_level &L, bool first)
{
    cudaStream_t st = L.ctx->stream;
    const long n = L.n;
    const double hi = 1.1 * L.lmax, lo = hi / 10.0;
    const double theta = 0.5 * (hi + lo), delta = 0.5 * (hi - lo), sigma = theta / delta;
    double rho = 1.0 / sigma;
    k_mg_jac<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, L.dinv, L.r, 1.0 / theta, L.d);
    for (int i = 0; i < MG_DEGREE; i++) {
        k_mg_add<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, L.d, L.x, first && i == 0);
        int rc = spmv(m, L, L.d, L.t);
        if (rc) return rc;
        const double rn = 1.0 / (2.0 * sigma - rho);
        k_mg_cheb<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, L.t, L.dinv, rn * rho, 2.0 * rn / delta, L.r, L.d,
                                                     i + 1 < MG_DEGREE);
        rho = rn;
        m->launches += 2;
    }
    m->launches++;
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

void zero_dirichlet(igab_mg *m, mg_level &L, double *v)
{
    if (L.ctx->nd > 0) {
        k_mg_zero_rows<<<(unsigned)((L.ctx->nd + 255) / 256), 256, 0, L.ctx->stream>>>(L.ctx->nd, L.ctx->d_drow, v);
        m->launches++;
    }
}

/* A (row-major n x n) from the structured CSR of the coarsest level: one thread per row */
__global__ void k_mg_dense(int n, const int *__restrict__ rowptr, const int *__restrict__ cols,
                           const double *__restrict__ vals, double *__restrict__ A)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n) return;
    for (int k = rowptr[r]; k < rowptr[r + 1]; k++) A[(size_t)r * n + cols[k]] = vals[k];
}

/* pivot row and column 0 into the step buffers */
__global__ void k_mg_gj_init(int n, const double *__restrict__ A, double *__restrict__ row, double *__restrict__ col)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    row[i] = A[i];
    col[i] = A[(size_t)i * n];
}

/* Gauss-Jordan step k in place (row-major A), from the old pivot row / column (row, col);
 * writes row / column k + 1 of the result into (nrow, ncol) for the next step.  Each
 * entry is computed by one thread from the old values only. */
__global__ void k_mg_gj_step(int n, int k, double *__restrict__ A, const double *__restrict__ row,
                             const double *__restrict__ col, double *__restrict__ nrow, double *__restrict__ ncol,
                             int *__restrict__ flag)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= n || j >= n) return;
    const double p = col[k];
    if (i == k && j == k && !(p > 0.0 && isfinite(p))) *flag = 1;
    const double ip = 1.0 / p;
    double v;
    if (i == k) v = j == k ? ip : row[j] * ip;
    else if (j == k) v = -col[i] * ip;
    else v = A[(size_t)i * n + j] - col[i] * (row[j] * ip);
    A[(size_t)i * n + j] = v;
    if (i == k + 1) nrow[j] = v;
    if (j == k + 1) ncol[i] = v;
}

/* x = Ainv b: one warp per row, lane-strided partial sums then a fixed shuffle tree */
__global__ void k_mg_gemv(long n, const double *__restrict__ Ai, const double *__restrict__ b, double *__restrict__ x)
{
    const long r = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (r >= n) return;
    double s = 0.0;
    for (long j = lane; j < n; j += 32) s += Ai[r * n + j] * b[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) x[r] = s;
}

/* x_l = V-cycle approximation of K_l^-1 b_l (b in L.b, result in L.x) */
int vcycle(igab_mg *m, int l)
{
    mg_level &L = m->L[l];
    cudaStream_t st = L.ctx->stream;
    if (l == m->nlev - 1) {
        if (m->direct && m->dev_inv) {
            k_mg_gemv<<<(unsigned)((L.n + 7) / 8), 256, 0, st>>>(L.n, m->inv, L.b, L.x);
            m->launches++;
        } else if (m->direct) {
            IGAB_CUDA_TRY(cudaMemcpyAsync(m->h_vec, L.b, (size_t)L.n * sizeof(double), cudaMemcpyDeviceToHost, st));
            IGAB_CUDA_TRY(cudaStreamSynchronize(st));
            lu_solve(m->nd, m->lu, m->piv, m->h_vec);
            IGAB_CUDA_TRY(cudaMemcpyAsync(L.x, m->h_vec, (size_t)L.n * sizeof(double), cudaMemcpyHostToDevice, st));
        } else {
            k_mg_jac<<<MG_BLOCKS, MG_THREADS, 0, st>>>(L.n, L.dinv, L.b, 1.0, L.x);
            m->launches++;
        }
        return 0;
    }
    mg_level &C = m->L[l + 1];
    k_mg_copy<<<MG_BLOCKS, MG_THREADS, 0, st>>>(L.n, L.b, L.r);
    m->launches++;
    int rc = chebyshev(m, L, true);
    if (rc) return rc;
    /* coarse correction with the Dirichlet rows of both levels masked (symmetric) */
    zero_dirichlet(m, L, L.r);
    const mg_dirs_dev D = dirs_view(C);
    k_mg_restrict<<<MG_BLOCKS, MG_THREADS, 0, st>>>(D, L.r, C.b);
    m->launches++;
    zero_dirichlet(m, C, C.b);
    if ((rc = vcycle(m, l + 1))) return rc;
    zero_dirichlet(m, C, C.x);
    IGAB_CUDA_TRY(cudaMemsetAsync(L.t, 0, (size_t)L.n * sizeof(double), st));
    k_mg_prolong<<<MG_BLOCKS, MG_THREADS, 0, st>>>(D, C.x, L.t);
    m->launches++;
    zero_dirichlet(m, L, L.t);
    k_mg_axpby<<<MG_BLOCKS, MG_THREADS, 0, st>>>(L.n, 1.0, L.t, 1.0, L.x);
    /* r = b - K x, then the same smoother again */
    if ((rc = spmv(m, L, L.x, L.t))) return rc;
    k_mg_sub<<<MG_BLOCKS, MG_THREADS, 0, st>>>(L.n, L.b, L.t, L.r);
    m->launches += 2;
    if ((rc = chebyshev(m, L, false))) return rc;
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

/* the coarse levels for the context's current parameters */
int mg_build(igab_ctx *c, igab_mg *m)
{
    for (int l = 1; l < m->nlev; l++) mg_free_level(m->L[l], true);
    m->nlev = 1;
    m->direct = false;
    mg_level &F = m->L[0];
    F.ctx = c;
    F.n = c->ndof;
    if (!F.x) {
        int rc = mg_vectors(F);
        if (rc) return rc;
    }
    /* the preconditioner's fine operator: the caller's tangent at the zero state (FP32),
     * symmetric positive definite for a stable material whatever the current state is */
    if (!m->zero || m->zero_n < F.n) {
        cudaFree(m->zero);
        m->zero = nullptr;
        IGAB_CUDA_TRY(cudaMalloc((void **)&m->zero, (size_t)F.n * sizeof(double)));
        IGAB_CUDA_TRY(cudaMemset(m->zero, 0, (size_t)F.n * sizeof(double)));
        m->zero_n = F.n;
    }
    if (!m->fine_vals) IGAB_CUDA_TRY(cudaMalloc(&m->fine_vals, (size_t)c->nnz * sizeof(float)));
    {
        int rc = igab_launch_tangent(c, m->zero, m->fine_vals, IGAB_PREC_FP32);
        if (rc) return rc;
    }
    F.vals = m->fine_vals;
    F.prec = IGAB_PREC_FP32;
    k_mg_diag_inv<<<(unsigned)((F.n + 255) / 256), 256, 0, c->stream>>>(c->geom(), F.vals, F.prec, F.dinv);
    IGAB_CUDA_TRY(cudaGetLastError());
    {
        int rc = estimate_lmax(m, F);
        if (rc) return rc;
    }
    /* element log-scales of the caller's context (averaged per coarse element below) */
    std::vector<double> s_f;
    if (c->escale_on) {
        s_f.resize((size_t)c->nel);
        IGAB_CUDA_TRY(cudaMemcpy(s_f.data(), c->d_escale, (size_t)c->nel * sizeof(double), cudaMemcpyDeviceToHost));
    }
    while (m->nlev < MG_MAX_LEVELS) {
        igab_ctx *f = m->L[m->nlev - 1].ctx;
        if (f->ndof <= MG_COARSE_DOF) break;
        bool ok = true;
        for (int d = 0; d < 3; d++) ok = ok && f->ne[d] % 2 == 0 && f->ne[d] >= 4;
        if (!ok) break;
        igab_mesh_desc desc;
        memset(&desc, 0, sizeof(desc));
        desc.phys = f->phys;
        std::vector<double> kn;
        std::vector<double> knc[3], ins[3];
        for (int d = 0; d < 3; d++) {
            const std::vector<double> &kf = f->knots[d];
            const int n = f->ne[d];
            desc.nelem[d] = n / 2;
            knc[d].assign(kf.begin(), kf.begin() + 3);
            for (int i = 1; i < n; i++) {   /* interior knot i sits at kf[2 + i] */
                if (i % 2 == 0) knc[d].push_back(kf[2 + i]);
                else ins[d].push_back(kf[2 + i]);
            }
            knc[d].insert(knc[d].end(), kf.end() - 3, kf.end());
            kn.insert(kn.end(), knc[d].begin(), knc[d].end());
        }
        desc.knots = kn.data();
        memcpy(desc.par_mat, f->par_mat, sizeof(desc.par_mat));
        memcpy(desc.bc_type, f->bc_type, sizeof(desc.bc_type));
        memcpy(desc.par_periodic, f->par_periodic, sizeof(desc.par_periodic));
        memcpy(desc.par_dirichlet, f->par_dirichlet, sizeof(desc.par_dirichlet));
        igab_ctx *cc = nullptr;
        int rc = igab_create(&desc, f->device, &cc);
        if (rc) return rc;
        mg_level &C = m->L[m->nlev];
        C.ctx = cc;
        m->nlev++;
        if ((rc = igab_set_stream(cc, c->stream))) return rc;
        C.n = cc->ndof;
        C.prec = IGAB_PREC_FP64;
        for (int d = 0; d < 3; d++) {
            std::vector<double> P;
            int nbf = 0, nbc = 0;
            igab_mg_knot_prolongation(knc[d], ins[d], P, nbf, nbc);
            if (nbf != f->nb[d] || nbc != cc->nb[d]) {
                igab_set_error("multigrid: prolongation size %d x %d, expected %d x %d", nbf, nbc, f->nb[d], cc->nb[d]);
                return IGAB_ERR_ARG;
            }
            if ((rc = mg_upload_dir(C.dir[d], P, nbf, nbc))) return rc;
        }
        if ((rc = mg_vectors(C))) return rc;
        /* element scales: the mean of the eight fine elements of each coarse element */
        if (!s_f.empty()) {
            const int *nf = f->ne, *nc = cc->ne;
            std::vector<double> gc((size_t)cc->nel);
            for (int ex = 0; ex < nc[0]; ex++)
                for (int ey = 0; ey < nc[1]; ey++)
                    for (int ez = 0; ez < nc[2]; ez++) {
                        double sum = 0.0;
                        for (int k = 0; k < 8; k++) {
                            const long fe = ((long)(2 * ex + (k >> 2)) * nf[1] + 2 * ey + ((k >> 1) & 1)) * nf[2] +
                                            2 * ez + (k & 1);
                            sum += s_f[(size_t)fe];
                        }
                        gc[((size_t)ex * nc[1] + ey) * nc[2] + ez] = std::log(sum / 8.0);
                    }
            std::vector<double> sc((size_t)cc->nel);
            for (size_t e = 0; e < sc.size(); e++) sc[e] = std::exp(gc[e]);
            s_f.swap(sc);
            if ((rc = igab_set_element_log_scale(cc, gc.data(), 0))) return rc;
        }
        /* the coarse tangent at the zero state (m->zero holds the fine level's zeros) */
        IGAB_CUDA_TRY(cudaMalloc((void **)&C.own_vals, (size_t)cc->nnz * sizeof(double)));
        if ((rc = igab_launch_tangent(cc, m->zero, C.own_vals, IGAB_PREC_FP64))) return rc;
        C.vals = C.own_vals;
        k_mg_diag_inv<<<(unsigned)((C.n + 255) / 256), 256, 0, c->stream>>>(cc->geom(), C.vals, C.prec, C.dinv);
        IGAB_CUDA_TRY(cudaGetLastError());
        if ((rc = estimate_lmax(m, C))) return rc;
    }
    /* the coarsest level directly, when small: the device inverse */
    mg_level &B = m->L[m->nlev - 1];
    m->dev_inv = false;
    if (m->nlev > 1 && B.n <= MG_COARSE_DOF) {
        igab_ctx *cc = B.ctx;
        const int n = (int)B.n;
        cudaFree(m->inv);
        cudaFree(m->gj);
        m->inv = nullptr;
        m->gj = nullptr;
        IGAB_CUDA_TRY(cudaMalloc((void **)&m->inv, (size_t)n * n * sizeof(double)));
        IGAB_CUDA_TRY(cudaMalloc((void **)&m->gj, (size_t)4 * n * sizeof(double)));
        if (!m->gj_flag) IGAB_CUDA_TRY(cudaMalloc((void **)&m->gj_flag, sizeof(int)));
        int *dcols = nullptr;
        IGAB_CUDA_TRY(cudaMalloc((void **)&dcols, (size_t)cc->nnz * sizeof(int)));
        int rc = igab_launch_csr_cols(cc, dcols);
        if (!rc) {
            cudaStream_t st = c->stream;
            cudaError_t e = cudaMemsetAsync(m->inv, 0, (size_t)n * n * sizeof(double), st);
            if (e == cudaSuccess) e = cudaMemsetAsync(m->gj_flag, 0, sizeof(int), st);
            if (e == cudaSuccess) {
                k_mg_dense<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, cc->d_rowptr, dcols, B.own_vals, m->inv);
                k_mg_gj_init<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, m->inv, m->gj, m->gj + n);
                const dim3 grid((unsigned)((n + 15) / 16), (unsigned)((n + 15) / 16)), blk(16, 16);
                for (int k = 0; k < n; k++) {
                    double *rk = m->gj + (size_t)(k & 1) * 2 * n, *nx = m->gj + (size_t)((k + 1) & 1) * 2 * n;
                    k_mg_gj_step<<<grid, blk, 0, st>>>(n, k, m->inv, rk, rk + n, nx, nx + n, m->gj_flag);
                }
                e = cudaGetLastError();
            }
            int flag = 1;
            if (e == cudaSuccess) e = cudaMemcpyAsync(&flag, m->gj_flag, sizeof(int), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) {
                igab_set_error("multigrid coarse inverse: %s", cudaGetErrorString(e));
                rc = IGAB_ERR_CUDA;
            } else if (!flag) {
                m->dev_inv = true;
            }
        }
        cudaFree(dcols);
        if (rc) return rc;
    }
    if (m->nlev > 1 && B.n <= MG_COARSE_DOF && m->dev_inv) {
        m->direct = true;
        m->nd = (int)B.n;
    } else if (m->nlev > 1 && B.n <= MG_COARSE_DOF) {   /* not positive definite: host LU */
        igab_ctx *cc = B.ctx;
        const int n = (int)B.n;
        std::vector<int> cols((size_t)cc->nnz);
        int rc = igab_csr_pattern(cc, nullptr, cols.data());
        if (rc) return rc;
        std::vector<double> v((size_t)cc->nnz);
        IGAB_CUDA_TRY(cudaStreamSynchronize(c->stream));
        IGAB_CUDA_TRY(cudaMemcpy(v.data(), B.vals, (size_t)cc->nnz * sizeof(double), cudaMemcpyDeviceToHost));
        m->lu.assign((size_t)n * n, 0.0);
        for (int r = 0; r < n; r++)
            for (int k = cc->rowptr_h[r]; k < cc->rowptr_h[r + 1]; k++) m->lu[(size_t)cols[k] * n + r] = v[k];
        if (!lu_factor(n, m->lu, m->piv)) {
            igab_set_error("multigrid: the coarsest tangent is singular");
            return IGAB_ERR_NONFINITE;
        }
        m->direct = true;
        m->nd = n;
        cudaFreeHost(m->h_vec);
        m->h_vec = nullptr;
        IGAB_CUDA_TRY(cudaMallocHost((void **)&m->h_vec, (size_t)n * sizeof(double)));
    }
    m->version = c->param_version;
    return 0;
}

} /* namespace */

void igab_mg_release(igab_ctx *c)
{
    mg_free(c->mg);
    c->mg = nullptr;
}

int igab_mg_levels(igab_ctx *c, int *levels)
{
    *levels = c->mg ? c->mg->nlev : 0;
    return 0;
}


namespace {

#define GM_RESTART 50          /* GMRES restart length */

/* partial sums of V_i . w, i < k (V_i = V + i n), per block into part[i][RD_BLOCKS] */
__global__ void __launch_bounds__(RD_THREADS) k_md_partial(long n, const double *__restrict__ V, int k,
                                                           const double *__restrict__ w, double *part)
{
    __shared__ double red[RD_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = 0; i < k; i++) {
        const double *v = V + (size_t)i * n;
        double s0 = 0.0;
        for (long t = blockIdx.x * (long)RD_THREADS + threadIdx.x; t < n; t += (long)RD_BLOCKS * RD_THREADS)
            s0 += v[t] * w[t];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        if (lane == 0) red[warp] = s0;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int q = 0; q < RD_THREADS / 32; q++) s += red[q];
            part[(size_t)i * RD_BLOCKS + blockIdx.x] = s;
        }
        __syncthreads();
    }
}

/* out[i] = sum of part[i][0..RD_BLOCKS) in a fixed order, one block per i */
__global__ void __launch_bounds__(RD_THREADS) k_md_finish(const double *part, double *out)
{
    __shared__ double red[RD_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double s = 0.0;
    for (int b = threadIdx.x; b < RD_BLOCKS; b += RD_THREADS) s += part[(size_t)blockIdx.x * RD_BLOCKS + b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < RD_THREADS / 32; q++) t += red[q];
        out[blockIdx.x] = t;
    }
}

/* w -= sum_{i<k} h_i V_i  (h on the device) */
__global__ void k_md_update(long n, const double *__restrict__ V, int k, const double *__restrict__ h, double *w)
{
    MG_LOOP(t, n)
    {
        double s = w[t];
        for (int i = 0; i < k; i++) s -= h[i] * V[(size_t)i * n + t];
        w[t] = s;
    }
}

/* u = sum_{i<k} y_i V_i  (y on the device) */
__global__ void k_md_combine(long n, const double *__restrict__ V, int k, const double *__restrict__ y, double *u)
{
    MG_LOOP(t, n)
    {
        double s = 0.0;
        for (int i = 0; i < k; i++) s += y[i] * V[(size_t)i * n + t];
        u[t] = s;
    }
}

/* h = V[0..k)^T w on the host (and on the device at dev_h) */
cudaError_t mdot(igab_mg *m, cudaStream_t st, long n, const double *V, int k, const double *w, double *h)
{
    double *dev_out = m->mpart + (size_t)(GM_RESTART + 1) * RD_BLOCKS;
    k_md_partial<<<RD_BLOCKS, RD_THREADS, 0, st>>>(n, V, k, w, m->mpart);
    k_md_finish<<<k, RD_THREADS, 0, st>>>(m->mpart, dev_out);
    m->launches += 2;
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(m->h_md, dev_out, (size_t)k * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) memcpy(h, m->h_md, (size_t)k * sizeof(double));
    return e;
}

/* the V-cycle as the preconditioner: z = M r */
int precond(igab_mg *m, const double *r, double *z)
{
    mg_level &F = m->L[0];
    cudaStream_t st = F.ctx->stream;
    k_mg_copy<<<MG_BLOCKS, MG_THREADS, 0, st>>>(F.n, r, F.b);
    int rc = vcycle(m, 0);
    if (rc) return rc;
    k_mg_copy<<<MG_BLOCKS, MG_THREADS, 0, st>>>(F.n, F.x, z);
    m->launches += 2;
    return 0;
}

int dot1(igab_mg *m, cudaStream_t st, long n, const double *a, const double *b, double *out)
{
    double d2[2];
    IGAB_CUDA_TRY(rd_dot2(st, n, a, b, nullptr, nullptr, m->part, m->dots, m->h_dots, d2));
    *out = d2[0];
    return 0;
}

/* preconditioned CG on K (vals, prec); breakdown when p.Kp <= 0 */
int solve_cg(igab_mg *m, igab_ctx *c, const void *vals, int prec, const double *b, double *x, double tol, int maxit,
             int *iterations, int *converged, double *rnorm, int *breakdown)
{
    cudaStream_t st = c->stream;
    const long n = c->ndof;
    double *r = m->kv, *z = r + n, *p = z + n, *q = p + n;
    int rc = 0;
    k_mg_copy<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, b, r);
    if ((rc = precond(m, r, z))) return rc;
    k_mg_copy<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, z, p);
    double rz = 0.0;
    if ((rc = dot1(m, st, n, r, z, &rz))) return rc;
    for (int it = 1; it <= maxit; it++) {
        if ((rc = igab_launch_spmv(c, vals, prec, p, q))) return rc;
        double pq = 0.0, rr = 0.0;
        if ((rc = dot1(m, st, n, p, q, &pq))) return rc;
        if (!(pq > 0.0) || !(rz > 0.0)) {
            *breakdown = 1;
            return 0;
        }
        const double alpha = rz / pq;
        k_mg_axpby<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, alpha, p, 1.0, x);
        k_mg_axpby<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, -alpha, q, 1.0, r);
        if ((rc = dot1(m, st, n, r, r, &rr))) return rc;
        *iterations = it;
        *rnorm = std::sqrt(rr);
        if (*rnorm <= tol) {
            *converged = 1;
            return 0;
        }
        if ((rc = precond(m, r, z))) return rc;
        double rz1 = 0.0;
        if ((rc = dot1(m, st, n, r, z, &rz1))) return rc;
        k_mg_axpby<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, 1.0, z, rz1 / rz, p);
        rz = rz1;
        m->launches += 4;
    }
    return 0;
}

/* right-preconditioned GMRES(GM_RESTART) on K with the V-cycle M: x = M u, u in the
 * Krylov space of K M; classical Gram-Schmidt with one reorthogonalisation (CGS2), Givens
 * rotations; the true residual is recomputed at every restart */
int solve_gmres(igab_mg *m, igab_ctx *c, const void *vals, int prec, const double *b, double *x, double tol,
                int maxit, int *iterations, int *converged, double *rnorm)
{
    cudaStream_t st = c->stream;
    const long n = c->ndof;
    const int mr = GM_RESTART;
    double *V = m->kv, *t = V + (size_t)(mr + 1) * n, *w = t + n, *r = w + n;
    double *dev_coef = m->mpart + (size_t)(GM_RESTART + 1) * RD_BLOCKS + (GM_RESTART + 1);
    std::vector<double> H((size_t)(mr + 1) * mr), cs(mr), sn(mr), g(mr + 1), h(mr + 1), h2(mr + 1), y(mr);
    int rc = 0, its = 0;
    k_mg_copy<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, b, r);
    double beta = 0.0;
    if ((rc = dot1(m, st, n, r, r, &beta))) return rc;
    beta = std::sqrt(beta);
    *rnorm = beta;
    while (its < maxit) {
        if (beta <= tol) {
            *converged = 1;
            break;
        }
        k_mg_axpby<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, 1.0 / beta, r, 0.0, V);
        std::fill(g.begin(), g.end(), 0.0);
        g[0] = beta;
        int j = 0;
        for (; j < mr && its < maxit; j++) {
            if ((rc = precond(m, V + (size_t)j * n, t))) return rc;
            if ((rc = igab_launch_spmv(c, vals, prec, t, w))) return rc;
            /* CGS2: h = V^T w, w -= V h, twice */
            IGAB_CUDA_TRY(mdot(m, st, n, V, j + 1, w, h.data()));
            IGAB_CUDA_TRY(cudaMemcpyAsync(dev_coef, h.data(), (size_t)(j + 1) * sizeof(double), cudaMemcpyHostToDevice, st));
            k_md_update<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, V, j + 1, dev_coef, w);
            IGAB_CUDA_TRY(mdot(m, st, n, V, j + 1, w, h2.data()));
            IGAB_CUDA_TRY(cudaMemcpyAsync(dev_coef, h2.data(), (size_t)(j + 1) * sizeof(double), cudaMemcpyHostToDevice, st));
            k_md_update<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, V, j + 1, dev_coef, w);
            for (int i = 0; i <= j; i++) h[i] += h2[i];
            double hn = 0.0;
            if ((rc = dot1(m, st, n, w, w, &hn))) return rc;
            hn = std::sqrt(hn);
            m->launches += 3;
            its++;
            /* apply the previous rotations, then a new one that zeroes hn */
            for (int i = 0; i < j; i++) {
                const double a = h[i], bb = h[i + 1];
                h[i] = cs[i] * a + sn[i] * bb;
                h[i + 1] = -sn[i] * a + cs[i] * bb;
            }
            const double den = std::sqrt(h[j] * h[j] + hn * hn);
            if (den == 0.0) {
                cs[j] = 1.0;
                sn[j] = 0.0;
            } else {
                cs[j] = h[j] / den;
                sn[j] = hn / den;
            }
            h[j] = den;
            for (int i = 0; i <= j; i++) H[(size_t)i * mr + j] = h[i];
            g[j + 1] = -sn[j] * g[j];
            g[j] = cs[j] * g[j];
            *rnorm = std::fabs(g[j + 1]);
            if (*rnorm <= tol || hn == 0.0) {
                j++;
                break;
            }
            k_mg_axpby<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, 1.0 / hn, w, 0.0, V + (size_t)(j + 1) * n);
        }
        /* y = H^-1 g, x += M (V y) */
        for (int i = j - 1; i >= 0; i--) {
            double sacc = g[i];
            for (int k = i + 1; k < j; k++) sacc -= H[(size_t)i * mr + k] * y[k];
            y[i] = H[(size_t)i * mr + i] != 0.0 ? sacc / H[(size_t)i * mr + i] : 0.0;
        }
        IGAB_CUDA_TRY(cudaMemcpyAsync(dev_coef, y.data(), (size_t)j * sizeof(double), cudaMemcpyHostToDevice, st));
        k_md_combine<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, V, j, dev_coef, w);
        if ((rc = precond(m, w, t))) return rc;
        k_mg_axpby<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, 1.0, t, 1.0, x);
        /* true residual */
        if ((rc = igab_launch_spmv(c, vals, prec, x, w))) return rc;
        k_mg_sub<<<MG_BLOCKS, MG_THREADS, 0, st>>>(n, b, w, r);
        m->launches += 4;
        if ((rc = dot1(m, st, n, r, r, &beta))) return rc;
        beta = std::sqrt(beta);
        *rnorm = beta;
    }
    if (beta <= tol) *converged = 1;
    *iterations = its;
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

} /* namespace */

int igab_mg_solve(igab_ctx *c, int method, const void *vals, int prec, const double *b, double *x, double rtol,
                  double atol, int maxit, int *iterations, int *converged, double *rnorm, double *bnorm, int *breakdown)
{
    if (!c->mg) {
        c->mg = new igab_mg();
        IGAB_CUDA_TRY(cudaMalloc((void **)&c->mg->part, (2 * RD_BLOCKS + 2) * sizeof(double)));
        c->mg->dots = c->mg->part + 2 * RD_BLOCKS;
        IGAB_CUDA_TRY(cudaMallocHost((void **)&c->mg->h_dots, 2 * sizeof(double)));
        IGAB_CUDA_TRY(cudaMalloc((void **)&c->mg->mpart,
                                 ((size_t)(GM_RESTART + 1) * RD_BLOCKS + 2 * (GM_RESTART + 1)) * sizeof(double)));
        IGAB_CUDA_TRY(cudaMallocHost((void **)&c->mg->h_md, (GM_RESTART + 1) * sizeof(double)));
    }
    igab_mg *m = c->mg;
    m->launches = 0;
    int rc = 0;
    if (m->version != c->param_version || m->nlev == 0)
        if ((rc = mg_build(c, m))) return rc;
    const long n = c->ndof;
    const long need = (long)(GM_RESTART + 4) * n;
    if (m->kv_n != need) {
        cudaFree(m->kv);
        m->kv = nullptr;
        m->kv_n = 0;
        IGAB_CUDA_TRY(cudaMalloc((void **)&m->kv, (size_t)need * sizeof(double)));
        m->kv_n = need;
    }
    cudaStream_t st = c->stream;
    IGAB_CUDA_TRY(cudaMemsetAsync(x, 0, (size_t)n * sizeof(double), st));
    double bb = 0.0;
    if ((rc = dot1(m, st, n, b, b, &bb))) return rc;
    const double bn = std::sqrt(bb);
    const double tol = std::max(rtol * bn, atol);
    *bnorm = bn;
    *rnorm = bn;
    *iterations = 0;
    *converged = bn <= tol ? 1 : 0;
    *breakdown = 0;
    if (!*converged) {
        if (method == IGAB_KSP_MG_CG)
            rc = solve_cg(m, c, vals, prec, b, x, tol, maxit, iterations, converged, rnorm, breakdown);
        else
            rc = solve_gmres(m, c, vals, prec, b, x, tol, maxit, iterations, converged, rnorm);
        if (rc) return rc;
    }
    IGAB_CUDA_TRY(cudaGetLastError());
    IGAB_CUDA_TRY(cudaStreamSynchronize(st));
    c->last_launches = m->launches;
    return 0;
}

extern "C" int igab_mg_prolongation_1d(const double *coarse_knots, int n_coarse_elements, const double *inserted,
                                       int n_inserted, double *P)
{
    if (!coarse_knots || !P || n_coarse_elements < 1 || n_inserted < 0 || (n_inserted > 0 && !inserted)) {
        igab_set_error("igab_mg_prolongation_1d: bad argument");
        return IGAB_ERR_ARG;
    }
    std::vector<double> kc(coarse_knots, coarse_knots + n_coarse_elements + 5);
    std::vector<double> ins(inserted, inserted + n_inserted);
    for (int i = 0; i < n_inserted; i++)
        if (!(ins[i] > kc[2] && ins[i] < kc[kc.size() - 3]) || (i > 0 && ins[i] < ins[i - 1])) {
            igab_set_error("igab_mg_prolongation_1d: inserted knots must be ascending and interior");
            return IGAB_ERR_ARG;
        }
    std::vector<double> M;
    int nbf = 0, nbc = 0;
    igab_mg_knot_prolongation(kc, ins, M, nbf, nbc);
    memcpy(P, M.data(), M.size() * sizeof(double));
    return 0;
}
