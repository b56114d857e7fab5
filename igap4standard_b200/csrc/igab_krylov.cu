/*
 * Device-resident linear solve on the assembled tangent: right-preconditioned
 * BiCGStab with the Jacobi preconditioner M = diag(K), x0 = 0, stopping when
 * ||b - K x|| <= max(rtol ||b||, atol) -- the Krylov step of the Newton solve
 * (PETSc KSP in the reference application, src/snes_init.c), kept on the GPU
 * so no tangent leaves the device.
 *
 * Everything lives in device memory: the vectors, the scalars (rho, alpha,
 * omega, beta, the tolerance) and a stop flag.  One iteration is 11 kernels:
 *   p = r + beta (p - omega v), p^ = D^-1 p | v = K p^ | (r^, v) | alpha |
 *   s = r - alpha v, s^ = D^-1 s, ||s|| | test ||s|| | t = K s^ | (t, t), (t, s) |
 *   omega | x += alpha p^ + omega s^, r = s - omega t, ||r||, (r^, r) | tests, beta
 * Dot products are per-block partial sums over a fixed grid, finished by one
 * block in a fixed order, so a solve is bitwise repeatable.  Every kernel
 * returns at once when the stop flag is set, so a CUDA graph of 8 iterations
 * can be replayed until the host sees the flag (one read of the state per
 * replay) and the result equals a solve tested after every iteration.
 *
 * K x: one warp per control point, i.e. its three rows, which share their
 * columns: nxb * nyb (<= 25) runs of L = 3 nzb values whose columns are
 * consecutive (z fastest, then the component).  Lane j holds the first column of
 * run j; an entry's run is p / L by a multiply-shift reciprocal and its column is
 * fetched from that lane by a shuffle; one gathered x value serves the three
 * rows.  The warp sums its lanes in a fixed shuffle order per row.
 */
#include <cuda_runtime.h>
#include <vector>
#include "igab_device.cuh"

namespace {

#define KV_THREADS 256
#define KV_BLOCKS 296           /* dot-product grid: 2 x 148 SMs */
#define KV_GRAPH_ITERS 8
#define KV_KERNELS_PER_ITER 11

struct bcg_state {
    double rho, rho_new, alpha, omega, beta, tol, snorm, rnorm, bnorm;
    int it, maxit, stop, converged, half;
};

__device__ __forceinline__ bool halted(const bcg_state *S) { return S->stop != 0; }
__device__ __forceinline__ bool halted_or_half(const bcg_state *S) { return S->stop != 0 || S->half != 0; }

/* the window of control points a row couples to (csr_pos) */
__device__ __forceinline__ void row_window(const igab_geom &g, long r, int &x0, int &y0, int &z0, int &nxb, int &nyb,
                                           int &nzb, int &x1, int &y1, int &z1, int &k1)
{
    const long cp = r / 3;
    k1 = (int)(r % 3);
    z1 = (int)(cp % g.nb[2]);
    y1 = (int)((cp / g.nb[2]) % g.nb[1]);
    x1 = (int)(cp / ((long)g.nb[2] * g.nb[1]));
    x0 = x1 > 2 ? x1 - 2 : 0;
    y0 = y1 > 2 ? y1 - 2 : 0;
    z0 = z1 > 2 ? z1 - 2 : 0;
    const int xe = x1 + 2 < g.nb[0] - 1 ? x1 + 2 : g.nb[0] - 1;
    const int ye = y1 + 2 < g.nb[1] - 1 ? y1 + 2 : g.nb[1] - 1;
    const int ze = z1 + 2 < g.nb[2] - 1 ? z1 + 2 : g.nb[2] - 1;
    nxb = xe - x0 + 1;
    nyb = ye - y0 + 1;
    nzb = ze - z0 + 1;
}

template <typename T>
__global__ void __launch_bounds__(KV_THREADS) k_spmv(igab_geom g, const T *__restrict__ vals,
                                                     const double *__restrict__ x, double *__restrict__ y,
                                                     const bcg_state *S, int skip_half)
{
    if (S && (skip_half ? halted_or_half(S) : halted(S))) return;
    const long cp = (long)blockIdx.x * (KV_THREADS / 32) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (3 * cp >= g.ndof) return;   /* warp-uniform */
    int x0, y0, z0, nxb, nyb, nzb, x1, y1, z1, k1;
    row_window(g, 3 * cp, x0, y0, z0, nxb, nyb, nzb, x1, y1, z1, k1);
    const int L = 3 * nzb, total = nxb * nyb * L;   /* L in {9, 12, 15}, total <= 375 */
    /* lane j < nxb * nyb (<= 25) holds the first column of run j */
    const long base_own = lane < nxb * nyb ? 3 * cp_index(g, x0 + lane / nyb, y0 + lane % nyb, z0) : 0;
    /* run = p / L as (p * ceil(2^16 / L)) >> 16, exact for L in {9, 12, 15} and p < 375 */
    const unsigned invL = (65536u + (unsigned)L - 1u) / (unsigned)L;
    /* the three rows of the control point share the columns; row k starts k * total later */
    const T *v0 = vals + g.rowptr[3 * cp], *v1 = v0 + total, *v2 = v1 + total;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    /* four 32-entry chunks per pass: every load of the pass is issued before the first
     * multiply, so a warp keeps 16 loads in flight; the additions keep the chunk order */
    for (int p0 = 0; p0 < total; p0 += 128) {
        double xv[4];
        T w0[4], w1[4], w2[4];
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const int p = p0 + 32 * c + lane;
            const bool in = p < total;
            const int run = (int)(((unsigned)(in ? p : 0) * invL) >> 16);
            const long base = __shfl_sync(0xffffffffu, base_own, run);
            xv[c] = in ? x[base + (p - run * L)] : 0.0;
            w0[c] = in ? v0[p] : T(0);
            w1[c] = in ? v1[p] : T(0);
            w2[c] = in ? v2[p] : T(0);
        }
#pragma unroll
        for (int c = 0; c < 4; c++) {
            if (p0 + 32 * c + lane < total) {
                a0 += double(w0[c]) * xv[c];
                a1 += double(w1[c]) * xv[c];
                a2 += double(w2[c]) * xv[c];
            }
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    }
    if (lane == 0) {
        y[3 * cp] = a0;
        y[3 * cp + 1] = a1;
        y[3 * cp + 2] = a2;
    }
}

/* dinv = 1 / K_ii (1 where K_ii = 0) */
template <typename T>
__global__ void k_jacobi(igab_geom g, const T *__restrict__ vals, double *__restrict__ dinv)
{
    const long r = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (r >= g.ndof) return;
    int x0, y0, z0, nxb, nyb, nzb, x1, y1, z1, k1;
    row_window(g, r, x0, y0, z0, nxb, nyb, nzb, x1, y1, z1, k1);
    const long pos = (((long)(x1 - x0) * nyb + (y1 - y0)) * nzb + (z1 - z0)) * 3 + k1;
    const double d = double(vals[g.rowptr[r] + pos]);
    dinv[r] = d != 0.0 ? 1.0 / d : 1.0;
}

/* fixed-order block sum of NV values per thread into part[NV][blockIdx] */
template <int NV>
__device__ __forceinline__ void block_part(const double (&v)[NV], double *part)
{
    __shared__ double red[NV][KV_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; i++) {
        double s = v[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[i][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        for (int w = 0; w < KV_THREADS / 32; w++) s += red[threadIdx.x][w];
        part[threadIdx.x * KV_BLOCKS + blockIdx.x] = s;
    }
}

/* one block: the sum of part[i][0..KV_BLOCKS) for i < NV, in a fixed order */
template <int NV>
__device__ __forceinline__ void finish_part(const double *part, double (&out)[NV])
{
    __shared__ double red[NV][KV_THREADS / 32];
    __shared__ double res[NV];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int i = 0; i < NV; i++) {
        double s = 0.0;
        for (int b = threadIdx.x; b < KV_BLOCKS; b += KV_THREADS) s += part[i * KV_BLOCKS + b];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[i][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x < NV) {
        double s = 0.0;
        for (int w = 0; w < KV_THREADS / 32; w++) s += red[threadIdx.x][w];
        res[threadIdx.x] = s;
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < NV; i++) out[i] = res[i];
}

#define GRID_LOOP(i, n) for (long i = blockIdx.x * (long)KV_THREADS + threadIdx.x; i < (n); i += (long)KV_BLOCKS * KV_THREADS)

/* r = b, r^ = b, x = p = v = 0, partial ||b||^2 */
__global__ void __launch_bounds__(KV_THREADS) k_bcg_init(long n, const double *__restrict__ b, double *r,
                                                         double *rh, double *x, double *p, double *v, double *part)
{
    double s[1] = {0.0};
    GRID_LOOP(i, n)
    {
        const double bi = b[i];
        r[i] = bi;
        rh[i] = bi;
        x[i] = 0.0;
        p[i] = 0.0;
        v[i] = 0.0;
        s[0] += bi * bi;
    }
    block_part<1>(s, part);
}

__global__ void __launch_bounds__(KV_THREADS) k_bcg_init_end(const double *part, bcg_state *S, double rtol,
                                                             double atol, int maxit)
{
    double bb[1];
    finish_part<1>(part, bb);
    if (threadIdx.x == 0) {
        const double bn = sqrt(bb[0]);
        S->bnorm = bn;
        S->tol = rtol * bn > atol ? rtol * bn : atol;
        S->rho = S->alpha = S->omega = 1.0;
        S->beta = 0.0;
        S->rho_new = bb[0];   /* (r^, r) with r = r^ = b */
        S->snorm = S->rnorm = bn;
        S->it = bn == 0.0 ? 0 : 1;
        S->maxit = maxit;
        S->half = 0;
        S->converged = bn == 0.0 ? 1 : 0;
        S->stop = bn == 0.0 ? 1 : 0;
    }
}

/* p = r + beta (p - omega v) (p = r on the first iteration), p^ = D^-1 p */
__global__ void __launch_bounds__(KV_THREADS) k_bcg_p(long n, const double *__restrict__ r, double *p,
                                                      const double *__restrict__ v, const double *__restrict__ dinv,
                                                      double *ph, const bcg_state *S)
{
    if (halted(S)) return;
    const bool first = S->it == 1;
    const double beta = S->beta, omega = S->omega;
    GRID_LOOP(i, n)
    {
        const double pi = first ? r[i] : r[i] + beta * (p[i] - omega * v[i]);
        p[i] = pi;
        ph[i] = dinv[i] * pi;
    }
}

/* partial (a0, b0) and, for NV = 2, (a1, b1) */
template <int NV>
__global__ void __launch_bounds__(KV_THREADS) k_bcg_dot(long n, const double *__restrict__ a0,
                                                        const double *__restrict__ b0, const double *__restrict__ a1,
                                                        const double *__restrict__ b1, double *part,
                                                        const bcg_state *S, int skip_half)
{
    if (skip_half ? halted_or_half(S) : halted(S)) return;
    double s[NV];
#pragma unroll
    for (int i = 0; i < NV; i++) s[i] = 0.0;
    GRID_LOOP(i, n)
    {
        s[0] += a0[i] * b0[i];
        if (NV > 1) s[NV - 1] += a1[i] * b1[i];
    }
    block_part<NV>(s, part);
}

/* alpha = rho_new / (r^, v) */
__global__ void __launch_bounds__(KV_THREADS) k_bcg_alpha(const double *part, bcg_state *S)
{
    if (halted(S)) return;
    double d[1];
    finish_part<1>(part, d);
    if (threadIdx.x == 0) {
        if (d[0] == 0.0)
            S->stop = 1;   /* breakdown */
        else
            S->alpha = S->rho_new / d[0];
    }
}

/* s = r - alpha v, s^ = D^-1 s, partial ||s||^2 */
__global__ void __launch_bounds__(KV_THREADS) k_bcg_s(long n, const double *__restrict__ r,
                                                      const double *__restrict__ v, const double *__restrict__ dinv,
                                                      double *s, double *sh, double *part, const bcg_state *S)
{
    if (halted(S)) return;
    const double alpha = S->alpha;
    double ss[1] = {0.0};
    GRID_LOOP(i, n)
    {
        const double si = r[i] - alpha * v[i];
        s[i] = si;
        sh[i] = dinv[i] * si;
        ss[0] += si * si;
    }
    block_part<1>(ss, part);
}

/* ||s|| <= tol: converged after the half step */
__global__ void __launch_bounds__(KV_THREADS) k_bcg_scheck(const double *part, bcg_state *S)
{
    if (halted(S)) return;
    double ss[1];
    finish_part<1>(part, ss);
    if (threadIdx.x == 0) {
        S->snorm = sqrt(ss[0]);
        if (S->snorm <= S->tol) S->half = 1;
    }
}

/* omega = (t, s) / (t, t) (0 when t = 0) */
__global__ void __launch_bounds__(KV_THREADS) k_bcg_omega(const double *part, bcg_state *S)
{
    if (halted_or_half(S)) return;
    double d[2];
    finish_part<2>(part, d);
    if (threadIdx.x == 0) S->omega = d[0] > 0.0 ? d[1] / d[0] : 0.0;
}

/* x += alpha p^ (+ omega s^), r = s - omega t, partial ||r||^2 and (r^, r) */
__global__ void __launch_bounds__(KV_THREADS) k_bcg_xr(long n, double *x, const double *__restrict__ ph,
                                                       const double *__restrict__ sh, const double *__restrict__ s,
                                                       const double *__restrict__ t, double *r,
                                                       const double *__restrict__ rh, double *part, const bcg_state *S)
{
    if (halted(S)) return;
    const double alpha = S->alpha;
    if (S->half) {
        GRID_LOOP(i, n) x[i] += alpha * ph[i];
        return;
    }
    const double omega = S->omega;
    double acc[2] = {0.0, 0.0};
    GRID_LOOP(i, n)
    {
        x[i] += alpha * ph[i] + omega * sh[i];
        const double ri = s[i] - omega * t[i];
        r[i] = ri;
        acc[0] += ri * ri;
        acc[1] += rh[i] * ri;
    }
    block_part<2>(acc, part);
}

/* tests after the full step, next rho and beta */
__global__ void __launch_bounds__(KV_THREADS) k_bcg_end(const double *part, bcg_state *S)
{
    if (halted(S)) return;
    if (S->half) {
        if (threadIdx.x == 0) {
            S->converged = 1;
            S->rnorm = S->snorm;
            S->stop = 1;
        }
        return;
    }
    double d[2];
    finish_part<2>(part, d);
    if (threadIdx.x == 0) {
        S->rnorm = sqrt(d[0]);
        if (S->rnorm <= S->tol) {
            S->converged = 1;
            S->stop = 1;
        } else if (S->omega == 0.0) {
            S->stop = 1;   /* stagnation */
        } else if (S->it >= S->maxit) {
            S->stop = 1;   /* iteration limit */
        } else {
            S->it += 1;
            S->rho = S->rho_new;
            S->rho_new = d[1];
            if (S->rho_new == 0.0)
                S->stop = 1;   /* breakdown at the start of the next iteration */
            else
                S->beta = (S->rho_new / S->rho) * (S->alpha / S->omega);
        }
    }
}

struct bcg_work {
    long n = 0;
    double *vec = nullptr;    /* r, r^, p, p^, v, s, s^, t, x, dinv */
    double *part = nullptr;   /* [2][KV_BLOCKS] */
    bcg_state *S = nullptr;
    bcg_state *S_host = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    const void *g_vals = nullptr;
    int g_prec = -1;
};

template <typename T>
void launch_iteration(igab_ctx *c, const igab_geom &g, bcg_work &w, const T *vals)
{
    const long n = w.n;
    double *r = w.vec, *rh = w.vec + n, *p = w.vec + 2 * n, *ph = w.vec + 3 * n, *v = w.vec + 4 * n;
    double *s = w.vec + 5 * n, *sh = w.vec + 6 * n, *t = w.vec + 7 * n, *x = w.vec + 8 * n, *dinv = w.vec + 9 * n;
    const unsigned rows_blocks = (unsigned)((n / 3 + KV_THREADS / 32 - 1) / (KV_THREADS / 32));
    cudaStream_t st = c->stream;
    k_bcg_p<<<KV_BLOCKS, KV_THREADS, 0, st>>>(n, r, p, v, dinv, ph, w.S);
    k_spmv<T><<<rows_blocks, KV_THREADS, 0, st>>>(g, vals, ph, v, w.S, 0);
    k_bcg_dot<1><<<KV_BLOCKS, KV_THREADS, 0, st>>>(n, rh, v, nullptr, nullptr, w.part, w.S, 0);
    k_bcg_alpha<<<1, KV_THREADS, 0, st>>>(w.part, w.S);
    k_bcg_s<<<KV_BLOCKS, KV_THREADS, 0, st>>>(n, r, v, dinv, s, sh, w.part, w.S);
    k_bcg_scheck<<<1, KV_THREADS, 0, st>>>(w.part, w.S);
    k_spmv<T><<<rows_blocks, KV_THREADS, 0, st>>>(g, vals, sh, t, w.S, 1);
    k_bcg_dot<2><<<KV_BLOCKS, KV_THREADS, 0, st>>>(n, t, t, t, s, w.part, w.S, 1);
    k_bcg_omega<<<1, KV_THREADS, 0, st>>>(w.part, w.S);
    k_bcg_xr<<<KV_BLOCKS, KV_THREADS, 0, st>>>(n, x, ph, sh, s, t, r, rh, w.part, w.S);
    k_bcg_end<<<1, KV_THREADS, 0, st>>>(w.part, w.S);
}

std::vector<std::pair<const igab_ctx *, bcg_work>> g_work;

bcg_work &work_of(igab_ctx *c)
{
    for (auto &e : g_work)
        if (e.first == c) return e.second;
    g_work.emplace_back(c, bcg_work());
    return g_work.back().second;
}

} /* namespace */

void igab_krylov_release(igab_ctx *c)
{
    for (size_t i = 0; i < g_work.size(); i++)
        if (g_work[i].first == c) {
            bcg_work &w = g_work[i].second;
            if (w.exec) cudaGraphExecDestroy(w.exec);
            if (w.graph) cudaGraphDestroy(w.graph);
            cudaFree(w.vec);
            cudaFree(w.part);
            cudaFree(w.S);
            cudaFreeHost(w.S_host);
            g_work.erase(g_work.begin() + i);
            return;
        }
}

int igab_launch_spmv(igab_ctx *c, const void *dvals, int prec, const double *dx, double *dy)
{
    igab_geom g = c->geom();
    const unsigned rows_blocks = (unsigned)((c->ndof / 3 + KV_THREADS / 32 - 1) / (KV_THREADS / 32));
    if (prec == IGAB_PREC_FP64)
        k_spmv<double><<<rows_blocks, KV_THREADS, 0, c->stream>>>(g, (const double *)dvals, dx, dy, nullptr, 0);
    else
        k_spmv<float><<<rows_blocks, KV_THREADS, 0, c->stream>>>(g, (const float *)dvals, dx, dy, nullptr, 0);
    c->last_launches++;
    IGAB_CUDA_TRY(cudaGetLastError());
    return 0;
}

int igab_krylov_solve(igab_ctx *c, const void *dvals, int prec, const double *db, double *dx, double rtol,
                      double atol, int maxit, int *iterations, int *converged, double *rnorm, double *bnorm)
{
    igab_geom g = c->geom();
    bcg_work &w = work_of(c);
    const long n = c->ndof;
    if (w.n != n) {
        cudaFree(w.vec);
        w.vec = nullptr;
        IGAB_CUDA_TRY(cudaMalloc((void **)&w.vec, (size_t)10 * n * sizeof(double)));
        if (!w.part) IGAB_CUDA_TRY(cudaMalloc((void **)&w.part, 2 * KV_BLOCKS * sizeof(double)));
        if (!w.S) IGAB_CUDA_TRY(cudaMalloc((void **)&w.S, sizeof(bcg_state)));
        if (!w.S_host) IGAB_CUDA_TRY(cudaMallocHost((void **)&w.S_host, sizeof(bcg_state)));
        w.n = n;
        if (w.exec) { cudaGraphExecDestroy(w.exec); w.exec = nullptr; }
        if (w.graph) { cudaGraphDestroy(w.graph); w.graph = nullptr; }
    }
    double *r = w.vec, *rh = w.vec + n, *p = w.vec + 2 * n, *v = w.vec + 4 * n, *x = w.vec + 8 * n,
           *dinv = w.vec + 9 * n;
    cudaStream_t st = c->stream;
    /* the graph of KV_GRAPH_ITERS iterations, captured once per (values, precision) */
    if (!w.exec || w.g_vals != dvals || w.g_prec != prec) {
        if (w.exec) { cudaGraphExecDestroy(w.exec); w.exec = nullptr; }
        if (w.graph) { cudaGraphDestroy(w.graph); w.graph = nullptr; }
        IGAB_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < KV_GRAPH_ITERS; i++) {
            if (prec == IGAB_PREC_FP64)
                launch_iteration<double>(c, g, w, (const double *)dvals);
            else
                launch_iteration<float>(c, g, w, (const float *)dvals);
        }
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(st, &graph);
        if (e != cudaSuccess) {
            igab_set_error("igab_solve_device: graph capture failed: %s", cudaGetErrorString(e));
            return IGAB_ERR_CUDA;
        }
        w.graph = graph;
        IGAB_CUDA_TRY(cudaGraphInstantiate(&w.exec, w.graph, 0));
        w.g_vals = dvals;
        w.g_prec = prec;
    }
    c->last_launches = 0;
    if (prec == IGAB_PREC_FP64)
        k_jacobi<double><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, (const double *)dvals, dinv);
    else
        k_jacobi<float><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(g, (const float *)dvals, dinv);
    k_bcg_init<<<KV_BLOCKS, KV_THREADS, 0, st>>>(n, db, r, rh, x, p, v, w.part);
    k_bcg_init_end<<<1, KV_THREADS, 0, st>>>(w.part, w.S, rtol, atol, maxit);
    c->last_launches += 3;
    IGAB_CUDA_TRY(cudaGetLastError());
    /* replay until the device raises the stop flag (at most maxit iterations run) */
    const long max_replays = maxit / KV_GRAPH_ITERS + 2;
    for (long k = 0;; k++) {
        IGAB_CUDA_TRY(cudaMemcpyAsync(w.S_host, w.S, sizeof(bcg_state), cudaMemcpyDeviceToHost, st));
        IGAB_CUDA_TRY(cudaStreamSynchronize(st));
        if (w.S_host->stop || k >= max_replays) break;
        IGAB_CUDA_TRY(cudaGraphLaunch(w.exec, st));
        c->last_launches += KV_GRAPH_ITERS * KV_KERNELS_PER_ITER;
    }
    IGAB_CUDA_TRY(cudaMemcpyAsync(dx, x, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, st));
    IGAB_CUDA_TRY(cudaStreamSynchronize(st));
    const bcg_state &S = *w.S_host;
    if (iterations) *iterations = S.it;
    if (converged) *converged = S.converged;
    if (rnorm) *rnorm = S.rnorm;
    if (bnorm) *bnorm = S.bnorm;
    return 0;
}
