/*
 * Time stepping of the transient physics (phys/getime) on the device, and its discrete
 * adjoint with state checkpoints.
 *
 * The reference application advances one step as example/ex1/main.c:48-56 does: the
 * initial guess is U_hist[1] (initguess), snes_solve runs the Newton loop, then the history
 * shifts (U_hist[2] <- U_hist[1] <- U).  igab_transient_run repeats that step on the
 * device: the context's history levels are the U_hist levels, each solve is
 * igab_newton_solve, the Neumann values follow the traction amplitude * sin(2 pi t) of the
 * time-stepping workload.  No state leaves the GPU unless the caller asks for it.
 *
 * The adjoint (no reference counterpart) runs the same steps forward with checkpoints and
 * sweeps them backward (see include/igab.h); every vector operation is a kernel on the
 * context stream and every reduction of the linear solves is fixed-order, so a gradient is
 * bitwise repeatable.
 */
#include <algorithm>
#include <chrono>
#include <cmath>
#include <vector>
#include <cuda_runtime.h>
#include "igab_internal.h"

namespace {

using clk = std::chrono::steady_clock;
double ms_since(clk::time_point t0)
{
    return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
}

constexpr double TWO_PI = 6.283185307179586;

/* v[rows[i]] = 0 */
__global__ void k_zero_at(long n, const int *__restrict__ rows, double *__restrict__ v)
{
    const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) v[rows[i]] = 0.0;
}

/* y += s x */
__global__ void k_axpy(long n, double s, const double *__restrict__ x, double *__restrict__ y)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        y[i] += s * x[i];
}

/* y = s x */
__global__ void k_scale_to(long n, double s, const double *__restrict__ x, double *__restrict__ y)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        y[i] = s * x[i];
}

unsigned vec_blocks(long n)
{
    const long b = (n + 255) / 256;
    return (unsigned)(b < 1184 ? (b < 1 ? 1 : b) : 1184);   /* 8 x 148 SMs */
}

int check_opts(const igab_ctx *ctx, const igab_transient_opts *o, const char *who)
{
    if (!ctx || !o) {
        igab_set_error("%s: null argument", who);
        return IGAB_ERR_ARG;
    }
    if (ctx->phys != IGAB_PHYS_GETIME || ctx->torder < 2) {
        igab_set_error("%s: needs the transient physics (phys/getime)", who);
        return IGAB_ERR_ARG;
    }
    if (o->nsteps < 0 || !(o->dt >= 0.0) || !std::isfinite(o->amplitude)) {
        igab_set_error("%s: bad options (nsteps %d, dt %g)", who, o->nsteps, o->dt);
        return IGAB_ERR_ARG;
    }
    if (!ctx->stream) {
        igab_set_error("%s: needs a non-default stream (igab_set_stream)", who);
        return IGAB_ERR_ARG;
    }
    return 0;
}

/* the traction of the workload at the Neumann points: amplitude sin(2 pi t) on the points
 * of the chosen (face, order, dof) combination */
struct traction {
    std::vector<char> on;
    std::vector<double> val;
    double amplitude = 0.0, dt = 0.0;

    int init(igab_ctx *ctx, const igab_transient_opts *o)
    {
        long n = 0;
        int rc = igab_neumann_points(ctx, &n, nullptr, nullptr);
        if (rc) return rc;
        std::vector<int> meta((size_t)(3 * n + 1));
        if (n > 0 && (rc = igab_neumann_points(ctx, &n, nullptr, meta.data()))) return rc;
        on.assign((size_t)n, 0);
        for (long i = 0; i < n; i++)
            on[i] = meta[3 * i] == o->face && meta[3 * i + 1] == o->order && meta[3 * i + 2] == o->dof;
        val.assign((size_t)n, 0.0);
        amplitude = o->amplitude;
        dt = o->dt > 0.0 ? o->dt : ctx->par_mat[7];
        return 0;
    }
    /* the values of step n (t = (n + 1) dt) into the context */
    int apply(igab_ctx *ctx, int n)
    {
        if (val.empty()) return 0;
        const double a = amplitude * std::sin(TWO_PI * (n + 1) * dt);
        for (size_t i = 0; i < val.size(); i++) val[i] = on[i] ? a : 0.0;
        return igab_set_neumann_values(ctx, val.data());
    }
};

/* history levels 1 and 2 of the context <- (h1, h2); h2 NULL = zero */
int set_levels(igab_ctx *c, const double *h1, const double *h2)
{
    const size_t bytes = (size_t)c->ndof * sizeof(double);
    IGAB_CUDA_TRY(cudaMemcpyAsync(c->d_hist, h1, bytes, cudaMemcpyDeviceToDevice, c->stream));
    if (h2)
        IGAB_CUDA_TRY(cudaMemcpyAsync(c->d_hist + c->ndof, h2, bytes, cudaMemcpyDeviceToDevice, c->stream));
    else
        IGAB_CUDA_TRY(cudaMemsetAsync(c->d_hist + c->ndof, 0, bytes, c->stream));
    return 0;
}

} /* namespace */

extern "C" void igab_transient_defaults(igab_transient_opts *o)
{
    if (!o) return;
    o->nsteps = 1;
    o->dt = 0.0;
    o->amplitude = 0.01;
    o->face = 1;
    o->order = 0;
    o->dof = 0;
    igab_newton_defaults(&o->newton);
    o->newton.prec = IGAB_PREC_FP32;
    o->newton.ksp = IGAB_KSP_BICGSTAB;
}

extern "C" int igab_transient_run(igab_ctx *ctx, const igab_transient_opts *o, double *U_dev, const double *U_prev_dev,
                                  double *U_steps_host, igab_newton_info *step_info, igab_transient_info *info)
{
    IGAB_NO_PERIODIC(ctx, "igab_transient_run");
    int rc = check_opts(ctx, o, "igab_transient_run");
    if (rc) return rc;
    if (!U_dev || !info) {
        igab_set_error("igab_transient_run: null argument");
        return IGAB_ERR_ARG;
    }
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    const auto t0 = clk::now();
    traction tr;
    if ((rc = tr.init(ctx, o))) return rc;
    *info = igab_transient_info();
    const long n = ctx->ndof;
    const size_t bytes = (size_t)n * sizeof(double);
    if ((rc = set_levels(ctx, U_dev, U_prev_dev))) return rc;
    for (int step = 0; step < o->nsteps; step++) {
        if ((rc = tr.apply(ctx, step))) return rc;
        igab_newton_info ni;
        /* initial guess: U = U_hist[1], which U_dev already holds */
        if ((rc = igab_newton_solve(ctx, U_dev, &o->newton, &ni, nullptr, nullptr, 0))) return rc;
        /* history shift: level 2 <- level 1 <- U */
        IGAB_CUDA_TRY(cudaMemcpyAsync(ctx->d_hist + n, ctx->d_hist, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        IGAB_CUDA_TRY(cudaMemcpyAsync(ctx->d_hist, U_dev, bytes, cudaMemcpyDeviceToDevice, ctx->stream));
        if (U_steps_host)
            IGAB_CUDA_TRY(cudaMemcpyAsync(U_steps_host + (size_t)step * n, U_dev, bytes, cudaMemcpyDeviceToHost,
                                          ctx->stream));
        if (step_info) step_info[step] = ni;
        info->steps++;
        info->steps_converged += ni.converged;
        info->newton_iterations += ni.iterations;
        info->krylov_iterations += ni.krylov_iterations;
        info->n_residual += ni.n_residual;
        info->n_tangent += ni.n_tangent;
        info->launches += ni.launches;
    }
    IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    info->ms_total = ms_since(t0);
    return 0;
}

/* ------------------------------------------------------------------ adjoint */

struct igab_tadj {
    igab_ctx *c = nullptr;
    igab_transient_opts o;
    int every = 1;
    traction tr;
    long n = 0;
    /* checkpoints: states (U_{s-1}, U_s) at s = 0, every, 2 every, ... */
    std::vector<double *> ckpt;
    /* a segment's states U_{s-1} .. U_{s+every}, the Newton iterate, adjoint vectors */
    std::vector<double *> seg;
    double *X = nullptr, *lam = nullptr, *cvec = nullptr, *gstep = nullptr;
    double *b[3] = {nullptr, nullptr, nullptr};   /* pending right-hand sides, b_k in b[k % 3] */
    double *V = nullptr, *Vj = nullptr;           /* FP64 tangent and history Jacobian values */
    bool forward_done = false;
    igab_tadj_info_t info{};

    ~igab_tadj()
    {
        for (double *p : ckpt) cudaFree(p);
        for (double *p : seg) cudaFree(p);
        cudaFree(X);
        cudaFree(lam);
        cudaFree(cvec);
        cudaFree(gstep);
        for (double *p : b) cudaFree(p);
        cudaFree(V);
        cudaFree(Vj);
    }

    /* steps k0 .. k1-1 from seg states (U_{k0-1}, U_{k0}) at seg[k0 - s0 + 1 - 1] .. ; fills
     * the states U_{k0+1} .. U_{k1}; seg[j] holds U_{s0 - 1 + j} */
    int steps(int s0, int k0, int k1, int *converged)
    {
        const size_t bytes = (size_t)n * sizeof(double);
        int rc = 0;
        for (int k = k0; k < k1; k++) {
            double *Um = seg[k - s0], *Uk = seg[k - s0 + 1], *Up = seg[k - s0 + 2];
            if ((rc = tr.apply(c, k))) return rc;
            if ((rc = set_levels(c, Uk, Um))) return rc;
            IGAB_CUDA_TRY(cudaMemcpyAsync(X, Uk, bytes, cudaMemcpyDeviceToDevice, c->stream));
            igab_newton_info ni;
            if ((rc = igab_newton_solve(c, X, &o.newton, &ni, nullptr, nullptr, 0))) return rc;
            IGAB_CUDA_TRY(cudaMemcpyAsync(Up, X, bytes, cudaMemcpyDeviceToDevice, c->stream));
            if (converged) *converged += ni.converged;
        }
        return 0;
    }
};

extern "C" int igab_tadj_create(igab_ctx *ctx, const igab_transient_opts *o, int every, igab_tadj **out)
{
    IGAB_NO_PERIODIC(ctx, "igab_tadj_create");
    int rc = check_opts(ctx, o, "igab_tadj_create");
    if (rc) return rc;
    if (!out || every < 1 || o->nsteps < 1) {
        igab_set_error("igab_tadj_create: bad argument (every %d, nsteps %d)", every, o->nsteps);
        return IGAB_ERR_ARG;
    }
    *out = nullptr;
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    igab_tadj *t = new igab_tadj();
    t->c = ctx;
    t->o = *o;
    t->every = every;
    t->n = ctx->ndof;
    if ((rc = t->tr.init(ctx, o))) {
        delete t;
        return rc;
    }
    const size_t bytes = (size_t)t->n * sizeof(double);
    const int nck = (o->nsteps + every - 1) / every;
    cudaError_t e = cudaSuccess;
    t->ckpt.assign((size_t)2 * nck, nullptr);
    t->seg.assign((size_t)every + 2, nullptr);
    for (double *&p : t->ckpt)
        if (e == cudaSuccess) e = cudaMalloc((void **)&p, bytes);
    for (double *&p : t->seg)
        if (e == cudaSuccess) e = cudaMalloc((void **)&p, bytes);
    for (double **p : {&t->X, &t->lam, &t->cvec, &t->b[0], &t->b[1], &t->b[2]})
        if (e == cudaSuccess) e = cudaMalloc((void **)p, bytes);
    if (e == cudaSuccess) e = cudaMalloc((void **)&t->gstep, (size_t)ctx->nel * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void **)&t->V, (size_t)ctx->nnz * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc((void **)&t->Vj, (size_t)ctx->nnz * sizeof(double));
    if (e != cudaSuccess) {
        igab_set_error("igab_tadj_create: %s", cudaGetErrorString(e));
        delete t;
        return IGAB_ERR_NOMEM;
    }
    long nd = 0;   /* builds the Dirichlet rows if they are not yet */
    if ((rc = igab_dirichlet_rows(ctx, &nd, nullptr))) {
        delete t;
        return rc;
    }
    *out = t;
    return 0;
}

extern "C" int igab_tadj_forward(igab_tadj *t, const double *U_init_dev, const double *U_prev_dev, double *U_final_dev)
{
    if (!t || !U_init_dev) {
        igab_set_error("igab_tadj_forward: null argument");
        return IGAB_ERR_ARG;
    }
    igab_ctx *c = t->c;
    IGAB_CUDA_TRY(cudaSetDevice(c->device));
    const auto t0 = clk::now();
    const size_t bytes = (size_t)t->n * sizeof(double);
    const int N = t->o.nsteps;
    t->forward_done = false;
    t->info = igab_tadj_info_t();
    /* seg[0] = U_{-1}, seg[1] = U_0 */
    if (U_prev_dev)
        IGAB_CUDA_TRY(cudaMemcpyAsync(t->seg[0], U_prev_dev, bytes, cudaMemcpyDeviceToDevice, c->stream));
    else
        IGAB_CUDA_TRY(cudaMemsetAsync(t->seg[0], 0, bytes, c->stream));
    IGAB_CUDA_TRY(cudaMemcpyAsync(t->seg[1], U_init_dev, bytes, cudaMemcpyDeviceToDevice, c->stream));
    int rc = 0, conv = 0;
    for (int s = 0, ck = 0; s < N; s += t->every, ck++) {
        const int e = std::min(s + t->every, N);
        IGAB_CUDA_TRY(cudaMemcpyAsync(t->ckpt[2 * ck], t->seg[0], bytes, cudaMemcpyDeviceToDevice, c->stream));
        IGAB_CUDA_TRY(cudaMemcpyAsync(t->ckpt[2 * ck + 1], t->seg[1], bytes, cudaMemcpyDeviceToDevice, c->stream));
        if ((rc = t->steps(s, s, e, &conv))) return rc;
        /* the segment's last two states start the next one */
        IGAB_CUDA_TRY(cudaMemcpyAsync(t->seg[0], t->seg[e - s], bytes, cudaMemcpyDeviceToDevice, c->stream));
        IGAB_CUDA_TRY(cudaMemcpyAsync(t->seg[1], t->seg[e - s + 1], bytes, cudaMemcpyDeviceToDevice, c->stream));
        t->info.checkpoints++;
    }
    if (U_final_dev) IGAB_CUDA_TRY(cudaMemcpyAsync(U_final_dev, t->seg[1], bytes, cudaMemcpyDeviceToDevice, c->stream));
    IGAB_CUDA_TRY(cudaStreamSynchronize(c->stream));
    t->info.forward_steps = N;
    t->info.forward_converged = conv;
    t->info.ms_forward = ms_since(t0);
    t->forward_done = true;
    return 0;
}

extern "C" int igab_tadj_backward(igab_tadj *t, const double *dJdU_dev, double *grad_dev)
{
    if (!t || !dJdU_dev || !grad_dev) {
        igab_set_error("igab_tadj_backward: null argument");
        return IGAB_ERR_ARG;
    }
    if (!t->forward_done) {
        igab_set_error("igab_tadj_backward: no forward pass");
        return IGAB_ERR_ARG;
    }
    igab_ctx *c = t->c;
    IGAB_CUDA_TRY(cudaSetDevice(c->device));
    const auto t0 = clk::now();
    const long n = t->n;
    const size_t bytes = (size_t)n * sizeof(double);
    const int N = t->o.nsteps, every = t->every;
    const unsigned nbv = vec_blocks(n), nbg = vec_blocks(c->nel);
    std::vector<char> live((size_t)N, 0);
    IGAB_CUDA_TRY(cudaMemcpyAsync(t->b[(N - 1) % 3], dJdU_dev, bytes, cudaMemcpyDeviceToDevice, c->stream));
    live[N - 1] = 1;
    IGAB_CUDA_TRY(cudaMemsetAsync(grad_dev, 0, (size_t)c->nel * sizeof(double), c->stream));
    int rc = 0;
    const int nck = (N + every - 1) / every;
    for (int ck = nck - 1; ck >= 0; ck--) {
        const int s = ck * every, e = std::min(s + every, N);
        IGAB_CUDA_TRY(cudaMemcpyAsync(t->seg[0], t->ckpt[2 * ck], bytes, cudaMemcpyDeviceToDevice, c->stream));
        IGAB_CUDA_TRY(cudaMemcpyAsync(t->seg[1], t->ckpt[2 * ck + 1], bytes, cudaMemcpyDeviceToDevice, c->stream));
        if ((rc = t->steps(s, s, e, nullptr))) return rc;
        t->info.recomputed_steps += e - s;
        for (int k = e - 1; k >= s; k--) {
            if (!live[k]) continue;   /* no objective dependence reaches this step */
            live[k] = 0;
            double *bk = t->b[k % 3];
            const double *Um = t->seg[k - s], *Uk = t->seg[k - s + 1], *Up = t->seg[k - s + 2];
            if (c->nd > 0) {
                k_zero_at<<<(unsigned)((c->nd + 255) / 256), 256, 0, c->stream>>>(c->nd, c->d_drow, bk);
                IGAB_CUDA_TRY(cudaGetLastError());
            }
            if ((rc = set_levels(c, Uk, Um))) return rc;
            /* K_k at U_{k+1}; K lam = b_k (K symmetric: Dirichlet rows and columns eliminated) */
            if ((rc = igab_launch_tangent(c, Up, t->V, IGAB_PREC_FP64))) return rc;
            int its = 0, conv = 0;
            double rn = 0.0, bn = 0.0;
            if ((rc = igab_krylov_solve(c, t->V, IGAB_PREC_FP64, bk, t->lam, t->o.newton.ksp_rtol, 0.0,
                                        t->o.newton.ksp_maxit, &its, &conv, &rn, &bn)))
                return rc;
            t->info.krylov_iterations_backward += its;
            t->info.adjoint_solves++;
            t->info.adjoint_solves_converged += conv;
            if (c->nd > 0) {
                k_zero_at<<<(unsigned)((c->nd + 255) / 256), 256, 0, c->stream>>>(c->nd, c->d_drow, t->lam);
                IGAB_CUDA_TRY(cudaGetLastError());
            }
            /* grad += lam . dR_k/dg */
            if ((rc = igab_adjoint_backward(c, Up, nullptr, IGAB_PREC_FP64, t->lam, nullptr, t->gstep))) return rc;
            k_axpy<<<nbg, 256, 0, c->stream>>>(c->nel, 1.0, t->gstep, grad_dev);
            /* b_{k-1} -= J1_k^T lam, b_{k-2} -= J0_k^T lam */
            for (int level = 1; level <= 2; level++) {
                const int tgt = k - level;
                if (tgt < 0) continue;
                if ((rc = igab_history_jacobian_device(c, Up, t->Vj, IGAB_PREC_FP64, level))) return rc;
                if ((rc = igab_adjoint_backward(c, nullptr, t->Vj, IGAB_PREC_FP64, t->lam, t->cvec, nullptr)))
                    return rc;
                double *bt = t->b[tgt % 3];
                if (live[tgt])
                    k_axpy<<<nbv, 256, 0, c->stream>>>(n, -1.0, t->cvec, bt);
                else
                    k_scale_to<<<nbv, 256, 0, c->stream>>>(n, -1.0, t->cvec, bt);
                IGAB_CUDA_TRY(cudaGetLastError());
                live[tgt] = 1;
            }
        }
    }
    /* dJ/dg = -sum lam . dR/dg */
    k_scale_to<<<nbg, 256, 0, c->stream>>>(c->nel, -1.0, grad_dev, grad_dev);
    IGAB_CUDA_TRY(cudaGetLastError());
    IGAB_CUDA_TRY(cudaStreamSynchronize(c->stream));
    t->info.ms_backward = ms_since(t0);
    return 0;
}

extern "C" int igab_tadj_info(const igab_tadj *t, igab_tadj_info_t *info)
{
    if (!t || !info) {
        igab_set_error("igab_tadj_info: null argument");
        return IGAB_ERR_ARG;
    }
    *info = t->info;
    return 0;
}

extern "C" void igab_tadj_destroy(igab_tadj *t)
{
    if (!t) return;
    cudaSetDevice(t->c->device);
    cudaStreamSynchronize(t->c->stream);
    delete t;
}
