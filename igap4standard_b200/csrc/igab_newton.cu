/*
 * Newton solve on the device: the reference application's solver loop
 * (src/snes_solve.c:10-36) with the SNES configuration of src/snes_init.c:8-47,
 * driving the GPU assembly without moving a residual or a tangent to the host.
 *
 * The loop repeats one-step Newton solves (SNESSetTolerances(abstol 1e-10,
 * rtol 1e-20, stol 1e-20, max_it 1), src/snes_init.c:18) until the reason is
 * not "max iterations"; it also stops when ||F|| stagnates, |F_old - F_new| /
 * F_old < 1e-6 with F_old = 999 before the first pass (src/snes_solve.c:28-32).
 * One step (SNESNEWTONLS, src/snes_init.c:19):
 *   F = R(X); stop if ||F|| < abstol; J = K(X) (Dirichlet rows and columns
 *   zeroed, unit diagonal, as the tangent callback leaves it); J Y = F by the
 *   device Krylov solve (igab_krylov_solve, stands in for PETSc's KSP);
 *   backtracking line search of cubic order along X - lambda Y
 *   (SNESLINESEARCHBT, src/snes_init.c:21-22).
 * The line search is the algorithm of Dennis and Schnabel, "Numerical Methods
 * for Unconstrained Optimization and Nonlinear Equations" (1983), A6.3.1: a
 * full step, then a quadratic backtrack, then cubic ones, each new lambda held
 * in [0.1, 0.5] of the previous one, sufficient decrease with alpha = 1e-4,
 * minimum lambda 1e-12, steps longer than 1e8 scaled down, the initial slope
 * -(F, J Y) forced negative.
 *
 * Vectors live on the device; every norm and dot product is a fixed-order
 * two-pass reduction (per-block partial sums over a fixed grid, then one block),
 * so a solve is bitwise repeatable.  The host holds only the scalars of the
 * line search and the convergence tests.
 *
 * With opts.use_graph each assembly (the residual at the iterate, the residual at
 * the line-search point, the tangent at the iterate) is replayed from a CUDA graph
 * kept on the context: captured on first use (that call runs eagerly once, then is
 * captured), replayed while its pointers, kind and the context's schedule version
 * are unchanged, so a sequence of solves (time steps) captures each once.
 */
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cuda_runtime.h>
#include "igab_internal.h"
#include "igab_reduce.cuh"

namespace {

#define NL_THREADS 256
#define NL_BLOCKS RD_BLOCKS

constexpr double NL_F_OLD0 = 999.0;   /* src/snes_solve.c:22 */

/* W = X - lam Y */
__global__ void k_nl_step(long n, const double *__restrict__ X, const double *__restrict__ Y, double lam,
                          double *__restrict__ W)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        W[i] = X[i] - lam * Y[i];
}

/* Y *= s */
__global__ void k_nl_scale(long n, double *__restrict__ Y, double s)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) Y[i] *= s;
}

/* one captured assembly of the Newton loop */
struct nl_graph {
    cudaGraphExec_t exec = nullptr;
    const void *in = nullptr, *out = nullptr;
    int kind = 0;           /* -1 residual, else the tangent precision */
    long version = -1;      /* igab_ctx::sched_version at capture */
    int launches = 0;       /* kernels in the graph */
};

} /* namespace */

struct igab_nl_graphs {
    nl_graph slot[3];       /* residual at the iterate, residual at the trial point, tangent at the iterate */
};

namespace {

struct nl_work {
    igab_ctx *c;
    bool use_graph;
    long n;
    double *F, *G, *Y, *JY, *W;   /* residual at X, at the trial point, step, J Y, trial point */
    double *part, *dots;          /* reduction scratch (device) */
    double *h_dots;               /* pinned host copy of dots[2] */
    void *vals;
    int prec;
    int launches;

    /* (a0, b0) [and (a1, b1)] on the device, both results on the host */
    int dot(const double *a0, const double *b0, const double *a1, const double *b1, double out[2])
    {
        launches += 2;
        IGAB_CUDA_TRY(rd_dot2(c->stream, n, a0, b0, a1, b1, part, dots, h_dots, out));
        return 0;
    }
    int norm(const double *a, double *out)
    {
        double d[2];
        int rc = dot(a, a, nullptr, nullptr, d);
        *out = std::sqrt(d[0]);
        return rc;
    }
    void step(const double *X, double lam, double *Wout)
    {
        k_nl_step<<<NL_BLOCKS, NL_THREADS, 0, c->stream>>>(n, X, Y, lam, Wout);
        launches++;
    }
};

using clk = std::chrono::steady_clock;
double ms_since(clk::time_point t0)
{
    return std::chrono::duration<double, std::milli>(clk::now() - t0).count();
}

struct nl_counters {
    int nres = 0, ntan = 0, ntan64 = 0;
    long kits = 0;
    double ms_res = 0.0, ms_tan = 0.0, ms_ksp = 0.0;
};

int launch_assembly(igab_ctx *c, int kind, const double *in, void *out)
{
    return kind < 0 ? igab_launch_residual(c, in, (double *)out) : igab_launch_tangent(c, in, out, kind);
}

/* one assembly (kind -1: the residual, else the tangent in that precision) of `in` into
 * `out`: replayed from the graph of `slot` when that was captured for the same pointers,
 * kind and schedule version, else run eagerly (this call's result; it also sets the
 * kernel attributes outside the capture) and captured for the next calls */
int nl_assemble(nl_work &w, int slot, int kind, const double *in, void *out)
{
    igab_ctx *c = w.c;
    if (!w.use_graph) {
        const int rc = launch_assembly(c, kind, in, out);
        w.launches += c->last_launches;
        return rc;
    }
    if (!c->nlg) c->nlg = new igab_nl_graphs();
    nl_graph &G = c->nlg->slot[slot];
    if (G.exec && G.in == in && G.out == out && G.kind == kind && G.version == c->sched_version) {
        IGAB_CUDA_TRY(cudaGraphLaunch(G.exec, c->stream));
        w.launches += G.launches;
        return 0;
    }
    if (G.exec) cudaGraphExecDestroy(G.exec);
    G = nl_graph();
    /* a graph always runs the Neumann kernel: zero values that the last upload skipped */
    if (!c->neumann_nonzero && c->d_hval)
        IGAB_CUDA_TRY(cudaMemsetAsync(c->d_hval, 0, (size_t)c->n_neu_points * sizeof(double), c->stream));
    const bool prof = c->profiling;
    c->profiling = false;
    c->force_neumann = true;
    int rc = launch_assembly(c, kind, in, out);
    w.launches += c->last_launches;
    if (!rc) {
        cudaGraph_t gr = nullptr;
        cudaError_t e = cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            rc = launch_assembly(c, kind, in, out);
            const int n = c->last_launches;
            e = cudaStreamEndCapture(c->stream, &gr);
            if (!rc && e == cudaSuccess) e = cudaGraphInstantiate(&G.exec, gr, 0);
            if (gr) cudaGraphDestroy(gr);
            if (!rc && e == cudaSuccess) {
                G.in = in;
                G.out = out;
                G.kind = kind;
                G.version = c->sched_version;
                G.launches = n;
            }
        }
        if (!rc && e != cudaSuccess) {
            igab_set_error("igab_newton_solve: assembly graph: %s", cudaGetErrorString(e));
            rc = IGAB_ERR_CUDA;
        }
    }
    c->profiling = prof;
    c->force_neumann = false;
    return rc;
}

/* F = R(X) and ||F|| (slot 0: F at the iterate, 1: G at the trial point) */
int eval_residual(nl_work &w, int slot, const double *X, double *F, double *fnorm, nl_counters &k)
{
    const auto t0 = clk::now();
    int rc = nl_assemble(w, slot, -1, X, F);
    if (!rc) rc = w.norm(F, fnorm);
    k.nres++;
    k.ms_res += ms_since(t0);
    return rc;
}

/* backtracking line search along X - lambda Y (the caller has J Y in w.JY).
 * On return w.W holds the accepted point and w.G its residual. */
int line_search(nl_work &w, const double *X, double fnorm, double &gnorm, double &lam, bool &ok, nl_counters &k)
{
    const double alpha = 1e-4, minlambda = 1e-12, maxstep = 1e8;
    const int max_its = 40;
    double d[2];
    int rc = w.norm(w.Y, &d[0]);
    if (rc) return rc;
    const double ynorm = d[0];
    if (ynorm > maxstep) {
        k_nl_scale<<<NL_BLOCKS, NL_THREADS, 0, w.c->stream>>>(w.n, w.Y, maxstep / ynorm);
        k_nl_scale<<<NL_BLOCKS, NL_THREADS, 0, w.c->stream>>>(w.n, w.JY, maxstep / ynorm);
        w.launches += 2;
    }
    if ((rc = w.dot(w.F, w.JY, nullptr, nullptr, d))) return rc;
    double initslope = d[0];
    if (initslope > 0.0) initslope = -initslope;
    if (initslope == 0.0) initslope = -1.0;
    const double f2 = fnorm * fnorm;
    auto accept = [&](double gn, double l) { return std::isfinite(gn) && 0.5 * gn * gn <= 0.5 * f2 + l * alpha * initslope; };
    lam = 1.0;
    w.step(X, lam, w.W);
    if ((rc = eval_residual(w, 1, w.W, w.G, &gnorm, k))) return rc;
    if (!std::isfinite(gnorm)) {
        ok = false;
        return 0;
    }
    if (accept(gnorm, lam)) {
        ok = true;
        return 0;
    }
    /* quadratic first backtrack */
    double lamtemp = -initslope / (gnorm * gnorm - f2 - 2.0 * lam * initslope);
    lamtemp = std::min(lamtemp, 0.5 * lam);
    lam = lamtemp <= 0.1 * lam ? 0.1 * lam : lamtemp;
    w.step(X, lam, w.W);
    double gprev = gnorm, lamprev = 1.0;
    if ((rc = eval_residual(w, 1, w.W, w.G, &gnorm, k))) return rc;
    if (accept(gnorm, lam)) {
        ok = true;
        return 0;
    }
    /* cubic backtracks */
    for (int it = 0; it < max_its; it++) {
        if (lam <= minlambda) break;
        const double t1 = 0.5 * (gnorm * gnorm - f2) - lam * initslope;
        const double t2 = 0.5 * (gprev * gprev - f2) - lamprev * initslope;
        const double a = (t1 / (lam * lam) - t2 / (lamprev * lamprev)) / (lam - lamprev);
        const double b = (-lamprev * t1 / (lam * lam) + lam * t2 / (lamprev * lamprev)) / (lam - lamprev);
        const double disc = std::max(b * b - 3.0 * a * initslope, 0.0);
        lamtemp = a == 0.0 ? -initslope / (2.0 * b) : (-b + std::sqrt(disc)) / (3.0 * a);
        lamprev = lam;
        gprev = gnorm;
        lamtemp = std::min(lamtemp, 0.5 * lam);
        lam = lamtemp <= 0.1 * lam ? 0.1 * lam : lamtemp;
        w.step(X, lam, w.W);
        if ((rc = eval_residual(w, 1, w.W, w.G, &gnorm, k))) return rc;
        if (accept(gnorm, lam)) {
            ok = true;
            return 0;
        }
    }
    ok = false;
    return 0;
}

} /* namespace */

void igab_newton_release(igab_ctx *c)
{
    if (c->nlg) {
        for (nl_graph &G : c->nlg->slot)
            if (G.exec) cudaGraphExecDestroy(G.exec);
        delete c->nlg;
        c->nlg = nullptr;
    }
    cudaFree(c->d_nl);
    cudaFree(c->d_nl_vals);
    cudaFreeHost(c->h_nl);
    c->d_nl = nullptr;
    c->d_nl_vals = nullptr;
    c->h_nl = nullptr;
    c->nl_vals_bytes = 0;
}

extern "C" void igab_newton_defaults(igab_newton_opts *o)
{
    if (!o) return;
    o->prec = IGAB_PREC_FP64;
    o->abstol = 1e-10;
    o->rtol = 1e-20;
    o->stol = 1e-20;
    o->stagnation = 1e-6;
    o->max_subiter = 10000;
    o->ksp_rtol = 1e-5;
    o->ksp_maxit = 100000;
    o->ksp = IGAB_KSP_MG_GMRES;
    o->verbose = 0;
    o->fp64_polish = 0;
    o->use_graph = 1;
}

extern "C" int igab_newton_solve(igab_ctx *ctx, double *U_dev, const igab_newton_opts *opts, igab_newton_info *info,
                                 double *fnorm_history, int *krylov_history, int history_cap)
{
    IGAB_NO_PERIODIC(ctx, "igab_newton_solve");
    if (!ctx || !U_dev || !opts || !info) {
        igab_set_error("igab_newton_solve: null argument");
        return IGAB_ERR_ARG;
    }
    if ((opts->prec != IGAB_PREC_FP64 && opts->prec != IGAB_PREC_FP32) || opts->max_subiter < 1 ||
        (opts->ksp != IGAB_KSP_BICGSTAB && opts->ksp != IGAB_KSP_MG_CG && opts->ksp != IGAB_KSP_MG_GMRES) ||
        opts->ksp_maxit < 1 || !(opts->ksp_rtol >= 0.0) || !(opts->abstol >= 0.0)) {
        igab_set_error("igab_newton_solve: bad options");
        return IGAB_ERR_ARG;
    }
    if (history_cap < 0 || (history_cap > 0 && !fnorm_history && !krylov_history)) {
        igab_set_error("igab_newton_solve: bad history buffers");
        return IGAB_ERR_ARG;
    }
    if (!ctx->stream) {
        igab_set_error("igab_newton_solve: needs a non-default stream (igab_set_stream)");
        return IGAB_ERR_ARG;
    }
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    const auto t_start = clk::now();
    const long n = ctx->ndof;
    const size_t es = opts->prec == IGAB_PREC_FP64 ? sizeof(double) : sizeof(float);
    if (!ctx->d_nl) IGAB_CUDA_TRY(cudaMalloc((void **)&ctx->d_nl, ((size_t)5 * n + 2 * NL_BLOCKS + 2) * sizeof(double)));
    if (!ctx->h_nl) IGAB_CUDA_TRY(cudaMallocHost((void **)&ctx->h_nl, 2 * sizeof(double)));
    const size_t es_max = opts->fp64_polish ? sizeof(double) : es;   /* the polish steps need FP64 values */
    if (ctx->nl_vals_bytes < (size_t)ctx->nnz * es_max) {
        cudaFree(ctx->d_nl_vals);
        ctx->d_nl_vals = nullptr;
        ctx->nl_vals_bytes = 0;
        IGAB_CUDA_TRY(cudaMalloc(&ctx->d_nl_vals, (size_t)ctx->nnz * es_max));
        ctx->nl_vals_bytes = (size_t)ctx->nnz * es_max;
    }
    nl_work w;
    w.c = ctx;
    w.use_graph = opts->use_graph != 0;
    w.n = n;
    w.F = ctx->d_nl;
    w.G = w.F + n;
    w.Y = w.G + n;
    w.JY = w.Y + n;
    w.W = w.JY + n;
    w.part = w.W + n;
    w.dots = w.part + 2 * NL_BLOCKS;
    w.h_dots = ctx->h_nl;
    w.vals = ctx->d_nl_vals;
    w.prec = opts->prec;
    w.launches = 0;

    nl_counters k;
    double *X = U_dev;
    double f_old = NL_F_OLD0, fnorm = 0.0;
    int reason = IGAB_SNES_DIVERGED_MAX_IT, its = 0, rc = 0;
    for (int sub = 0; sub < opts->max_subiter; sub++) {
        /* one SNESSolve with max_it = 1 */
        int kits = 0;
        if ((rc = eval_residual(w, 0, X, w.F, &fnorm, k))) return rc;
        const double fprev = fnorm;
        if (!std::isfinite(fnorm)) {
            reason = IGAB_SNES_DIVERGED_FNORM_NAN;
        } else if (fnorm < opts->abstol) {
            reason = IGAB_SNES_CONVERGED_FNORM_ABS;
        } else {
            const double ttol = fnorm * opts->rtol;
            auto t0 = clk::now();
            rc = nl_assemble(w, 2, w.prec, X, w.vals);
            if (!rc) {
                cudaError_t e = cudaStreamSynchronize(ctx->stream);
                if (e != cudaSuccess) {
                    igab_set_error("igab_newton_solve: tangent: %s", cudaGetErrorString(e));
                    return IGAB_ERR_CUDA;
                }
                rc = igab_check_status(ctx);
            }
            if (rc) return rc;
            k.ntan++;
            if (w.prec == IGAB_PREC_FP64) k.ntan64++;
            k.ms_tan += ms_since(t0);
            t0 = clk::now();
            int conv = 0, brk = 1;
            double rn = 0.0, bn = 0.0;
            if (opts->ksp != IGAB_KSP_BICGSTAB && ctx->phys == IGAB_PHYS_GE) {
                rc = igab_mg_solve(ctx, opts->ksp, w.vals, w.prec, w.F, w.Y, opts->ksp_rtol, 0.0, opts->ksp_maxit, &kits,
                                   &conv, &rn, &bn, &brk);
                w.launches += ctx->last_launches;
                if (rc) return rc;
            }
            if (brk) {   /* BiCGStab: requested, transient physics, or CG met non-positive curvature */
                int k2 = 0;
                rc = igab_krylov_solve(ctx, w.vals, w.prec, w.F, w.Y, opts->ksp_rtol, 0.0, opts->ksp_maxit, &k2, &conv,
                                       &rn, &bn);
                w.launches += ctx->last_launches;
                if (rc) return rc;
                kits += k2;
            }
            k.kits += kits;
            k.ms_ksp += ms_since(t0);
            /* J Y with the Jacobian of the solve (line-search slope) */
            if ((rc = igab_launch_spmv(ctx, w.vals, w.prec, w.Y, w.JY))) return rc;
            w.launches++;
            double xn = 0.0;
            if ((rc = w.norm(X, &xn))) return rc;
            double gnorm = 0.0, lam = 1.0;
            bool ok = false;
            if ((rc = line_search(w, X, fnorm, gnorm, lam, ok, k))) return rc;
            /* the accepted (or last tried) point becomes the iterate, as in SNESNEWTONLS */
            IGAB_CUDA_TRY(cudaMemcpyAsync(X, w.W, (size_t)n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
            fnorm = gnorm;
            its++;
            double yn = 0.0;
            if ((rc = w.norm(w.Y, &yn))) return rc;
            const double snorm = lam * yn;
            if (!ok)
                reason = IGAB_SNES_DIVERGED_LINE_SEARCH;
            else if (!std::isfinite(fnorm))
                reason = IGAB_SNES_DIVERGED_FNORM_NAN;
            else if (fnorm < opts->abstol)
                reason = IGAB_SNES_CONVERGED_FNORM_ABS;
            else if (fnorm <= ttol)
                reason = IGAB_SNES_CONVERGED_FNORM_RELATIVE;
            else if (snorm < opts->stol * xn)
                reason = IGAB_SNES_CONVERGED_SNORM_RELATIVE;
            else
                reason = IGAB_SNES_DIVERGED_MAX_IT;
            /* FP32 tangent whose error now limits the step: polish in FP64 */
            if (opts->fp64_polish && w.prec == IGAB_PREC_FP32 && reason == IGAB_SNES_DIVERGED_MAX_IT &&
                fnorm > 0.1 * fprev)
                w.prec = IGAB_PREC_FP64;
        }
        /* src/snes_solve.c:28-32: stagnation ends the loop */
        if (std::fabs(f_old - fnorm) / f_old < opts->stagnation) reason = IGAB_SNES_DIVERGED_LINE_SEARCH;
        f_old = fnorm;
        if (sub < history_cap) {
            if (fnorm_history) fnorm_history[sub] = fnorm;
            if (krylov_history) krylov_history[sub] = kits;
        }
        if (opts->verbose) {
            printf("%6d: Fnorm = %e, #lin.ite.= %6d, (%08.2f[min])\n", sub + 1, fnorm, kits,
                   ms_since(t_start) / 60000.0);
            fflush(stdout);
        }
        if (reason != IGAB_SNES_DIVERGED_MAX_IT) break;
    }
    IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    info->iterations = its;
    info->reason = reason;
    info->converged = reason > 0;
    info->krylov_iterations = k.kits;
    info->n_residual = k.nres;
    info->n_tangent = k.ntan;
    info->n_tangent_fp64 = k.ntan64;
    info->fnorm = fnorm;
    info->ms_residual = k.ms_res;
    info->ms_tangent = k.ms_tan;
    info->ms_krylov = k.ms_ksp;
    info->ms_total = ms_since(t_start);
    info->launches = w.launches;
    return 0;
}
