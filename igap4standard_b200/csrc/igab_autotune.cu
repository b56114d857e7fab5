/*
 * Autotuner of the assembly schedule (no reference counterpart: the reference
 * has one fixed CPU loop).  Every candidate is timed on the caller's own mesh
 * (or batch) and state with CUDA events on the library stream; the fastest is
 * kept and left applied.
 *
 * Single mesh (igab_autotune):
 *   residual       elements per block: tile edge 2 or 4 of the 8-colour schedule
 *   FP64 tangent   FP64 tensor path (mma f64) or FP64 FMA pipe
 *   FP32 tangent   tcgen05 tensor cores (TF32 hi/lo) or FP32 FMA pipe
 *   colour order   natural, mirrored or Gray (igab_colour_at), on the sum of the
 *                  kernels chosen above
 * Batch (igab_batch_autotune):
 *   CTAs per SM of the persistent residual and FP64 tangent kernels (1 or as many
 *   as fit; the FP32 kernel runs one CTA per work item), the instance
 *   order of the colour-major work list (natural or largest first) and the
 *   colour order.
 * Tile size, CTA count and instance order leave every per-entry summation order
 * as it is; the kernel variant and the colour order change results by rounding.
 */
#include <algorithm>
#include <vector>
#include <cuda_runtime.h>
#include "igab_internal.h"

namespace {

struct event_pair {
    cudaEvent_t a = nullptr, b = nullptr;
    ~event_pair()
    {
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
    }
};

template <typename F>
int time_ms(cudaStream_t s, int reps, F &&run, double *ms)
{
    event_pair ev;
    IGAB_CUDA_TRY(cudaEventCreate(&ev.a));
    IGAB_CUDA_TRY(cudaEventCreate(&ev.b));
    int rc = run();   /* warm-up (also sets kernel attributes outside the timed region) */
    if (rc) return rc;
    IGAB_CUDA_TRY(cudaEventRecord(ev.a, s));
    for (int r = 0; r < reps; r++)
        if ((rc = run())) return rc;
    IGAB_CUDA_TRY(cudaEventRecord(ev.b, s));
    IGAB_CUDA_TRY(cudaEventSynchronize(ev.b));
    float t = 0.f;
    IGAB_CUDA_TRY(cudaEventElapsedTime(&t, ev.a, ev.b));
    *ms = (double)t / reps;
    return 0;
}

struct dev_buf {
    void *p = nullptr;
    ~dev_buf() { cudaFree(p); }
};

} /* namespace */

extern "C" int igab_autotune(igab_ctx *ctx, const double *U_dev, int what, int reps, igab_tune_result *out)
{
    if (!ctx || !out || reps < 1 || (what & ~15)) {
        igab_set_error("igab_autotune: bad argument");
        return IGAB_ERR_ARG;
    }
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    dev_buf U0, R, V;
    if (!U_dev) {
        IGAB_CUDA_TRY(cudaMalloc(&U0.p, (size_t)ctx->ndof * sizeof(double)));
        IGAB_CUDA_TRY(cudaMemsetAsync(U0.p, 0, (size_t)ctx->ndof * sizeof(double), ctx->stream));
        U_dev = (const double *)U0.p;
    }
    IGAB_CUDA_TRY(cudaMalloc(&R.p, (size_t)ctx->ndof * sizeof(double)));
    if (what & 14) IGAB_CUDA_TRY(cudaMalloc(&V.p, (size_t)ctx->nnz * sizeof(double)));
    const bool prof = ctx->profiling;
    ctx->profiling = false;
    int rc = 0;
    out->residual_tile = ctx->tile_res;
    out->tangent_fp64_kernel = ctx->tan_kernel;
    out->tangent_fp32_kernel = ctx->tan32_kernel;
    out->colour_order = ctx->colour_order;
    out->residual_ms = out->tangent_fp64_ms = out->tangent_fp32_ms = -1.0;
    if (what & 1) {
        double best = 1e300;
        for (int te : {2, 4}) {
            ctx->tile_res = te;
            double t = 0.0;
            if ((rc = time_ms(ctx->stream, reps, [&] { return igab_launch_residual(ctx, U_dev, (double *)R.p); }, &t)))
                break;
            if (t < best) { best = t; out->residual_tile = te; }
        }
        ctx->tile_res = out->residual_tile;
        out->residual_ms = best;
    }
    for (int prec = 0; prec < 2 && !rc; prec++) {
        if (!(what & (2 << prec))) continue;
        int &knob = prec == 0 ? ctx->tan_kernel : ctx->tan32_kernel;
        int &pick = prec == 0 ? out->tangent_fp64_kernel : out->tangent_fp32_kernel;
        double &tms = prec == 0 ? out->tangent_fp64_ms : out->tangent_fp32_ms;
        double best = 1e300;
        for (int k : {1, 0}) {
            if (ctx->phys != IGAB_PHYS_GE && k != knob) continue;   /* getime has one tangent kernel */
            knob = k;
            double t = 0.0;
            if ((rc = time_ms(ctx->stream, reps, [&] { return igab_launch_tangent(ctx, U_dev, V.p, prec); }, &t)))
                break;
            if (t < best) { best = t; pick = k; }
        }
        knob = pick;
        tms = best;
    }
    if ((what & 8) && !rc) {
        /* colour order: the kernels chosen above (all three when none was tuned), summed */
        const int kern = (what & 7) ? (what & 7) : 7;
        double best = 1e300;
        for (int order = 0; order < 3 && !rc; order++) {
            ctx->colour_order = order;
            double total = 0.0;
            for (int k = 0; k < 3 && !rc; k++) {
                if (!(kern & (1 << k))) continue;
                double t = 0.0;
                if (k == 0)
                    rc = time_ms(ctx->stream, reps, [&] { return igab_launch_residual(ctx, U_dev, (double *)R.p); }, &t);
                else
                    rc = time_ms(ctx->stream, reps, [&] { return igab_launch_tangent(ctx, U_dev, V.p, k - 1); }, &t);
                total += t;
            }
            if (!rc && total < best) {
                best = total;
                out->colour_order = order;
            }
        }
        ctx->colour_order = out->colour_order;
    }
    ctx->profiling = prof;
    ctx->sched_version++;
    IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    return rc;
}

/* ---------------------------------------------------------------- batch */

extern "C" int igab_batch_autotune(igab_batch *b, const double *U_dev, int what, int reps, igab_batch_tune_result *out)
{
    if (!b || !out || reps < 1 || (what & ~15)) {
        igab_set_error("igab_batch_autotune: bad argument");
        return IGAB_ERR_ARG;
    }
    long ndof = 0, nnz = 0;
    int rc = igab_batch_sizes(b, &ndof, &nnz, nullptr, nullptr, nullptr);
    if (rc) return rc;
    igab_ctx *c0 = igab_batch_instance(b, 0);
    IGAB_CUDA_TRY(cudaSetDevice(c0->device));
    cudaStream_t s = c0->stream;   /* the batch stream */
    dev_buf U0, R, V;
    if (!U_dev) {
        IGAB_CUDA_TRY(cudaMalloc(&U0.p, (size_t)ndof * sizeof(double)));
        IGAB_CUDA_TRY(cudaMemsetAsync(U0.p, 0, (size_t)ndof * sizeof(double), s));
        U_dev = (const double *)U0.p;
    }
    IGAB_CUDA_TRY(cudaMalloc(&R.p, (size_t)ndof * sizeof(double)));
    if (what & 14) IGAB_CUDA_TRY(cudaMalloc(&V.p, (size_t)nnz * sizeof(double)));
    int occ[3] = {0, 0, 0};
    if ((rc = igab_batch_occupancy_res(&occ[0])) || (rc = igab_batch_occupancy_dmma(&occ[1])) ||
        (rc = igab_batch_occupancy_tc32(&occ[2])))
        return rc;
    int cur[4];
    if ((rc = igab_batch_get_schedule(b, &cur[0], &cur[1], &cur[2], &cur[3]))) return rc;
    /* per order: the best CTA count of each timed kernel; the order with the least total wins */
    double best_total = 1e300;
    int best[4] = {cur[0], cur[1], cur[2], cur[3]};
    double best_ms[3] = {-1.0, -1.0, -1.0};
    for (int order : {0, 1}) {
        int pick[3] = {cur[0], cur[1], cur[2]};
        double ms[3] = {-1.0, -1.0, -1.0}, total = 0.0;
        for (int k = 0; k < 3 && !rc; k++) {
            if (!(what & (1 << k))) continue;
            std::vector<int> cands = {0};
            if (k != 2)   /* the FP32 batch kernel runs one CTA per work item: no CTA count to choose */
                for (int c = 1; c < occ[k]; c++) cands.push_back(c);
            double bk = 1e300;
            for (int cand : cands) {
                int sch[3] = {pick[0], pick[1], pick[2]};
                sch[k] = cand;
                if ((rc = igab_batch_set_schedule(b, sch[0], sch[1], sch[2], order))) break;
                double t = 0.0;
                auto run = [&]() -> int {
                    if (k == 0) return igab_batch_residual_device(b, U_dev, (double *)R.p);
                    return igab_batch_tangent_device(b, U_dev, V.p, k == 1 ? IGAB_PREC_FP64 : IGAB_PREC_FP32);
                };
                if ((rc = time_ms(s, reps, run, &t))) break;
                if (t < bk) { bk = t; pick[k] = cand; }
            }
            ms[k] = bk;
            total += bk;
        }
        if (rc) break;
        if (total < best_total) {
            best_total = total;
            best[0] = pick[0]; best[1] = pick[1]; best[2] = pick[2]; best[3] = order;
            std::copy(ms, ms + 3, best_ms);
        }
    }
    int rc2 = igab_batch_set_schedule(b, best[0], best[1], best[2], best[3]);
    if (rc) return rc;
    if (rc2) return rc2;
    int corder = 0;
    if ((rc = igab_batch_get_colour_order(b, &corder))) return rc;
    if (what & 8) {
        /* colour order on the chosen schedule: the selected kernels (all three when none), summed */
        const int kern = (what & 7) ? (what & 7) : 7;
        double best_total_c = 1e300;
        int pick = corder;
        for (int co = 0; co < 3 && !rc; co++) {
            if ((rc = igab_batch_set_colour_order(b, co))) break;
            double total = 0.0;
            for (int k = 0; k < 3 && !rc; k++) {
                if (!(kern & (1 << k))) continue;
                double t = 0.0;
                auto run = [&]() -> int {
                    if (k == 0) return igab_batch_residual_device(b, U_dev, (double *)R.p);
                    return igab_batch_tangent_device(b, U_dev, V.p, k == 1 ? IGAB_PREC_FP64 : IGAB_PREC_FP32);
                };
                rc = time_ms(s, reps, run, &t);
                total += t;
            }
            if (!rc && total < best_total_c) {
                best_total_c = total;
                pick = co;
            }
        }
        rc2 = igab_batch_set_colour_order(b, pick);
        if (rc) return rc;
        if (rc2) return rc2;
        corder = pick;
    }
    out->colour_order = corder;
    out->ctas_res = best[0];
    out->ctas_tan64 = best[1];
    out->ctas_tan32 = best[2];
    out->order = best[3];
    out->residual_ms = best_ms[0];
    out->tangent_fp64_ms = best_ms[1];
    out->tangent_fp32_ms = best_ms[2];
    return igab_batch_sync(b);
}
