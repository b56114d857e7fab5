/*
 * igab_residual_noalloc: the host-pointer residual without any device allocation.
 *
 * igab_residual stages U and R in device buffers that the context allocates
 * with cudaMalloc on first use.  Some callers cannot let a library allocate
 * device memory at that point: a process whose device memory is already
 * reserved in full by another allocator (a framework's caching allocator or
 * a pool sized to the whole GPU), or a solver callback that runs under a fixed
 * device-memory budget.  This entry point stages U and R in a file-scope
 * __device__ array instead, so a call performs no cudaMalloc, cudaFree or
 * other allocating call.
 *
 * Limits and sharing:
 *  - at most IGAB_NOALLOC_MAX_DOF dofs (2 x 8 MiB of FP64 staging); larger
 *    meshes are rejected with IGAB_ERR_ARG.  Every GPU that loads the library
 *    holds the 16 MiB array until the process exits.
 *  - all calls share the one array; calls that overlap on the GPU (several
 *    host threads, or several contexts on one device at once) race.
 *  - in host code the array's name only stands for it: its device address
 *    belongs to the CUDA context that loaded this module, so every call looks
 *    it up with cudaGetSymbolAddress on the context's device (a lookup, not an
 *    allocation) instead of keeping it from an earlier call, which would go
 *    stale after cudaDeviceReset or under another context.
 */
#include <cuda_runtime.h>
#include <math.h>
#include "igab_internal.h"

#define IGAB_NOALLOC_MAX_DOF (1L << 20)
/* staging: [0, MAX) holds U, [MAX, 2 MAX) holds R */
static __device__ __align__(256) double g_noalloc_stage[2 * IGAB_NOALLOC_MAX_DOF];

/* device address of the staging array in the current context (the caller has
 * made the context's device current) */
static int stage_address(double **out)
{
    double *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_stage);
    if (e != cudaSuccess || !p) {
        igab_set_error("igab_residual_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        return IGAB_ERR_CUDA;
    }
    *out = p;
    return 0;
}

extern "C" int igab_residual_noalloc(igab_ctx *ctx, const double *U_host, double *R_host)
{
    IGAB_NO_PERIODIC(ctx, "igab_residual_noalloc");
    if (!ctx || !U_host || !R_host) {
        igab_set_error("igab_residual_noalloc: null argument");
        return IGAB_ERR_ARG;
    }
    if (ctx->ndof > IGAB_NOALLOC_MAX_DOF) {
        igab_set_error("igab_residual_noalloc: %ld dofs exceed the %ld-dof staging array; use igab_residual",
                       ctx->ndof, (long)IGAB_NOALLOC_MAX_DOF);
        return IGAB_ERR_ARG;
    }
    if (ctx->phys != IGAB_PHYS_GE) {
        igab_set_error("igab_residual_noalloc: only phys/ge is built in this version");
        return IGAB_ERR_ARG;
    }
    IGAB_CUDA_TRY(cudaSetDevice(ctx->device));
    double *stage = nullptr;
    int rc = stage_address(&stage);
    if (rc) return rc;
    double *dU = stage;
    double *dR = stage + IGAB_NOALLOC_MAX_DOF;
    size_t bytes = (size_t)ctx->ndof * sizeof(double);
    IGAB_CUDA_TRY(cudaMemcpyAsync(dU, U_host, bytes, cudaMemcpyHostToDevice, ctx->stream));
    /* the residual launcher zeroes dR before accumulating, so stale contents never leak */
    rc = igab_launch_residual(ctx, dU, dR);
    if (rc) return rc;
    IGAB_CUDA_TRY(cudaMemcpyAsync(R_host, dR, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    IGAB_CUDA_TRY(cudaStreamSynchronize(ctx->stream));
    for (long i = 0; i < ctx->ndof; i++)
        if (!isfinite(R_host[i])) {
            igab_set_error("igab_residual_noalloc: non-finite entry at %ld", i);
            return IGAB_ERR_NONFINITE;
        }
    return 0;
}
