/*
 * igab_reduce.cuh -- fixed-order dot products over device vectors: per-block partial
 * sums over a fixed grid, then one block sums the partials in a fixed order, so a
 * result is bitwise repeatable (used by the Newton driver and the multigrid solver).
 */
#ifndef IGAB_REDUCE_CUH
#define IGAB_REDUCE_CUH

#include <cuda_runtime.h>

namespace {

constexpr int RD_THREADS = 256;
constexpr int RD_BLOCKS = 296;   /* 2 x 148 SMs */

/* partial sums of (a0, b0) [and (a1, b1) when a1 != nullptr] per block into part[2][RD_BLOCKS] */
__global__ void __launch_bounds__(RD_THREADS) k_rd_dot(long n, const double *__restrict__ a0,
                                                       const double *__restrict__ b0, const double *__restrict__ a1,
                                                       const double *__restrict__ b1, double *part)
{
    double s0 = 0.0, s1 = 0.0;
    for (long i = blockIdx.x * (long)RD_THREADS + threadIdx.x; i < n; i += (long)RD_BLOCKS * RD_THREADS) {
        s0 += a0[i] * b0[i];
        if (a1) s1 += a1[i] * b1[i];
    }
    __shared__ double red[2][RD_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        s0 += __shfl_xor_sync(0xffffffffu, s0, o);
        s1 += __shfl_xor_sync(0xffffffffu, s1, o);
    }
    if (lane == 0) {
        red[0][warp] = s0;
        red[1][warp] = s1;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double s = 0.0;
        for (int w = 0; w < RD_THREADS / 32; w++) s += red[threadIdx.x][w];
        part[threadIdx.x * RD_BLOCKS + blockIdx.x] = s;
    }
}

/* one block: out[k] = sum of part[k][0..RD_BLOCKS) in a fixed order, k = 0, 1 */
__global__ void __launch_bounds__(RD_THREADS) k_rd_finish(const double *part, double *out)
{
    __shared__ double red[2][RD_THREADS / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < 2; k++) {
        double s = 0.0;
        for (int b = threadIdx.x; b < RD_BLOCKS; b += RD_THREADS) s += part[k * RD_BLOCKS + b];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) red[k][warp] = s;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        double s = 0.0;
        for (int w = 0; w < RD_THREADS / 32; w++) s += red[threadIdx.x][w];
        out[threadIdx.x] = s;
    }
}

/* both dot products on the host: part needs 2 * RD_BLOCKS doubles, dots 2 (device),
 * h_dots 2 (pinned host); synchronises the stream */
inline cudaError_t rd_dot2(cudaStream_t st, long n, const double *a0, const double *b0, const double *a1,
                           const double *b1, double *part, double *dots, double *h_dots, double out[2])
{
    k_rd_dot<<<RD_BLOCKS, RD_THREADS, 0, st>>>(n, a0, b0, a1, b1, part);
    k_rd_finish<<<1, RD_THREADS, 0, st>>>(part, dots);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(h_dots, dots, 2 * sizeof(double), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) {
        out[0] = h_dots[0];
        out[1] = h_dots[1];
    }
    return e;
}

} /* namespace */

#endif
