/*
 * igab_device.cuh -- device helpers shared by the assembly kernels: the
 * derivative multi-index tables, the 8-colour tile decode and the closed-form
 * CSR positions of the structured AIJ pattern.
 */
#ifndef IGAB_DEVICE_CUH
#define IGAB_DEVICE_CUH

#include "igab_internal.h"

namespace {

/* derivative multi-index of component alpha (eval_Bspline order):
 * 0:(0,0,0) 1:(1,0,0) 2:(0,1,0) 3:(0,0,1) 4:(2,0,0) 5:(1,1,0) 6:(1,0,1) 7:(0,2,0) 8:(0,1,1) 9:(0,0,2) */
__host__ __device__ constexpr int a_kx(int a) { return a == 1 || a == 5 || a == 6 ? 1 : (a == 4 ? 2 : 0); }
__host__ __device__ constexpr int a_ky(int a) { return a == 2 || a == 5 || a == 8 ? 1 : (a == 7 ? 2 : 0); }
__host__ __device__ constexpr int a_kz(int a) { return a == 3 || a == 6 || a == 8 ? 1 : (a == 9 ? 2 : 0); }
/* (ky,kz) pair index: 0:(0,0) 1:(1,0) 2:(0,1) 3:(2,0) 4:(1,1) 5:(0,2) */
__host__ __device__ constexpr int kk_of(int ky, int kz)
{
    return (ky == 0 && kz == 0) ? 0 : (ky == 1 && kz == 0) ? 1 : (ky == 0 && kz == 1) ? 2
         : (ky == 2 && kz == 0) ? 3 : (ky == 1 && kz == 1) ? 4 : 5;
}
__host__ __device__ constexpr int kk_ky(int kk) { return kk == 1 || kk == 4 ? 1 : (kk == 3 ? 2 : 0); }
__host__ __device__ constexpr int kk_kz(int kk) { return kk == 2 || kk == 4 ? 1 : (kk == 5 ? 2 : 0); }
__host__ __device__ constexpr int a_kk(int a) { return kk_of(a_ky(a), a_kz(a)); }

__device__ __forceinline__ void group_sync(int group)
{
    asm volatile("bar.sync %0, %1;" ::"r"(group + 1), "r"(64) : "memory");
}

__device__ __forceinline__ double shfl_xor(double v, int m) { return __shfl_xor_sync(0xffffffffu, v, m); }

/* tile bookkeeping for one colour */
struct tile_t {
    int t[3];   /* tile coordinates */
    int e0[3];  /* first element */
    int nv[3];  /* valid elements per direction */
};

/* Colour = 4 px + 2 py + pz, p the parities of the tile coordinates; tile ids of a
 * colour run with x slowest.  With the x parity most significant, the tiles of
 * one colour inside an x-range of tiles are a contiguous range of ids, and
 * launching the colours slab by slab along x, each slab starting on an odd tile,
 * adds into every CSR entry in the same order as launching each colour over the
 * whole mesh: an entry is touched by at most two x-tiles t, t+1, and across a slab
 * boundary t is even (colours 0-3, first in either order). */
__device__ __forceinline__ bool decode_tile(const igab_geom &g, int TE, int colour, int bid, tile_t &T)
{
    int c[3] = {(colour >> 2) & 1, (colour >> 1) & 1, colour & 1};
    int nc[3];
    for (int d = 0; d < 3; d++) {
        int nt = (g.ne[d] + TE - 1) / TE;
        nc[d] = nt > c[d] ? (nt - c[d] + 1) / 2 : 0;
    }
    int i2 = bid % nc[2];
    int i1 = (bid / nc[2]) % nc[1];
    int i0 = bid / (nc[2] * nc[1]);
    if (i0 >= nc[0]) return false;
    T.t[0] = 2 * i0 + c[0]; T.t[1] = 2 * i1 + c[1]; T.t[2] = 2 * i2 + c[2];
    for (int d = 0; d < 3; d++) {
        T.e0[d] = T.t[d] * TE;
        int r = g.ne[d] - T.e0[d];
        T.nv[d] = r < TE ? r : TE;
    }
    return true;
}

__device__ __forceinline__ long cp_index(const igab_geom &g, int x, int y, int z)
{
    return ((long)x * g.nb[1] + y) * g.nb[2] + z;
}

/* position of column (cx,cy,cz,k2) inside the CSR row of control point (x,y,z) */
__device__ __forceinline__ int csr_pos(const igab_geom &g, int x, int y, int z, int cx, int cy, int cz, int k2)
{
    int x0 = x > 2 ? x - 2 : 0;
    int y0 = y > 2 ? y - 2 : 0, y1 = y + 2 < g.nb[1] - 1 ? y + 2 : g.nb[1] - 1;
    int z0 = z > 2 ? z - 2 : 0, z1 = z + 2 < g.nb[2] - 1 ? z + 2 : g.nb[2] - 1;
    int nyb = y1 - y0 + 1, nzb = z1 - z0 + 1;
    return (((cx - x0) * nyb + (cy - y0)) * nzb + (cz - z0)) * 3 + k2;
}

/* CSR bases of row c1 (= 3 a1 + k1) of the element matrix of the element whose first
 * control point is (ex, ey, ez): entry (c1, c2), c2 = 3 (9 ax + 3 ay + az) + k2, lies at
 *   rb + ax * rsx + ay * rsy + 3 az + k2
 * (csr_pos with the row's window fixed; one rowptr load per row instead of per entry). */
__device__ __forceinline__ void elem_row_base(const igab_geom &g, int ex, int ey, int ez, int c1, long &rb, int &rsx,
                                              int &rsy)
{
    const int a1 = c1 / 3, k1 = c1 % 3;
    const int x1 = ex + a1 / 9, y1 = ey + (a1 / 3) % 3, z1 = ez + a1 % 3;
    const int x0 = x1 > 2 ? x1 - 2 : 0;
    const int y0 = y1 > 2 ? y1 - 2 : 0, ye = y1 + 2 < g.nb[1] - 1 ? y1 + 2 : g.nb[1] - 1;
    const int z0 = z1 > 2 ? z1 - 2 : 0, ze = z1 + 2 < g.nb[2] - 1 ? z1 + 2 : g.nb[2] - 1;
    const int nyb = ye - y0 + 1, nzb = ze - z0 + 1;
    rb = (long)g.rowptr[3 * cp_index(g, x1, y1, z1) + k1] + (((ex - x0) * nyb + (ey - y0)) * nzb + (ez - z0)) * 3;
    rsx = nyb * nzb * 3;
    rsy = nzb * 3;
}

/* per-element integrand scale (1 when no scaling is set) */
__device__ __forceinline__ double elem_scale(const igab_geom &g, int ex, int ey, int ez)
{
    return g.escale ? g.escale[((long)ex * g.ne[1] + ey) * g.ne[2] + ez] : 1.0;
}

/* ---- persistent batched launches: one work item (a tile of one instance) at a time */
#define IGAB_BATCH_SPIN (1L << 22)   /* polls (with a 128 ns sleep) before a dependency wait gives up */

/* one thread: wait until every sweep position before `colour` (a position in the
 * batch's colour order) of instance `inst` is complete.  Each wait polls at most B.spin_limit times (128 ns sleep between
 * polls), then sets bit 2 of the status word and moves on; B.hold raises the
 * count that colour 0 of instance 0 must reach, so that the waits on it cannot
 * finish (a host-set test switch that exercises the give-up path). */
__device__ __forceinline__ void batch_wait_colours(const igab_batch_dev &B, int inst, int colour)
{
    int *done = B.done + 8 * inst;
    const int *need = B.need + 8 * inst;
    for (int c = 0; c < colour; c++) {
        const int target = need[c] + (inst == 0 && c == 0 ? B.hold : 0);
        long spins = 0;
        while (atomicOr(&done[c], 0) < target) {
            if (++spins > B.spin_limit) {
                atomicOr(B.status, 2);
                break;
            }
            __nanosleep(128);
        }
    }
}

struct batch_slot {
    igab_geom g;      /* geometry of the current item's instance */
    int item, inst, colour, tile;
    int pos;          /* position of the colour in the batch's colour order */
};

/* all threads: fetch the next item, wait until every earlier colour of its
 * instance is complete, stage the instance geometry in shared memory.
 * Returns false when the list is exhausted (block-uniform). */
__device__ __forceinline__ bool batch_next(const igab_batch_dev &B, batch_slot &sl)
{
    if (threadIdx.x == 0) {
        const int it = atomicAdd(B.counter, 1);
        sl.item = it;
        if (it < B.nitems) {
            const int4 w = B.items[it];
            sl.inst = w.x;
            sl.pos = w.y;
            sl.tile = w.z;
            sl.colour = w.w;
            batch_wait_colours(B, w.x, w.y);
            __threadfence();
        }
    }
    __syncthreads();
    if (sl.item >= B.nitems) return false;
    const int *src = reinterpret_cast<const int *>(B.geoms + sl.inst);
    int *dst = reinterpret_cast<int *>(&sl.g);
    for (int i = threadIdx.x; i < (int)(sizeof(igab_geom) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    return true;
}

/* all threads, after the item's last global write: publish the finished tile */
__device__ __forceinline__ void batch_done(const igab_batch_dev &B, const batch_slot &sl)
{
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(&B.done[8 * sl.inst + sl.pos], 1);
}

long tiles_of_colour(const igab_geom &g, int TE, int colour)
{
    long n = 1;
    for (int d = 0; d < 3; d++) {
        int c = (colour >> (2 - d)) & 1;
        int nt = (g.ne[d] + TE - 1) / TE;
        n *= nt > c ? (nt - c + 1) / 2 : 0;
    }
    return n;
}

/* the tiles of a colour whose x tile coordinate lies in [tx0, tx1): ids
 * *first .. *first + return value - 1 (decode_tile numbering) */
long tiles_of_colour_in(const igab_geom &g, int TE, int colour, int tx0, int tx1, long *first)
{
    const int cx = (colour >> 2) & 1;
    long plane = 1;
    for (int d = 1; d < 3; d++) {
        int c = (colour >> (2 - d)) & 1;
        int nt = (g.ne[d] + TE - 1) / TE;
        plane *= nt > c ? (nt - c + 1) / 2 : 0;
    }
    const int ntx = (g.ne[0] + TE - 1) / TE;
    const int ncx = ntx > cx ? (ntx - cx + 1) / 2 : 0;
    int i0 = (tx0 - cx + 1) / 2, i1 = (tx1 - cx + 1) / 2;   /* tx = 2 i + cx in [tx0, tx1) */
    if (i0 < 0) i0 = 0;
    if (i1 > ncx) i1 = ncx;
    *first = (long)i0 * plane;
    return i1 > i0 ? (long)(i1 - i0) * plane : 0;
}

} /* namespace */

#endif
