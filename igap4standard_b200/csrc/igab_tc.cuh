/*
 * igab_tc.cuh -- inline-PTX wrappers for the sm_100a tensor-core path
 * (tcgen05: tensor-memory allocation, MMA issue, commit to an mbarrier,
 * tensor-memory loads) and the shared-memory operand layout the kernels use.
 *
 * Operand layout (K-major, no swizzle).  A chunk holds KC = 32 K-slots of an
 * operand with R rows; element (row r, slot j) sits at byte
 *     (r / 8) * 1024 + (j / 4) * 128 + (r % 8) * 16 + (j % 4) * 4,
 * i.e. 8-row x 16-byte core matrices, adjacent along K (leading byte offset
 * 128) and 1024 bytes apart along M/N (stride byte offset).  One MMA k-step
 * (8 TF32 values of K) is two core matrices, so k-step kk starts 256 bytes
 * after the chunk start.
 *
 * Every wait on an mbarrier is bounded: tc_mbar_wait gives up after a fixed
 * number of polls and returns false, and the kernels then record an error
 * status, release their tensor memory and return.
 */
#ifndef IGAB_TC_CUH
#define IGAB_TC_CUH

#include <stdint.h>

namespace {

constexpr int TC_KC = 32;          /* K slots per operand chunk */
constexpr int TC_SBO = 1024;       /* bytes between 8-row groups of a chunk */
constexpr int TC_LBO = 128;        /* bytes between K-adjacent core matrices */
constexpr int TC_KSTEP_BYTES = 256;
constexpr long TC_WAIT_POLLS = 1L << 22;

/* Instruction descriptor of tcgen05.mma kind::tf32: D f32 (bits 4-5 = 1),
 * A and B tf32 (bits 7-9, 10-12 = 2), negate A (bit 13, optional), both
 * K-major (bits 15, 16 = 0), N >> 3 in bits 17-22, M >> 4 in bits 24-28, dense. */
__host__ __device__ constexpr uint32_t tc_idesc_tf32(int M, int N, bool negate_a = false)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | (negate_a ? (1u << 13) : 0u) | ((uint32_t)(N >> 3) << 17) |
           ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t tc_smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

/* byte offset of (row r, slot j) inside a chunk */
__device__ __forceinline__ uint32_t tc_off(int r, int j)
{
    return (uint32_t)((r >> 3) * TC_SBO + (j >> 2) * TC_LBO + (r & 7) * 16 + (j & 3) * 4);
}

/* Shared-memory matrix descriptor (tcgen05): start address >> 4 in bits 0-13,
 * leading byte offset >> 4 in bits 16-29, stride byte offset >> 4 in bits
 * 32-45, descriptor version 1 in bits 46-47, base offset 0, no swizzle. */
__device__ __forceinline__ uint64_t tc_sdesc(uint32_t saddr)
{
    return (uint64_t)((saddr & 0x3FFFFu) >> 4) | ((uint64_t)(TC_LBO >> 4) << 16) |
           ((uint64_t)(TC_SBO >> 4) << 32) | (1ull << 46);
}

__device__ __forceinline__ float tc_tf32(float x)
{
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

/* x = hi + lo with hi, lo exactly representable in TF32 (|lo| <= 2^-11 |hi|) */
__device__ __forceinline__ void tc_split(float x, float &hi, float &lo)
{
    hi = tc_tf32(x);
    lo = tc_tf32(x - hi);
}

__device__ __forceinline__ void tc_mbar_init(unsigned long long *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(tc_smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void tc_fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

/* bounded wait for the completion of the phase with the given parity */
__device__ __forceinline__ bool tc_mbar_wait(unsigned long long *bar, uint32_t parity)
{
    const uint32_t a = tc_smem_u32(bar);
    for (long i = 0; i < TC_WAIT_POLLS; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

/* bounded wait that also gives up as soon as *abort is set (another role gave up) */
__device__ __forceinline__ bool tc_mbar_wait_abortable(unsigned long long *bar, uint32_t parity,
                                                       const volatile int *abort)
{
    const uint32_t a = tc_smem_u32(bar);
    for (long i = 0; i < TC_WAIT_POLLS; i++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(a), "r"(parity)
            : "memory");
        if (ok) return true;
        if ((i & 63) == 63 && *abort) return false;
    }
    return false;
}

/* one arrival on *bar (release: this thread's prior shared-memory writes are visible to the waiter) */
__device__ __forceinline__ void tc_mbar_arrive(unsigned long long *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(tc_smem_u32(bar)) : "memory");
}

/* named barrier among `count` threads (a role's threads, not the whole block) */
__device__ __forceinline__ void tc_bar_sync(int id, int count)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

/* named barrier with an AND vote over `count` threads */
__device__ __forceinline__ bool tc_bar_and(int id, int count, bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id), "r"(count)
        : "memory");
    return r != 0;
}

/* generic-proxy shared-memory writes -> visible to the tensor core (async proxy) */
__device__ __forceinline__ void tc_fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_before_sync()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void tc_fence_after_sync()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

/* whole warp: allocate ncols tensor-memory columns, base address written to *dst */
__device__ __forceinline__ void tc_alloc(uint32_t *dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_u32(dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tc_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

/* single thread: D[tmem] (+)= A * B^T, A M x 8 and B N x 8 from shared memory */
__device__ __forceinline__ void tc_mma_tf32(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                            uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}"
        ::"r"(dtmem), "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
        : "memory");
}

/* single thread: arrive on *bar once every MMA this thread issued so far has completed */
__device__ __forceinline__ void tc_commit(unsigned long long *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     tc_smem_u32(bar))
                 : "memory");
}

/* whole warp: 16 consecutive 32-bit columns of the warp's 32 lanes (one lane per thread) */
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    /* load and wait in one statement: the registers are valid when the asm ends */
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

} /* namespace */

#endif
