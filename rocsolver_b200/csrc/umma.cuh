// umma.cuh -- the 5th-generation tensor-core path (tcgen05) for FP32 products at FP32-level
// accuracy: split-TF32 operands in shared memory, accumulators in tensor memory (TMEM).
//
// Operands are stored in the no-swizzle K-major canonical layout of tcgen05 shared-memory
// descriptors: core matrices of 8 rows x 16 bytes (8 rows x 4 TF32), the two 16-byte K
// halves of one 8-deep MMA step LBO = 128 bytes apart, consecutive 8-row groups SBO bytes
// apart.  With K = kk elements per row, element (r, k) sits at
//     (r % 8) * 16 + (r / 8) * (kk / 4) * 128 + (k / 4) * 128 + (k % 4) * 4   bytes,
// so K step s (k = 8s .. 8s+7) starts 256 * s bytes into the buffer (kmaj_off below).
//
// Split TF32: x = hi + lo with hi = x rounded to TF32 and lo = (x - hi) rounded to TF32, both
// exact TF32 values (so the tensor core's handling of the low mantissa bits does not
// matter); a*b ~ a_lo*b_hi + a_hi*b_lo + a_hi*b_hi, accumulated in FP32 in TMEM (the dropped
// a_lo*b_lo is below 2^-21 |a||b|).
//
// Every wait on an MMA completion is bounded: after UMMA_WAIT_LIMIT polls the caller sees
// `false`, records the failure and stops issuing tensor work (it still frees its TMEM).
#pragma once

#include <stdint.h>

namespace rsb {
namespace umma {

#ifndef UMMA_WAIT_LIMIT
#define UMMA_WAIT_LIMIT (1 << 22)
#endif

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// byte offset of element (r, k) of a K-major operand with kk elements per row
__host__ __device__ __forceinline__ uint32_t kmaj_off(int r, int k, int kk)
{
    return (uint32_t)((r & 7) * 16 + (r >> 3) * (kk >> 2) * 128 + (k >> 2) * 128 + (k & 3) * 4);
}

// shared-memory matrix descriptor (no swizzle, version 1 = sm100)
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo)
{
    return (uint64_t)((addr >> 4) & 0x3fff) | ((uint64_t)((lbo >> 4) & 0x3fff) << 16)
           | ((uint64_t)((sbo >> 4) & 0x3fff) << 32) | ((uint64_t)1 << 46);
}

// instruction descriptor of kind::tf32: FP32 accumulate, TF32 A and B, both K-major
__host__ __device__ constexpr uint32_t idesc_tf32(int m, int n)
{
    return (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(n >> 3) << 17)
           | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
                 ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(accumulate), "r"(0), "r"(0),
                 "r"(0), "r"(0));
}

// arrive on the mbarrier once every tensor operation this thread issued has completed
__device__ __forceinline__ void commit(uint64_t* mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(mbar)) : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count));
}

// bounded wait for the mbarrier phase with parity `parity` to complete
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity)
{
    uint32_t done = 0;
    for(int it = 0; it < UMMA_WAIT_LIMIT && !done; ++it)
        asm volatile("{\n\t.reg .pred P1;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t}"
                     : "=r"(done)
                     : "r"(smem_u32(mbar)), "r"(parity)
                     : "memory");
    return done != 0;
}

// make this thread's generic-proxy shared-memory writes visible to the tensor core
__device__ __forceinline__ void fence_async_shared()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
__device__ __forceinline__ void fence_before_sync()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// TMEM allocation by one whole warp; the base address is written to *slot
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 ::"r"(smem_u32(slot)), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base),
                 "r"(ncols));
}

// 16 consecutive FP32 columns of this thread's TMEM lane (lane = 32 * (warp % 4) + lane id)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for(int j = 0; j < 16; ++j)
        v[j] = __uint_as_float(r[j]);
}

// split x into TF32 hi and lo (both exact TF32 bit patterns), rounding to nearest
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo)
{
    hi = (__float_as_uint(x) + 0x1000u) & 0xffffe000u;
    lo = (__float_as_uint(x - __uint_as_float(hi)) + 0x1000u) & 0xffffe000u;
}

// smallest power of two >= n and >= 32 (TMEM allocation granularity)
__host__ __device__ constexpr uint32_t tmem_cols(uint32_t n)
{
    uint32_t c = 32;
    while(c < n)
        c <<= 1;
    return c;
}

} // namespace umma
} // namespace rsb
