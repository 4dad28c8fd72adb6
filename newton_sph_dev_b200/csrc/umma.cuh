// umma.cuh — 5th-generation tensor core (tcgen05) building blocks for sm_100a,
// written as inline PTX: shared-memory operand descriptors, the instruction
// descriptor of kind::f16 (bf16 x bf16 -> f32), TMEM allocation, MMA issue,
// commit to an mbarrier, bounded waits and accumulator loads.
//
// Operand layout: K-major, no swizzle. A tile of R rows x K bf16 columns is
// stored as 8x8 "core matrices" (8 rows x 16 bytes, 128 contiguous bytes):
// core matrix (r/8, k/8) at byte ((r/8)*(K/8) + k/8)*128, element (r, k)
// inside it at (r%8)*16 + (k%8)*2. In the descriptor the leading byte
// offset (LBO) is the stride between core matrices adjacent in K (128 B) and
// the stride byte offset (SBO) the stride between 8-row groups ((K/8)*128 B).
// One MMA consumes K = 16, i.e. two core matrices along K, so the k-th MMA of
// a chain starts 256*k bytes further.
//
// Accumulator (M = 128, cta_group::1): row m of D is TMEM lane m, column n
// is TMEM column (base + n), fp32. Warp w of the CTA reads lanes
// [32*(w%4), 32*(w%4) + 32) with tcgen05.ld.32x32b.
#pragma once

#include <cstdint>

namespace nsph {
namespace umma {

__host__ __device__ __forceinline__ uint32_t core_offset(int row, int k, int K)
{
    return (uint32_t)((((row >> 3) * (K >> 3) + (k >> 3)) << 7) + ((row & 7) << 4) + ((k & 7) << 1));
}

// shared-memory matrix descriptor: start address, LBO, SBO (bytes), version 1, no swizzle
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    uint64_t d = (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;
    return d;
}

// instruction descriptor, kind::f16: D f32, A and B bf16, both K-major, M x N
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// whole warp: allocate `ncols` TMEM columns (power of two >= 32); the base
// address is written to *slot (shared memory)
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)), "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}

// whole warp
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_smem_to_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// one thread: D (+)= A * B^T over one K = 16 slice
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

// one thread: arrive on `bar` when all MMAs issued so far by this thread complete
__device__ __forceinline__ void mma_commit(uint64_t* bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_addr(bar))
                 : "memory");
}

// wait for the phase with parity `parity` to complete; gives up after
// `limit` polls and returns false (the caller records the error)
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int limit)
{
    const uint32_t a = smem_addr(bar);
    for (int it = 0; it < limit; ++it) {
        uint32_t done;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// this warp's 32 lanes x 16 fp32 columns starting at `taddr` (lane offset included)
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
          "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

}  // namespace umma
}  // namespace nsph
