// umma.cuh -- 5th-generation tensor-core (tcgen05) building blocks for sm_100a:
// tensor-memory allocation, shared-memory operand descriptors in the
// no-swizzle K-major layout, the BF16 x BF16 -> FP32 MMA issued by one thread,
// completion through an mbarrier, and accumulator reads.
//
// Operand layout in shared memory (K-major, no swizzle).  An R x K bf16 tile
// (R a multiple of 8, K a multiple of 16) is stored as "core matrices" of
// 8 rows x 16 bytes (8 elements of K), 128 contiguous bytes each; core matrix
// (r/8, k/8) sits at ((r/8) * (K/8) + k/8) * 128 bytes.  In descriptor terms
// the leading-dimension byte offset (next 8 elements of K) is 128 and the
// stride-dimension byte offset (next 8 rows) is K/8 * 128.  One MMA consumes
// K = 16 (two core matrices along K), so k-step s starts 256 * s bytes in.
//
// The descriptor and instruction-descriptor bit fields follow the PTX ISA
// description of tcgen05 matrix descriptors (start address >> 4 in bits 0-13,
// leading byte offset >> 4 in 16-29, stride byte offset >> 4 in 32-45,
// version 1 in 46-47, layout type 0 = no swizzle in 61-63) and of the
// kind::f16 instruction descriptor (D format F32 in bits 4-5, A and B format
// BF16 in 7-9 and 10-12, K-major A and B, N >> 3 in 17-22, M >> 4 in 24-28).
#pragma once

#include <cstdint>

#include "aco_device.cuh"

namespace aco {
namespace umma {

// Byte offset of element (r, k) of an R x K tile in the layout above.
__device__ __forceinline__ uint32_t kmajor_offset(int r, int k, int K)
{
    return ((uint32_t)(((r >> 3) * (K >> 3) + (k >> 3))) << 7) + ((uint32_t)(r & 7) << 4) + ((uint32_t)(k & 7) << 1);
}

// Shared-memory matrix descriptor of the tile at smem address `addr` (K columns), k-step s.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, int K, int s)
{
    const uint32_t a = addr + 256u * (uint32_t)s;
    const uint64_t lbo = 128u >> 4, sbo = (uint64_t)((K >> 3) * 128) >> 4;
    return (uint64_t)((a >> 4) & 0x3FFFu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// Instruction descriptor: D F32, A/B BF16, both K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ uint16_t bf16_bits(float x) // round to nearest even
{
    const __nv_bfloat16 b = __float2bfloat16_rn(x);
    return *reinterpret_cast<const uint16_t *>(&b);
}

// Tensor-memory allocation by one whole warp; the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Generic-proxy shared-memory writes become visible to the tensor core (async proxy).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T for one k-step; issued by a single thread.
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, bool acc)
{
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
                 "l"(adesc), "l"(bdesc), "r"(idesc), "r"((uint32_t)acc)
                 : "memory");
}

// Arrive on the mbarrier once every MMA issued so far by this thread is done.
__device__ __forceinline__ void commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

// 16 consecutive fp32 accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// TMEM address of lane `lane`, column `col` relative to the allocation base.
__device__ __forceinline__ uint32_t taddr(uint32_t base, int lane, int col)
{
    return base + ((uint32_t)lane << 16) + (uint32_t)col;
}

} // namespace umma
} // namespace aco
