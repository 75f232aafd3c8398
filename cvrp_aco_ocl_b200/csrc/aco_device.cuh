// aco_device.cuh -- device helpers shared by the sm_100a kernels.
//
// Arithmetic rules (they are what makes the CUDA path bit-exact against the
// reference): every fp32 operation that the reference writes as a separate
// expression is issued with an explicit round-to-nearest intrinsic
// (__fadd_rn/__fmul_rn/__fdiv_rn) so that nvcc cannot contract it into an FMA,
// and the Park-Miller stream is advanced with exact 64-bit modular
// multiplication instead of Schrage's decomposition (both compute
// 16807 * x mod (2^31 - 1) for x in [0, 2^31 - 1)).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/cvrp_aco.h"

namespace aco {

constexpr uint32_t kPM = 2147483647u; // Park-Miller modulus
constexpr float kEps = 0.001f;        // EPSILON (utilities.h:19, kernel.cl:6)

// a * b mod (2^31 - 1) for a, b < 2^31 - 1.
__device__ __forceinline__ uint32_t pm_mul(uint32_t a, uint32_t b)
{
    const uint64_t p = (uint64_t)a * b;
    uint32_t r = (uint32_t)(p & kPM) + (uint32_t)(p >> 31);
    r = (r & kPM) + (r >> 31);
    return r >= kPM ? r - kPM : r;
}

// ran01's return value for a state x already advanced (kernel.cl:50).  AM = 2^-31.
__device__ __forceinline__ float pm_uniform(uint32_t x)
{
    return __fmul_rn(__int2float_rn((int)x), 4.656612873077392578125e-10f);
}

// Sticky error: the first failing kernel's code wins.
__device__ __forceinline__ void set_status(int *status, int code)
{
    atomicCAS(status, 0, code);
}

// pow(x, e) with the oracle's rule: exact left-to-right products for integer
// 0 <= e <= 8, powf otherwise (non-integer exponents are outside parity).
__device__ __forceinline__ float pow_rule(float x, float e, int e_int)
{
    if (e_int == 1) return x;
    if (e_int >= 0) {
        if (e_int == 0) return 1.0f;
        float r = x;
        for (int i = 1; i < e_int; i++) r = __fmul_rn(r, x);
        return r;
    }
    return powf(x, e);
}

// ---- TMA bulk copies (1-D cp.async.bulk, no multicast) and mbarriers ------
__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
}

// Bulk global -> shared copy completing on `bar`.  dst, src 16-byte aligned,
// bytes a multiple of 16.
__device__ __forceinline__ void tma_bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile("cp.async.bulk.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Bounded wait on phase `parity` of `bar`.  Returns false after ~`limit`
// polls (the caller reports ACO_ERR_TIMEOUT); never spins forever.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit = 1u << 24)
{
    const uint32_t addr = smem_u32(bar);
    for (uint32_t it = 0; it < limit; it++) {
        uint32_t done;
        asm volatile("{\n\t.reg .pred p;\n\t"
                     "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                     "selp.u32 %0, 1, 0, p;\n\t}"
                     : "=r"(done)
                     : "r"(addr), "r"(parity)
                     : "memory");
        if (done) return true;
        if (it > 64) __nanosleep(64);
    }
    return false;
}

__device__ __forceinline__ void named_barrier(int id, int threads)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(threads) : "memory");
}

__device__ __forceinline__ uint64_t globaltimer_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

} // namespace aco
