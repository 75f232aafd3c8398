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

// 16807^e mod (2^31 - 1): the jump of a Park-Miller state over e draws.
__device__ __forceinline__ uint32_t pm_pow16807(long long e)
{
    uint32_t r = 1u, b = 16807u;
    for (; e > 0; e >>= 1) {
        if (e & 1) r = pm_mul(r, b);
        b = pm_mul(b, b);
    }
    return r;
}

// ran01's return value for a state x already advanced (kernel.cl:50).  AM = 2^-31.
__device__ __forceinline__ float pm_uniform(uint32_t x)
{
    return __fmul_rn(__int2float_rn((int)x), 4.656612873077392578125e-10f);
}

// The throughput sampler's exponential clock: E = -ln(u) ~ Exp(1) for u
// uniform in (0, 1], without a division, written out so that the host
// restatement computes the same bits.  u = m * 2^e with m in [sqrt(1/2),
// sqrt(2)), t = m - 1, ln(m) = t + t^2 * Q(t) with Q the degree-6 polynomial
// fitted by least squares on Chebyshev nodes of that interval to
// (ln(1+t) - t) / t^2, weighted for relative error (|relative error of ln(m)|
// below 3e-7 in fp32), evaluated by Horner with fused multiply-adds.
// u = 1 gives E = +0.
__device__ __forceinline__ float race_exp1(float u)
{
    const uint32_t b = __float_as_uint(u);
    int e = (int)(b >> 23) - 127;
    float m = __uint_as_float((b & 0x007fffffu) | 0x3f800000u);
    if (m > 1.41421354f) {
        m = __fmul_rn(m, 0.5f);
        e += 1;
    }
    const float t = __fsub_rn(m, 1.0f);
    float q = __fmaf_rn(-0.098038554f, t, 0.16080461f);
    q = __fmaf_rn(q, t, -0.172902f);
    q = __fmaf_rn(q, t, 0.19920385f);
    q = __fmaf_rn(q, t, -0.24968483f);
    q = __fmaf_rn(q, t, 0.333343f);
    q = __fmaf_rn(q, t, -0.5000038f);
    const float lm = __fmaf_rn(t, __fmul_rn(t, q), t);
    return __fsub_rn(0.0f, __fmaf_rn((float)e, 0.693147182f, lm)); // 0 - x: +0 at u = 1, not -0
}

// Race key of a lane: the bits of E / weight = E * (1 / weight) (non-negative,
// so ordered as unsigned) with the low 5 bits replaced by the lane, so that one
// unsigned min reduction yields the winner -- the smallest E_j / w_j, which
// selects candidate j with probability w_j / sum(w) -- and equal keys go to the
// lowest lane.  The candidate tables hold 1 / weight; a candidate of weight 0
// (reciprocal +inf) cannot win: kNoKey.
constexpr uint32_t kNoKey = 0xffffffffu;

__device__ __forceinline__ uint32_t race_key(float e, float winv, int lane)
{
    return (__float_as_uint(__fmul_rn(e, winv)) & ~31u) | (uint32_t)lane;
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

constexpr uint32_t kWaitPolls = 1u << 24; // default poll limit of a bounded wait (about a second)

// The poll limit a kernel was given (a device word; <= 0 or null: the default).
__device__ __forceinline__ uint32_t wait_polls(const int *limit)
{
    const int v = limit ? *limit : 0;
    return v > 0 ? (uint32_t)v : kWaitPolls;
}

// Bounded wait on phase `parity` of `bar`.  Returns false after `limit` polls
// (the caller reports ACO_ERR_TIMEOUT); never spins forever.  The first poll
// does not block (test_wait), the later ones may suspend briefly (try_wait).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, uint32_t limit = kWaitPolls)
{
    const uint32_t addr = smem_u32(bar);
    for (uint32_t it = 0; it < limit; it++) {
        uint32_t done;
        if (it == 0)
            asm volatile("{\n\t.reg .pred p;\n\t"
                         "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                         "selp.u32 %0, 1, 0, p;\n\t}"
                         : "=r"(done)
                         : "r"(addr), "r"(parity)
                         : "memory");
        else
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
