// pheromone.cu -- route-cost reduction, best-so-far bookkeeping, elite
// selection and the fused pheromone pass.
//
// stats_kernel (one CTA) restates, in one launch, best_solution_phase_0/1
// (kernel.cl:594-665), update_best_so_far (:546-586), get_elites (:717-741)
// and the gathering half of pheromone_deposit (:747-776): it turns the elite
// tours into per-node successor lists so that the deposit can be applied inside
// the streaming pass in a fixed order (elite 0, 1, ..., ras_ranks-1) instead of
// with unordered float atomics.
//
// pheromone_update_kernel is evaporation (kernel.cl:685-692) + deposit +
// compute_total_info (:782-789) as one float4 pass over the n x ld matrices:
// read tau and heur (= eta^beta, precomputed once), write tau and total_info:
// 16 bytes of HBM traffic per element.
#include <cuda_runtime.h>

#include "aco_device.cuh"
#include "kernels.h"

namespace aco {

namespace {

__device__ __forceinline__ unsigned long long block_min_u64(unsigned long long v, unsigned long long *red)
{
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = lane < nw ? red[lane] : ~0ull;
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v; // every thread holds the block minimum
}

__global__ void __launch_bounds__(1024) stats_kernel(StatsArgs a, const unsigned long long *t0_ns)
{
    extern __shared__ float s_hb[]; // help_b[n_ants] of get_elites
    __shared__ unsigned long long red[32];
    __shared__ int s_best, s_flag;
    __shared__ float s_minval;
    const int A = a.n_ants, T = a.T, tid = threadIdx.x, bs = blockDim.x;
    const int lg = a.log2_nloc;
    const int iter = *a.iteration;

    // iteration best: min over (length, work-group, bit-reversed lane).  Phase 0
    // halves a power-of-two group keeping the left operand on ties, so inside a
    // group the survivor among equal lengths is the lowest bit-reversed lane;
    // phase 1 scans groups in order with a strict <.
    unsigned long long best = ~0ull;
    for (int k = tid; k < A; k += bs) {
        const unsigned g = (unsigned)k >> lg, lid = (unsigned)k & ((1u << lg) - 1u);
        const unsigned rank = (g << lg) | (__brev(lid) >> (32 - lg));
        const unsigned long long key = ((unsigned long long)__float_as_uint(a.lens[k]) << 32) | rank;
        best = key < best ? key : best;
    }
    best = block_min_u64(best, red);
    if (tid == 0) {
        const unsigned rank = (unsigned)(best & 0xffffffffu);
        const unsigned g = rank >> lg, br = rank & ((1u << lg) - 1u);
        const int idx = (int)((g << lg) | (__brev(br) >> (32 - lg)));
        const float minval = a.lens[idx];
        a.solutions[(size_t)T * (A + 1)] = idx;
        s_best = idx;
        s_minval = minval;
        s_flag = __fsub_rn(minval, a.lens[A]) < -kEps; // kernel.cl:660
    }
    __syncthreads();
    if (s_flag) { // update_best_so_far (kernel.cl:551-585)
        const int *it = a.solutions + (size_t)T * s_best;
        int *bt = a.solutions + (size_t)T * A;
        const int size = it[T - 1];
        for (int p = tid; p < size; p += bs) bt[p] = it[p];
        if (tid == 0) {
            bt[T - 1] = size;
            a.lens[A] = s_minval;
            const int pos = *a.num_bsf;
            if (pos < a.record_cap) {
                aco_record r;
                r.iter = iter;
                r.length = s_minval;
                r.time = (float)((double)(globaltimer_ns() - *t0_ns) * 1e-9);
                a.records[pos] = r;
            } else {
                set_status(a.status, ACO_ERR_RECORD_OVERFLOW);
            }
            *a.num_bsf = pos + 1;
        }
    }
    if (a.do_elites) {
        // get_elites (kernel.cl:717-741): elite 0 is the best-so-far slot, then
        // ras_ranks-1 first-occurrence minima with knock-out.
        for (int k = tid; k < A; k += bs) s_hb[k] = a.lens[k];
        if (tid == 0) a.elites[0] = A;
        __syncthreads();
        for (int r = 1; r < a.ras_ranks; r++) {
            unsigned long long m = ~0ull;
            for (int k = tid; k < A; k += bs) {
                const unsigned long long key = ((unsigned long long)__float_as_uint(s_hb[k]) << 32) | (unsigned)k;
                m = key < m ? key : m;
            }
            m = block_min_u64(m, red);
            if (tid == 0) {
                const int target = A > 0 ? (int)(m & 0xffffffffu) : 0;
                s_hb[target] = __int_as_float(0x7f800000);
                a.elites[r] = target;
            }
            __syncthreads();
        }
        // deposit list: successor of every customer in each elite tour and the
        // depot -> customer edges as a per-customer bit mask.
        const int n = a.n, R = a.ras_ranks;
        for (int e = tid; e < R * n; e += bs) a.succ[e] = -1;
        for (int e = tid; e < n; e += bs) a.depmask[e] = 0u;
        if (tid < R) a.d_tau[tid] = __fdiv_rn((float)(R - tid), a.lens[a.elites[tid]]); // kernel.cl:767-768
        __syncthreads();
        for (int r = 0; r < R; r++) {
            const int *tour = a.solutions + (size_t)T * a.elites[r];
            const int size = tour[T - 1];
            for (int k = tid; k < size - 1; k += bs) {
                const int u = tour[k], v = tour[k + 1];
                if (u != 0) a.succ[(size_t)r * n + u] = v;
                else atomicOr(&a.depmask[v], 1u << r);
            }
        }
    }
    if (tid == 0) *a.iteration = iter + 1; // main.cpp:86 (Problem::iteration++)
}

__global__ void __launch_bounds__(256) pheromone_update_kernel(UpdateArgs a)
{
    const unsigned units = (unsigned)a.n * (unsigned)a.q;
    const unsigned stride = gridDim.x * blockDim.x;
    const int R = a.ras_ranks;
    for (unsigned u = blockIdx.x * blockDim.x + threadIdx.x; u < units; u += stride) {
        const unsigned i = (unsigned)(((unsigned long long)u * a.qinv) >> 40);
        const unsigned c4 = (u - i * (unsigned)a.q) * 4u;
        const size_t off = (size_t)i * a.ld + c4;
        const float4 t = *reinterpret_cast<const float4 *>(a.tau + off);
        const float4 h = __ldg(reinterpret_cast<const float4 *>(a.heur + off));
        float v0 = __fmul_rn(a.evap, t.x), v1 = __fmul_rn(a.evap, t.y);
        float v2 = __fmul_rn(a.evap, t.z), v3 = __fmul_rn(a.evap, t.w);
        if (i != 0) {
            for (int r = 0; r < R; r++) {
                const unsigned d = (unsigned)(__ldg(a.succ + (size_t)r * a.n + i) - (int)c4);
                if (d < 4u) {
                    const float dt = __ldg(a.d_tau + r);
                    if (d == 0) v0 = __fadd_rn(v0, dt);
                    else if (d == 1) v1 = __fadd_rn(v1, dt);
                    else if (d == 2) v2 = __fadd_rn(v2, dt);
                    else v3 = __fadd_rn(v3, dt);
                }
            }
        } else {
            const uint32_t m0 = c4 + 0 < (unsigned)a.n ? __ldg(a.depmask + c4 + 0) : 0u;
            const uint32_t m1 = c4 + 1 < (unsigned)a.n ? __ldg(a.depmask + c4 + 1) : 0u;
            const uint32_t m2 = c4 + 2 < (unsigned)a.n ? __ldg(a.depmask + c4 + 2) : 0u;
            const uint32_t m3 = c4 + 3 < (unsigned)a.n ? __ldg(a.depmask + c4 + 3) : 0u;
            for (int r = 0; r < R; r++) {
                const float dt = __ldg(a.d_tau + r);
                if ((m0 >> r) & 1u) v0 = __fadd_rn(v0, dt);
                if ((m1 >> r) & 1u) v1 = __fadd_rn(v1, dt);
                if ((m2 >> r) & 1u) v2 = __fadd_rn(v2, dt);
                if ((m3 >> r) & 1u) v3 = __fadd_rn(v3, dt);
            }
        }
        float4 o, tot;
        o.x = v0; o.y = v1; o.z = v2; o.w = v3;
        tot.x = __fmul_rn(pow_rule(v0, a.alpha, a.alpha_int), h.x);
        tot.y = __fmul_rn(pow_rule(v1, a.alpha, a.alpha_int), h.y);
        tot.z = __fmul_rn(pow_rule(v2, a.alpha, a.alpha_int), h.z);
        tot.w = __fmul_rn(pow_rule(v3, a.alpha, a.alpha_int), h.w);
        *reinterpret_cast<float4 *>(a.tau + off) = o;
        *reinterpret_cast<float4 *>(a.total + off) = tot;
    }
}

// pheromone_init (kernel.cl:672-679); trail_0 = 1/(rho * best length) when
// from_bsf is set (g_aco.cpp:89).  Columns n..ld-1 stay zero.
__global__ void __launch_bounds__(256) pheromone_init_kernel(InitArgs a)
{
    const float trail = a.from_bsf ? __fdiv_rn(1.0f, __fmul_rn(a.rho, *a.bsf_len)) : a.trail;
    const float pa = pow_rule(trail, a.alpha, a.alpha_int);
    const size_t total = (size_t)a.n * a.ld;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
        const int col = (int)(g % (size_t)a.ld);
        const bool in = col < a.n;
        a.tau[g] = in ? trail : 0.f;
        a.total[g] = in ? __fmul_rn(pa, a.heur[g]) : 0.f;
    }
}

// eta^beta = (1/(d + 0.1f))^beta, once per instance (kernel.cl:678,788).
__global__ void __launch_bounds__(256) heur_kernel(const float *dist, float *heur, int n, int ld, float beta, int beta_int)
{
    const size_t total = (size_t)n * ld;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < total; g += (size_t)gridDim.x * blockDim.x) {
        const int col = (int)(g % (size_t)ld);
        heur[g] = col < n ? pow_rule(__fdiv_rn(1.0f, __fadd_rn(dist[g], 0.1f)), beta, beta_int) : 0.f;
    }
}

__global__ void t0_kernel(unsigned long long *t0) { *t0 = globaltimer_ns(); }

} // namespace

cudaError_t launch_heur(const float *dist, float *heur, int n, int ld, float beta, int beta_int, cudaStream_t st)
{
    const size_t total = (size_t)n * ld;
    const int blocks = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
    heur_kernel<<<blocks, 256, 0, st>>>(dist, heur, n, ld, beta, beta_int);
    return cudaGetLastError();
}

cudaError_t launch_pheromone_init(const InitArgs &a, cudaStream_t st)
{
    const size_t total = (size_t)a.n * a.ld;
    const int blocks = (int)((total + 255) / 256 < 4096 ? (total + 255) / 256 : 4096);
    pheromone_init_kernel<<<blocks, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_stats(const StatsArgs &a, cudaStream_t st)
{
    const size_t smem = (size_t)(a.n_ants > 0 ? a.n_ants : 1) * sizeof(float);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(stats_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    stats_kernel<<<1, 1024, smem, st>>>(a, a.t0_ns);
    return cudaGetLastError();
}

cudaError_t launch_pheromone_update(const UpdateArgs &a, int sm_count, cudaStream_t st)
{
    const unsigned units = (unsigned)a.n * (unsigned)a.q;
    int blocks = (int)((units + 255) / 256);
    const int cap = sm_count * 8; // 8 CTAs of 256 threads per SM, grid-stride beyond that
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    pheromone_update_kernel<<<blocks, 256, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_t0(unsigned long long *t0, cudaStream_t st)
{
    t0_kernel<<<1, 1, 0, st>>>(t0);
    return cudaGetLastError();
}

} // namespace aco
