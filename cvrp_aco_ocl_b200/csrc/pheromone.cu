// pheromone.cu -- route-cost reduction, best-so-far bookkeeping, elite
// selection and the row passes over the n x ld matrices (heuristic matrix,
// pheromone init, the fused update, the candidate gather).
//
// stats_kernel (one CTA per instance) restates, in one launch,
// best_solution_phase_0/1 (kernel.cl:594-665), update_best_so_far (:546-586),
// get_elites (:717-741) and the gathering half of pheromone_deposit
// (:747-776): it turns the elite tours into per-node successor lists so that
// the deposit can be applied inside the streaming pass in a fixed order
// (elite 0, 1, ..., ras_ranks-1) instead of with unordered float atomics.
//
// rows_kernel (ROW_UPDATE) is evaporation (kernel.cl:685-692) + deposit +
// compute_total_info (:782-789) as one pass: one warp per matrix row, float4
// loads and stores; it reads tau and heur (= eta^beta, precomputed once) and
// writes tau and total_info -- 16 bytes of HBM traffic per element -- and, in
// throughput mode, the total_info of the row's candidates (staged in shared
// memory) into the compact candidate table the construct kernel loads by TMA.
#include <cuda_runtime.h>

#include "aco_device.cuh"
#include "kernels.h"

namespace aco {

namespace {

constexpr unsigned FULL = 0xffffffffu;

__device__ __forceinline__ unsigned long long block_min_u64(unsigned long long v, unsigned long long *red)
{
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(FULL, v, o);
        v = w < v ? w : v;
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = lane < nw ? red[lane] : ~0ull;
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(FULL, v, o);
        v = w < v ? w : v;
    }
    return v; // every thread holds the block minimum
}

__global__ void __launch_bounds__(1024) stats_kernel(const StatsArgs *args, int do_elites)
{
    extern __shared__ float s_hb[]; // help_b[n_ants] of get_elites
    __shared__ unsigned long long red[32];
    __shared__ int s_best, s_flag;
    __shared__ float s_minval;
    const StatsArgs a = args[blockIdx.x];
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
        const unsigned rank = (g << lg) | (lg ? (__brev(lid) >> (32 - lg)) : 0u);
        const unsigned long long key = ((unsigned long long)__float_as_uint(a.lens[k]) << 32) | rank;
        best = key < best ? key : best;
    }
    best = block_min_u64(best, red);
    if (tid == 0) {
        const unsigned rank = (unsigned)(best & 0xffffffffu);
        const unsigned g = rank >> lg, br = rank & ((1u << lg) - 1u);
        const int idx = (int)((g << lg) | (lg ? (__brev(br) >> (32 - lg)) : 0u));
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
                r.time = (float)((double)(globaltimer_ns() - *a.t0_ns) * 1e-9);
                a.records[pos] = r;
            } else {
                set_status(a.status, ACO_ERR_RECORD_OVERFLOW);
            }
            *a.num_bsf = pos + 1;
        }
    }
    if (do_elites) {
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

// One warp, row i of instance a.  Columns are walked as float4 (ld is a
// multiple of 32); columns n..ld-1 stay zero.
__device__ __forceinline__ void row_pass(const UpdateArgs &a, int i, int mode, float trail, float *srow, int lane)
{
    const int n = a.n, q4 = (n + 3) >> 2;
    const size_t off = (size_t)i * a.ld;
    if (mode == ROW_HEUR) {
        for (int q = lane; q < q4; q += 32) {
            const float4 d = *reinterpret_cast<const float4 *>(a.dist + off + 4 * q);
            const int c = 4 * q;
            float4 h;
            h.x = c + 0 < n ? pow_rule(__fdiv_rn(1.0f, __fadd_rn(d.x, 0.1f)), a.beta, a.beta_int) : 0.f;
            h.y = c + 1 < n ? pow_rule(__fdiv_rn(1.0f, __fadd_rn(d.y, 0.1f)), a.beta, a.beta_int) : 0.f;
            h.z = c + 2 < n ? pow_rule(__fdiv_rn(1.0f, __fadd_rn(d.z, 0.1f)), a.beta, a.beta_int) : 0.f;
            h.w = c + 3 < n ? pow_rule(__fdiv_rn(1.0f, __fadd_rn(d.w, 0.1f)), a.beta, a.beta_int) : 0.f;
            *reinterpret_cast<float4 *>(a.heur + off + 4 * q) = h;
        }
        return;
    }
    if (mode == ROW_INIT_TRAIL || mode == ROW_INIT_BSF) { // pheromone_init (kernel.cl:672-679)
        const float tr = mode == ROW_INIT_BSF ? __fdiv_rn(1.0f, __fmul_rn(a.rho, *a.bsf_len)) : trail;
        const float pa = pow_rule(tr, a.alpha, a.alpha_int);
        for (int q = lane; q < q4; q += 32) {
            const float4 h = *reinterpret_cast<const float4 *>(a.heur + off + 4 * q);
            const int c = 4 * q;
            float4 t, o;
            t.x = c + 0 < n ? tr : 0.f; o.x = c + 0 < n ? __fmul_rn(pa, h.x) : 0.f;
            t.y = c + 1 < n ? tr : 0.f; o.y = c + 1 < n ? __fmul_rn(pa, h.y) : 0.f;
            t.z = c + 2 < n ? tr : 0.f; o.z = c + 2 < n ? __fmul_rn(pa, h.z) : 0.f;
            t.w = c + 3 < n ? tr : 0.f; o.w = c + 3 < n ? __fmul_rn(pa, h.w) : 0.f;
            *reinterpret_cast<float4 *>(a.tau + off + 4 * q) = t;
            *reinterpret_cast<float4 *>(a.total + off + 4 * q) = o;
            if (a.chc) *reinterpret_cast<float4 *>(srow + 4 * q) = o;
        }
    } else if (mode == ROW_UPDATE) {
        // deposit columns of this row: the successor of customer i in each elite
        // tour, read once and broadcast (elite order kept when adding)
        const int R = a.ras_ranks;
        int mys = -1;
        float myd = 0.f;
        if (lane < R && i != 0) {
            mys = __ldg(a.succ + (size_t)lane * n + i);
            myd = __ldg(a.d_tau + lane);
        }
        int sr[8];
        float dr[8];
#pragma unroll
        for (int r = 0; r < 8; r++) {
            sr[r] = __shfl_sync(FULL, mys, r);
            dr[r] = __shfl_sync(FULL, myd, r);
        }
        for (int q = lane; q < q4; q += 32) {
            const float4 t = *reinterpret_cast<const float4 *>(a.tau + off + 4 * q);
            const float4 h = __ldg(reinterpret_cast<const float4 *>(a.heur + off + 4 * q));
            float v0 = __fmul_rn(a.evap, t.x), v1 = __fmul_rn(a.evap, t.y);
            float v2 = __fmul_rn(a.evap, t.z), v3 = __fmul_rn(a.evap, t.w);
            const int c4 = 4 * q;
            if (i != 0) {
#pragma unroll
                for (int r = 0; r < 8; r++) {
                    const unsigned d = (unsigned)(sr[r] - c4);
                    if (r < R && d < 4u) {
                        if (d == 0) v0 = __fadd_rn(v0, dr[r]);
                        else if (d == 1) v1 = __fadd_rn(v1, dr[r]);
                        else if (d == 2) v2 = __fadd_rn(v2, dr[r]);
                        else v3 = __fadd_rn(v3, dr[r]);
                    }
                }
                for (int r = 8; r < R; r++) { // more than 8 ranks: read the rest directly
                    const unsigned d = (unsigned)(__ldg(a.succ + (size_t)r * n + i) - c4);
                    if (d < 4u) {
                        const float dt = __ldg(a.d_tau + r);
                        if (d == 0) v0 = __fadd_rn(v0, dt);
                        else if (d == 1) v1 = __fadd_rn(v1, dt);
                        else if (d == 2) v2 = __fadd_rn(v2, dt);
                        else v3 = __fadd_rn(v3, dt);
                    }
                }
            } else { // depot row: depot -> customer edges from the per-column masks
                const uint32_t m0 = c4 + 0 < n ? __ldg(a.depmask + c4 + 0) : 0u;
                const uint32_t m1 = c4 + 1 < n ? __ldg(a.depmask + c4 + 1) : 0u;
                const uint32_t m2 = c4 + 2 < n ? __ldg(a.depmask + c4 + 2) : 0u;
                const uint32_t m3 = c4 + 3 < n ? __ldg(a.depmask + c4 + 3) : 0u;
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
            *reinterpret_cast<float4 *>(a.tau + off + 4 * q) = o;
            *reinterpret_cast<float4 *>(a.total + off + 4 * q) = tot;
            if (a.chc) *reinterpret_cast<float4 *>(srow + 4 * q) = tot;
        }
    } else if (mode == ROW_GATHER) {
        if (a.chc)
            for (int q = lane; q < q4; q += 32)
                *reinterpret_cast<float4 *>(srow + 4 * q) = *reinterpret_cast<const float4 *>(a.total + off + 4 * q);
    }
    if (a.chc) { // compact candidate table: chc[i][j] = total[i][nn[i][j]]
        __syncwarp();
        for (int j = lane; j < a.K; j += 32) a.chc[(size_t)i * a.Kp + j] = srow[a.nn16[(size_t)i * a.Kp + j]];
        __syncwarp();
    }
}

__global__ void __launch_bounds__(256) rows_kernel(const UpdateArgs *args, const int *row_base, int n_inst,
                                                   int total_rows, int mode, float trail, int ld_max)
{
    extern __shared__ __align__(16) float s_rows[];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    float *srow = s_rows + (size_t)wib * ld_max;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    int b = 0;
    for (int g = gw; g < total_rows; g += nw) {
        if (n_inst > 1) { // instance of global row g: binary search over the first rows
            int lo = 0, hi = n_inst;
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (__ldg(row_base + mid) <= g) lo = mid;
                else hi = mid;
            }
            b = lo;
        }
        row_pass(args[b], g - __ldg(row_base + b), mode, trail, srow, lane);
    }
}

__global__ void t0_kernel(unsigned long long *t0) { *t0 = globaltimer_ns(); }

} // namespace

cudaError_t launch_stats(const StatsArgs *d_args, int n_inst, int do_elites, size_t smem, cudaStream_t st)
{
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(stats_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    stats_kernel<<<n_inst, 1024, smem, st>>>(d_args, do_elites);
    return cudaGetLastError();
}

size_t rows_smem(int ld_max) { return (size_t)8 * ld_max * sizeof(float); }

cudaError_t launch_rows(const UpdateArgs *d_args, const int *d_row_base, int n_inst, int total_rows, int mode,
                        float trail, int ld_max, int sm_count, cudaStream_t st)
{
    const size_t smem = rows_smem(ld_max);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    int blocks = (total_rows + 7) / 8; // 8 warps (rows) per CTA
    const int cap = sm_count * 8;      // grid-stride beyond 8 CTAs per SM
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    rows_kernel<<<blocks, 256, smem, st>>>(d_args, d_row_base, n_inst, total_rows, mode, trail, ld_max);
    return cudaGetLastError();
}

cudaError_t launch_t0(unsigned long long *t0, cudaStream_t st)
{
    t0_kernel<<<1, 1, 0, st>>>(t0);
    return cudaGetLastError();
}

} // namespace aco
