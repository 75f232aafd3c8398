// swap.cu -- the inter-route swap stage after 2-opt: LocalSearch::swap
// (localSearch.cpp:301-410) on every ant's tour, then the tour length as
// compute_tour_length sums it (vrpHelper.cpp:244-253).
//
// The reference scans positions i < j in order and applies the first exchange
// of two customers whose gain is below -EPSILON and that keeps both routes
// within capacity and max_distance, then resumes the scan at the same i.  One
// warp per ant: for position i the lanes evaluate 32 candidate positions j at
// a time and a ballot picks the lowest qualifying one, which is the one the
// sequential scan would take.  Depot positions never move (only customers are
// exchanged), so each position's route index is fixed for the whole stage.
// Every float expression keeps the reference's evaluation order.
//
// One CTA per construct work item (instance, first ant): its ants share the
// instance, whose distance matrix is staged in shared memory when it fits.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/cvrp_aco.h"
#include "aco_device.cuh"
#include "kernels.h"

namespace aco {
namespace {

constexpr unsigned FULL = 0xffffffffu;

// Per-warp shared arrays: tour (T ints), route index of every position (T
// ints), route loads and lengths (n each).
__host__ __device__ inline size_t swap_warp_bytes(int n) { return (size_t)(2 * 2 * n + 2 * n) * 4; }

__host__ __device__ inline bool swap_stage_matrix(int n, int ld, int apc)
{
    return (size_t)n * ld * 4 + (size_t)apc * swap_warp_bytes(n) <= (size_t)200 * 1024;
}

template <bool SMAT>
__device__ void swap_ant(const ConstructArgs &a, int ant, const float *D, int ldd, int *tour, int *rpos, int *rload,
                         float *rdist, int max_swaps)
{
    const int lane = threadIdx.x & 31, n = a.n, T = a.T;
    int *gt = a.solutions + (size_t)ant * T;
    const int size = gt[T - 1];
    if (size < 2) return; // a failed construction: nothing to do (its status is already set)
    for (int p = lane; p < size; p += 32) tour[p] = gt[p];
    __syncwarp();
    // route index of every position (depots at or before it, counted from position 1)
    int base = 0;
    for (int p0 = 0; p0 < size; p0 += 32) {
        const int p = p0 + lane;
        const bool dep = p >= 1 && p < size && tour[p] == 0;
        const unsigned m = __ballot_sync(FULL, dep);
        if (p < size) rpos[p] = base + __popc(m & ((1u << lane) - 1u));
        base += __popc(m);
    }
    __syncwarp();
    // route loads and lengths (localSearch.cpp:322-341): one lane per route
    // walks it; the route of a depot position p >= 1 ends there
    for (int p0 = 1; p0 < size; p0 += 32) {
        const int p = p0 + lane;
        if (p < size && tour[p] == 0) {
            const int k = rpos[p];
            int beg = p - 1;
            while (beg > 0 && tour[beg] != 0) beg--;
            int load = 0;
            float dd = 0.f;
            for (int q = beg + 1; q <= p; q++) {
                load += a.demand[tour[q]];
                dd = __fadd_rn(dd, D[(size_t)tour[q - 1] * ldd + tour[q]]);
            }
            rload[k] = load;
            rdist[k] = __fadd_rn(dd, __fmul_rn(a.serv_time, (float)(p - beg - 1)));
        }
    }
    __syncwarp();
    int swaps = 0;
    bool over = false;
    for (int i = 1; i < size && !over;) {
        const int n1 = tour[i];
        if (n1 == 0) {
            i++;
            continue;
        }
        const int p_n1 = tour[i - 1], s_n1 = tour[i + 1], p1 = rpos[i];
        const float d_pn1_n1 = D[(size_t)p_n1 * ldd + n1], d_n1_sn1 = D[(size_t)n1 * ldd + s_n1];
        bool moved = false;
        for (int j0 = i + 1; j0 < size; j0 += 32) {
            const int j = j0 + lane;
            int n2 = 0;
            bool cand = false;
            int load1 = 0, load2 = 0;
            float dist1 = 0.f, dist2 = 0.f;
            if (j < size) n2 = tour[j];
            if (j < size && n2 != 0) {
                const int p_n2 = tour[j - 1], s_n2 = tour[j + 1], p2 = rpos[j];
                const float d_pn1_n2 = D[(size_t)p_n1 * ldd + n2], d_n1_sn2 = D[(size_t)n1 * ldd + s_n2];
                const float d_n2_sn2 = D[(size_t)n2 * ldd + s_n2];
                float gain;
                float d_pn2_n2 = 0.f, d_n2_sn1 = 0.f, d_pn2_n1 = 0.f;
                if (j == i + 1) {
                    gain = __fadd_rn(-__fadd_rn(d_pn1_n1, d_n2_sn2), __fadd_rn(d_pn1_n2, d_n1_sn2));
                } else {
                    d_pn2_n2 = D[(size_t)p_n2 * ldd + n2];
                    d_n2_sn1 = D[(size_t)n2 * ldd + s_n1];
                    d_pn2_n1 = D[(size_t)p_n2 * ldd + n1];
                    const float rem = __fadd_rn(__fadd_rn(__fadd_rn(d_pn1_n1, d_n1_sn1), d_pn2_n2), d_n2_sn2);
                    const float add = __fadd_rn(__fadd_rn(__fadd_rn(d_pn1_n2, d_n2_sn1), d_pn2_n1), d_n1_sn2);
                    gain = __fadd_rn(-rem, add);
                }
                if (gain < -kEps) {
                    if (p1 != p2) {
                        load1 = rload[p1] - a.demand[n1] + a.demand[n2];
                        load2 = rload[p2] - a.demand[n2] + a.demand[n1];
                        dist1 = __fadd_rn(__fsub_rn(rdist[p1], __fadd_rn(d_pn1_n1, d_n1_sn1)),
                                          __fadd_rn(d_pn1_n2, d_n2_sn1));
                        dist2 = __fadd_rn(__fsub_rn(rdist[p2], __fadd_rn(d_pn2_n2, d_n2_sn2)),
                                          __fadd_rn(d_pn2_n1, d_n1_sn2));
                        cand = !((load1 > a.capacity || load2 > a.capacity) || (dist1 > a.max_dist || dist2 > a.max_dist));
                    } else {
                        load1 = load2 = rload[p1];
                        dist1 = dist2 = __fadd_rn(rdist[p1], gain);
                        cand = true;
                    }
                }
            }
            const unsigned m = __ballot_sync(FULL, cand);
            if (m) {
                const int src = __ffs(m) - 1;
                const int jj = __shfl_sync(FULL, j, src), nn2 = __shfl_sync(FULL, n2, src);
                const int l1 = __shfl_sync(FULL, load1, src), l2 = __shfl_sync(FULL, load2, src);
                const float e1 = __shfl_sync(FULL, dist1, src), e2 = __shfl_sync(FULL, dist2, src);
                if (lane == 0) {
                    const int p2 = rpos[jj];
                    tour[i] = nn2;
                    tour[jj] = n1;
                    rload[p1] = l1;
                    rload[p2] = l2;
                    rdist[p1] = e1;
                    rdist[p2] = e2;
                }
                __syncwarp();
                moved = true;
                if (++swaps > max_swaps) over = true;
                break;
            }
        }
        if (!moved) i++; // an accepted swap re-examines position i (the reference's i--)
    }
    if (over && lane == 0) set_status(a.status, ACO_ERR_LS_LIMIT);
    for (int p = lane; p < size; p += 32) gt[p] = tour[p];
    // compute_tour_length: fp32 sum of the edges in position order
    float len = 0.f;
    for (int b0 = 0; b0 < size - 1; b0 += 32) {
        const int p = b0 + lane;
        const float e = p < size - 1 ? D[(size_t)tour[p] * ldd + tour[p + 1]] : 0.f;
        const int m = size - 1 - b0 < 32 ? size - 1 - b0 : 32;
#pragma unroll
        for (int k = 0; k < 32; k++) {
            const float y = __shfl_sync(FULL, e, k);
            if (k < m) len = __fadd_rn(len, y);
        }
    }
    if (lane == 0) a.lens[ant] = len;
    (void)n;
}

__global__ void __launch_bounds__(512) swap_kernel(const ConstructArgs *args, const int2 *items, int apc,
                                                   int max_swaps_per_node)
{
    extern __shared__ __align__(16) unsigned char sm[];
    const int2 it = items[blockIdx.x];
    const ConstructArgs a = args[it.x];
    const int n = a.n, warp = threadIdx.x >> 5;
    const bool stage = swap_stage_matrix(n, a.ld, apc);
    const float *D = a.dist;
    int ldd = a.ld;
    size_t off = 0;
    if (stage) { // whole matrix, rows of n (only the first n columns are read)
        float *sd = reinterpret_cast<float *>(sm);
        for (int e = threadIdx.x; e < n * n; e += blockDim.x) sd[e] = a.dist[(size_t)(e / n) * a.ld + (e % n)];
        D = sd;
        ldd = n;
        off = ((size_t)n * n * 4 + 15) & ~(size_t)15;
        __syncthreads();
    }
    const int ant = it.y + warp;
    if (warp >= apc || ant >= a.n_ants) return;
    int *w = reinterpret_cast<int *>(sm + off + (size_t)warp * swap_warp_bytes(n));
    int *tour = w, *rpos = w + 2 * n, *rload = w + 4 * n;
    float *rdist = reinterpret_cast<float *>(w + 5 * n);
    const int limit = max_swaps_per_node * n;
    if (stage) swap_ant<true>(a, ant, D, ldd, tour, rpos, rload, rdist, limit);
    else swap_ant<false>(a, ant, D, ldd, tour, rpos, rload, rdist, limit);
}

} // namespace

size_t swap_smem(int n, int ld, int apc)
{
    return (swap_stage_matrix(n, ld, apc) ? (((size_t)n * n * 4 + 15) & ~(size_t)15) : 0) +
           (size_t)apc * swap_warp_bytes(n);
}

cudaError_t launch_swap(const ConstructArgs *d_args, const int2 *d_items, int n_items, int apc, size_t smem,
                        int max_swaps_per_node, cudaStream_t st)
{
    const cudaError_t e = cudaFuncSetAttribute(swap_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    swap_kernel<<<n_items, apc * 32, smem, st>>>(d_args, d_items, apc, max_swaps_per_node);
    return cudaGetLastError();
}

} // namespace aco
