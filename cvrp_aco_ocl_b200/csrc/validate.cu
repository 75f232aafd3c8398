// validate.cu -- every tour of a colony checked on the device, so a batch of
// many instances can be validated without copying its tours to the host.
//
// The check is check_solution / check_route (problem.cpp:226-319) as the
// host's check_solution states it: the tour starts at the depot; every
// customer appears exactly once; every route between two depot visits has at
// least one customer, a load within capacity and a length (fp32 sum of its
// edges in order, plus service time per customer) within max_distance.  Two
// checks are added: node ids are in range, and the stored length equals the
// fp32 sum of the tour's edges in order (compute_tour_length,
// vrpHelper.cpp:244-253) bit for bit.
//
// One warp per tour slot (the ants and the best-so-far slot of every
// instance).  The lanes mark the visited set in shared memory with atomics
// (a set bit found set again is a repeat); lane 0 walks the tour once for the
// route loads and lengths, the order of the fp32 sums fixing it to one lane.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/cvrp_aco.h"
#include "kernels.h"

namespace aco {
namespace {

constexpr int kWarps = 4;

__global__ void __launch_bounds__(kWarps * 32) validate_kernel(const ConstructArgs *args, int *flags,
                                                                const int *slot_base, int *invalid)
{
    extern __shared__ uint32_t bits_all[];
    const int b = blockIdx.y;
    const ConstructArgs a = args[b];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int s = blockIdx.x * kWarps + warp; // slot: ants 0..A-1, best-so-far A
    if (s > a.n_ants) return;
    const int n = a.n, T = a.T, words = (n + 31) >> 5;
    uint32_t *bits = bits_all + (size_t)warp * words;
    const int *tour = a.solutions + (size_t)s * T;
    const int size = tour[T - 1];
    bool ok = size >= 2 && size <= T - 1 && tour[0] == 0;
    for (int w = lane; w < words; w += 32) bits[w] = w == 0 ? 1u : 0u; // the depot counts as used
    __syncwarp();
    if (ok) {
        bool bad = false;
        for (int p = 1 + lane; p < size; p += 32) {
            const int c = tour[p];
            if (c < 0 || c >= n) {
                bad = true;
            } else if (c != 0) {
                const uint32_t bit = 1u << (c & 31);
                if (atomicOr(&bits[c >> 5], bit) & bit) bad = true;
            }
        }
        ok = !__any_sync(0xffffffffu, bad);
        __syncwarp();
        bool all = true;
        for (int w = lane; w < words; w += 32) {
            const uint32_t want = w == words - 1 && (n & 31) ? (1u << (n & 31)) - 1u : 0xffffffffu;
            if (bits[w] != want) all = false;
        }
        ok = ok && __all_sync(0xffffffffu, all);
    }
    if (ok && lane == 0) {
        int rbeg = 0, load = 0;
        float rlen = 0.f, tlen = 0.f;
        for (int p = 1; p < size && ok; p++) {
            const int prev = tour[p - 1], c = tour[p];
            const float e = a.dist[(size_t)prev * a.ld + c];
            rlen = __fadd_rn(rlen, e);
            tlen = __fadd_rn(tlen, e);
            if (c != 0) {
                load += a.demand[c];
                continue;
            }
            // route [rbeg, p] (check_route, problem.cpp:291-319)
            const float d = __fadd_rn(rlen, __fmul_rn(a.serv_time, (float)(p - rbeg - 1)));
            if (p - rbeg < 2 || load > a.capacity || d > a.max_dist) ok = false;
            rbeg = p;
            load = 0;
            rlen = 0.f;
        }
        if (ok && __float_as_uint(tlen) != __float_as_uint(a.lens[s])) ok = false;
    }
    ok = __shfl_sync(0xffffffffu, ok, 0);
    if (lane == 0) {
        flags[slot_base[b] + s] = ok ? 1 : 0;
        if (!ok) atomicAdd(&invalid[b], 1);
    }
}

// The best-so-far slot of every instance packed into one buffer: instance b's
// tour (2n ints, the reference layout of slot A) at tour_base[b], its size and
// length at [b].  One CTA per instance.
__global__ void __launch_bounds__(256) gather_best_kernel(const ConstructArgs *args, const int *tour_base,
                                                          int *tours, int *sizes, float *lens)
{
    const int b = blockIdx.x;
    const ConstructArgs &a = args[b];
    const int T = a.T, A = a.n_ants;
    const int *src = a.solutions + (size_t)A * T;
    int *dst = tours + tour_base[b];
    for (int p = threadIdx.x; p < T; p += blockDim.x) dst[p] = src[p];
    if (threadIdx.x == 0) {
        sizes[b] = src[T - 1];
        lens[b] = a.lens[A];
    }
}

} // namespace

cudaError_t launch_gather_best(const ConstructArgs *d_args, int n_inst, const int *d_tour_base, int *tours,
                               int *sizes, float *lens, cudaStream_t st)
{
    gather_best_kernel<<<n_inst, 256, 0, st>>>(d_args, d_tour_base, tours, sizes, lens);
    return cudaGetLastError();
}

cudaError_t launch_validate(const ConstructArgs *d_args, int n_inst, int max_slots, int max_n, int *flags,
                            const int *slot_base, int *invalid, cudaStream_t st)
{
    const size_t smem = (size_t)kWarps * ((max_n + 31) / 32) * 4;
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(validate_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                   (int)smem);
        if (e != cudaSuccess) return e;
    }
    const dim3 grid((max_slots + kWarps - 1) / kWarps, n_inst);
    validate_kernel<<<grid, kWarps * 32, smem, st>>>(d_args, flags, slot_base, invalid);
    return cudaGetLastError();
}

} // namespace aco
