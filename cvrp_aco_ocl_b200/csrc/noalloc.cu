// noalloc.cu -- aco_pheromone_update_noalloc: the pheromone update
// (evaporation, rank-based deposit, total_info) for callers that must not have
// this library allocate device memory.
//
// Who needs it: hosts whose own memory manager owns every byte of device memory
// and forbids libraries from calling cudaMalloc (fixed memory budgets, pooled
// allocators), and loops that cannot afford the device-wide synchronisation that
// cudaMalloc / cudaFree imply.  Such a caller passes its own device buffers for
// the inputs and outputs; the only other memory this entry point touches is the
// fixed scratch array below, which lives in the library image and is reserved on
// every GPU that loads the library until the process exits.
//
// Limits: n <= kMaxNodes (4096) nodes and ras_ranks <= kMaxRanks (8); larger
// problems are rejected with ACO_ERR_CAPACITY.  All calls share the one scratch
// array (it keeps the last call's contents; each call re-initialises what it
// reads), so calls that overlap on the GPU -- on different streams, or from
// different threads -- race and must be serialised by the caller.
//
// The elite tours come from the caller's buffers, so they are checked before
// any scratch write: an elite whose tour size lies outside [2, 2n-1] or that
// holds a node id outside [0, n) deposits nothing, and its elites_out entry
// reads ACO_ERR_INVALID instead of the ant id.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/cvrp_aco.h"
#include "aco_device.cuh"

namespace aco {
namespace {

constexpr int kMaxNodes = 4096;
constexpr int kMaxRanks = 8;

struct NoAllocScratch {
    int succ[kMaxRanks * kMaxNodes]; // successor of customer i in elite r's tour, -1 if none
    uint32_t depmask[kMaxNodes];     // bit r: elite r's tour goes depot -> i
    float d_tau[kMaxRanks];          // (ras_ranks - r) / length of elite r
    int elites[kMaxRanks];           // elite ant ids, [0] = best-so-far slot
};

// The scratch: 148 KB of device memory in the library image, no allocation.
static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// Device address of g_noalloc_scratch per device, looked up once per device and
// context: a context that is destroyed and created again (cudaDeviceReset) may
// load the module at another address, so the cached address is keyed on the
// context it was looked up in.
std::mutex g_scratch_mu;
NoAllocScratch *g_scratch_ptr[64] = {};
CUcontext g_scratch_ctx[64] = {};

__device__ __forceinline__ unsigned long long block_min_key(unsigned long long v, unsigned long long *red)
{
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    __syncthreads();
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    const int nw = (blockDim.x + 31) >> 5;
    v = (int)(threadIdx.x & 31) < nw ? red[threadIdx.x & 31] : ~0ull;
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

// Elites (kernel.cl:717-741) and the per-node deposit lists, written into the
// scratch.  One CTA.
__global__ void __launch_bounds__(1024) noalloc_deposit_list_kernel(NoAllocScratch *sc, int n, int n_ants,
                                                                     int ras_ranks, const int *solutions,
                                                                     const float *lens, int *elites_out)
{
    __shared__ unsigned long long red[32];
    __shared__ int s_knocked[kMaxRanks];
    const int A = n_ants, T = 2 * n, tid = threadIdx.x, bs = blockDim.x;
    if (tid == 0) sc->elites[0] = A;
    for (int r = 1; r < ras_ranks; r++) {
        unsigned long long m = ~0ull;
        for (int k = tid; k < A; k += bs) {
            bool out = false;
            for (int q = 1; q < r; q++) out = out || (s_knocked[q] == k);
            const float v = out ? __int_as_float(0x7f800000) : lens[k];
            const unsigned long long key = ((unsigned long long)__float_as_uint(v) << 32) | (unsigned)k;
            m = key < m ? key : m;
        }
        m = block_min_key(m, red);
        if (tid == 0) {
            const int target = (int)(m & 0xffffffffu);
            s_knocked[r] = target;
            sc->elites[r] = target;
        }
        __syncthreads();
    }
    for (int e = tid; e < ras_ranks * n; e += bs) sc->succ[e] = -1; // clear what the last call left
    for (int e = tid; e < n; e += bs) sc->depmask[e] = 0u;
    // Check every elite tour before it is read as indices: size in [2, T-1],
    // every node id in [0, n).  A failing elite deposits nothing (d_tau = 0 and
    // no list entries) and is reported as ACO_ERR_INVALID.
    __shared__ int s_bad[kMaxRanks];
    if (tid < ras_ranks) s_bad[tid] = 0;
    __syncthreads();
    for (int r = 0; r < ras_ranks; r++) {
        const int *tour = solutions + (size_t)T * sc->elites[r];
        const int size = tour[T - 1];
        if (size < 2 || size > T - 1) {
            if (tid == 0) s_bad[r] = 1;
            continue;
        }
        for (int k = tid; k < size; k += bs) {
            const int u = tour[k];
            if (u < 0 || u >= n) s_bad[r] = 1;
        }
    }
    __syncthreads();
    if (tid < ras_ranks) {
        const bool bad = s_bad[tid] != 0;
        sc->d_tau[tid] = bad ? 0.0f : __fdiv_rn((float)(ras_ranks - tid), lens[sc->elites[tid]]);
        if (elites_out) elites_out[tid] = bad ? ACO_ERR_INVALID : sc->elites[tid];
    }
    for (int r = 0; r < ras_ranks; r++) {
        if (s_bad[r]) continue;
        const int *tour = solutions + (size_t)T * sc->elites[r];
        const int size = tour[T - 1];
        for (int k = tid; k < size - 1; k += bs) {
            const int u = tour[k], v = tour[k + 1];
            if (u != 0) sc->succ[(size_t)r * n + u] = v;
            else atomicOr(&sc->depmask[v], 1u << r);
        }
    }
}

// Evaporation + deposit (elite order) + total_info, one element per thread, any
// row pitch; eta^beta is recomputed from the distance (kernel.cl:782-789).
__global__ void __launch_bounds__(256) noalloc_pass_kernel(const NoAllocScratch *sc, int n, int ld, int ras_ranks,
                                                            float evap, float alpha, int alpha_int, float beta,
                                                            int beta_int, float *tau, float *total,
                                                            const float *dist)
{
    const size_t count = (size_t)n * n;
    for (size_t g = blockIdx.x * (size_t)blockDim.x + threadIdx.x; g < count; g += (size_t)gridDim.x * blockDim.x) {
        const int i = (int)(g / (size_t)n), j = (int)(g - (size_t)i * n);
        const size_t off = (size_t)i * ld + j;
        float v = __fmul_rn(evap, tau[off]);
        if (i != 0) {
            for (int r = 0; r < ras_ranks; r++)
                if (sc->succ[(size_t)r * n + i] == j) v = __fadd_rn(v, sc->d_tau[r]);
        } else {
            const uint32_t m = sc->depmask[j];
            for (int r = 0; r < ras_ranks; r++)
                if ((m >> r) & 1u) v = __fadd_rn(v, sc->d_tau[r]);
        }
        const float eta = __fdiv_rn(1.0f, __fadd_rn(dist[off], 0.1f));
        tau[off] = v;
        total[off] = __fmul_rn(pow_rule(v, alpha, alpha_int), pow_rule(eta, beta, beta_int));
    }
}

int exp_int(float e)
{
    if (e >= 0.0f && e <= 8.0f && e == (float)(int)e) return (int)e;
    return -1;
}

// Set-up, once per device and context, with that device current: the device
// address of the scratch array (its host-side name is only a stand-in, not a
// device address).  The current context comes from the driver's
// cuCtxGetCurrent, reached through cudaGetDriverEntryPoint so the library
// needs no link against libcuda.
using CtxGetCurrentFn = CUresult (*)(CUcontext *);

CtxGetCurrentFn ctx_get_current()
{
    static CtxGetCurrentFn fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<CtxGetCurrentFn>(p);
    }();
    return fn;
}

int scratch_address(NoAllocScratch **out)
{
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return ACO_ERR_CUDA;
    const CtxGetCurrentFn get = ctx_get_current();
    CUcontext ctx = nullptr; // null until the runtime has made the device's primary context current
    if (!get || get(&ctx) != CUDA_SUCCESS) return ACO_ERR_CUDA;
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (ctx == nullptr || !g_scratch_ptr[dev] || g_scratch_ctx[dev] != ctx) {
        void *p = nullptr; // the lookup also initialises the primary context when needed
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || p == nullptr) return ACO_ERR_CUDA;
        if (ctx == nullptr && (get(&ctx) != CUDA_SUCCESS || ctx == nullptr)) return ACO_ERR_CUDA;
        g_scratch_ptr[dev] = static_cast<NoAllocScratch *>(p);
        g_scratch_ctx[dev] = ctx;
    }
    *out = g_scratch_ptr[dev];
    return ACO_OK;
}

} // namespace
} // namespace aco

extern "C" int aco_pheromone_update_noalloc(int n, int ld, int n_ants, int ras_ranks, float rho, float alpha,
                                            float beta, float *tau, float *total_info, const float *dist,
                                            const int *solutions, const float *lens, int *elites_out, void *stream)
{
    using namespace aco;
    if (n < 2 || ld < n || n_ants < 1 || ras_ranks < 1 || !tau || !total_info || !dist || !solutions || !lens)
        return ACO_ERR_INVALID;
    if (!(rho > 0.0f && rho <= 1.0f)) return ACO_ERR_INVALID;
    if (n > kMaxNodes || ras_ranks > kMaxRanks) return ACO_ERR_CAPACITY; // beyond the fixed scratch array
    NoAllocScratch *sc = nullptr;
    const int rc = scratch_address(&sc);
    if (rc != ACO_OK) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    noalloc_deposit_list_kernel<<<1, 1024, 0, st>>>(sc, n, n_ants, ras_ranks, solutions, lens, elites_out);
    if (cudaGetLastError() != cudaSuccess) return ACO_ERR_CUDA;
    const size_t count = (size_t)n * n;
    const int blocks = (int)((count + 255) / 256 < 2048 ? (count + 255) / 256 : 2048);
    noalloc_pass_kernel<<<blocks, 256, 0, st>>>(sc, n, ld, ras_ranks, 1.0f - rho, alpha, exp_int(alpha), beta,
                                                exp_int(beta), tau, total_info, dist);
    if (cudaGetLastError() != cudaSuccess) return ACO_ERR_CUDA;
    return ACO_OK;
}
