// local_search.cu -- 2-opt of every route of every ant, first improvement in
// sequence order with don't-look bits: a warp-cooperative restatement of
// local_search / two_opt_solution / two_opt_single_route
// (cvrp_ocl/gpu/kernel.cl:126-319, 500-539).
//
// One warp per ant.  The ant's tour, node positions, edge lengths
// (dist_tour_wrk) and don't-look / route-membership bits live in shared memory.
// Every distance a route's 2-opt reads joins two nodes of that route (the depot
// included), so the route's distance sub-matrix is gathered once into a
// shared-memory tile (routes longer than rmax read the L2-resident matrix).
// The neighbour scan of one node takes 32 list entries per warp step and keeps
// the reference's first-improvement order: the first entry (in list order) that
// either ends the scan (radius test fails, kernel.cl:197,229) or improves wins,
// found with ballot + find-first-set.  Moves are applied by all lanes at once.
#include <cuda_runtime.h>

#include "aco_device.cuh"
#include "kernels.h"

namespace aco {

namespace {

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }

struct WarpLayout {
    size_t tour, pos, li, rnode, dlb, map, dt, tile, bytes;
};

__host__ __device__ inline WarpLayout warp_layout(int n, int T, int rmax)
{
    const size_t words = (size_t)((n + 31) / 32);
    WarpLayout L;
    size_t o = 0;
    L.tour = o; o = al16(o + (size_t)T * 2);
    L.pos = o; o = al16(o + (size_t)n * 2);
    L.li = o; o = al16(o + (size_t)n * 2);
    L.rnode = o; o = al16(o + (size_t)rmax * 2);
    L.dlb = o; o = al16(o + words * 4);
    L.map = o; o = al16(o + words * 4);
    L.dt = o; o = al16(o + (size_t)T * 4);
    L.tile = o; o = al16(o + (size_t)rmax * rmax * 4);
    L.bytes = o;
    return L;
}

__host__ __device__ inline size_t ls_total_smem(int n, int T, int nn_ls, int rmax, int apc, bool snn)
{
    size_t head = snn ? al16((size_t)n * nn_ls * 2) : 0;
    return head + (size_t)apc * warp_layout(n, T, rmax).bytes;
}

struct Ctx {
    uint16_t *tour, *pos, *li, *rnode;
    uint32_t *dlb, *map;
    float *dt, *tile;
    const float *dist;
    const int *nn_g;
    const uint16_t *nn_s;
    int ld, nn_ls, R, lane;
    bool tiled;

    __device__ __forceinline__ float D(int a, int b) const
    {
        if (tiled) return tile[li[a] * R + li[b]];
        return __ldg(dist + (size_t)a * ld + b);
    }
    __device__ __forceinline__ int NN(int a, int h) const
    {
        return nn_s ? (int)nn_s[(size_t)a * nn_ls + h] : __ldg(nn_g + (size_t)a * nn_ls + h);
    }
    __device__ __forceinline__ bool in_route(int v) const { return (map[v >> 5] >> (v & 31)) & 1u; }
    __device__ __forceinline__ bool dlb_get(int v) const { return (dlb[v >> 5] >> (v & 31)) & 1u; }
};

constexpr unsigned FULL = 0xffffffffu;

// Apply the exchange (kernel.cl:235-270) with all lanes.
__device__ __forceinline__ void apply_move(Ctx &c, int h1, int h2, int h3, int h4)
{
    if (c.lane == 0) {
        c.dlb[h1 >> 5] &= ~(1u << (h1 & 31));
        c.dlb[h2 >> 5] &= ~(1u << (h2 & 31));
        c.dlb[h3 >> 5] &= ~(1u << (h3 & 31));
        c.dlb[h4 >> 5] &= ~(1u << (h4 & 31));
    }
    if (c.pos[h3] < c.pos[h1]) {
        int t = h1; h1 = h3; h3 = t;
        t = h2; h2 = h4; h4 = t;
    }
    const int i = c.pos[h1], j = c.pos[h3];
    const int a = c.pos[h2];
    const float d13 = c.D(h1, h3), d24 = c.D(h2, h4);
    __syncwarp();
    if (c.lane == 0) {
        c.dt[i] = d13;
        c.dt[j] = d24;
    }
    const int L1 = j - i - 1; // reverse dist_tour_wrk[i+1 .. j-1]
    for (int k = c.lane; k < L1 / 2; k += 32) {
        const int x = i + 1 + k, y = j - 1 - k;
        const float tx = c.dt[x];
        c.dt[x] = c.dt[y];
        c.dt[y] = tx;
    }
    const int L2 = j - a + 1; // reverse tour[pos[h2] .. pos[h3]]
    for (int k = c.lane; k < L2 / 2; k += 32) {
        const int x = a + k, y = j - k;
        const uint16_t tx = c.tour[x], ty = c.tour[y];
        c.tour[x] = ty;
        c.tour[y] = tx;
        c.pos[ty] = (uint16_t)x;
        c.pos[tx] = (uint16_t)y;
    }
    __syncwarp();
}

// two_opt_single_route (kernel.cl:126-277) for the route at positions [rb, re].
__device__ int two_opt_route(Ctx &c, int rb, int re, int pass_limit)
{
    const int lane = c.lane;
    const int nr = re - rb + 1;
    int passes = 0;
    bool imp = true;
    while (imp) {
        if (pass_limit > 0 && passes >= pass_limit) return ACO_ERR_LS_LIMIT;
        passes++;
        imp = false;
        for (int l = 0; l < nr; l++) {
            const int pos1 = rb + l;
            const int n1 = c.tour[pos1];
            if (c.dlb_get(n1)) continue;
            const int s1 = pos1 == re ? c.tour[rb] : c.tour[pos1 + 1];
            float radius = c.D(n1, s1);
            bool found = false;
            int h1 = 0, h2 = 0, h3 = 0, h4 = 0;
            // successor search (kernel.cl:180-198)
            for (int h0 = 0; h0 < c.nn_ls; h0 += 32) {
                const int h = h0 + lane;
                const bool valid = h < c.nn_ls;
                const int n2 = valid ? c.NN(n1, h) : 0;
                const bool inr = valid && c.in_route(n2);
                bool cond = false, okm = false;
                int s2 = 0;
                if (inr) {
                    const float d12 = c.D(n1, n2);
                    cond = __fsub_rn(radius, d12) > kEps;
                    if (cond) {
                        const int p2 = c.pos[n2];
                        s2 = p2 == re ? c.tour[rb] : c.tour[p2 + 1];
                        const float g = __fsub_rn(__fadd_rn(__fadd_rn(-radius, d12), c.D(s1, s2)), c.dt[p2]);
                        okm = g < -kEps;
                    }
                }
                const unsigned stop = __ballot_sync(FULL, inr && (!cond || okm));
                if (stop) {
                    const int f = __ffs(stop) - 1;
                    if (__shfl_sync(FULL, (int)cond, f)) {
                        found = true;
                        h1 = n1;
                        h2 = s1;
                        h3 = __shfl_sync(FULL, n2, f);
                        h4 = __shfl_sync(FULL, s2, f);
                    }
                    break;
                }
            }
            if (!found) { // predecessor search (kernel.cl:202-230)
                const int p1 = pos1 == rb ? c.tour[re] : c.tour[pos1 - 1];
                radius = c.D(p1, n1);
                for (int h0 = 0; h0 < c.nn_ls; h0 += 32) {
                    const int h = h0 + lane;
                    const bool valid = h < c.nn_ls;
                    const int n2 = valid ? c.NN(n1, h) : 0;
                    const bool inr = valid && c.in_route(n2);
                    bool cond = false, okm = false;
                    int pp2 = 0;
                    if (inr) {
                        const float d12 = c.D(n1, n2);
                        cond = __fsub_rn(radius, d12) > kEps;
                        if (cond) {
                            const int p2 = c.pos[n2];
                            pp2 = p2 == rb ? c.tour[re] : c.tour[p2 - 1];
                            if (!(pp2 == n1 || p1 == n2)) {
                                const float g =
                                    __fsub_rn(__fadd_rn(__fadd_rn(-radius, d12), c.D(p1, pp2)), c.dt[p2 - 1]);
                                okm = g < -kEps;
                            }
                        }
                    }
                    const unsigned stop = __ballot_sync(FULL, inr && (!cond || okm));
                    if (stop) {
                        const int f = __ffs(stop) - 1;
                        if (__shfl_sync(FULL, (int)cond, f)) {
                            found = true;
                            h1 = p1;
                            h2 = n1;
                            h3 = __shfl_sync(FULL, pp2, f);
                            h4 = __shfl_sync(FULL, n2, f);
                        }
                        break;
                    }
                }
            }
            if (!found) { // dlb[n1] = TRUE (kernel.cl:232)
                if (lane == 0) c.dlb[n1 >> 5] |= 1u << (n1 & 31);
                __syncwarp();
                continue;
            }
            imp = true;
            apply_move(c, h1, h2, h3, h4);
        }
    }
    return ACO_OK;
}

template <bool SNN>
__global__ void __launch_bounds__(512) local_search_kernel(LocalSearchArgs a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int n = a.n, T = a.T;
    const int apc = blockDim.x >> 5;
    const int slot = threadIdx.x >> 5, lane = threadIdx.x & 31;
    uint16_t *s_nn = reinterpret_cast<uint16_t *>(smem);
    const size_t head = SNN ? al16((size_t)n * a.nn_ls * 2) : 0;
    if (SNN) {
        for (int e = threadIdx.x; e < n * a.nn_ls; e += blockDim.x) s_nn[e] = (uint16_t)__ldg(a.nn_list + e);
        __syncthreads();
    }
    const WarpLayout W = warp_layout(n, T, a.rmax);
    unsigned char *ws = smem + head + (size_t)slot * W.bytes;
    Ctx c;
    c.tour = reinterpret_cast<uint16_t *>(ws + W.tour);
    c.pos = reinterpret_cast<uint16_t *>(ws + W.pos);
    c.li = reinterpret_cast<uint16_t *>(ws + W.li);
    c.rnode = reinterpret_cast<uint16_t *>(ws + W.rnode);
    c.dlb = reinterpret_cast<uint32_t *>(ws + W.dlb);
    c.map = reinterpret_cast<uint32_t *>(ws + W.map);
    c.dt = reinterpret_cast<float *>(ws + W.dt);
    c.tile = reinterpret_cast<float *>(ws + W.tile);
    c.dist = a.dist;
    c.nn_g = a.nn_list;
    c.nn_s = SNN ? s_nn : nullptr;
    c.ld = a.ld;
    c.nn_ls = a.nn_ls;
    c.lane = lane;
    c.R = 0;
    c.tiled = false;

    const int ant = blockIdx.x * apc + slot;
    if (ant >= a.n_ants) return;
    int *gtour = a.solutions + (size_t)ant * T;
    const int size = gtour[T - 1];
    if (size < 2) return; // a failed construction has nothing to improve

    // local_search (kernel.cl:517-523) + two_opt_solution set-up (:293-300)
    const int words = (n + 31) >> 5;
    for (int w = lane; w < words; w += 32) {
        c.dlb[w] = 0u;
        c.map[w] = 0u;
    }
    for (int p = lane; p < size; p += 32) {
        const int v = gtour[p];
        c.tour[p] = (uint16_t)v;
        if (v != 0) c.pos[v] = (uint16_t)p;
    }
    __syncwarp();
    for (int p = lane; p < size - 1; p += 32)
        c.dt[p] = __ldg(a.dist + (size_t)c.tour[p] * a.ld + c.tour[p + 1]);
    __syncwarp();

    // routes in tour order (kernel.cl:302-318)
    int status = ACO_OK;
    int rb = 0;
    for (int base = 1; base < size; base += 32) {
        const int p = base + lane;
        unsigned dep = __ballot_sync(FULL, p < size && c.tour[p] == 0);
        while (dep) {
            const int i = base + __ffs(dep) - 1;
            dep &= dep - 1;
            const int re = i - 1;
            for (int q = rb + 1 + lane; q <= re; q += 32) {
                const int v = c.tour[q];
                atomicOr(&c.map[v >> 5], 1u << (v & 31));
            }
            if (lane == 0) c.pos[0] = (uint16_t)rb;
            const int R = re - rb + 1;
            c.R = R;
            c.tiled = R <= a.rmax;
            if (c.tiled) {
                for (int k = lane; k < R; k += 32) {
                    const int v = c.tour[rb + k];
                    c.li[v] = (uint16_t)k;
                    c.rnode[k] = (uint16_t)v;
                }
                __syncwarp();
                for (int e = lane; e < R * R; e += 32) {
                    const int k1 = e / R, k2 = e - (e / R) * R;
                    c.tile[e] = __ldg(a.dist + (size_t)c.rnode[k1] * a.ld + c.rnode[k2]);
                }
            }
            __syncwarp();
            const int st = two_opt_route(c, rb, re, a.pass_limit);
            if (st != ACO_OK && status == ACO_OK) status = st;
            for (int q = rb + 1 + lane; q <= re; q += 32) {
                const int v = c.tour[q];
                atomicAnd(&c.map[v >> 5], ~(1u << (v & 31)));
            }
            __syncwarp();
            rb = i;
        }
    }

    for (int p = lane; p < size; p += 32) gtour[p] = c.tour[p]; // kernel.cl:530-532
    if (lane == 0) {                                             // kernel.cl:534-538
        float len = 0.f;
        for (int p = 0; p < size - 1; p++) len = __fadd_rn(len, c.dt[p]);
        a.lens[ant] = len;
        if (status != ACO_OK) set_status(a.status, status);
    }
}

template <bool SNN>
cudaError_t launch_ls_t(const LocalSearchArgs &a, int apc, cudaStream_t st)
{
    const size_t bytes = ls_total_smem(a.n, a.T, a.nn_ls, a.rmax, apc, SNN);
    auto kern = local_search_kernel<SNN>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    const int blocks = (a.n_ants + apc - 1) / apc;
    kern<<<blocks, apc * 32, bytes, st>>>(a);
    return cudaGetLastError();
}

} // namespace

size_t local_search_smem(int n, int nn_ls, int rmax, int apc, bool snn)
{
    return ls_total_smem(n, 2 * n, nn_ls, rmax, apc, snn);
}

cudaError_t launch_local_search(const LocalSearchArgs &a, int apc, bool snn, cudaStream_t st)
{
    return snn ? launch_ls_t<true>(a, apc, st) : launch_ls_t<false>(a, apc, st);
}

} // namespace aco
