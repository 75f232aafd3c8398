// local_search.cu -- 2-opt of every route of every ant, first improvement in
// sequence order with don't-look bits: a restatement of local_search /
// two_opt_solution / two_opt_single_route (cvrp_ocl/gpu/kernel.cl:126-319, 500-539).
//
// Route-parallel.  two_opt_solution runs the routes of a tour one after the
// other, but they share no state except the depot's don't-look bit: customers,
// tour positions, edge lengths (dist_tour_wrk) and route membership all belong
// to exactly one route.  The depot's bit enters the first route cleared
// (kernel.cl:293-296) and leaves every route set: the improvement loop only ends
// after a pass without a move, and in that pass the depot -- always at the
// route's first position -- is either skipped with its bit set or examined
// without a move, which sets it (kernel.cl:232).  So route r starts with the
// depot bit = (r > 0), and the routes of a tour can run concurrently, each on
// one warp, with results identical to the sequential order.  (When a route stops
// at the pass budget the bit may still be clear; that error path reports
// ACO_ERR_LS_LIMIT and its tours are valid but not matched bit for bit.)
//
// One CTA per ant, W warps, routes dealt round-robin to the warps.  The tour,
// node positions, edge lengths, don't-look bytes and route ids live in shared
// memory; every distance a route's 2-opt reads joins two of its nodes (depot
// included), so each warp gathers its route's distance sub-matrix into a
// shared-memory tile once (routes longer than rmax read the L2-resident matrix).
// A node's neighbour scan takes 32 list entries per warp step and keeps the
// reference's order: the first entry that ends the scan (radius test fails,
// kernel.cl:197,229) or improves wins, found with ballot + find-first-set.
#include <cuda_runtime.h>

#include "aco_device.cuh"
#include "kernels.h"

namespace aco {

namespace {

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }

struct LsLayout {
    size_t tour, pos, li, rid, dlb, rstart, dt, tiles, rnodes, bytes;
};

__host__ __device__ inline LsLayout ls_layout(int n, int T, int rmax, int warps)
{
    LsLayout L;
    size_t o = 0;
    L.tour = o; o = al16(o + (size_t)T * 2);
    L.pos = o; o = al16(o + (size_t)n * 2);
    L.li = o; o = al16(o + (size_t)n * 2);
    L.rid = o; o = al16(o + (size_t)n * 2);
    L.dlb = o; o = al16(o + (size_t)n);
    L.rstart = o; o = al16(o + (size_t)(n + 1) * 2);
    L.dt = o; o = al16(o + (size_t)T * 4);
    L.tiles = o; o = al16(o + (size_t)warps * rmax * rmax * 4);
    L.rnodes = o; o = al16(o + (size_t)warps * rmax * 2);
    L.bytes = o;
    return L;
}

constexpr unsigned FULL = 0xffffffffu;

struct Route {
    uint16_t *tour, *pos, *li, *rid, *rnode;
    uint8_t *dlb;
    float *dt, *tile;
    const float *dist;
    const int *nn;
    int ld, nn_ls, lane, r, rb, re, R;
    bool tiled, dlb0; // dlb0: the depot's don't-look bit inside this route

    __device__ __forceinline__ float D(int a, int b) const
    {
        if (tiled) return tile[li[a] * R + li[b]];
        return __ldg(dist + (size_t)a * ld + b);
    }
    __device__ __forceinline__ int P(int v) const { return v == 0 ? rb : (int)pos[v]; } // tour_node_pos[0] = route_beg
    __device__ __forceinline__ bool in_route(int v) const { return v != 0 && rid[v] == r; }
    __device__ __forceinline__ bool dlb_get(int v) const { return v == 0 ? dlb0 : dlb[v] != 0; }
};

// kernel.cl:235-270 with all lanes.
__device__ __forceinline__ void apply_move(Route &c, int h1, int h2, int h3, int h4)
{
    if (h1 == 0 || h2 == 0 || h3 == 0 || h4 == 0) c.dlb0 = false;
    if (c.lane == 0) {
        if (h1) c.dlb[h1] = 0;
        if (h2) c.dlb[h2] = 0;
        if (h3) c.dlb[h3] = 0;
        if (h4) c.dlb[h4] = 0;
    }
    if (c.P(h3) < c.P(h1)) {
        int t = h1; h1 = h3; h3 = t;
        t = h2; h2 = h4; h4 = t;
    }
    const int i = c.P(h1), j = c.P(h3), a = c.P(h2);
    const float d13 = c.D(h1, h3), d24 = c.D(h2, h4);
    __syncwarp();
    if (c.lane == 0) {
        c.dt[i] = d13;
        c.dt[j] = d24;
    }
    const int L1 = j - i - 1; // dist_tour_wrk[i+1 .. j-1] reversed
    for (int k = c.lane; k < L1 / 2; k += 32) {
        const int x = i + 1 + k, y = j - 1 - k;
        const float tx = c.dt[x];
        c.dt[x] = c.dt[y];
        c.dt[y] = tx;
    }
    const int L2 = j - a + 1; // tour[pos[h2] .. pos[h3]] reversed
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

// two_opt_single_route (kernel.cl:126-277).
__device__ int two_opt_route(Route &c, int pass_limit)
{
    const int lane = c.lane, rb = c.rb, re = c.re;
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
                const int n2 = valid ? __ldg(c.nn + (size_t)n1 * c.nn_ls + h) : 0;
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
                    const int n2 = valid ? __ldg(c.nn + (size_t)n1 * c.nn_ls + h) : 0;
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
                if (n1 == 0) c.dlb0 = true;
                else if (lane == 0) c.dlb[n1] = 1;
                __syncwarp();
                continue;
            }
            imp = true;
            apply_move(c, h1, h2, h3, h4);
        }
    }
    return ACO_OK;
}

__global__ void __launch_bounds__(512) local_search_kernel(LocalSearchArgs a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int n = a.n, T = a.T;
    const int W = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const LsLayout L = ls_layout(n, T, a.rmax, W);
    uint16_t *tour = reinterpret_cast<uint16_t *>(smem + L.tour);
    uint16_t *pos = reinterpret_cast<uint16_t *>(smem + L.pos);
    uint16_t *li = reinterpret_cast<uint16_t *>(smem + L.li);
    uint16_t *rid = reinterpret_cast<uint16_t *>(smem + L.rid);
    uint8_t *dlb = reinterpret_cast<uint8_t *>(smem + L.dlb);
    uint16_t *rstart = reinterpret_cast<uint16_t *>(smem + L.rstart);
    float *dt = reinterpret_cast<float *>(smem + L.dt);
    __shared__ int s_routes;

    const int ant = blockIdx.x;
    int *gtour = a.solutions + (size_t)ant * T;
    const int size = gtour[T - 1];
    if (size < 2) return; // a failed construction has nothing to improve (uniform over the CTA)

    // local_search (kernel.cl:517-523) + two_opt_solution set-up (:293-300)
    for (int p = threadIdx.x; p < size; p += blockDim.x) {
        const int v = gtour[p];
        tour[p] = (uint16_t)v;
        if (v != 0) pos[v] = (uint16_t)p;
    }
    for (int v = threadIdx.x; v < n; v += blockDim.x) dlb[v] = 0;
    if (threadIdx.x == 0) li[0] = 0; // the depot is local node 0 of every route tile
    __syncthreads();
    for (int p = threadIdx.x; p < size - 1; p += blockDim.x)
        dt[p] = __ldg(a.dist + (size_t)tour[p] * a.ld + tour[p + 1]);
    // route table: positions of the depots, in order (warp 0 compacts with ballots)
    if (warp == 0) {
        int count = 0;
        for (int base = 0; base < size; base += 32) {
            const int p = base + lane;
            const bool dep = p < size && tour[p] == 0;
            const unsigned m = __ballot_sync(FULL, dep);
            if (dep) rstart[count + __popc(m & ((1u << lane) - 1u))] = (uint16_t)p;
            count += __popc(m);
        }
        if (lane == 0) s_routes = count - 1; // depots at both ends of each route
    }
    __syncthreads();
    const int routes = s_routes;
    for (int r = warp; r < routes; r += W) // route id of every customer
        for (int p = rstart[r] + 1 + lane; p < rstart[r + 1]; p += 32) rid[tour[p]] = (uint16_t)r;
    __syncthreads();

    Route c;
    c.tour = tour; c.pos = pos; c.li = li; c.rid = rid; c.dlb = dlb; c.dt = dt;
    c.tile = reinterpret_cast<float *>(smem + L.tiles) + (size_t)warp * a.rmax * a.rmax;
    c.rnode = reinterpret_cast<uint16_t *>(smem + L.rnodes) + (size_t)warp * a.rmax;
    c.dist = a.dist; c.nn = a.nn_list; c.ld = a.ld; c.nn_ls = a.nn_ls; c.lane = lane;
    int status = ACO_OK;
    for (int r = warp; r < routes; r += W) {
        c.r = r;
        c.rb = rstart[r];
        c.re = rstart[r + 1] - 1;
        c.R = c.re - c.rb + 1;
        c.dlb0 = r > 0;
        c.tiled = c.R <= a.rmax;
        if (c.tiled) {
            for (int k = lane; k < c.R; k += 32) {
                const int v = tour[c.rb + k];
                if (v != 0) li[v] = (uint16_t)k;
                c.rnode[k] = (uint16_t)v;
            }
            __syncwarp();
            for (int e = lane; e < c.R * c.R; e += 32) {
                const int k1 = e / c.R, k2 = e - (e / c.R) * c.R;
                c.tile[e] = __ldg(a.dist + (size_t)c.rnode[k1] * a.ld + c.rnode[k2]);
            }
            __syncwarp();
        }
        const int st = two_opt_route(c, a.pass_limit);
        if (st != ACO_OK && status == ACO_OK) status = st;
    }
    if (status != ACO_OK && lane == 0) set_status(a.status, status);
    __syncthreads();

    for (int p = threadIdx.x; p < size; p += blockDim.x) gtour[p] = tour[p]; // kernel.cl:530-532
    if (threadIdx.x == 0) {                                                  // kernel.cl:534-538
        float len = 0.f;
        for (int p = 0; p < size - 1; p++) len = __fadd_rn(len, dt[p]);
        a.lens[ant] = len;
    }
}

} // namespace

size_t local_search_smem(int n, int /*nn_ls*/, int rmax, int warps, bool /*stage_nn*/)
{
    return ls_layout(n, 2 * n, rmax, warps).bytes;
}

cudaError_t launch_local_search(const LocalSearchArgs &a, int warps, bool /*stage_nn*/, cudaStream_t st)
{
    const size_t bytes = ls_layout(a.n, a.T, a.rmax, warps).bytes;
    cudaError_t e = cudaFuncSetAttribute(local_search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    local_search_kernel<<<a.n_ants, warps * 32, bytes, st>>>(a);
    return cudaGetLastError();
}

} // namespace aco
