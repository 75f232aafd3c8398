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
// depot bit = (r > 0), and the routes of a tour can run concurrently with
// results identical to the sequential order.  (When a route stops at the pass
// budget the bit may still be clear; that error path reports ACO_ERR_LS_LIMIT
// and its tours are valid but not matched bit for bit.)
//
// local_search_kernel: CTAs of 1-8 ants whose warps pull the routes of all of
// them from a shared counter, longest first; route_opt_kernel: a persistent
// grid over the construct's list of every ant's routes (see below).  A route of
// at most 32 nodes (depot included) runs entirely in one warp's registers: lane q
// holds the local node at route position q, its edge length, and the position
// of local node q; the don't-look bits are one warp-uniform mask; the route's
// distance sub-matrix is a 32x32 shared tile; and every node's neighbour list
// is pre-filtered to the neighbours inside the route, in list order.  The scan
// of kernel.cl:180-230 only ever stops on an in-route entry (others `continue`),
// so the filtered list visits exactly the entries that decide the outcome: the
// first that ends the scan (radius test fails) or improves, found with ballot +
// find-first-set.  A move reverses a position range with shuffles.  Longer
// routes take the generic path over shared-memory arrays and the L2-resident
// distance matrix.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>

#include "aco_device.cuh"
#include "kernels.h"
#include "two_opt.cuh"

namespace aco {

namespace {

__host__ __device__ inline size_t al16(size_t x) { return (x + 15) & ~(size_t)15; }


// Shared memory: one block per ant of the CTA (sized for the colony's largest
// instance), then one block per warp.
struct LsAnt {
    size_t tour, pos, li, rid, dlb, rstart, dt, bytes;
};

__host__ __device__ inline LsAnt ls_ant_layout(int n)
{
    const int T = 2 * n;
    LsAnt L;
    size_t o = 0;
    L.tour = o; o = al16(o + (size_t)T * 2);
    L.pos = o; o = al16(o + (size_t)n * 2);
    L.li = o; o = al16(o + (size_t)n);
    L.rid = o; o = al16(o + (size_t)n * 2);
    L.dlb = o; o = al16(o + (size_t)n);
    L.rstart = o; o = al16(o + (size_t)(n + 1) * 2);
    L.dt = o; o = al16(o + (size_t)T * 4);
    L.bytes = o;
    return L;
}

// per warp: distance tile, in-route neighbour lists (local indices), list counts
constexpr size_t kLsWarp = kRL * kRL * 4 + kRL * kRL + kRL;
constexpr int kLsRows = 8; // tile rows loaded per round
constexpr int kMaxLsAnts = 8;
constexpr int kLsOrder = 128; // routes of a CTA ordered longest first when at most this many
constexpr unsigned FULL = 0xffffffffu;

__host__ __device__ inline size_t ls_smem_bytes(int n_max, int apc, int warps)
{
    return (size_t)apc * ls_ant_layout(n_max).bytes + (size_t)warps * kLsWarp;
}

// ---------------------------------------------------------------------------
// Generic path: any route length, shared-memory arrays, global distances.
// ---------------------------------------------------------------------------
struct Route {
    uint16_t *tour, *pos, *rid;
    uint8_t *dlb;
    float *dt;
    const float *dist;
    const int *nn;
    int ld, nn_ls, lane, r, rb, re;
    bool dlb0; // the depot's don't-look bit inside this route

    __device__ __forceinline__ float D(int a, int b) const { return __ldg(dist + (size_t)a * ld + b); }
    __device__ __forceinline__ int P(int v) const { return v == 0 ? rb : (int)pos[v]; } // tour_node_pos[0] = route_beg
    __device__ __forceinline__ bool in_route(int v) const { return v != 0 && rid[v] == r; }
    __device__ __forceinline__ bool dlb_get(int v) const { return v == 0 ? dlb0 : dlb[v] != 0; }
};

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
    const int L1 = j - i - 1;
    for (int k = c.lane; k < L1 / 2; k += 32) {
        const int x = i + 1 + k, y = j - 1 - k;
        const float tx = c.dt[x];
        c.dt[x] = c.dt[y];
        c.dt[y] = tx;
    }
    const int L2 = j - a + 1;
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

__device__ int two_opt_route_generic(Route &c, int pass_limit)
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
            if (c.nn_ls <= 32) {
                // one list of at most 32 entries: both searches from one load of it, the
                // predecessor's result used only when the successor search finds no move
                const int p1 = pos1 == rb ? c.tour[re] : c.tour[pos1 - 1];
                const float rp = c.D(p1, n1);
                const bool valid = lane < c.nn_ls;
                const int n2 = valid ? __ldg(c.nn + (size_t)n1 * c.nn_ls + lane) : 0;
                const bool inr = valid && c.in_route(n2);
                bool sc = false, sok = false, pc = false, pok = false;
                int s2 = 0, pp2 = 0;
                if (inr) {
                    const float d12 = c.D(n1, n2);
                    sc = __fsub_rn(radius, d12) > kEps;
                    pc = __fsub_rn(rp, d12) > kEps;
                    const int p2 = c.pos[n2];
                    if (sc) {
                        s2 = p2 == re ? c.tour[rb] : c.tour[p2 + 1];
                        const float g = __fsub_rn(__fadd_rn(__fadd_rn(-radius, d12), c.D(s1, s2)), c.dt[p2]);
                        sok = g < -kEps;
                    }
                    if (pc) {
                        pp2 = p2 == rb ? c.tour[re] : c.tour[p2 - 1];
                        if (!(pp2 == n1 || p1 == n2)) {
                            const float g = __fsub_rn(__fadd_rn(__fadd_rn(-rp, d12), c.D(p1, pp2)), c.dt[p2 - 1]);
                            pok = g < -kEps;
                        }
                    }
                }
                const unsigned sstop = __ballot_sync(FULL, inr && (!sc || sok));
                const unsigned pstop = __ballot_sync(FULL, inr && (!pc || pok));
                if (sstop) { // successor search
                    const int f = __ffs(sstop) - 1;
                    if (__shfl_sync(FULL, (int)sc, f)) {
                        found = true;
                        h1 = n1;
                        h2 = s1;
                        h3 = __shfl_sync(FULL, n2, f);
                        h4 = __shfl_sync(FULL, s2, f);
                    }
                }
                if (!found && pstop) { // predecessor search
                    const int f = __ffs(pstop) - 1;
                    if (__shfl_sync(FULL, (int)pc, f)) {
                        found = true;
                        h1 = p1;
                        h2 = n1;
                        h3 = __shfl_sync(FULL, pp2, f);
                        h4 = __shfl_sync(FULL, n2, f);
                    }
                }
            } else {
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
                if (!found) {
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
            }
            if (!found) {
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

// Grid mode (list == null): CTA b improves the global ants [b * apc, b * apc +
// apc).  List mode: a persistent grid takes groups of apc ants from the list
// the construct kernel wrote (the ants flagged in `only`, list_ctr[0] of them),
// so the CTAs see only those ants; the last CTA rewinds the list.
__global__ void __launch_bounds__(1024) local_search_kernel(const LocalSearchArgs *args, const int *ant_inst,
                                                             const int *ant_base, const uint8_t *only, int apc,
                                                             int n_max, int total_ants, const int *list,
                                                             int *list_ctr)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_inst[kMaxLsAnts], s_ant[kMaxLsAnts], s_size[kMaxLsAnts], s_routes[kMaxLsAnts + 1];
    __shared__ int s_only[kMaxLsAnts]; // 1: the short routes of this ant are done already
    __shared__ uint16_t s_order[kLsOrder], s_rlen[kLsOrder]; // routes, longest first
    __shared__ int s_next;
    const int W = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const LsAnt AL = ls_ant_layout(n_max);
    unsigned char *wbase = smem + (size_t)apc * AL.bytes + (size_t)warp * kLsWarp;
    float *tile = reinterpret_cast<float *>(wbase);
    uint8_t *lnn = wbase + kRL * kRL * 4;
    uint8_t *lcnt = lnn + kRL * kRL;
    auto ant_ptr = [&](int j, size_t off) { return smem + (size_t)j * AL.bytes + off; };
    __shared__ int s_group;
    const int listed = list ? min(list_ctr[0], total_ants) : 0;
    for (int grp = blockIdx.x;;) {
    if (list) {
        __syncthreads(); // the previous group is done with shared memory
        if (threadIdx.x == 0) s_group = atomicAdd(list_ctr + 1, 1);
        __syncthreads();
        grp = s_group;
        if (grp * apc >= listed) break;
    }

    // the CTA's ants: global ants [grp * apc, ... + apc), or entries of the list
    if (threadIdx.x < apc) {
        const int j = threadIdx.x;
        const int g = list ? (grp * apc + j < listed ? __ldg(list + grp * apc + j) : total_ants) : grp * apc + j;
        int inst = -1, ant = 0, size = 0;
        if (g < total_ants && (!only || only[g])) { // `only`: the ants a fused construct left to this kernel
            inst = __ldg(ant_inst + g);
            ant = g - __ldg(ant_base + inst);
            const LocalSearchArgs &a = args[inst];
            size = a.solutions[(size_t)ant * a.T + a.T - 1];
            if (size < 2) inst = -1; // a failed construction has nothing to improve
        }
        s_inst[j] = inst;
        s_ant[j] = ant;
        s_only[j] = only && g < total_ants ? only[g] : 0;
        s_size[j] = inst >= 0 ? size : 0;
    }
    __syncthreads();

    // local_search (kernel.cl:517-523) + two_opt_solution set-up (:293-300): the
    // tours are staged by the whole CTA, then warp j makes one pass over ant j's:
    // node positions, depot positions (route table) and every customer's route id
    // and index inside its route, from one ballot per 32 positions.  Edge lengths
    // (dist_tour_wrk) are filled per route: by the register path from its tile,
    // by the others from the matrix.
    for (int j = 0; j < apc; j++) {
        if (s_inst[j] < 0) continue;
        const LocalSearchArgs &a = args[s_inst[j]];
        const int *gtour = a.solutions + (size_t)s_ant[j] * a.T;
        uint16_t *tour = reinterpret_cast<uint16_t *>(ant_ptr(j, AL.tour));
        uint8_t *dlb = ant_ptr(j, AL.dlb);
        for (int p = threadIdx.x; p < s_size[j]; p += blockDim.x) tour[p] = (uint16_t)gtour[p];
        for (int v = threadIdx.x; v < a.n; v += blockDim.x) dlb[v] = 0;
    }
    __syncthreads();
    if (warp < apc) {
        const int j = warp;
        int count = 0;
        if (s_inst[j] >= 0) {
            const uint16_t *tour = reinterpret_cast<const uint16_t *>(ant_ptr(j, AL.tour));
            uint16_t *pos = reinterpret_cast<uint16_t *>(ant_ptr(j, AL.pos));
            uint16_t *rstart = reinterpret_cast<uint16_t *>(ant_ptr(j, AL.rstart));
            uint16_t *rid = reinterpret_cast<uint16_t *>(ant_ptr(j, AL.rid));
            uint8_t *li = ant_ptr(j, AL.li);
            const int size = s_size[j];
            int last = 0; // position of the last depot before this chunk
            for (int base = 0; base < size; base += 32) {
                const int p = base + lane;
                const int v = p < size ? (int)tour[p] : -1;
                const bool dep = v == 0;
                const unsigned m = __ballot_sync(FULL, dep);
                const unsigned lt = m & ((1u << lane) - 1u);
                if (p < size) {
                    if (dep) {
                        rstart[count + __popc(lt)] = (uint16_t)p;
                    } else {
                        const int r = count + __popc(lt) - 1;     // depots before p, less the first
                        const int rb = lt ? base + 31 - __clz(lt) : last; // the depot opening p's route
                        pos[v] = (uint16_t)p;
                        rid[v] = (uint16_t)r;
                        li[v] = (uint8_t)(p - rb < 256 ? p - rb : 0);
                    }
                }
                count += __popc(m);
                if (m) last = base + 31 - __clz(m);
            }
            count -= 1;
        }
        if (lane == 0) s_routes[j] = count;
    }
    __syncthreads();
    if (threadIdx.x == 0) { // routes of ant j are flattened after those of ants < j
        int acc = 0;
        for (int j = 0; j < apc; j++) {
            const int c = s_routes[j];
            s_routes[j] = acc;
            acc += c;
        }
        s_routes[apc] = acc;
        s_next = W;
    }
    __syncthreads();
    const int total_routes = s_routes[apc];
    auto locate = [&](int f, int &j, int &r) { // flattened route f -> (ant j, route r)
        j = 0;
        while (j + 1 < apc && s_routes[j + 1] <= f) j++;
        r = f - s_routes[j];
    };
    // Longest routes first: the warps take routes in this order, so a warp that
    // finishes early picks up a short one and the CTA ends with its longest
    // route rather than with a second route behind it (results do not depend on
    // the order: routes are independent).
    const bool ordered = total_routes <= kLsOrder && total_routes <= (int)blockDim.x;
    if (ordered) {
        if (threadIdx.x < total_routes) {
            int j, r;
            locate(threadIdx.x, j, r);
            const uint16_t *rstart = reinterpret_cast<const uint16_t *>(ant_ptr(j, AL.rstart));
            s_rlen[threadIdx.x] = (uint16_t)(rstart[r + 1] - rstart[r]);
        }
        __syncthreads();
        if (threadIdx.x < total_routes) {
            const int f = threadIdx.x, lf = s_rlen[f];
            int rank = 0;
            for (int g = 0; g < total_routes; g++) {
                const int lg = s_rlen[g];
                rank += lg > lf || (lg == lf && g < f);
            }
            s_order[rank] = (uint16_t)f;
        }
        __syncthreads();
    }

    int status = ACO_OK, status_inst = 0;
    for (int f = warp; f < total_routes;) {
        int j, r;
        locate(ordered ? (int)s_order[f] : f, j, r);
        const LocalSearchArgs a = args[s_inst[j]];
        uint16_t *tour = reinterpret_cast<uint16_t *>(ant_ptr(j, AL.tour));
        uint16_t *pos = reinterpret_cast<uint16_t *>(ant_ptr(j, AL.pos));
        uint8_t *li = ant_ptr(j, AL.li);
        uint16_t *rid = reinterpret_cast<uint16_t *>(ant_ptr(j, AL.rid));
        uint8_t *dlb = ant_ptr(j, AL.dlb);
        const uint16_t *rstart = reinterpret_cast<const uint16_t *>(ant_ptr(j, AL.rstart));
        float *dt = reinterpret_cast<float *>(ant_ptr(j, AL.dt));
        const int rb = rstart[r], re = rstart[r + 1] - 1, R = re - rb + 1;
        int st = ACO_OK;
        if (R <= kRL && s_only[j] == 1) {
            // routes of at most 32 nodes improved already (fused construct or
            // route-level kernel); only the longer ones of this ant are left
            // here.  Their edge lengths still enter the tour length.
            for (int p = rb + lane; p <= re; p += 32) dt[p] = __ldg(a.dist + (size_t)tour[p] * a.ld + tour[p + 1]);
        } else if (R <= kRL) {
            // route-local state: the distance tile (row k1 = distances from route
            // node k1, lane k2 its column) and every route node's neighbour list
            // filtered to the route, in list order.  Lane q holds route node q; row
            // nodes come by shuffle, so the loads of a round of kLsRows rows depend
            // on nothing in shared memory and are all in flight together.
            const int v = lane < R ? (int)tour[rb + lane] : 0;
            for (int k0 = 0; k0 < R; k0 += kLsRows) {
                float d[kLsRows];
                int nb[kLsRows];
#pragma unroll
                for (int u = 0; u < kLsRows; u++) {
                    const int k1 = k0 + u;
                    const int node1 = __shfl_sync(FULL, v, k1 & 31);
                    d[u] = (k1 < R && lane < R) ? __ldg(a.dist + (size_t)node1 * a.ld + v) : 0.f;
                    nb[u] = (k1 < R && lane < a.nn_ls) ? __ldg(a.nn_list + (size_t)node1 * a.nn_ls + lane) : 0;
                }
#pragma unroll
                for (int u = 0; u < kLsRows; u++) {
                    const int k1 = k0 + u;
                    if (k1 >= R) break; // warp-uniform
                    tile[k1 * kRL + lane] = d[u];
                    const int n2 = nb[u];
                    const bool in = n2 != 0 && rid[n2] == r;
                    const unsigned m = __ballot_sync(FULL, in);
                    const int slot = __popc(m & ((1u << lane) - 1u));
                    if (in && slot < kRL) lnn[k1 * kRL + slot] = li[n2];
                    int cnt = __popc(m);
                    // lists deeper than 32: the rest while the route may still gain entries
                    const int node1 = __shfl_sync(FULL, v, k1 & 31);
                    for (int h0 = 32; h0 < a.nn_ls && cnt < R - 1; h0 += 32) {
                        const int h = h0 + lane;
                        const int n3 = h < a.nn_ls ? __ldg(a.nn_list + (size_t)node1 * a.nn_ls + h) : 0;
                        const bool in3 = n3 != 0 && rid[n3] == r;
                        const unsigned m3 = __ballot_sync(FULL, in3);
                        const int slot3 = cnt + __popc(m3 & ((1u << lane) - 1u));
                        if (in3 && slot3 < kRL) lnn[k1 * kRL + slot3] = li[n3];
                        cnt += __popc(m3);
                    }
                    if (lane == 0) lcnt[k1] = (uint8_t)(cnt < R - 1 ? cnt : R - 1);
                }
            }
            __syncwarp();
            int tq = lane < R ? lane : 0;
            int pk = lane < R ? lane : 0;
            // edge lengths: position q -> q+1, the last one back to the next depot (node 0 = local 0)
            float dq = lane < R ? tile[lane * kRL + (lane + 1 < R ? lane + 1 : 0)] : 0.f;
            st = a.best ? two_opt_route_best(lane, R, tile, lnn, tq, pk, dq, a.pass_limit)
                        : two_opt_route_regs(lane, R, r == 0, tile, lnn, lcnt, tq, pk, dq, a.pass_limit);
            const int node = __shfl_sync(FULL, v, tq);
            if (lane < R) {
                tour[rb + lane] = (uint16_t)node;
                dt[rb + lane] = dq;
            }
            __syncwarp();
        } else {
            for (int p = rb + lane; p <= re; p += 32) dt[p] = __ldg(a.dist + (size_t)tour[p] * a.ld + tour[p + 1]);
            __syncwarp();
            Route c;
            c.tour = tour; c.pos = pos; c.rid = rid; c.dlb = dlb; c.dt = dt;
            c.dist = a.dist; c.nn = a.nn_list; c.ld = a.ld; c.nn_ls = a.nn_ls; c.lane = lane;
            c.r = r; c.rb = rb; c.re = re; c.dlb0 = r > 0;
            st = two_opt_route_generic(c, a.pass_limit);
        }
        if (st != ACO_OK && status == ACO_OK) {
            status = st;
            status_inst = s_inst[j];
        }
        int nxt = 0;
        if (lane == 0) nxt = atomicAdd(&s_next, 1);
        f = __shfl_sync(FULL, nxt, 0);
    }
    if (status != ACO_OK && lane == 0) set_status(args[status_inst].status, status);
    __syncthreads();

    for (int j = 0; j < apc; j++) {
        if (s_inst[j] < 0) continue;
        const LocalSearchArgs &a = args[s_inst[j]];
        int *gtour = a.solutions + (size_t)s_ant[j] * a.T;
        const uint16_t *tour = reinterpret_cast<const uint16_t *>(ant_ptr(j, AL.tour));
        for (int p = threadIdx.x; p < s_size[j]; p += blockDim.x) gtour[p] = tour[p]; // kernel.cl:530-532
    }
    if (warp < apc && s_inst[warp] >= 0) { // kernel.cl:534-538: fp32 sum of dist_tour_wrk in position order
        const int j = warp, size = s_size[j];
        const float *dt = reinterpret_cast<const float *>(ant_ptr(j, AL.dt));
        float len = 0.f;
        for (int base = 0; base < size - 1; base += 32) {
            const float e = base + lane < size - 1 ? dt[base + lane] : 0.f;
            const int m = size - 1 - base < 32 ? size - 1 - base : 32;
#pragma unroll
            for (int k = 0; k < 32; k++) {
                const float x = __shfl_sync(FULL, e, k);
                if (k < m) len = __fadd_rn(len, x);
            }
        }
        if (lane == 0) args[s_inst[j]].lens[s_ant[j]] = len;
    }
    if (!list) break;
    }
    if (list) { // the last CTA to finish rewinds the list for the next construct
        __syncthreads();
        if (threadIdx.x == 0) {
            __threadfence();
            if (atomicAdd(list_ctr + 2, 1) == (int)gridDim.x - 1) {
                list_ctr[0] = 0;
                list_ctr[1] = 0;
                list_ctr[2] = 0;
            }
        }
    }
}

} // namespace

// ---------------------------------------------------------------------------
// Route-level 2-opt (throughput construct): every route of every ant (of at
// most 255 nodes) is one entry of the list the construct kernel wrote, and the
// warps of a persistent grid take entries from a counter, so the routes of
// one ant spread over all SMs instead of queueing in one CTA.  A route needs
// no state of its ant beyond its own nodes: its membership test is a per-warp
// node -> local index map in shared memory, set for the route and cleared
// after it.  Routes of at most 32 nodes run in registers (two_opt.cuh), longer
// ones through two_opt_route_local.  The warp that improves an ant's last listed route sums the ant's
// tour length (kernel.cl:534-538) from the distances of its final tour edges,
// which equal the 2-opt's edge lengths for a symmetric matrix (the only case
// this kernel is used for); ants flagged for the per-ant kernel get their
// length there.
// ---------------------------------------------------------------------------
constexpr int kRouteRows = 4; // tile rows loaded per round (register budget of two CTAs per SM)

// Routes of 33..255 nodes in the route-level kernel: kernel.cl:126-277 with
// the route's state in the warp's shared memory (the area of the register
// path's distance tile) and local node ids: nodes[k] is the global node of
// local id k (0: the depot), tk[p] the local id at route position p, pk[k] the
// position of local id k, dq[p] dist_tour_wrk of position p, dlb[k] the
// don't-look bits; loc[node] is the local id of a customer of the route (0:
// not in it).  Positions are scanned in order; for each examined node, the
// warp evaluates 32 entries of its neighbour list at a time, and the first
// entry that ends the search (past the radius, or an improving move) decides,
// as in the sequential code; the exchange reverses position ranges pairwise.
__device__ int two_opt_route_local(int lane, int R, const float *dist, int ld, const int *nn, int nn_ls,
                                   const uint8_t *loc, const uint16_t *nodes, uint8_t *tk, uint8_t *pk, uint8_t *dlb,
                                   float *dq, int pass_limit)
{
    auto D = [&](int a, int b) { return __ldg(dist + (size_t)a * ld + b); };
    int passes = 0;
    bool imp = true;
    while (imp) {
        if (pass_limit > 0 && passes >= pass_limit) return ACO_ERR_LS_LIMIT;
        passes++;
        imp = false;
        for (int l = 0; l < R; l++) {
            const int k1 = tk[l];
            if (dlb[k1]) continue;
            const int n1 = nodes[k1];
            int h1 = 0, h2 = 0, h3 = 0, h4 = 0;
            bool found = false;
            if (nn_ls <= 32) {
                // one list of at most 32 entries: both searches from one load of it, the
                // predecessor's result used only when the successor search finds no move
                const int ks1 = tk[l + 1 < R ? l + 1 : 0], kp1 = tk[l > 0 ? l - 1 : R - 1];
                const int ns1 = nodes[ks1], np1 = nodes[kp1];
                const float rs = D(n1, ns1), rp = D(np1, n1);
                const int n2 = lane < nn_ls ? __ldg(nn + (size_t)n1 * nn_ls + lane) : 0;
                const int kk2 = loc[n2];
                bool sc = false, sok = false, pc = false, pok = false;
                int ks2 = 0, kpp2 = 0;
                if (kk2 != 0) {
                    const float d12 = D(n1, n2);
                    sc = __fsub_rn(rs, d12) > kEps;
                    pc = __fsub_rn(rp, d12) > kEps;
                    const int p2 = pk[kk2];
                    if (sc) {
                        ks2 = tk[p2 + 1 < R ? p2 + 1 : 0];
                        const float g = __fsub_rn(__fadd_rn(__fadd_rn(-rs, d12), D(ns1, nodes[ks2])), dq[p2]);
                        sok = g < -kEps;
                    }
                    if (pc) {
                        kpp2 = tk[p2 > 0 ? p2 - 1 : R - 1];
                        if (!(kpp2 == k1 || kp1 == kk2)) {
                            const float g = __fsub_rn(__fadd_rn(__fadd_rn(-rp, d12), D(np1, nodes[kpp2])), dq[p2 - 1]);
                            pok = g < -kEps;
                        }
                    }
                }
                const unsigned sstop = __ballot_sync(FULL, kk2 != 0 && (!sc || sok));
                const unsigned pstop = __ballot_sync(FULL, kk2 != 0 && (!pc || pok));
                if (sstop) { // successor search (kernel.cl:180-198)
                    const int f = __ffs(sstop) - 1;
                    if (__shfl_sync(FULL, (int)sc, f)) {
                        found = true;
                        h1 = k1;
                        h2 = ks1;
                        h3 = __shfl_sync(FULL, kk2, f);
                        h4 = __shfl_sync(FULL, ks2, f);
                    }
                }
                if (!found && pstop) { // predecessor search (kernel.cl:202-230)
                    const int f = __ffs(pstop) - 1;
                    if (__shfl_sync(FULL, (int)pc, f)) {
                        found = true;
                        h1 = kp1;
                        h2 = k1;
                        h3 = __shfl_sync(FULL, kpp2, f);
                        h4 = __shfl_sync(FULL, kk2, f);
                    }
                }
            } else {
                {   // successor search (kernel.cl:180-198)
                    const int ks1 = tk[l + 1 < R ? l + 1 : 0];
                    const float radius = D(n1, nodes[ks1]);
                    for (int h0 = 0; h0 < nn_ls; h0 += 32) {
                        const int h = h0 + lane;
                        const int n2 = h < nn_ls ? __ldg(nn + (size_t)n1 * nn_ls + h) : 0;
                        const int kk2 = loc[n2];
                        bool cond = false, okm = false;
                        int ks2 = 0;
                        if (kk2 != 0) {
                            const float d12 = D(n1, n2);
                            cond = __fsub_rn(radius, d12) > kEps;
                            if (cond) {
                                const int p2 = pk[kk2];
                                ks2 = tk[p2 + 1 < R ? p2 + 1 : 0];
                                const float g = __fsub_rn(__fadd_rn(__fadd_rn(-radius, d12), D(nodes[ks1], nodes[ks2])), dq[p2]);
                                okm = g < -kEps;
                            }
                        }
                        const unsigned stop = __ballot_sync(FULL, kk2 != 0 && (!cond || okm));
                        if (stop) {
                            const int f = __ffs(stop) - 1;
                            if (__shfl_sync(FULL, (int)cond, f)) {
                                found = true;
                                h1 = k1;
                                h2 = ks1;
                                h3 = __shfl_sync(FULL, kk2, f);
                                h4 = __shfl_sync(FULL, ks2, f);
                            }
                            break;
                        }
                    }
                }
                if (!found) { // predecessor search (kernel.cl:202-230)
                    const int kp1 = tk[l > 0 ? l - 1 : R - 1];
                    const float radius = D(nodes[kp1], n1);
                    for (int h0 = 0; h0 < nn_ls; h0 += 32) {
                        const int h = h0 + lane;
                        const int n2 = h < nn_ls ? __ldg(nn + (size_t)n1 * nn_ls + h) : 0;
                        const int kk2 = loc[n2];
                        bool cond = false, okm = false;
                        int kpp2 = 0;
                        if (kk2 != 0) {
                            const float d12 = D(n1, n2);
                            cond = __fsub_rn(radius, d12) > kEps;
                            if (cond) {
                                const int p2 = pk[kk2];
                                kpp2 = tk[p2 > 0 ? p2 - 1 : R - 1];
                                if (!(kpp2 == k1 || kp1 == kk2)) {
                                    const float g =
                                        __fsub_rn(__fadd_rn(__fadd_rn(-radius, d12), D(nodes[kp1], nodes[kpp2])), dq[p2 - 1]);
                                    okm = g < -kEps;
                                }
                            }
                        }
                        const unsigned stop = __ballot_sync(FULL, kk2 != 0 && (!cond || okm));
                        if (stop) {
                            const int f = __ffs(stop) - 1;
                            if (__shfl_sync(FULL, (int)cond, f)) {
                                found = true;
                                h1 = kp1;
                                h2 = k1;
                                h3 = __shfl_sync(FULL, kpp2, f);
                                h4 = __shfl_sync(FULL, kk2, f);
                            }
                            break;
                        }
                    }
                }
            }
            if (!found) {
                if (lane == 0) dlb[k1] = 1; // kernel.cl:232
                __syncwarp();
                continue;
            }
            // exchange (kernel.cl:235-270)
            imp = true;
            int p1 = pk[h1], p3 = pk[h3];
            if (p3 < p1) {
                int t = h1; h1 = h3; h3 = t;
                t = h2; h2 = h4; h4 = t;
                t = p1; p1 = p3; p3 = t;
            }
            const int i = p1, jj = p3, a = pk[h2];
            const float d13 = D(nodes[h1], nodes[h3]), d24 = D(nodes[h2], nodes[h4]);
            __syncwarp();
            if (lane == 0) {
                dlb[h1] = 0;
                dlb[h2] = 0;
                dlb[h3] = 0;
                dlb[h4] = 0;
                dq[i] = d13;
                dq[jj] = d24;
            }
            for (int k = lane; k < (jj - i - 1) / 2; k += 32) { // dist_tour_wrk (i, jj) reversed
                const int x = i + 1 + k, y = jj - 1 - k;
                const float t = dq[x];
                dq[x] = dq[y];
                dq[y] = t;
            }
            for (int k = lane; k < (jj - a + 1) / 2; k += 32) { // positions [a, jj] reversed
                const int x = a + k, y = jj - k;
                const uint8_t tx = tk[x], ty = tk[y];
                tk[x] = ty;
                tk[y] = tx;
                pk[ty] = (uint8_t)x;
                pk[tx] = (uint8_t)y;
            }
            __syncwarp();
        }
    }
    return ACO_OK;
}

__host__ __device__ inline size_t route_warp_bytes(int n_max)
{
    return kRL * kRL * 4 + kRL * kRL + kRL + al16((size_t)n_max);
}

__global__ void __launch_bounds__(512, 2) route_opt_kernel(const LocalSearchArgs *args, const int *ant_inst,
                                                           const int *ant_base, const int2 *desc, int *ctr, int cap,
                                                           int *rem, const uint8_t *flagged, int n_max)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    unsigned char *wbase = smem + (size_t)warp * route_warp_bytes(n_max);
    float *tile = reinterpret_cast<float *>(wbase);
    uint8_t *lnn = wbase + kRL * kRL * 4;
    uint8_t *lcnt = lnn + kRL * kRL;
    uint8_t *loc = lcnt + kRL; // node -> local index (0: not in the route)
    for (int i = lane; i < n_max; i += 32) loc[i] = 0;
    __syncwarp();
    const int total = min(ctr[0], cap);
    for (;;) {
        int idx = 0;
        if (lane == 0) idx = atomicAdd(&ctr[1], 1);
        idx = __shfl_sync(FULL, idx, 0);
        if (idx >= total) break;
        const int2 d = desc[idx];
        if (d.x < 0) continue; // an empty entry
        const int g = d.x, rb = d.y & 0xFFFF, R = d.y >> 16;
        const int b = __ldg(ant_inst + g), ant = g - __ldg(ant_base + b);
        const LocalSearchArgs a = args[b];
        int *gt = a.solutions + (size_t)ant * a.T;
        if (R > kRL) { // 33..255 nodes: the route-local generic path in the warp's tile area
            uint16_t *nodes = reinterpret_cast<uint16_t *>(wbase);
            uint8_t *tk = wbase + 512, *pk = tk + 256, *dlb = pk + 256;
            float *dq = reinterpret_cast<float *>(wbase + 1280);
            for (int k = lane; k < R; k += 32) {
                const int node = gt[rb + k];
                nodes[k] = (uint16_t)node;
                tk[k] = (uint8_t)k;
                pk[k] = (uint8_t)k;
                dlb[k] = (uint8_t)(k == 0 && rb != 0 ? 1 : 0); // the depot's bit: clear entering route 0 only
                if (k >= 1) loc[node] = (uint8_t)k;
            }
            __syncwarp();
            for (int k = lane; k < R; k += 32) dq[k] = __ldg(a.dist + (size_t)nodes[k] * a.ld + nodes[k + 1 < R ? k + 1 : 0]);
            __syncwarp();
            const int st = two_opt_route_local(lane, R, a.dist, a.ld, a.nn_list, a.nn_ls, loc, nodes, tk, pk, dlb, dq,
                                               a.pass_limit);
            if (st != ACO_OK && lane == 0) set_status(a.status, st);
            for (int k = lane; k < R; k += 32) __stcs(gt + rb + k, (int)nodes[tk[k]]);
            for (int k = 1 + lane; k < R; k += 32) loc[nodes[k]] = 0;
            __syncwarp();
        } else {
        const int v = lane < R ? gt[rb + lane] : 0;
        if (lane >= 1 && lane < R) loc[v] = (uint8_t)lane; // customers only (kernel.cl:293-300)
        __syncwarp();
        for (int k0 = 0; k0 < R; k0 += kRouteRows) {
            float dd[kRouteRows];
            int nb[kRouteRows];
#pragma unroll
            for (int u = 0; u < kRouteRows; u++) {
                const int k1 = k0 + u;
                const int node1 = __shfl_sync(FULL, v, k1 & 31);
                dd[u] = (k1 < R && lane < R) ? __ldg(a.dist + (size_t)node1 * a.ld + v) : 0.f;
                nb[u] = (k1 < R && lane < a.nn_ls) ? __ldg(a.nn_list + (size_t)node1 * a.nn_ls + lane) : 0;
            }
#pragma unroll
            for (int u = 0; u < kRouteRows; u++) {
                const int k1 = k0 + u;
                if (k1 >= R) break; // warp-uniform
                tile[k1 * kRL + lane] = dd[u];
                const int n2 = nb[u];
                const int l2 = n2 != 0 ? loc[n2] : 0;
                const unsigned m = __ballot_sync(FULL, l2 != 0);
                const int slot = __popc(m & ((1u << lane) - 1u));
                if (l2 != 0 && slot < kRL) lnn[k1 * kRL + slot] = (uint8_t)l2;
                int cnt = __popc(m);
                const int node1 = __shfl_sync(FULL, v, k1 & 31);
                for (int h0 = 32; h0 < a.nn_ls && cnt < R - 1; h0 += 32) { // lists deeper than 32
                    const int h = h0 + lane;
                    const int n3 = h < a.nn_ls ? __ldg(a.nn_list + (size_t)node1 * a.nn_ls + h) : 0;
                    const int l3 = n3 != 0 ? loc[n3] : 0;
                    const unsigned m3 = __ballot_sync(FULL, l3 != 0);
                    const int slot3 = cnt + __popc(m3 & ((1u << lane) - 1u));
                    if (l3 != 0 && slot3 < kRL) lnn[k1 * kRL + slot3] = (uint8_t)l3;
                    cnt += __popc(m3);
                }
                if (lane == 0) lcnt[k1] = (uint8_t)(cnt < R - 1 ? cnt : R - 1);
            }
        }
        __syncwarp();
        // edge lengths: position q -> q+1, the last one back to the next depot (node 0 = local 0)
        int tq = lane < R ? lane : 0, pk = lane < R ? lane : 0;
        float dq = lane < R ? tile[lane * kRL + (lane + 1 < R ? lane + 1 : 0)] : 0.f;
        const int st = a.best ? two_opt_route_best(lane, R, tile, lnn, tq, pk, dq, a.pass_limit)
                              : two_opt_route_regs(lane, R, rb == 0, tile, lnn, lcnt, tq, pk, dq, a.pass_limit);
        if (st != ACO_OK && lane == 0) set_status(a.status, st);
        const int node = __shfl_sync(FULL, v, tq);
        if (lane < R) __stcs(gt + rb + lane, node); // evict first: not read again before the statistics
        if (lane >= 1 && lane < R) loc[v] = 0;
        __syncwarp();
        }
        __threadfence();
        int last = 0;
        if (lane == 0) last = atomicSub(rem + g, 1) == 1;
        last = __shfl_sync(FULL, last, 0);
        if (last && !flagged[g]) { // every route of the ant is final: its length
            __threadfence();
            const int size = __ldcg(gt + a.T - 1);
            float len = 0.f;
            // four chunks of 32 edges: their tour and distance loads in flight before the sums
            for (int base = 0; base < size - 1; base += 128) {
                int u[4], w[4];
                float e[4];
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int p = base + 32 * c + lane;
                    u[c] = p < size - 1 ? __ldcg(gt + p) : 0;
                    w[c] = p < size - 1 ? __ldcg(gt + p + 1) : 0;
                }
#pragma unroll
                for (int c = 0; c < 4; c++) e[c] = __ldg(a.dist + (size_t)u[c] * a.ld + w[c]);
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int m = size - 1 - (base + 32 * c);
#pragma unroll
                    for (int k = 0; k < 32; k++) {
                        const float x = __shfl_sync(FULL, e[c], k);
                        if (k < m) len = __fadd_rn(len, x);
                    }
                }
            }
            if (lane == 0) a.lens[ant] = len;
        }
    }
    // the last CTA to finish rewinds the list for the next iteration
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(&ctr[2], 1) == (int)gridDim.x - 1) {
            ctr[0] = 0;
            ctr[1] = 0;
            ctr[2] = 0;
        }
    }
}

size_t local_search_smem(int n_max, int ants_per_cta, int warps) { return ls_smem_bytes(n_max, ants_per_cta, warps); }

int local_search_occupancy(int warps, size_t smem)
{
    // answers are kept per (device, warps, shared memory): a colony's shape
    // search asks a few hundred of them
    static std::mutex mu;
    static std::map<std::tuple<int, int, size_t>, int> memo;
    int dev = 0;
    cudaGetDevice(&dev);
    const auto key = std::make_tuple(dev, warps, smem);
    {
        std::lock_guard<std::mutex> lk(mu);
        const auto it = memo.find(key);
        if (it != memo.end()) return it->second;
    }
    if (cudaFuncSetAttribute(local_search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, local_search_kernel, warps * 32, smem) != cudaSuccess)
        return 0;
    std::lock_guard<std::mutex> lk(mu);
    memo[key] = blocks;
    return blocks;
}

size_t route_opt_smem(int n_max, int warps) { return (size_t)warps * route_warp_bytes(n_max); }

cudaError_t launch_route_opt(const LocalSearchArgs *d_args, const int *d_ant_inst, const int *d_ant_base,
                             const int2 *d_desc, int *d_ctr, int cap, int *d_rem, const uint8_t *d_flagged, int n_max,
                             int warps, int sm_count, cudaStream_t st)
{
    const size_t smem = route_opt_smem(n_max, warps);
    cudaError_t e = cudaFuncSetAttribute(route_opt_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, route_opt_kernel, warps * 32, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    route_opt_kernel<<<sm_count * per_sm, warps * 32, smem, st>>>(d_args, d_ant_inst, d_ant_base, d_desc, d_ctr, cap,
                                                                   d_rem, d_flagged, n_max);
    return cudaGetLastError();
}

cudaError_t launch_local_search(const LocalSearchArgs *d_args, const int *d_ant_inst, const int *d_ant_base,
                                int total_ants, int ants_per_cta, int n_max, int warps, size_t smem, cudaStream_t st,
                                const uint8_t *only, const int *list, int *list_ctr, int sm_count)
{
    if (ants_per_cta < 1 || ants_per_cta > kMaxLsAnts || warps < ants_per_cta) return cudaErrorInvalidValue;
    if ((list == nullptr) != (list_ctr == nullptr) || (list && !only)) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(local_search_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int blocks = (total_ants + ants_per_cta - 1) / ants_per_cta;
    if (list) { // persistent over the listed ants: as many CTAs as fit at once, at most one per group
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, local_search_kernel, warps * 32, smem);
        if (e != cudaSuccess) return e;
        if (per_sm < 1) return cudaErrorInvalidConfiguration;
        blocks = std::min(blocks, sm_count * per_sm);
    }
    local_search_kernel<<<blocks, warps * 32, smem, st>>>(d_args, d_ant_inst, d_ant_base, only, ants_per_cta, n_max,
                                                          total_ants, list, list_ctr);
    return cudaGetLastError();
}

} // namespace aco
