// ns.cu -- the random-descent stage: the reference's random neighbourhood
// moves (NeighbourSearch, neighbourSearch.cpp:40-446, and Move::apply,
// move.cpp:17-80) proposed `rounds` times on every ant's tour after the local
// search, the valid ones with a gain below -EPSILON applied, then the tour
// length recomputed as compute_tour_length sums it (vrpHelper.cpp:244-253).
//
// The moves draw from glibc's random() (additive feedback, degree 31,
// separation 3: r[k] = r[k-31] + r[k-3] mod 2^32, output r[k] >> 1, after
// srandom's Park-Miller fill of the first 31 words and 310 discarded outputs),
// seeded per ant and iteration.  The reference's rejection loops spin forever
// when no route qualifies; here each gives up after a bounded number of draws
// and the proposal is dropped.  Float expressions keep the reference's
// evaluation order.
//
// The proposals of one ant form a dependent chain (each may change the tour
// the next one reads), so lane 0 of the ant's warp runs it; the warp copies the
// tour in and out and sums the length.  One CTA per work item (instance,
// first ant), one warp per ant.
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/cvrp_aco.h"
#include "aco_device.cuh"
#include "kernels.h"

namespace aco {
namespace {

constexpr unsigned FULL = 0xffffffffu;
constexpr int kTries = 4096;

struct Rng {
    uint32_t r[31];
    int f, b;
};

__device__ __forceinline__ int32_t rng_next(Rng &g)
{
    const uint32_t v = g.r[g.f] += g.r[g.b];
    if (++g.f >= 31) g.f = 0;
    if (++g.b >= 31) g.b = 0;
    return (int32_t)(v >> 1);
}

__device__ void rng_seed(Rng &g, unsigned seed)
{
    int32_t word = (int32_t)(seed ? seed : 1u);
    g.r[0] = (uint32_t)word;
    for (int i = 1; i < 31; i++) {
        const long long hi = word / 127773, lo = word % 127773;
        long long w = 16807 * lo - 2836 * hi;
        if (w < 0) w += 2147483647;
        word = (int32_t)w;
        g.r[i] = (uint32_t)word;
    }
    g.f = 3;
    g.b = 0;
    for (int k = 0; k < 310; k++) (void)rng_next(g);
}

__device__ __forceinline__ unsigned ns_seed(int rnd_seed, int iteration, int ant)
{
    unsigned s = (unsigned)rnd_seed * 2654435761u + (unsigned)iteration * 40503u + (unsigned)ant * 2246822519u;
    s &= 0x7fffffffu;
    return s ? s : 1u;
}

struct Routes {
    int *beg, *end, *load;
    float *dist;
    int count;
};

struct Move {
    int type; // 0 exchange, 1 insertion, 2 inversion, -1 none
    bool valid;
    float gain;
    int p1, p2;
};

struct Ctx {
    const ConstructArgs *a;
    const int *tour;
    Routes rt;
    Rng *g;
    __device__ float D(int i, int j) const { return a->dist[(size_t)i * a->ld + j]; }
};

// reset_ant (neighbourSearch.cpp:40-70)
__device__ void reset_routes(const ConstructArgs &a, const int *tour, int size, Routes &rt)
{
    int k = 0, beg = 0, load = 0;
    float d = 0.f;
    for (int i = 1; i < size; i++) {
        load += a.demand[tour[i]];
        d = __fadd_rn(d, a.dist[(size_t)tour[i - 1] * a.ld + tour[i]]);
        if (tour[i] == 0) {
            rt.beg[k] = beg;
            rt.end[k] = i;
            rt.load[k] = load;
            rt.dist[k] = d;
            k++;
            beg = i;
            load = 0;
            d = 0.f;
        }
    }
    rt.count = k;
}

__device__ __forceinline__ int rnd_route(Rng &g, int nr) { return (int)rng_next(g) % nr; }
__device__ __forceinline__ int rnd_pos(Rng &g, const Routes &rt, int r)
{
    return rt.beg[r] + rng_next(g) % (rt.end[r] - rt.beg[r]);
}

__device__ int big_route(Rng &g, const Routes &rt)
{
    for (int t = 0; t < kTries; t++) {
        const int r = rnd_route(g, rt.count);
        if (rt.end[r] - rt.beg[r] + 1 > 3) return r;
    }
    return -1;
}

__device__ int customer_pos(Rng &g, const Routes &rt, int r, int avoid)
{
    for (int t = 0; t < kTries; t++) {
        const int p = rnd_pos(g, rt, r);
        if (p != rt.beg[r] && p != avoid) return p;
    }
    return -1;
}

// route length with its service time, the form the moves compare
__device__ __forceinline__ float route_base(const Routes &rt, int r, int extra, float serv)
{
    return __fadd_rn(rt.dist[r], __fmul_rn((float)(rt.end[r] - rt.beg[r] - 1 + extra), serv));
}

__device__ __forceinline__ float sum4(float a, float b, float c, float d)
{
    return __fadd_rn(__fadd_rn(__fadd_rn(a, b), c), d);
}
__device__ __forceinline__ float sum3(float a, float b, float c) { return __fadd_rn(__fadd_rn(a, b), c); }

__device__ void exchange_1(const Ctx &c, Move &m)
{
    const ConstructArgs &a = *c.a;
    const int *t = c.tour;
    const int r = big_route(*c.g, c.rt);
    if (r < 0) return;
    int p1 = customer_pos(*c.g, c.rt, r, -1);
    int p2 = p1 < 0 ? -1 : customer_pos(*c.g, c.rt, r, p1);
    if (p2 < 0) return;
    if (p1 > p2) { const int x = p1; p1 = p2; p2 = x; }
    const int n1 = t[p1], n2 = t[p2], p_n1 = t[p1 - 1], p_n2 = t[p2 - 1], s_n1 = t[p1 + 1], s_n2 = t[p2 + 1];
    float gain;
    if (p2 - p1 == 1)
        gain = __fadd_rn(-__fadd_rn(c.D(p_n1, n1), c.D(n2, s_n2)), __fadd_rn(c.D(p_n1, n2), c.D(n1, s_n2)));
    else
        gain = __fadd_rn(-sum4(c.D(p_n1, n1), c.D(n1, s_n1), c.D(p_n2, n2), c.D(n2, s_n2)),
                         sum4(c.D(p_n1, n2), c.D(n2, s_n1), c.D(p_n2, n1), c.D(n1, s_n2)));
    const float d = __fadd_rn(route_base(c.rt, r, 0, a.serv_time), gain);
    m = Move{0, !(d > a.max_dist), gain, p1, p2};
}

__device__ void exchange(const Ctx &c, Move &m)
{
    const ConstructArgs &a = *c.a;
    const int *t = c.tour;
    const int r1 = rnd_route(*c.g, c.rt.count), r2 = rnd_route(*c.g, c.rt.count);
    if (r1 == r2) {
        exchange_1(c, m);
        return;
    }
    int p1 = -1, p2 = -1, n1 = 0, n2 = 0;
    for (int k = 0; k < kTries && n1 == 0; k++) {
        p1 = rnd_pos(*c.g, c.rt, r1);
        n1 = t[p1];
    }
    for (int k = 0; k < kTries && n2 == 0; k++) {
        p2 = rnd_pos(*c.g, c.rt, r2);
        n2 = t[p2];
    }
    if (n1 == 0 || n2 == 0) return;
    const int p_n1 = t[p1 - 1], p_n2 = t[p2 - 1], s_n1 = t[p1 + 1], s_n2 = t[p2 + 1];
    const float gain = __fadd_rn(-sum4(c.D(p_n1, n1), c.D(n1, s_n1), c.D(p_n2, n2), c.D(n2, s_n2)),
                                 sum4(c.D(p_n1, n2), c.D(n2, s_n1), c.D(p_n2, n1), c.D(n1, s_n2)));
    const float d1 = __fadd_rn(__fsub_rn(route_base(c.rt, r1, 0, a.serv_time), __fadd_rn(c.D(p_n1, n1), c.D(n1, s_n1))),
                               __fadd_rn(c.D(p_n1, n2), c.D(n2, s_n1)));
    const float d2 = __fadd_rn(__fsub_rn(route_base(c.rt, r2, 0, a.serv_time), __fadd_rn(c.D(p_n2, n2), c.D(n2, s_n2))),
                               __fadd_rn(c.D(p_n2, n1), c.D(n1, s_n2)));
    const int l1 = c.rt.load[r1] - a.demand[n1] + a.demand[n2], l2 = c.rt.load[r2] - a.demand[n2] + a.demand[n1];
    m = Move{0, !((l1 > a.capacity || l2 > a.capacity) || (d1 > a.max_dist || d2 > a.max_dist)), gain, p1, p2};
}

__device__ float insertion_gain(const Ctx &c, int p1, int p2)
{
    const int *t = c.tour;
    const int n1 = t[p1], n2 = t[p2], p_n1 = t[p1 - 1], p_n2 = t[p2 - 1], s_n1 = t[p1 + 1], s_n2 = t[p2 + 1];
    if (p1 > p2)
        return __fadd_rn(-sum3(c.D(p_n1, n1), c.D(n1, s_n1), c.D(p_n2, n2)),
                         sum3(c.D(n1, n2), c.D(p_n2, n1), c.D(p_n1, s_n1)));
    return __fadd_rn(-sum3(c.D(p_n1, n1), c.D(n1, s_n1), c.D(n2, s_n2)),
                     sum3(c.D(n2, n1), c.D(n1, s_n2), c.D(p_n1, s_n1)));
}

__device__ void insertion_1(const Ctx &c, Move &m)
{
    const ConstructArgs &a = *c.a;
    const int r = big_route(*c.g, c.rt);
    if (r < 0) return;
    const int p1 = customer_pos(*c.g, c.rt, r, -1);
    const int p2 = p1 < 0 ? -1 : customer_pos(*c.g, c.rt, r, p1);
    if (p2 < 0) return;
    const float gain = insertion_gain(c, p1, p2);
    const float d = __fadd_rn(route_base(c.rt, r, 0, a.serv_time), gain);
    m = Move{1, !(d > a.max_dist), gain, p1, p2};
}

__device__ void insertion(const Ctx &c, Move &m)
{
    const ConstructArgs &a = *c.a;
    const int *t = c.tour;
    const int r1 = big_route(*c.g, c.rt);
    if (r1 < 0) return;
    const int r2 = rnd_route(*c.g, c.rt.count);
    if (r1 == r2) {
        insertion_1(c, m);
        return;
    }
    const int p1 = customer_pos(*c.g, c.rt, r1, -1), p2 = customer_pos(*c.g, c.rt, r2, -1);
    if (p1 < 0 || p2 < 0) return;
    const int n1 = t[p1], n2 = t[p2], p_n2 = t[p2 - 1], s_n2 = t[p2 + 1];
    const float gain = insertion_gain(c, p1, p2);
    const float base = route_base(c.rt, r2, 1, a.serv_time); // route 2 gains a customer
    float d2;
    if (p1 > p2)
        d2 = __fadd_rn(__fsub_rn(base, c.D(p_n2, n2)), __fadd_rn(c.D(n1, n2), c.D(p_n2, n1)));
    else
        d2 = __fadd_rn(__fsub_rn(base, c.D(n2, s_n2)), __fadd_rn(c.D(n2, n1), c.D(n1, s_n2)));
    const int l2 = c.rt.load[r2] + a.demand[n1];
    m = Move{1, !(l2 > a.capacity || d2 > a.max_dist), gain, p1, p2};
}

__device__ void inversion(const Ctx &c, Move &m)
{
    const ConstructArgs &a = *c.a;
    const int *t = c.tour;
    const int r = big_route(*c.g, c.rt);
    if (r < 0) return;
    int p1 = customer_pos(*c.g, c.rt, r, -1);
    int p2 = p1 < 0 ? -1 : customer_pos(*c.g, c.rt, r, p1);
    if (p2 < 0) return;
    if (p1 > p2) { const int x = p1; p1 = p2; p2 = x; }
    if (p2 == c.rt.end[r] - 1 && p1 == c.rt.beg[r] + 1) return; // the whole route: no move
    const int n1 = t[p1], n2 = t[p2], p_n1 = t[p1 - 1], s_n2 = t[p2 + 1];
    const float gain = __fadd_rn(-__fadd_rn(c.D(p_n1, n1), c.D(n2, s_n2)), __fadd_rn(c.D(p_n1, n2), c.D(n1, s_n2)));
    const float d = __fadd_rn(route_base(c.rt, r, 0, a.serv_time), gain);
    m = Move{2, !(d > a.max_dist), gain, p1, p2};
}

__device__ void apply_move(int *t, const Move &m)
{
    int p1 = m.p1, p2 = m.p2;
    if (m.type == 0) {
        const int x = t[p1];
        t[p1] = t[p2];
        t[p2] = x;
    } else if (m.type == 1) {
        const int x = t[p1];
        if (p1 < p2)
            for (int i = p1; i < p2; i++) t[i] = t[i + 1];
        else
            for (int i = p1; i > p2; i--) t[i] = t[i - 1];
        t[p2] = x;
    } else if (m.type == 2) {
        while (p1 < p2) {
            const int x = t[p1];
            t[p1] = t[p2];
            t[p2] = x;
            p1++;
            p2--;
        }
    }
}

__global__ void __launch_bounds__(256) ns_kernel(const ConstructArgs *args, const StatsArgs *sargs, const int2 *items,
                                                 int apc, int rounds, int rnd_seed)
{
    extern __shared__ __align__(16) unsigned char sm[];
    const int2 it = items[blockIdx.x];
    const ConstructArgs a = args[it.x];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ant = it.y + warp;
    if (warp >= apc || ant >= a.n_ants) return;
    const int n = a.n, T = a.T;
    int *w = reinterpret_cast<int *>(sm) + (size_t)warp * 6 * n;
    int *tour = w;
    Routes rt{w + 2 * n, w + 3 * n, w + 4 * n, reinterpret_cast<float *>(w + 5 * n), 0};
    int *gt = a.solutions + (size_t)ant * T;
    const int size = gt[T - 1];
    if (size < 2) return;
    for (int p = lane; p < size; p += 32) tour[p] = gt[p];
    __syncwarp();
    if (lane == 0) {
        Rng g;
        rng_seed(g, ns_seed(rnd_seed + it.x, *sargs[it.x].iteration, ant));
        const Ctx c{&a, tour, rt, &g};
        bool fresh = false;
        Ctx cc = c;
        for (int k = 0; k < rounds; k++) {
            if (!fresh) {
                reset_routes(a, tour, size, cc.rt);
                fresh = true;
            }
            if (cc.rt.count < 1) break;
            Move m{-1, false, 0.f, 0, 0};
            const int kind = rng_next(g) % 3;
            if (kind == 0) exchange(cc, m);
            else if (kind == 1) insertion(cc, m);
            else inversion(cc, m);
            if (m.type >= 0 && m.valid && m.gain < -kEps) {
                apply_move(tour, m);
                fresh = false; // the routes follow the tour
            }
        }
    }
    __syncwarp();
    for (int p = lane; p < size; p += 32) gt[p] = tour[p];
    float len = 0.f; // compute_tour_length: fp32 sum in position order
    for (int b0 = 0; b0 < size - 1; b0 += 32) {
        const int p = b0 + lane;
        const float e = p < size - 1 ? a.dist[(size_t)tour[p] * a.ld + tour[p + 1]] : 0.f;
        const int m = size - 1 - b0 < 32 ? size - 1 - b0 : 32;
#pragma unroll
        for (int k = 0; k < 32; k++) {
            const float y = __shfl_sync(FULL, e, k);
            if (k < m) len = __fadd_rn(len, y);
        }
    }
    if (lane == 0) a.lens[ant] = len;
}

} // namespace

size_t ns_smem(int n, int apc) { return (size_t)apc * 6 * n * 4; }

cudaError_t launch_ns(const ConstructArgs *d_args, const StatsArgs *d_sargs, const int2 *d_items, int n_items, int apc,
                      size_t smem, int rounds, int rnd_seed, cudaStream_t st)
{
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(ns_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    ns_kernel<<<n_items, apc * 32, smem, st>>>(d_args, d_sargs, d_items, apc, rounds, rnd_seed);
    return cudaGetLastError();
}

} // namespace aco
