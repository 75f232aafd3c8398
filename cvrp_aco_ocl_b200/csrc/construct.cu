// construct.cu -- route construction, one CVRP tour per ant.
//
// construct_parity_kernel restates construct_solution + independent_roulette
// (cvrp_ocl/gpu/kernel.cl:325-373, 382-493) bit for bit:
//   * The reference runs one work-group of nloc work-items per ant; work-item l
//     owns a Park-Miller state and draws one number for every node
//     i = l, l+nloc, ... at every step (kernel.cl:331-337).  Here an ant is
//     32*WPA threads; the node i of thread t is i = t + 32*WPA*j, its lane is
//     l = i mod nloc (thread t owns exactly the lanes l = t mod 32*WPA) and its
//     draw index inside the step is k = i / nloc, so the number is
//     state_l * 16807^(k+1) mod m.  After the step every lane jumps by
//     16807^(draws of lane l).
//   * The argmax tournament (kernel.cl:343-366) keeps the left operand on ties;
//     the winner among equal maxima is the node with the smallest tournament
//     rank, precomputed on the host.  A 32-bit key ((0xFFFF - rank) << 16 | node)
//     turns the tournament into two redux.sync.max reductions.
//   * value == 0 means "no candidate": return to the depot (kernel.cl:461-465).
// construct_nn_kernel is the throughput mode (no reference counterpart):
// warp-per-ant sampling over a nearest-neighbour candidate list staged in
// shared memory by TMA bulk copies.  The roulette is run as an exponential
// race: lane j draws u_j from its own Park-Miller stream and candidate j wins
// with the smallest -ln(u_j) / weight_j, which picks j with probability
// weight_j / sum(weight) like the roulette, in one warp min-reduction instead
// of a prefix scan (the draws are off the step's dependent chain).  The
// candidate tables hold 1 / weight, so a step needs no division.
//
// Rows of total_info and the lookup tables are staged into shared memory with
// 1-D cp.async.bulk copies (no cluster multicast) completing on an mbarrier.
#include <cuda_runtime.h>

#include "aco_device.cuh"
#include "kernels.h"
#include "two_opt.cuh"

namespace aco {

namespace {

__host__ __device__ inline size_t al128(size_t x) { return (x + 127) & ~(size_t)127; }

struct ParityLayout {
    size_t bar, dem, key, d0, jump, adv, state, red, mat, bytes;
};

__host__ __device__ inline ParityLayout parity_layout(int n, int nloc, int kmax, int wpa, int apc, bool smat)
{
    const size_t n4 = (size_t)((n + 3) & ~3), k4 = (size_t)((kmax + 3) & ~3);
    ParityLayout L;
    size_t o = 0;
    L.bar = o; o = al128(o + 16);
    L.dem = o; o = al128(o + n4 * 4);
    L.key = o; o = al128(o + n4 * 4);
    L.d0 = o; o = al128(o + n4 * 4);
    L.jump = o; o = al128(o + k4 * 4);
    L.adv = o; o = al128(o + (size_t)nloc * 4);
    L.state = o; o = al128(o + (size_t)apc * nloc * 4);
    L.red = o; o = al128(o + (size_t)apc * 2 * wpa * 2 * 4);
    L.mat = o;
    if (smat) o = al128(o + (size_t)n * n4 * 4);
    L.bytes = o;
    return L;
}

__device__ __forceinline__ uint32_t pm_norm(int x)
{
    long long r = (long long)x % (long long)kPM;
    if (r < 0) r += kPM;
    return (uint32_t)r;
}

template <int WPA, bool FIN, bool SMAT>
__global__ void __launch_bounds__(512) construct_parity_kernel(ConstructArgs a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    constexpr int TPA = 32 * WPA;
    const int n = a.n, ld = a.ld, nloc = a.nloc;
    const int n4 = (n + 3) & ~3, k4 = (a.kmax + 3) & ~3;
    const int apc = blockDim.x / TPA;
    const ParityLayout L = parity_layout(n, nloc, a.kmax, WPA, apc, SMAT);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L.bar);
    int *s_dem = reinterpret_cast<int *>(smem + L.dem);
    uint32_t *s_key = reinterpret_cast<uint32_t *>(smem + L.key);
    float *s_d0 = reinterpret_cast<float *>(smem + L.d0);
    uint32_t *s_jump = reinterpret_cast<uint32_t *>(smem + L.jump);
    uint32_t *s_adv = reinterpret_cast<uint32_t *>(smem + L.adv);
    uint32_t *s_state = reinterpret_cast<uint32_t *>(smem + L.state);
    uint32_t *s_red = reinterpret_cast<uint32_t *>(smem + L.red);
    float *s_mat = reinterpret_cast<float *>(smem + L.mat);

    // ---- stage instance-wide tables (and the whole total_info matrix when it fits)
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t bytes = (uint32_t)(2 * n4 * 4 + k4 * 4 + nloc * 4);
        if (SMAT) bytes += (uint32_t)(n * n4 * 4);
        mbar_arrive_expect_tx(bar, bytes);
        tma_bulk_g2s(s_dem, a.demand, n4 * 4, bar);
        tma_bulk_g2s(s_key, a.tiekey, n4 * 4, bar);
        tma_bulk_g2s(s_jump, a.jump, k4 * 4, bar);
        tma_bulk_g2s(s_adv, a.adv, nloc * 4, bar);
    }
    if (SMAT)
        for (int r = threadIdx.x; r < n; r += blockDim.x)
            tma_bulk_g2s(s_mat + (size_t)r * n4, a.total + (size_t)r * ld, n4 * 4, bar);
    for (int i = threadIdx.x; i < n; i += blockDim.x) s_d0[i] = a.dist[(size_t)i * ld]; // column 0
    const bool ok = mbar_wait(bar, 0, wait_polls(a.wait_limit));
    if (__syncthreads_or(!ok)) { // give up, but let the copies in flight land first (default bound)
        if (threadIdx.x == 0) set_status(a.status, ACO_ERR_TIMEOUT);
        if (!ok) mbar_wait(bar, 0);
        return;
    }

    // ---- one ant per 32*WPA threads
    const int slot = threadIdx.x / TPA;
    const int t = threadIdx.x - slot * TPA;
    const int lane = threadIdx.x & 31;
    const int wsl = t >> 5;
    const int ant = blockIdx.x * apc + slot;
    if (ant >= a.n_ants) return;
    const int nlanes = n < nloc ? n : nloc;
    uint32_t *st = s_state + (size_t)slot * nloc;
    int *seeds = a.seeds + (size_t)ant * nloc;
    for (int l = t; l < nlanes; l += TPA) st[l] = pm_norm(seeds[l]);

    const int J = (n + TPA - 1) / TPA; // nodes per thread (<= 32: visited bits fit one register)
    uint32_t vis = (t == 0) ? 1u : 0u; // node 0 (the depot) starts visited (kernel.cl:431)
    int cur = 0, step = 0, vcnt = 1, load = 0, err = 0;
    float rdist = 0.f, tdist = 0.f, pend = 0.f;
    int *tour = a.solutions + (size_t)ant * a.T;
    if (t == 0) tour[0] = 0;
    const float *base = SMAT ? s_mat : a.total;
    const size_t stride = SMAT ? (size_t)n4 : (size_t)ld;
    const int lmask = nloc - 1;

    while (vcnt < n) {
        if (step >= a.T - 3) { // 2n-3 steps is the longest valid tour
            err = ACO_ERR_STEP_LIMIT;
            break;
        }
        const float *trow = base + (size_t)cur * stride;
        const float *drow = a.dist + (size_t)cur * ld;
        uint32_t bhi = 0u, blo = 0u;
#pragma unroll 4
        for (int j = 0; j < J; j++) {
            const int i = t + TPA * j;
            if (i < n) {
                const uint32_t x = pm_mul(st[i & lmask], s_jump[i >> a.log2_nloc]);
                const float r = __fadd_rn(pm_uniform(x), 0.001f);  // ran01 + 0.001f
                const float p = __fmul_rn(trow[i], 100.0f);         // total_info * 100
                const float v = __fmul_rn(r, p);
                bool c = !((vis >> j) & 1u) && (load + s_dem[i] <= a.capacity);
                if (FIN)
                    c = c && (__fadd_rn(__fadd_rn(rdist, __fadd_rn(drow[i], a.serv_time)), s_d0[i]) <= a.max_dist);
                const uint32_t vb = c ? __float_as_uint(v) : 0u; // r*p*c with c in {0,1}
                const uint32_t key = s_key[i];
                if (vb > bhi || (vb == bhi && key > blo)) {
                    bhi = vb;
                    blo = key;
                }
            }
        }
        uint32_t whi = __reduce_max_sync(0xffffffffu, bhi);
        uint32_t wlo = __reduce_max_sync(0xffffffffu, bhi == whi ? blo : 0u);
        if (WPA > 1) {
            uint32_t *red = s_red + ((size_t)(slot * 2 + (step & 1)) * WPA) * 2;
            if (lane == 0) {
                red[2 * wsl] = whi;
                red[2 * wsl + 1] = wlo;
            }
            named_barrier(1 + slot, TPA);
            whi = 0u;
            wlo = 0u;
#pragma unroll
            for (int w = 0; w < WPA; w++) {
                const uint32_t h = red[2 * w], l2 = red[2 * w + 1];
                if (h > whi || (h == whi && l2 > wlo)) {
                    whi = h;
                    wlo = l2;
                }
            }
        }
        step++;
        int nxt;
        if (whi == 0u) { // no candidate: back to the depot (kernel.cl:461-465)
            nxt = 0;
            load = 0;
            rdist = 0.f;
        } else {
            nxt = (int)(wlo & 0xFFFFu);
            load += s_dem[nxt];
            if (FIN) rdist = __fadd_rn(rdist, __fadd_rn(drow[nxt], a.serv_time));
            vcnt++;
            if (nxt % TPA == t) vis |= 1u << (nxt / TPA);
        }
        if (t == 0) { // tour_dist += dist_wrk[nxt] one step late, in the same order
            tdist = __fadd_rn(tdist, pend);
            pend = __ldg(drow + nxt);
            tour[step] = nxt;
        }
        cur = nxt;
        for (int l = t; l < nlanes; l += TPA) st[l] = pm_mul(st[l], s_adv[l]);
    }

    if (err) {
        if (t == 0) {
            tour[a.T - 1] = 0;
            a.lens[ant] = __int_as_float(0x7f800000);
            set_status(a.status, err);
        }
    } else if (t == 0) { // kernel.cl:482-488
        tdist = __fadd_rn(tdist, pend);
        tdist = __fadd_rn(tdist, s_d0[cur]);
        step++;
        tour[step] = 0;
        tour[a.T - 1] = step + 1;
        a.lens[ant] = tdist;
    }
    if (step > 0) // rnd_seeds[gid] = rnd_seed (kernel.cl:492) for every lane that drew
        for (int l = t; l < nlanes; l += TPA) seeds[l] = (int)st[l];
}

// ---------------------------------------------------------------------------
// Throughput mode.  A persistent kernel: each CTA pulls work items (instance,
// group of `apc` ants) from a device queue, stages the instance's demand,
// candidate table (cand32 packed as node | demand << 16, or uint16 nodes),
// candidate choice_info (chc) and -- when it fits (smat) -- the whole
// total_info matrix into shared memory with TMA bulk copies, then runs one
// warp per ant.  Per ant:
//   * lane l draws from the ant's Park-Miller state l, one number a step, and
//     turns it into its exponential clock E = -ln(u) (race_exp1);
//   * with helper warps (draw), a second warp per ant makes those draws and
//     rates 16 steps ahead into a double-buffered shared ring, handing over at
//     a two-warp named barrier every 16 steps, so the ant's warp keeps only the
//     dependent chain of the step: candidate row, visited bit, key, one redux;
//   * with n <= 1024 the visited set lives in registers (lane l holds bit j for
//     node l + 32j): a candidate's bit is one shuffle away, the update needs no
//     memory operation, and the full-row fallback tests its own bits;
//   * the tour goes to a shared buffer and its length is summed after the last
//     step, in step order.
// ---------------------------------------------------------------------------
struct NNLayout {
    size_t bar, dem, d0, cand, chc, vis, tour, mat, rid, li, dt, pend, cnt, q, ready, ls, ring, flag, bytes;
    int qcap;
};

// Helper-warp draws: steps per hand-over (the ring holds two such chunks per ant).
constexpr int kDrawChunk = 16;

// Shared memory of one 2-opt warp of the fused construct: distance tile,
// in-route neighbour lists and counts, route node ids.
constexpr size_t kLsWarpBytes = 32 * 32 * 4 + 32 * 32 + 32 + 64 + 32 * 32 * 2;

// gtab: the candidate table is read from global memory (L2) instead of being
// staged (instances whose table does not fit next to the per-ant buffers).
// lsw > 0: the fused 2-opt (lsw improving warps): per ant the route id and
// local index of every node and the edge lengths, the route queue.
__host__ __device__ inline NNLayout nn_layout(int n, int K, int Kp, int apc, bool smat, bool packed, bool gtab,
                                              int lsw = 0, bool draw = false)
{
    const size_t n4 = (size_t)((n + 3) & ~3);
    const size_t words = (size_t)((n + 31) / 32);
    NNLayout L;
    size_t o = 0;
    L.bar = o; o = al128(o + 16);
    L.dem = o; o = al128(o + n4 * 4);
    L.d0 = o; o = al128(o + n4 * 4);
    L.cand = o; if (!gtab) o = al128(o + (size_t)n * Kp * (packed ? 4 : 2));
    L.chc = o; if (!gtab) o = al128(o + (size_t)n * Kp * 4);
    L.vis = o; o = al128(o + (size_t)apc * words * 4);
    L.tour = o; o = al128(o + (size_t)apc * 2 * n * 2);
    L.mat = o;
    if (smat) o = al128(o + (size_t)n * n4 * 4);
    L.qcap = apc * n + 64;
    L.rid = L.li = L.dt = L.pend = L.cnt = L.q = L.ready = L.ls = o;
    if (lsw > 0) {
        L.rid = o; o = al128(o + (size_t)apc * n * 2);
        L.li = o; o = al128(o + (size_t)apc * n);
        L.dt = o; o = al128(o + (size_t)apc * 2 * n * 4);
        L.pend = o; o = al128(o + (size_t)2 * apc * 4); // pending routes, deferred flag
        L.cnt = o; o = al128(o + 4 * 4);                // slots allocated, tickets, construct warps done
        L.q = o; o = al128(o + (size_t)L.qcap * 8);
        L.ready = o; o = al128(o + (size_t)L.qcap * 4);
        L.ls = o; o = al128(o + (size_t)lsw * kLsWarpBytes);
    }
    L.ring = L.flag = o;
    if (draw) { // per ant: two chunks of rates, two hand-over flags
        L.ring = o; o = al128(o + (size_t)apc * 2 * kDrawChunk * 32 * 4);
        L.flag = o; o = al128(o + (size_t)apc * 2 * 4);
    }
    L.bytes = o;
    (void)K;
    return L;
}

// One work item: ants [ant0, ant0 + apc) of instance a.  Returns false if the
// staging copies did not arrive in time (uniform over the CTA).
__device__ __forceinline__ int ld_volatile(const int *p) { return *reinterpret_cast<const volatile int *>(p); }

constexpr uint32_t kSpinLimit = 1u << 26; // polls before a wait gives up (with 128 ns sleeps: seconds)

// The 2-opt warps of the fused construct: take tickets in order, wait until
// the route with that index is published (or every construct warp is done and
// no route is left), improve it in registers (two_opt.cuh) and write it back
// in place.  Routes of more than 32 nodes mark their ant for the 2-opt kernel.
__device__ void fused_ls_warp(const ConstructArgs &a, unsigned char *smem, const NNLayout &L, int apc, int lsw_index,
                              int ncw)
{
    const int lane = threadIdx.x & 31, n = a.n;
    int *cnt = reinterpret_cast<int *>(smem + L.cnt);
    int *pend = reinterpret_cast<int *>(smem + L.pend); // [0, apc) pending routes, [apc, 2 apc) deferred
    const int2 *q = reinterpret_cast<const int2 *>(smem + L.q);
    const int *ready = reinterpret_cast<const int *>(smem + L.ready);
    unsigned char *w = smem + L.ls + (size_t)lsw_index * kLsWarpBytes;
    float *tile = reinterpret_cast<float *>(w);
    uint8_t *lnn = w + 32 * 32 * 4;
    uint8_t *lcnt = lnn + 32 * 32;
    uint16_t *rnode = reinterpret_cast<uint16_t *>(lcnt + 32);
    uint16_t *nnbuf = rnode + 32;
    int status = ACO_OK;
    for (;;) {
        int t = 0, state = 0; // state: 1 route ready, 2 nothing left, 3 timed out
        if (lane == 0) {
            t = atomicAdd(&cnt[1], 1);
            for (uint32_t it = 0;; it++) {
                if (t < L.qcap && ld_volatile(&ready[t])) { state = 1; break; }
                if (ld_volatile(&cnt[2]) >= ncw && ld_volatile(&cnt[0]) <= t) { state = 2; break; }
                if (it > kSpinLimit) { state = 3; break; }
                if (it > 32) __nanosleep(128);
            }
        }
        state = __shfl_sync(kFullMask, state, 0);
        t = __shfl_sync(kFullMask, t, 0);
        if (state == 3) {
            status = ACO_ERR_TIMEOUT;
            break;
        }
        if (state == 2) break;
        __threadfence_block();
        const volatile int *qe = reinterpret_cast<const volatile int *>(q + t);
        const int2 e = make_int2(qe[0], qe[1]);
        const int j = e.x & 0xff, r = e.x >> 8, rb = e.y & 0xffff, R = e.y >> 16;
        uint16_t *tb = reinterpret_cast<uint16_t *>(smem + L.tour) + (size_t)j * 2 * n;
        const uint16_t *rid = reinterpret_cast<const uint16_t *>(smem + L.rid) + (size_t)j * n;
        const uint8_t *li = reinterpret_cast<const uint8_t *>(smem + L.li) + (size_t)j * n;
        float *dt = reinterpret_cast<float *>(smem + L.dt) + (size_t)j * 2 * n;
        if (R > kRL) { // longer routes: the whole ant goes to the 2-opt kernel
            if (lane == 0) pend[apc + j] = 1;
        } else {
            // route-local state, as the 2-opt kernel builds it (local_search.cu)
            const int v = lane < R ? (int)tb[rb + lane] : 0;
            if (lane < R) rnode[lane] = (uint16_t)v;
            __syncwarp();
#pragma unroll 8
            for (int x = lane; x < R * kRL; x += 32) {
                const int k1 = x >> 5, k2 = x & 31;
                tile[x] = k2 < R ? __ldg(a.dist + (size_t)rnode[k1] * a.ld + rnode[k2]) : 0.f;
                nnbuf[x] = k2 < a.nn_ls ? (uint16_t)__ldg(a.nn_list + (size_t)rnode[k1] * a.nn_ls + k2) : 0;
            }
            __syncwarp();
            for (int k = 0; k < R; k++) {
                const int node = rnode[k];
                int c = 0;
                for (int h0 = 0; h0 < a.nn_ls && c < R - 1; h0 += 32) {
                    const int h = h0 + lane;
                    const int n2 = h >= a.nn_ls ? 0
                                   : h0 == 0 ? (int)nnbuf[k * kRL + lane]
                                             : __ldg(a.nn_list + (size_t)node * a.nn_ls + h);
                    const bool in = h < a.nn_ls && n2 != 0 && rid[n2] == r;
                    const unsigned m = __ballot_sync(kFullMask, in);
                    const int slot = c + __popc(m & ((1u << lane) - 1u));
                    if (in && slot < kRL) lnn[k * kRL + slot] = li[n2];
                    c += __popc(m);
                }
                if (lane == 0) lcnt[k] = (uint8_t)(c < R - 1 ? c : R - 1);
            }
            __syncwarp();
            int tq = lane < R ? lane : 0, pk = lane < R ? lane : 0;
            float dq = lane < R ? tile[lane * kRL + (lane + 1 < R ? lane + 1 : 0)] : 0.f; // dist_tour_wrk
            const int st = a.ls_best ? two_opt_route_best(lane, R, tile, lnn, tq, pk, dq, a.pass_limit)
                                     : two_opt_route_regs(lane, R, r == 0, tile, lnn, lcnt, tq, pk, dq, a.pass_limit);
            if (st != ACO_OK) status = st;
            const int node = __shfl_sync(kFullMask, v, tq);
            if (lane < R) {
                tb[rb + lane] = (uint16_t)node;
                dt[rb + lane] = dq;
            }
        }
        __syncwarp();
        __threadfence_block();
        if (lane == 0) atomicSub(&pend[j], 1);
    }
    if (status != ACO_OK && lane == 0) set_status(a.status, status);
}

// Barrier `id` shared by exactly two warps (an ant's warp and its helper).
__device__ __forceinline__ void pair_barrier(int id) { asm volatile("bar.sync %0, 64;" ::"r"(id) : "memory"); }

// Helper warp of one ant: the race clocks of chunk c go to ring half c & 1; at
// hand-over c both warps meet at the pair barrier, after which the ant's warp
// has set flag[c & 1] (1 = the ant is done, 0 = continue).  The ant's warp
// reads flag-free: it only waits at the same barriers.
__device__ __forceinline__ uint32_t draw_chunk(uint32_t xs, float *buf, int lane)
{
#pragma unroll 4
    for (int k = 0; k < kDrawChunk; k++) {
        xs = pm_mul(xs, 16807u);
        buf[k * 32 + lane] = race_exp1(pm_uniform(xs));
    }
    return xs;
}

// xs: the lane's state after chunk 0, which the helper fills while the item's
// tables are still being staged.
__device__ __forceinline__ void draw_warp(uint32_t xs, float *ring, const int *flag, int bar_id, int lane)
{
    for (int c = 0;; c++) {
        if (c > 0) xs = draw_chunk(xs, ring + (c & 1) * kDrawChunk * 32, lane);
        pair_barrier(bar_id);
        if (*reinterpret_cast<const volatile int *>(flag + (c & 1))) break;
    }
}

// The route list entries of one finished ant (warp-wide): route r is the
// positions [depot r, depot r+1) of its tour, listed as {ant, first position |
// nodes << 16} for the route-level 2-opt, which improves routes of at most
// kListedRoute nodes (its local node ids are bytes).  An ant with a longer
// route, or whose routes do not fit the list, lists none and is flagged
// (ls_needed 2) for the per-ant kernel, which improves all of its routes.
constexpr int kListedRoute = 255;

__device__ __forceinline__ void emit_routes(const ConstructArgs &a, const uint16_t *tbuf, int size, int g, int lane)
{
    const unsigned FULL = 0xffffffffu;
    int nr = 0, prev = 0;
    bool toolong = false;
    for (int base = 0; base < size; base += 32) { // count
        const int p = base + lane;
        unsigned m = __ballot_sync(FULL, p >= 1 && p < size && tbuf[p < size ? p : 0] == 0);
        while (m) {
            const int q = base + __ffs(m) - 1;
            m &= m - 1;
            nr++;
            toolong = toolong || q - prev > kListedRoute;
            prev = q;
        }
    }
    int rbase = 0;
    if (lane == 0 && !toolong) rbase = atomicAdd(a.route_ctr, nr);
    rbase = __shfl_sync(FULL, rbase, 0);
    const bool fits = !toolong && rbase + nr <= a.route_cap;
    if (fits) { // write
        int k = 0;
        prev = 0;
        for (int base = 0; base < size; base += 32) {
            const int p = base + lane;
            unsigned m = __ballot_sync(FULL, p >= 1 && p < size && tbuf[p < size ? p : 0] == 0);
            while (m) {
                const int q = base + __ffs(m) - 1;
                m &= m - 1;
                if (lane == (k & 31)) a.route_desc[rbase + k] = make_int2(g, prev | ((q - prev) << 16));
                k++;
                prev = q;
            }
        }
    } else if (!toolong) { // entries of this reservation below the capacity are read: mark them empty
        for (int k = lane; k < nr && rbase + k < a.route_cap; k += 32) a.route_desc[rbase + k] = make_int2(-1, 0);
    }
    if (lane == 0) {
        a.route_rem[g] = fits ? nr : 0;
        a.ls_needed[g] = (uint8_t)(fits ? 0 : 2);
        if (!fits) { // one entry per ant and construct: the list holds every ant of the colony
            const int k = atomicAdd(a.ls_list_ctr, 1);
            a.ls_list[k] = g;
        }
    }
}

// Register visited set (n <= 1024): bit k of a lane's word is node lane + 32k.
// The lane's unvisited customers: its in-range bits not yet set (node 0, the
// depot, is bit 0 of lane 0 and always set).
__device__ __forceinline__ uint32_t open_bits(uint32_t vis, int n, int lane)
{
    const int cnt = lane < n ? (n - lane + 31) >> 5 : 0; // nodes lane, lane + 32, ... below n
    const uint32_t valid = cnt >= 32 ? 0xffffffffu : (1u << cnt) - 1u;
    return ~vis & valid;
}

// Smallest demand among the unvisited customers of an ant (warp-wide result).
template <bool REGVIS>
__device__ __forceinline__ int min_open_demand(const int *s_dem, uint32_t vis, const uint32_t *vism, int n, int words,
                                               int lane)
{
    int m = 0x7fffffff;
    if (REGVIS) { // only this lane's unvisited nodes
        for (uint32_t o = open_bits(vis, n, lane); o; o &= o - 1u) m = min(m, s_dem[lane + 32 * (__ffs(o) - 1)]);
    } else {
        for (int k = 0; k < words; k++) {
            const int i = lane + 32 * k;
            if (i > 0 && i < n && !((vism[k] >> lane) & 1u)) m = min(m, s_dem[i]);
        }
    }
    return (int)__reduce_min_sync(0xffffffffu, (unsigned)m);
}

// The same with the number of unvisited customers that have it (0 when none
// is left): visiting one of them lowers the count, and only when it reaches 0
// can the smallest demand have changed.
template <bool REGVIS>
__device__ __forceinline__ int min_open_demand_count(const int *s_dem, uint32_t vis, const uint32_t *vism, int n,
                                                     int words, int lane, int &count)
{
    int m = 0x7fffffff, c = 0;
    if (REGVIS) {
        for (uint32_t o = open_bits(vis, n, lane); o; o &= o - 1u) {
            const int d = s_dem[lane + 32 * (__ffs(o) - 1)];
            c = d < m ? 1 : c + (d == m ? 1 : 0);
            m = min(m, d);
        }
    } else {
        for (int k = 0; k < words; k++) {
            const int i = lane + 32 * k;
            if (i > 0 && i < n && !((vism[k] >> lane) & 1u)) {
                const int d = s_dem[i];
                c = d < m ? 1 : c + (d == m ? 1 : 0);
                m = min(m, d);
            }
        }
    }
    const int gm = (int)__reduce_min_sync(0xffffffffu, (unsigned)m);
    count = (int)__reduce_add_sync(0xffffffffu, (unsigned)(m == gm ? c : 0));
    return gm;
}

// The feasible customer of the full row with the largest total_info (ties:
// lowest index), -1 if none: the step's path when no listed candidate fits.
// PRUNE (register visited set only): test the demands first, from shared
// memory, and read row values only for the nodes that fit; a route's last step
// (nothing fits) then ends without reading the row.  Measured: it pays where the
// row is read from L2 by few warps (the helper-warp kernel on large instances)
// and costs where the row is staged or many warps share the SM.
template <bool FIN, bool REGVIS, bool PRUNE = false>
__device__ __forceinline__ int best_of_row(const float *row, const int *s_dem, const float *s_d0, const float *drow,
                                           uint32_t vis, const uint32_t *vism, int n, int words, int lane, int load,
                                           int cap, float rdist, float serv, float maxd)
{
    const unsigned FULL = 0xffffffffu;
    uint32_t bk = 0u, bi = 0xffffffffu;
    if (REGVIS) {
        const int capleft = cap - load;
        uint32_t open = open_bits(vis, n, lane);
        if (PRUNE) { // the lane's unvisited nodes whose demand fits, eight a round
            uint32_t fit = 0u;
            const int rounds = ((int)__reduce_max_sync(FULL, (unsigned)__popc(open)) + 7) >> 3;
            for (int r = 0; r < rounds; r++) {
                int kb[8], dm[8];
#pragma unroll
                for (int u = 0; u < 8; u++) {
                    kb[u] = open ? __ffs(open) - 1 : 0;
                    dm[u] = open ? s_dem[lane + 32 * kb[u]] : 0x7fffffff; // no node: does not fit
                    open &= open - 1u;
                }
#pragma unroll
                for (int u = 0; u < 8; u++) fit |= (dm[u] <= capleft ? 1u : 0u) << kb[u];
            }
            if (!__any_sync(FULL, fit != 0u)) return -1;
            open = fit;
        }
        // Only the lane's unvisited (PRUNE: and fitting) nodes, lowest first (so a
        // strict > keeps the lowest index of a lane's equal values), four a round
        // with their loads issued first; rounds until the lane with the most such
        // nodes is done.
        const int rounds = ((int)__reduce_max_sync(FULL, (unsigned)__popc(open)) + 3) >> 2;
        for (int r = 0; r < rounds; r++) {
            int idx[4], dm[4];
            float rv[4], dv[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                const int i = open ? lane + 32 * (__ffs(open) - 1) : -1;
                open &= open - 1u;
                const int ic = i >= 0 ? i : 0;
                idx[u] = i;
                rv[u] = row[ic];
                dm[u] = i < 0 ? 0x7fffffff : PRUNE ? 0 : s_dem[ic]; // no node: fails the capacity test
                if (FIN) dv[u] = __ldg(drow + ic);
            }
#pragma unroll
            for (int u = 0; u < 4; u++) {
                bool ff = dm[u] <= capleft;
                if (FIN) ff = ff && __fadd_rn(__fadd_rn(rdist, __fadd_rn(dv[u], serv)), s_d0[idx[u] >= 0 ? idx[u] : 0]) <= maxd;
                const uint32_t kk = ff ? __float_as_uint(rv[u]) + 1u : 0u;
                const bool better = kk > bk;
                bk = better ? kk : bk;
                bi = better ? (uint32_t)idx[u] : bi;
            }
        }
        const uint32_t hk = __reduce_max_sync(FULL, bk);
        if (hk == 0u) return -1;
        return (int)__reduce_min_sync(FULL, bk == hk ? bi : 0xffffffffu);
    }
    constexpr int G = FIN ? 4 : 8;
    for (int k0 = 0; k0 < words; k0 += G) { // branch-free: every lane tests its own nodes
        // G nodes a lane at a time, all loads first (indices clamped into range)
        float rv[G], dv[G];
        int dm[G];
#pragma unroll
        for (int u = 0; u < G; u++) {
            const int i = lane + 32 * (k0 + u);
            const int ic = i < n ? i : 0;
            rv[u] = row[ic];
            dm[u] = s_dem[ic];
            if (FIN) dv[u] = __ldg(drow + ic);
        }
#pragma unroll
        for (int u = 0; u < G; u++) {
            const int k = k0 + u, i = lane + 32 * k;
            const uint32_t vk = REGVIS ? vis : (k < words ? vism[k] : ~0u);
            bool ff = i > 0 && i < n && !((vk >> (REGVIS ? (k & 31) : lane)) & 1u) && load + dm[u] <= cap;
            if (FIN) ff = ff && __fadd_rn(__fadd_rn(rdist, __fadd_rn(dv[u], serv)), s_d0[i < n ? i : 0]) <= maxd;
            const uint32_t kk = ff ? __float_as_uint(rv[u]) + 1u : 0u;
            const bool better = kk > bk; // strictly: the lowest k of a lane wins ties
            bk = better ? kk : bk;
            bi = better ? (uint32_t)i : bi;
        }
    }
    const uint32_t hk = __reduce_max_sync(FULL, bk);
    if (hk == 0u) return -1;
    return (int)__reduce_min_sync(FULL, bk == hk ? bi : 0xffffffffu);
}

struct FallbackPick {
    int nxt, mind, mcnt; // nxt -1: no customer fits
};

// best_of_row out of line, for the kernel without helper warps (many ants per
// SM), with a shortcut: mind is the smallest demand among unvisited customers
// and mcnt the number of them that have it (recounted here when it has dropped
// to 0); when even mind does not fit, no customer does and the row is not
// scanned.  Measured: the shortcut and the call pay off there,
// while in the helper-warp kernel (one ant warp per SMSP, latency bound) the
// plain inline scan is faster, so that kernel keeps it.
template <bool FIN, bool REGVIS>
__device__ __noinline__ FallbackPick fallback_pick(const float *row, const int *s_dem, const float *s_d0,
                                                   const float *drow, uint32_t vis, const uint32_t *vism, int n,
                                                   int words, int lane, int load, int cap, float rdist, float serv,
                                                   float maxd, int mind, int mcnt)
{
    if (mcnt <= 0) mind = min_open_demand_count<REGVIS>(s_dem, vis, vism, n, words, lane, mcnt);
    if (mind > cap - load) return {-1, mind, mcnt};
    return {best_of_row<FIN, REGVIS>(row, s_dem, s_d0, drow, vis, vism, n, words, lane, load, cap, rdist, serv, maxd),
            mind, mcnt};
}

// lens_later: the route-level 2-opt follows and writes every listed ant's
// length, so the construct leaves it out (error paths still write +inf).
template <bool FIN, bool SMAT, bool PACKED, bool REGVIS, bool GTAB = false, bool LSF = false, bool DRAW = false>
__device__ __forceinline__ bool construct_nn_item(const ConstructArgs &a, int apc, int ant0, unsigned char *smem, uint32_t phase,
                                  int lsw = 0, bool lens_later = false)
{
    const int n = a.n, ld = a.ld, K = a.K, Kp = a.Kp, T = a.T;
    const int n4 = (n + 3) & ~3;
    const NNLayout L = nn_layout(n, K, Kp, apc, SMAT, PACKED, GTAB, LSF ? lsw : 0, DRAW);
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem + L.bar);
    int *s_dem = reinterpret_cast<int *>(smem + L.dem);
    float *s_d0 = reinterpret_cast<float *>(smem + L.d0);
    // candidate table: staged copy, or the global one itself (generic loads either way)
    const uint32_t *s_cand = GTAB ? a.cand32 : reinterpret_cast<const uint32_t *>(smem + L.cand);
    const uint16_t *s_nn = GTAB ? a.nn16 : reinterpret_cast<const uint16_t *>(smem + L.cand);
    const float *s_chc = GTAB ? a.chc : reinterpret_cast<const float *>(smem + L.chc);
    uint32_t *s_vis = reinterpret_cast<uint32_t *>(smem + L.vis);
    uint16_t *s_tour = reinterpret_cast<uint16_t *>(smem + L.tour);
    float *s_mat = reinterpret_cast<float *>(smem + L.mat);
    const int words = (n + 31) >> 5;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const unsigned FULL = 0xffffffffu;

    const uint32_t cand_bytes = (uint32_t)(n * Kp * (PACKED ? 4 : 2));
    if (threadIdx.x == 0) {
        uint32_t bytes = (uint32_t)(n4 * 4) + (GTAB ? 0u : cand_bytes + (uint32_t)(n * Kp * 4));
        if (SMAT) bytes += (uint32_t)(n * n4 * 4);
        mbar_arrive_expect_tx(bar, bytes);
        tma_bulk_g2s(s_dem, a.demand, n4 * 4, bar);
        if (!GTAB) {
            tma_bulk_g2s(smem + L.cand, PACKED ? (const void *)a.cand32 : (const void *)a.nn16, cand_bytes, bar);
            tma_bulk_g2s(smem + L.chc, a.chc, n * Kp * 4, bar);
        }
    }
    if (SMAT)
        for (int r = threadIdx.x; r < n; r += blockDim.x)
            tma_bulk_g2s(s_mat + (size_t)r * n4, a.total + (size_t)r * ld, n4 * 4, bar);
    if (FIN)
        for (int i = threadIdx.x; i < n; i += blockDim.x) s_d0[i] = a.dist[(size_t)i * ld];
    if (LSF) { // fused 2-opt bookkeeping starts empty for this item
        uint16_t *rid_all = reinterpret_cast<uint16_t *>(smem + L.rid);
        for (int i = threadIdx.x; i < apc * n; i += blockDim.x) rid_all[i] = 0xFFFFu;
        int *ready_all = reinterpret_cast<int *>(smem + L.ready);
        for (int i = threadIdx.x; i < L.qcap; i += blockDim.x) ready_all[i] = 0;
        int *pend_all = reinterpret_cast<int *>(smem + L.pend);
        for (int i = threadIdx.x; i < 2 * apc; i += blockDim.x) pend_all[i] = 0;
        if (threadIdx.x < 4) reinterpret_cast<int *>(smem + L.cnt)[threadIdx.x] = 0;
    }
    float *ring = reinterpret_cast<float *>(smem + L.ring) + (size_t)(DRAW ? warp % apc : 0) * 2 * kDrawChunk * 32;
    int *hflag = reinterpret_cast<int *>(smem + L.flag) + (DRAW ? warp % apc : 0) * 2;
    // helper warps: warp apc + j draws for ant j, its first chunk during the staging
    const bool helper = DRAW && warp >= apc && warp < 2 * apc && ant0 + (warp - apc) < a.n_ants;
    uint32_t hx = 0;
    if (helper) hx = draw_chunk(pm_norm(a.seeds[(size_t)(ant0 + warp - apc) * a.nloc + lane]), ring, lane);
    // an ant warp's Park-Miller states, loaded while the tables are staged
    const int seed0 = warp < apc && ant0 + warp < a.n_ants ? a.seeds[(size_t)(ant0 + warp) * a.nloc + lane] : 0;
    const bool ok = mbar_wait(bar, phase, wait_polls(a.wait_limit));
    if (__syncthreads_or(!ok)) { // give up, but let the copies in flight land first (default bound)
        if (threadIdx.x == 0) set_status(a.status, ACO_ERR_TIMEOUT);
        if (!ok) mbar_wait(bar, phase);
        return false;
    }

    const int ant = ant0 + warp;
    if (DRAW && warp >= apc) {
        if (helper) draw_warp(hx, ring, hflag, 1 + warp - apc, lane);
        return true;
    }
    if (LSF && warp >= apc) {
        if (warp < apc + lsw) {
            const int ncw = a.n_ants - ant0 < apc ? a.n_ants - ant0 : apc;
            fused_ls_warp(a, smem, L, apc, warp - apc, ncw);
        }
        return true;
    }
    // fused 2-opt: publish route [rb, rb + R) of this ant for the improving warps
    int *f_cnt = reinterpret_cast<int *>(smem + L.cnt);
    int *f_pend = reinterpret_cast<int *>(smem + L.pend);
    auto publish = [&](int r, int rb, int R) {
        if (threadIdx.x % 32 == 0) {
            atomicAdd(&f_pend[warp], 1);
            const int slot = atomicAdd(&f_cnt[0], 1);
            if (slot < L.qcap) {
                reinterpret_cast<int2 *>(smem + L.q)[slot] = make_int2(warp | (r << 8), rb | (R << 16));
                __threadfence_block();
                atomicExch(reinterpret_cast<int *>(smem + L.ready) + slot, 1);
            } else {
                atomicSub(&f_pend[warp], 1); // cannot happen (capacity covers every route)
                set_status(a.status, ACO_ERR_CAPACITY);
            }
        }
    };
    if (warp < apc && ant < a.n_ants) {
        uint16_t *tbuf = s_tour + warp * 2 * n;
        uint16_t *f_rid = reinterpret_cast<uint16_t *>(smem + L.rid) + (size_t)warp * n;
        uint8_t *f_li = reinterpret_cast<uint8_t *>(smem + L.li) + (size_t)warp * n;
        int f_rb = 0, f_r = 0;
        (void)f_rid; (void)f_li;
        uint32_t *vism = s_vis + warp * words;
        uint32_t vis = lane == 0 ? 1u : 0u; // register visited set (REGVIS): node 0 = lane 0, bit 0
        if (!REGVIS) {
            for (int w = lane; w < words; w += 32) vism[w] = w == 0 ? 1u : 0u;
            __syncwarp();
        }
        if (lane == 0) tbuf[0] = 0;
        // smallest demand among the unvisited customers and how many have it
        // (fallback_pick): visits only raise it, so it is recounted lazily, on the
        // fallback path, once every customer holding it has been visited
        int mcnt = 1;
        int mind = DRAW ? 0 : min_open_demand_count<REGVIS>(s_dem, vis, vism, n, words, lane, mcnt);
        // lane l draws from the ant's Park-Miller state l (nloc >= 32), one number a step
        int *seedp = a.seeds + (size_t)ant * a.nloc;
        uint32_t xs = pm_norm(seed0);
        int hand = 0; // hand-overs passed (helper-warp draws)
        if (DRAW) {   // hand-over 0: the helper has filled chunk 0
            if (lane == 0) hflag[0] = 0;
            __syncwarp();
            pair_barrier(1 + warp);
            hand = 1;
        }
        int cur = 0, step = 0, vcnt = 1, load = 0, err = 0;
        float rdist = 0.f;
        const int cap = a.capacity;
        const int jl = lane < K ? lane : K - 1;

        while (vcnt < n) {
            if (step >= T - 3) {
                err = ACO_ERR_STEP_LIMIT;
                break;
            }
            float ex; // this lane's exponential clock for the step
            if (DRAW) {
                const int sc = step & (kDrawChunk - 1);
                if (sc == 0 && step > 0) { // next chunk: hand-over `hand`, continue
                    if (lane == 0) hflag[hand & 1] = 0;
                    __syncwarp();
                    pair_barrier(1 + warp);
                    hand++;
                }
                ex = ring[((hand - 1) & 1) * kDrawChunk * 32 + sc * 32 + lane];
            } else {
                xs = pm_mul(xs, 16807u);
                ex = race_exp1(pm_uniform(xs)); // off the dependent chain of the step
            }
            int c, dc;
            if (PACKED) {
                const uint32_t pk = s_cand[cur * Kp + jl];
                c = (int)(pk & 0xFFFFu);
                dc = (int)(pk >> 16);
            } else {
                c = s_nn[cur * Kp + jl];
                dc = s_dem[c];
            }
            const float winv = s_chc[cur * Kp + jl]; // 1 / total_info of the candidate
            const uint32_t vw = REGVIS ? __shfl_sync(FULL, vis, c & 31) : vism[c >> 5];
            bool f = lane < K && !((vw >> (REGVIS ? (c >> 5) : (c & 31))) & 1u) && (load + dc <= cap);
            if (FIN && f)
                f = __fadd_rn(__fadd_rn(rdist, __fadd_rn(__ldg(a.dist + (size_t)cur * ld + c), a.serv_time)),
                              s_d0[c]) <= a.max_dist;
            // exponential race: the smallest E / w wins (probability w / sum of w); weight 0 never wins
            const uint32_t hk = __reduce_min_sync(FULL, f && winv < INFINITY ? race_key(ex, winv, lane) : kNoKey);
            int nxt = -1, nd = 0;
            if (hk != kNoKey) {
                const uint32_t pick = __shfl_sync(FULL, (uint32_t)c | ((uint32_t)dc << 16), (int)(hk & 31u));
                nxt = (int)(pick & 0xFFFFu);
                nd = (int)(pick >> 16);
            } else if (DRAW) {
                nxt = best_of_row<FIN, REGVIS, !SMAT>(SMAT ? s_mat + cur * n4 : a.total + (size_t)cur * ld, s_dem, s_d0,
                                               a.dist + (size_t)cur * ld, vis, vism, n, words, lane, load, cap, rdist,
                                               a.serv_time, a.max_dist);
                if (nxt >= 0) nd = s_dem[nxt];
            } else {
                const FallbackPick fp = fallback_pick<FIN, REGVIS>(
                    SMAT ? s_mat + cur * n4 : a.total + (size_t)cur * ld, s_dem, s_d0, a.dist + (size_t)cur * ld, vis,
                    vism, n, words, lane, load, cap, rdist, a.serv_time, a.max_dist, mind, mcnt);
                mind = fp.mind;
                mcnt = fp.mcnt;
                nxt = fp.nxt;
                if (nxt >= 0) nd = s_dem[nxt];
            }
            step++;
            if (nxt < 0) {
                nxt = 0;
                load = 0;
                rdist = 0.f;
            } else {
                load += nd;
                if (FIN) rdist = __fadd_rn(rdist, __fadd_rn(__ldg(a.dist + (size_t)cur * ld + nxt), a.serv_time));
                vcnt++;
            }
            if (REGVIS) {
                if (lane == (nxt & 31)) vis |= 1u << (nxt >> 5);
            } else {
                if (lane == 0) vism[nxt >> 5] |= 1u << (nxt & 31);
                __syncwarp();
            }
            if (!DRAW && nxt != 0 && nd == mind) mcnt--; // one customer of the smallest demand fewer
            if (lane == 0) tbuf[step] = (uint16_t)nxt;
            if (LSF) {
                if (nxt != 0) {
                    if (lane == 0) {
                        f_rid[nxt] = (uint16_t)f_r;
                        f_li[nxt] = (uint8_t)(step - f_rb < 256 ? step - f_rb : 0);
                    }
                } else { // back at the depot: the route [f_rb, step) is complete
                    publish(f_r, f_rb, step - f_rb);
                    f_r++;
                    f_rb = step;
                }
            }
            cur = nxt;
        }
        if (DRAW) { // last hand-over: the helper stops
            if (lane == 0) hflag[hand & 1] = 1;
            __syncwarp();
            pair_barrier(1 + warp);
        }
        __syncwarp();
        int *tour = a.solutions + (size_t)ant * T;
        bool use_dt = false;
        if (LSF) {
            if (!err) {
                if (lane == 0) tbuf[step + 1] = 0;
                publish(f_r, f_rb, step + 1 - f_rb); // the last route ends at the final depot
            }
            if (lane == 0) { // this ant is done publishing; wait until its routes are improved
                __threadfence_block();
                atomicAdd(&f_cnt[2], 1);
                uint32_t it = 0;
                while (ld_volatile(&f_pend[warp]) > 0) {
                    if (++it > kSpinLimit) {
                        set_status(a.status, ACO_ERR_TIMEOUT);
                        break;
                    }
                    if (it > 32) __nanosleep(128);
                }
                __threadfence_block();
            }
            __syncwarp();
            const bool deferred = ld_volatile(&f_pend[apc + warp]) != 0;
            use_dt = !deferred;
            if (lane == 0) a.ls_needed[a.ant_base + ant] = (uint8_t)(!err && deferred ? 1 : 0);
        }
        if (err) {
            if (lane == 0) {
                tour[T - 1] = 0;
                a.lens[ant] = __int_as_float(0x7f800000);
                set_status(a.status, err);
                if (!LSF && a.route_desc) {
                    a.route_rem[a.ant_base + ant] = 0;
                    a.ls_needed[a.ant_base + ant] = 0;
                }
            }
        } else {
            const int size = step + 2;
            if (lane == 0) tbuf[step + 1] = 0;
            __syncwarp();
            for (int p = lane; p < size; p += 32) tour[p] = tbuf[p];
            // tour length: the fp32 sum of the edges in step order (kernel.cl:475,483); after the
            // fused 2-opt, of its edge lengths in position order (kernel.cl:534-538).  Four
            // chunks of 32 edges have their loads in flight before their sums.
            const float *f_dt = reinterpret_cast<const float *>(smem + L.dt) + (size_t)warp * 2 * n;
            float tdist = 0.f;
            if (!lens_later) {
                for (int base = 0; base < size - 1; base += 128) {
                    float e[4];
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        const int p = base + 32 * c + lane;
                        e[c] = p < size - 1
                                   ? (use_dt ? f_dt[p] : __ldg(a.dist + (size_t)tbuf[p] * ld + tbuf[p + 1]))
                                   : 0.f;
                    }
#pragma unroll
                    for (int c = 0; c < 4; c++) {
                        const int m = size - 1 - (base + 32 * c);
#pragma unroll
                        for (int k = 0; k < 32; k++) {
                            const float y = __shfl_sync(FULL, e[c], k);
                            if (k < m) tdist = __fadd_rn(tdist, y);
                        }
                    }
                }
            }
            if (lane == 0) {
                tour[T - 1] = size;
                if (!lens_later) a.lens[ant] = tdist;
            }
            if (!LSF && a.route_desc) emit_routes(a, tbuf, size, a.ant_base + ant, lane);
        }
        if (step > 0) // states after the last draw (the helper may have drawn further)
            seedp[lane] = (int)(DRAW ? pm_mul(xs, pm_pow16807(step)) : xs);
    }
    return true;
}

// The item without fused 2-opt: candidate table staged or in global memory,
// register or shared visited set, with or without helper-warp draws.
template <bool FIN, bool DRAW>
__device__ __forceinline__ bool construct_nn_plain(const ConstructArgs &a, int apc, int ant0, unsigned char *smem,
                                                   uint32_t phase, bool ll)
{
    if (a.gtab && a.n <= 1024)
        return a.packed ? construct_nn_item<FIN, false, true, true, true, false, DRAW>(a, apc, ant0, smem, phase, 0, ll)
                        : construct_nn_item<FIN, false, false, true, true, false, DRAW>(a, apc, ant0, smem, phase, 0, ll);
    if (a.gtab)
        return a.packed ? construct_nn_item<FIN, false, true, false, true, false, DRAW>(a, apc, ant0, smem, phase, 0, ll)
                        : construct_nn_item<FIN, false, false, false, true, false, DRAW>(a, apc, ant0, smem, phase, 0, ll);
    if (a.n <= 1024) {
        if (a.smat)
            return a.packed ? construct_nn_item<FIN, true, true, true, false, false, DRAW>(a, apc, ant0, smem, phase, 0, ll)
                            : construct_nn_item<FIN, true, false, true, false, false, DRAW>(a, apc, ant0, smem, phase, 0, ll);
        return a.packed ? construct_nn_item<FIN, false, true, true, false, false, DRAW>(a, apc, ant0, smem, phase, 0, ll)
                        : construct_nn_item<FIN, false, false, true, false, false, DRAW>(a, apc, ant0, smem, phase, 0, ll);
    }
    return a.packed ? construct_nn_item<FIN, false, true, false, false, false, DRAW>(a, apc, ant0, smem, phase, 0, ll)
                    : construct_nn_item<FIN, false, false, false, false, false, DRAW>(a, apc, ant0, smem, phase, 0, ll);
}

// The item of the two-CTA kernel: no staged distance matrix (it does not fit
// half of the shared memory at the sizes where it pays) and no staged table
// above 1024 nodes, which keeps every path within 64 registers.
template <bool FIN>
__device__ __forceinline__ bool construct_nn_wide(const ConstructArgs &a, int apc, int ant0, unsigned char *smem,
                                                  uint32_t phase, bool ll)
{
    if (a.n > 1024)
        return a.packed ? construct_nn_item<FIN, false, true, false, true>(a, apc, ant0, smem, phase, 0, ll)
                        : construct_nn_item<FIN, false, false, false, true>(a, apc, ant0, smem, phase, 0, ll);
    if (a.gtab)
        return a.packed ? construct_nn_item<FIN, false, true, true, true>(a, apc, ant0, smem, phase, 0, ll)
                        : construct_nn_item<FIN, false, false, true, true>(a, apc, ant0, smem, phase, 0, ll);
    return a.packed ? construct_nn_item<FIN, false, true, true, false>(a, apc, ant0, smem, phase, 0, ll)
                    : construct_nn_item<FIN, false, false, true, false>(a, apc, ant0, smem, phase, 0, ll);
}

// KIND: 0 = plain, 1 = helper-warp draws, 2 = fused 2-opt (lsw improving warps),
// 3 = plain at two CTAs per SM
template <bool FIN, int KIND>
__device__ __forceinline__ void construct_nn_body(const ConstructArgs *args, const int2 *items, int n_items, int *queue,
                                                  int apc, int lsw, bool lens_later)
{
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int s_item;
    uint64_t *bar = reinterpret_cast<uint64_t *>(smem); // offset 0 in every layout
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_mbar_init();
    }
    uint32_t phase = 0;
    for (;;) {
        __syncthreads(); // the previous item is done with shared memory
        if (threadIdx.x == 0) s_item = atomicAdd(queue, 1);
        __syncthreads();
        const int it = s_item;
        if (it >= n_items) break;
        const int2 code = __ldg(items + it); // {instance, first ant of the group}
        const ConstructArgs a = args[code.x];
        const int ant0 = code.y;
        bool ok;
        if (KIND == 2 && a.gtab) { // fused 2-opt, candidate table in global memory
            ok = a.packed ? construct_nn_item<FIN, false, true, true, true, true>(a, apc, ant0, smem, phase, lsw)
                          : construct_nn_item<FIN, false, false, true, true, true>(a, apc, ant0, smem, phase, lsw);
        } else if (KIND == 2) { // fused 2-opt (register visited set, staged tables)
            if (a.smat) ok = a.packed ? construct_nn_item<FIN, true, true, true, false, true>(a, apc, ant0, smem, phase, lsw)
                                      : construct_nn_item<FIN, true, false, true, false, true>(a, apc, ant0, smem, phase, lsw);
            else ok = a.packed ? construct_nn_item<FIN, false, true, true, false, true>(a, apc, ant0, smem, phase, lsw)
                               : construct_nn_item<FIN, false, false, true, false, true>(a, apc, ant0, smem, phase, lsw);
        } else if (KIND == 3) {
            ok = construct_nn_wide<FIN>(a, apc, ant0, smem, phase, lens_later && a.route_desc != nullptr);
        } else {
            ok = construct_nn_plain<FIN, KIND == 1>(a, apc, ant0, smem, phase, lens_later && a.route_desc != nullptr);
        }
        if (!ok) break; // uniform: decided by __syncthreads_or
        phase ^= 1u;
    }
    // the last CTA to finish rewinds the queue for the next launch: every CTA
    // has taken its final ticket before it counts itself out
    if (threadIdx.x == 0) {
        __threadfence();
        if (atomicAdd(queue + 1, 1) == (int)gridDim.x - 1) {
            queue[0] = 0;
            queue[1] = 0;
        }
    }
}

// Register budget: one CTA of the widest launch (16 warps) per SM, the
// residency the staged tables allow on the batched workloads.
template <bool FIN, int KIND>
__global__ void __launch_bounds__(512, 1) construct_nn_kernel(const ConstructArgs *args, const int2 *items, int n_items,
                                                           int *queue, int apc, int lsw, int lens_later)
{
    construct_nn_body<FIN, KIND>(args, items, n_items, queue, apc, lsw, lens_later != 0);
}

// Two CTAs per SM at 64 registers a thread: 32 ant warps an SM instead of 16,
// twice the warps to cover the latency of the candidate-table reads, which on
// the large instances of a batch come through L2 (tables beyond half of the
// SM's shared memory are not staged).
template <bool FIN>
__global__ void __launch_bounds__(512, 2) construct_nn_wide_kernel(const ConstructArgs *args, const int2 *items,
                                                                   int n_items, int *queue, int apc, int lsw,
                                                                   int lens_later)
{
    construct_nn_body<FIN, 3>(args, items, n_items, queue, apc, lsw, lens_later != 0);
}

// The helper-warp variant runs one CTA per SM (few ants, latency bound): its
// registers are not squeezed for a second CTA.
template <bool FIN>
__global__ void __launch_bounds__(512, 1) construct_nn_draw_kernel(const ConstructArgs *args, const int2 *items,
                                                                   int n_items, int *queue, int apc, int lsw,
                                                                   int lens_later)
{
    construct_nn_body<FIN, 1>(args, items, n_items, queue, apc, lsw, lens_later != 0);
}

template <int WPA, bool FIN, bool SMAT>
cudaError_t launch_parity_t(const ConstructArgs &a, int apc, cudaStream_t st)
{
    const ParityLayout L = parity_layout(a.n, a.nloc, a.kmax, WPA, apc, SMAT);
    auto kern = construct_parity_kernel<WPA, FIN, SMAT>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.bytes);
    if (e != cudaSuccess) return e;
    const int blocks = (a.n_ants + apc - 1) / apc;
    kern<<<blocks, apc * 32 * WPA, L.bytes, st>>>(a);
    return cudaGetLastError();
}

template <int WPA>
cudaError_t launch_parity_w(const ConstructArgs &a, int apc, bool smat, cudaStream_t st)
{
    const bool fin = !(a.max_dist == __builtin_huge_valf());
    if (fin) return smat ? launch_parity_t<WPA, true, true>(a, apc, st) : launch_parity_t<WPA, true, false>(a, apc, st);
    return smat ? launch_parity_t<WPA, false, true>(a, apc, st) : launch_parity_t<WPA, false, false>(a, apc, st);
}

} // namespace

size_t construct_parity_smem(int n, int nloc, int kmax, int wpa, int apc, bool stage_total, bool)
{
    return parity_layout(n, nloc, kmax, wpa, apc, stage_total).bytes;
}

size_t construct_nn_smem(int n, int K, int Kp, int apc, bool stage_total, bool packed, bool global_table, int ls_warps,
                         bool draw)
{
    return nn_layout(n, K, Kp, apc, stage_total, packed, global_table, ls_warps, draw && ls_warps == 0).bytes;
}

cudaError_t launch_construct_nn(const ConstructArgs *d_args, const int2 *d_items, int n_items, int *d_queue, int apc,
                                size_t smem, int sm_count, bool finite_maxd, cudaStream_t st, int ls_warps, bool draw,
                                bool lens_later, bool wide)
{
    if (ls_warps > 0) draw = false;
    if (ls_warps > 0 || draw) wide = false;
    auto kern = ls_warps > 0 ? (finite_maxd ? construct_nn_kernel<true, 2> : construct_nn_kernel<false, 2>)
                : draw       ? (finite_maxd ? construct_nn_draw_kernel<true> : construct_nn_draw_kernel<false>)
                : wide       ? (finite_maxd ? construct_nn_wide_kernel<true> : construct_nn_wide_kernel<false>)
                             : (finite_maxd ? construct_nn_kernel<true, 0> : construct_nn_kernel<false, 0>);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    int warps = apc < 8 ? 8 : apc; // helper warps share the staging of each item
    if (draw && warps < 2 * apc) warps = 2 * apc;
    if (ls_warps > 0) warps = apc + ls_warps;
    if (warps > 16) return cudaErrorInvalidValue;
    // a persistent grid: the CTAs that are resident at once (registers and shared memory)
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, warps * 32, smem);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    int blocks = sm_count * per_sm;
    if (blocks > n_items) blocks = n_items;
    if (blocks < 1) blocks = 1;
    kern<<<blocks, warps * 32, smem, st>>>(d_args, d_items, n_items, d_queue, apc, ls_warps, lens_later ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_construct_parity(const ConstructArgs &a, int wpa, int apc, bool smat, cudaStream_t st)
{
    switch (wpa) {
    case 1: return launch_parity_w<1>(a, apc, smat, st);
    case 2: return launch_parity_w<2>(a, apc, smat, st);
    case 4: return launch_parity_w<4>(a, apc, smat, st);
    case 8: return launch_parity_w<8>(a, apc, smat, st);
    default: return cudaErrorInvalidValue;
    }
}


} // namespace aco
