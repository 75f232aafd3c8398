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
// throughput mode, the reciprocal total_info of the row's candidates (re-read
// from L2 after the row is written) into the compact candidate table the
// construct kernel loads by TMA.  The deposit is added inside the stream: the
// lane holding a deposit column's float4 adds the elites' amounts in elite
// order before total_info is formed, so no column is read twice.
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

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v)
{
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned long long w = __shfl_xor_sync(FULL, v, o);
        v = w < v ? w : v;
    }
    return v;
}

// args: one block per instance (batches); null: the single instance `one`,
// passed by value so that its fields need no global load.
__global__ void __launch_bounds__(1024) stats_kernel(const StatsArgs *args, StatsArgs one, int do_elites)
{
    extern __shared__ float s_len[]; // lens[0..A) of this iteration
    __shared__ unsigned long long red[32], s_wmin[32], s_thr;
    __shared__ int s_best, s_flag, s_elite[32], s_size[32], s_ncand;
    __shared__ unsigned long long s_cand[1024]; // get_elites candidates (keys at most the threshold)
    __shared__ float s_minval, s_bsf;
    __shared__ const int *s_tour[32];
    const StatsArgs a = args ? args[blockIdx.x] : one;
    const int A = a.n_ants, T = a.T, tid = threadIdx.x, bs = blockDim.x, R = a.ras_ranks;
    const int lg = a.log2_nloc;
    // every global value the kernel needs is loaded up front, in parallel
    if (tid == 0) {
        s_bsf = a.lens[A];
        s_elite[0] = A;
    }
    for (int k = tid; k < A; k += bs) s_len[k] = a.lens[k];
    __syncthreads();
    const int iter = *a.iteration;

    // iteration best: min over (length, work-group, bit-reversed lane).  Phase 0
    // halves a power-of-two group keeping the left operand on ties, so inside a
    // group the survivor among equal lengths is the lowest bit-reversed lane;
    // phase 1 scans groups in order with a strict <.
    unsigned long long best = ~0ull;
    for (int k = tid; k < A; k += bs) {
        const unsigned g = (unsigned)k >> lg, lid = (unsigned)k & ((1u << lg) - 1u);
        const unsigned rank = (g << lg) | (lg ? (__brev(lid) >> (32 - lg)) : 0u);
        const unsigned long long key = ((unsigned long long)__float_as_uint(s_len[k]) << 32) | rank;
        best = key < best ? key : best;
    }
    best = block_min_u64(best, red);
    if (tid == 0) {
        const unsigned rank = (unsigned)(best & 0xffffffffu);
        const unsigned g = rank >> lg, br = rank & ((1u << lg) - 1u);
        const int idx = (int)((g << lg) | (lg ? (__brev(br) >> (32 - lg)) : 0u));
        const float minval = s_len[idx];
        a.solutions[(size_t)T * (A + 1)] = idx;
        s_best = idx;
        s_minval = minval;
        s_flag = __fsub_rn(minval, s_bsf) < -kEps; // kernel.cl:660
    }
    // get_elites (kernel.cl:717-741): elite 0 is the best-so-far slot, then
    // ras_ranks-1 rounds of "first minimum, knocked out to +inf".  The finite
    // lengths come out in (length, index) order; once they are used up every
    // entry is +inf and each further round takes index 0.  With all lengths in
    // one pass of the block, each entry's rank is the number of keys below its
    // own, and the first R-1 finite ranks place themselves.
    if (do_elites && A <= bs && R > 1) {
        // keys (length bits, index) are unique.  Threshold t: the (R-1)-th
        // smallest of the warps' minima (at least R-1 keys are at most t, so the
        // R-1 smallest all are); only keys up to t are ranked, among themselves.
        const int warp = tid >> 5, lane = tid & 31, nw = (A + 31) >> 5;
        const unsigned long long key =
            tid < A ? ((unsigned long long)__float_as_uint(s_len[tid]) << 32) | (unsigned)tid : ~0ull;
        const unsigned long long wm = warp_min_u64(key);
        if (lane == 0 && warp < nw) s_wmin[warp] = wm;
        if (tid == 0) {
            s_ncand = 0;
            s_thr = ~0ull;
        }
        __syncthreads();
        if (warp == 0 && lane < nw && nw >= R - 1 && R > 1) { // lane i ranks warp minimum i
            const unsigned long long mi = s_wmin[lane];
            int below = 0;
            for (int q = 0; q < nw; q++) below += s_wmin[q] < mi;
            if (below == R - 2) s_thr = mi;
        }
        __syncthreads();
        if (tid < A && key <= s_thr) s_cand[atomicAdd(&s_ncand, 1)] = key;
        const int nfin = __syncthreads_count(tid < A && __float_as_uint(s_len[tid]) < 0x7f800000u);
        const int nc = s_ncand;
        if (tid < nc) {
            const unsigned long long own = s_cand[tid];
            int rk = 0;
            for (int j = 0; j < nc; j++) rk += s_cand[j] < own;
            if ((unsigned)(own >> 32) < 0x7f800000u && rk < R - 1) s_elite[1 + rk] = (int)(own & 0xffffffffu);
        }
        if (tid >= 1 + nfin && tid < R) s_elite[tid] = 0;
    }
    __syncthreads();
    const bool flag = s_flag;
    if (flag) { // update_best_so_far (kernel.cl:551-585)
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
        if (A > bs) { // many ants: the knock-out rounds as written
            for (int r = 1; r < R; r++) {
                unsigned long long m = ~0ull;
                for (int k = tid; k < A; k += bs) {
                    const unsigned long long key = ((unsigned long long)__float_as_uint(s_len[k]) << 32) | (unsigned)k;
                    m = key < m ? key : m;
                }
                m = block_min_u64(m, red);
                if (tid == 0) {
                    const int target = A > 0 ? (int)(m & 0xffffffffu) : 0;
                    s_len[target] = __int_as_float(0x7f800000);
                    s_elite[r] = target;
                }
                __syncthreads();
            }
        }
        // deposit weights (kernel.cl:767-768) and the elite tours: elite 0 reads
        // the iteration best directly when it has just become the best-so-far
        if (tid < R) {
            const int e = s_elite[tid];
            a.elites[tid] = e;
            const int src = (tid == 0 && flag) ? s_best : e;
            const float len = tid == 0 ? (flag ? s_minval : s_bsf) : (A <= bs ? s_len[e] : a.lens[e]);
            a.d_tau[tid] = __fdiv_rn((float)(R - tid), len);
            const int *tour = a.solutions + (size_t)T * src;
            s_tour[tid] = tour;
            s_size[tid] = __ldg(tour + T - 1);
        }
        // deposit list: successor of every customer in each elite tour and the
        // depot -> customer edges as a per-customer bit mask.
        const int n = a.n;
        for (int e = tid; e < R * n; e += bs) a.succ[e] = -1;
        for (int e = tid; e < n; e += bs) a.depmask[e] = 0u;
        __syncthreads();
        // all elites at once: item e = (r, k), edge k of elite r's tour; four
        // items a thread at a time with their loads issued first
        const int items = R * (T - 1);
        for (int e0 = tid; e0 < items; e0 += 4 * bs) {
            int uu[4], vv[4], rr[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int e = e0 + q * bs;
                const int r = e < items ? e / (T - 1) : 0, k = e - r * (T - 1);
                rr[q] = e < items && k < s_size[r] - 1 ? r : -1;
                const int *tour = s_tour[r];
                uu[q] = rr[q] >= 0 ? __ldg(tour + k) : 0;
                vv[q] = rr[q] >= 0 ? __ldg(tour + k + 1) : 0;
            }
#pragma unroll
            for (int q = 0; q < 4; q++) {
                if (rr[q] < 0) continue;
                if (uu[q] != 0) a.succ[(size_t)rr[q] * n + uu[q]] = vv[q];
                else atomicOr(&a.depmask[vv[q]], 1u << rr[q]);
            }
        }
    }
    if (tid == 0) *a.iteration = iter + 1; // main.cpp:86 (Problem::iteration++)
}

// Deposit into one float4 of the depot row (columns c4..c4+3): depot ->
// customer edges from the per-column elite masks, in elite order 0, 1, ...,
// R-1 -- the order the oracle applies the deposit in.
__device__ __forceinline__ void deposit4_depot(const UpdateArgs &a, int c4, float &v0, float &v1, float &v2, float &v3)
{
    const int R = a.ras_ranks, n = a.n;
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

// Float4 per lane per chunk of the evaporation pass: every load of a chunk is
// issued before its arithmetic, so a lane keeps three float4 of each input
// matrix in flight (measured: 2% faster than four with the cache-policy stores).
constexpr int kU = 3;
constexpr int kRowWarps = 8; // warps (rows in flight) per CTA of the row kernel

// Evaporation + deposit + total_info over customer row i, U float4 per lane
// per chunk.  Lanes r < R first read elite r's successor column of node i and
// its amount into the warp's slots s_col / s_amt; every lane then marks which
// of its float4 (index k: columns 4 * (lane + 32k) .. + 3) hold a deposit
// column -- bit k for k < 32, one flag for all later ones (rows past 4096) --
// and only those take the deposit loop.
template <int U, bool A1>
__device__ __forceinline__ void update_row_stream(const UpdateArgs &a, int i, int lane, int q4, float4 *tau4,
                                                  const float4 *heur4, float4 *tot4, int *s_col, float *s_amt)
{
    const int R = a.ras_ranks, n = a.n;
    if (lane < R) {
        s_col[lane] = __ldg(a.succ + (size_t)lane * n + i);
        s_amt[lane] = __ldg(a.d_tau + lane);
    }
    __syncwarp();
    uint32_t depk = 0;
    bool depfar = false;
    for (int r = 0; r < R; r++) {
        const int c = s_col[r];
        if (c >= 0 && ((c >> 2) & 31) == lane) {
            if (c < 4096) depk |= 1u << (c >> 7);
            else depfar = true;
        }
    }
    const float evap = a.evap;
    float4 *tp = tau4 + lane, *op = tot4 + lane;
    const float4 *hp = heur4 + lane;
    int k0 = 0;
    for (int left = q4 - lane; left > 0; left -= 32 * U, tp += 32 * U, op += 32 * U, hp += 32 * U, k0 += U) {
        float4 t[U], h[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (32 * u < left) {
                t[u] = __ldcs(tp + 32 * u); // read once per pass: evict first
                h[u] = __ldcs(hp + 32 * u);
            }
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (32 * u < left) {
                float4 o, tot;
                o.x = __fmul_rn(evap, t[u].x);
                o.y = __fmul_rn(evap, t[u].y);
                o.z = __fmul_rn(evap, t[u].z);
                o.w = __fmul_rn(evap, t[u].w);
                if (k0 + u < 32 ? (depk >> (k0 + u)) & 1u : depfar) { // kernel.cl:747-776, elite order
                    const int c4 = 4 * (lane + 32 * (k0 + u));
                    for (int r = 0; r < R; r++) {
                        const unsigned d = (unsigned)(s_col[r] - c4);
                        if (d < 4u) {
                            const float dt = s_amt[r];
                            if (d == 0) o.x = __fadd_rn(o.x, dt);
                            else if (d == 1) o.y = __fadd_rn(o.y, dt);
                            else if (d == 2) o.z = __fadd_rn(o.z, dt);
                            else o.w = __fadd_rn(o.w, dt);
                        }
                    }
                }
                if (A1) {
                    tot.x = __fmul_rn(o.x, h[u].x);
                    tot.y = __fmul_rn(o.y, h[u].y);
                    tot.z = __fmul_rn(o.z, h[u].z);
                    tot.w = __fmul_rn(o.w, h[u].w);
                } else {
                    tot.x = __fmul_rn(pow_rule(o.x, a.alpha, a.alpha_int), h[u].x);
                    tot.y = __fmul_rn(pow_rule(o.y, a.alpha, a.alpha_int), h[u].y);
                    tot.z = __fmul_rn(pow_rule(o.z, a.alpha, a.alpha_int), h[u].z);
                    tot.w = __fmul_rn(pow_rule(o.w, a.alpha, a.alpha_int), h[u].w);
                }
                // tau is read again only in the next pass: evict first; total_info stays in L2
                // for the candidate gather below and the next construct
                __stcs(tp + 32 * u, o);
                __stcg(op + 32 * u, tot);
            }
        }
    }
    __syncwarp(); // s_col / s_amt are reused by the warp's next row
}

// Depot row: every column may receive deposits (depot -> customer edges of
// every route of every elite), so each float4 takes the mask check.
__device__ __forceinline__ void update_depot_row(const UpdateArgs &a, int lane, int q4, float4 *tau4,
                                                 const float4 *heur4, float4 *tot4)
{
    for (int q = lane; q < q4; q += 32) {
        const float4 t = tau4[q], h = heur4[q];
        float v0 = __fmul_rn(a.evap, t.x), v1 = __fmul_rn(a.evap, t.y);
        float v2 = __fmul_rn(a.evap, t.z), v3 = __fmul_rn(a.evap, t.w);
        deposit4_depot(a, 4 * q, v0, v1, v2, v3);
        float4 o, tot;
        o.x = v0; o.y = v1; o.z = v2; o.w = v3;
        tot.x = __fmul_rn(pow_rule(v0, a.alpha, a.alpha_int), h.x);
        tot.y = __fmul_rn(pow_rule(v1, a.alpha, a.alpha_int), h.y);
        tot.z = __fmul_rn(pow_rule(v2, a.alpha, a.alpha_int), h.z);
        tot.w = __fmul_rn(pow_rule(v3, a.alpha, a.alpha_int), h.w);
        tau4[q] = o;
        tot4[q] = tot;
    }
}

// One warp, row i of instance a.  Columns are walked as float4 (ld is a
// multiple of 32; columns n..ld-1 stay zero).  s_col / s_amt: the warp's
// deposit slots (32 entries each).
__device__ __forceinline__ void row_pass(const UpdateArgs &a, int i, int mode, float trail, int lane, int *s_col,
                                         float *s_amt)
{
    const int n = a.n, q4 = (n + 3) >> 2;
    // the row's candidate ids, fetched with the row's first loads (ROW_GATHER reads them after the row)
    const int cid = a.chc && lane < a.K ? (int)__ldg(a.nn16 + (size_t)i * a.Kp + lane) : 0;
    const size_t off = (size_t)i * a.ld;
    const float4 *heur4 = reinterpret_cast<const float4 *>(a.heur + off);
    float4 *tau4 = reinterpret_cast<float4 *>(a.tau + off);
    float4 *tot4 = reinterpret_cast<float4 *>(a.total + off);
    if (mode == ROW_HEUR || mode == ROW_PRIOR) {
        // eta^beta; ROW_PRIOR multiplies it by the prior the heuristic matrix holds on entry
        const float4 *dist4 = reinterpret_cast<const float4 *>(a.dist + off);
        float4 *h4 = reinterpret_cast<float4 *>(a.heur + off);
        for (int q = lane; q < q4; q += 32) {
            const float4 d = dist4[q];
            const int c = 4 * q;
            float4 h;
            h.x = c + 0 < n ? pow_rule(__fdiv_rn(1.0f, __fadd_rn(d.x, 0.1f)), a.beta, a.beta_int) : 0.f;
            h.y = c + 1 < n ? pow_rule(__fdiv_rn(1.0f, __fadd_rn(d.y, 0.1f)), a.beta, a.beta_int) : 0.f;
            h.z = c + 2 < n ? pow_rule(__fdiv_rn(1.0f, __fadd_rn(d.z, 0.1f)), a.beta, a.beta_int) : 0.f;
            h.w = c + 3 < n ? pow_rule(__fdiv_rn(1.0f, __fadd_rn(d.w, 0.1f)), a.beta, a.beta_int) : 0.f;
            if (mode == ROW_PRIOR) {
                const float4 pr = h4[q];
                h.x = __fmul_rn(h.x, pr.x);
                h.y = __fmul_rn(h.y, pr.y);
                h.z = __fmul_rn(h.z, pr.z);
                h.w = __fmul_rn(h.w, pr.w);
            }
            h4[q] = h;
        }
        return;
    }
    if (mode == ROW_TOTAL) { // compute_total_info (kernel.cl:782-789) from the current tau and heur
        for (int q = lane; q < q4; q += 32) {
            const float4 t = tau4[q], h = heur4[q];
            float4 o;
            o.x = __fmul_rn(pow_rule(t.x, a.alpha, a.alpha_int), h.x);
            o.y = __fmul_rn(pow_rule(t.y, a.alpha, a.alpha_int), h.y);
            o.z = __fmul_rn(pow_rule(t.z, a.alpha, a.alpha_int), h.z);
            o.w = __fmul_rn(pow_rule(t.w, a.alpha, a.alpha_int), h.w);
            tot4[q] = o;
        }
    }
    if (mode == ROW_INIT_TRAIL || mode == ROW_INIT_BSF) { // pheromone_init (kernel.cl:672-679)
        const float tr = mode == ROW_INIT_BSF ? __fdiv_rn(1.0f, __fmul_rn(a.rho, *a.bsf_len)) : trail;
        const float pa = pow_rule(tr, a.alpha, a.alpha_int);
        for (int q = lane; q < q4; q += 32) {
            const float4 h = heur4[q];
            const int c = 4 * q;
            float4 t, o;
            t.x = c + 0 < n ? tr : 0.f; o.x = c + 0 < n ? __fmul_rn(pa, h.x) : 0.f;
            t.y = c + 1 < n ? tr : 0.f; o.y = c + 1 < n ? __fmul_rn(pa, h.y) : 0.f;
            t.z = c + 2 < n ? tr : 0.f; o.z = c + 2 < n ? __fmul_rn(pa, h.z) : 0.f;
            t.w = c + 3 < n ? tr : 0.f; o.w = c + 3 < n ? __fmul_rn(pa, h.w) : 0.f;
            tau4[q] = t;
            tot4[q] = o;
        }
    } else if (mode == ROW_UPDATE) {
        if (i == 0) {
            update_depot_row(a, lane, q4, tau4, heur4, tot4);
        } else {
            if (a.alpha_int == 1) update_row_stream<kU, true>(a, i, lane, q4, tau4, heur4, tot4, s_col, s_amt);
            else update_row_stream<1, false>(a, i, lane, q4, tau4, heur4, tot4, s_col, s_amt);
        }
    }
    if (a.chc) { // compact candidate table: chc[i][j] = 1 / total[i][nn[i][j]] (the race's reciprocal weight)
        // the row was written by this warp; __syncwarp orders those stores before
        // the re-reads below, which read L2, where the lines were just written
        __syncwarp();
        if (lane < a.K) a.chc[(size_t)i * a.Kp + lane] = __fdiv_rn(1.0f, __ldcg(a.total + off + cid));
    }
}

// Global row g (over the instances' rows in order) belongs to instance
// row_inst[g] (null: a single instance); row_base[b] is instance b's first.
template <int MODE>
__global__ void __launch_bounds__(kRowWarps * 32, 4) rows_kernel(const UpdateArgs *args, const int *row_base,
                                                                 const int *row_inst, int total_rows, float trail)
{
    constexpr int mode = MODE;
    __shared__ int s_col[kRowWarps][32];
    __shared__ float s_amt[kRowWarps][32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nw = (gridDim.x * blockDim.x) >> 5;
    for (int g = gw; g < total_rows; g += nw) {
        const int b = row_inst ? __ldg(row_inst + g) : 0;
        row_pass(args[b], g - __ldg(row_base + b), mode, trail, lane, s_col[warp], s_amt[warp]);
    }
}

__global__ void t0_kernel(unsigned long long *t0) { *t0 = globaltimer_ns(); }

// init_aco's per-instance resets: no best-so-far yet (+inf), no records, iteration 0.
__global__ void reset_slots_kernel(const StatsArgs *args, int count)
{
    for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < count; b += gridDim.x * blockDim.x) {
        const StatsArgs a = args[b];
        a.lens[a.n_ants] = __int_as_float(0x7f800000);
        *a.num_bsf = 0;
        *a.iteration = 0;
    }
}

} // namespace

cudaError_t launch_stats(const StatsArgs *d_args, int n_inst, int do_elites, size_t smem, cudaStream_t st,
                         const StatsArgs *one)
{
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(stats_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    // the construct and 2-opt kernels before it run with the largest shared
    // memory carve-out; asking for the same avoids reconfiguring the SMs
    cudaError_t e = cudaFuncSetAttribute(stats_kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    // one thread per ant (smem holds one length per ant), at least 8 and at most 32 warps:
    // fewer warps make every block barrier cheaper
    int threads = (int)((smem / sizeof(float) + 31) / 32 * 32);
    threads = threads < 256 ? 256 : (threads > 1024 ? 1024 : threads);
    stats_kernel<<<n_inst, threads, smem, st>>>(one ? nullptr : d_args, one ? *one : StatsArgs{}, do_elites);
    return cudaGetLastError();
}

cudaError_t launch_rows(const UpdateArgs *d_args, const int *d_row_base, const int *d_row_inst, int total_rows,
                        int mode, float trail, int sm_count, cudaStream_t st)
{
    int blocks = (total_rows + kRowWarps - 1) / kRowWarps; // one warp per row
    const int cap = sm_count * 4;      // grid-stride beyond 4 CTAs (32 warps) per SM
    if (blocks > cap) blocks = cap;
    if (blocks < 1) blocks = 1;
    switch (mode) {
    case ROW_HEUR: rows_kernel<ROW_HEUR><<<blocks, kRowWarps * 32, 0, st>>>(d_args, d_row_base, d_row_inst, total_rows, trail); break;
    case ROW_INIT_TRAIL:
        rows_kernel<ROW_INIT_TRAIL><<<blocks, kRowWarps * 32, 0, st>>>(d_args, d_row_base, d_row_inst, total_rows, trail);
        break;
    case ROW_INIT_BSF:
        rows_kernel<ROW_INIT_BSF><<<blocks, kRowWarps * 32, 0, st>>>(d_args, d_row_base, d_row_inst, total_rows, trail);
        break;
    case ROW_UPDATE:
        rows_kernel<ROW_UPDATE><<<blocks, kRowWarps * 32, 0, st>>>(d_args, d_row_base, d_row_inst, total_rows, trail);
        break;
    case ROW_PRIOR:
        rows_kernel<ROW_PRIOR><<<blocks, kRowWarps * 32, 0, st>>>(d_args, d_row_base, d_row_inst, total_rows, trail);
        break;
    case ROW_TOTAL:
        rows_kernel<ROW_TOTAL><<<blocks, kRowWarps * 32, 0, st>>>(d_args, d_row_base, d_row_inst, total_rows, trail);
        break;
    default: rows_kernel<ROW_GATHER><<<blocks, kRowWarps * 32, 0, st>>>(d_args, d_row_base, d_row_inst, total_rows, trail); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_reset_slots(const StatsArgs *d_args, int count, cudaStream_t st)
{
    reset_slots_kernel<<<(count + 255) / 256, 256, 0, st>>>(d_args, count);
    return cudaGetLastError();
}

cudaError_t launch_t0(unsigned long long *t0, cudaStream_t st)
{
    t0_kernel<<<1, 1, 0, st>>>(t0);
    return cudaGetLastError();
}

} // namespace aco
