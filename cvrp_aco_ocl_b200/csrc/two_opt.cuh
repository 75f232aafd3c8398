// two_opt.cuh -- the register path of the route 2-opt (first improvement in
// sequence order with don't-look bits, kernel.cl:126-277) for routes of at most
// 32 nodes, shared by the 2-opt kernel and the construct kernel that improves
// routes while later ones are still being built.
//
// Lane q holds the local node at route position q (tq), the length of the edge
// leaving position q (dq, dist_tour_wrk) and the position of local node q (pk);
// the don't-look bits are one warp-uniform mask; `tile` is the route's 32x32
// distance sub-matrix; lnn / lcnt are every local node's neighbour list
// filtered to the route, in list order.  The scan only stops on in-route
// entries, so the filtered lists decide exactly as the full ones.
#pragma once

#include <cstdint>

#include "aco_device.cuh"

namespace aco {
namespace {

constexpr int kRL = 32; // largest route (nodes, depot included) of the register path

constexpr unsigned kFullMask = 0xffffffffu;

// The 2-opt move that replaces edges (h1,h2) and (h3,h4) by (h1,h3) and (h2,h4)
// (kernel.cl:235-270) on the lane-per-position state: the positions between
// the two edges are reversed and dist_tour_wrk follows them.
__device__ __forceinline__ void route_exchange(int lane, const float *tile, int h1, int h2, int h3, int h4, int &tq,
                                               int &pk, float &dq)
{
    const unsigned FULLM = 0xffffffffu;
    int p1 = __shfl_sync(FULLM, pk, h1), p3 = __shfl_sync(FULLM, pk, h3);
    if (p3 < p1) {
        int t = h1; h1 = h3; h3 = t;
        t = h2; h2 = h4; h4 = t;
        t = p1; p1 = p3; p3 = t;
    }
    const int i = p1, jj = p3, a = __shfl_sync(FULLM, pk, h2);
    const float d13 = tile[h1 * kRL + h3], d24 = tile[h2 * kRL + h4];
    // dist_tour_wrk: [i] = d(h1,h3), [jj] = d(h2,h4), (i, jj) reversed
    const float dsrc = __shfl_sync(FULLM, dq, (lane > i && lane < jj) ? i + jj - lane : lane);
    if (lane == jj) dq = d24; // written after [i], as kernel.cl:249-250
    else if (lane == i) dq = d13;
    else if (lane > i && lane < jj) dq = dsrc;
    // tour positions [a, jj] reversed; positions of the moved nodes mirrored
    const int tsrc = __shfl_sync(FULLM, tq, (lane >= a && lane <= jj) ? a + jj - lane : lane);
    if (lane >= a && lane <= jj) tq = tsrc;
    if (pk >= a && pk <= jj) pk = a + jj - pk;
}

// ---------------------------------------------------------------------------
// Register path: routes of at most 32 nodes.
// ---------------------------------------------------------------------------
__device__ int two_opt_route_regs(int lane, int R, bool first_route, const float *tile, const uint8_t *lnn,
                                  const uint8_t *lcnt, int &tq, int &pk, float &dq, int pass_limit)
{
    // lane q: tq = local node at position q, dq = dist_tour_wrk of position q;
    // lane k: pk = position of local node k.  Local node 0 is the depot at position 0.
    //
    // The scan visits positions q1 = 0, 1, ..., R-1 and skips a node whose
    // don't-look bit is set.  `open` holds one bit per position whose node's bit
    // is clear, rebuilt whenever a move changes the tour or the bits, so the next
    // position to examine is a bit operation away.  For each examined node the
    // successor and the predecessor searches (kernel.cl:180-198, 202-230) are
    // evaluated together; the predecessor result is used only when the successor
    // search finds no move, as in the sequential code.
    const unsigned FULLM = 0xffffffffu;
    const unsigned rmask = R >= 32 ? FULLM : ((1u << R) - 1u);
    // lane k, by local node: the nodes after and before it on the tour, and the
    // dist_tour_wrk entries at its position and the one before (position 0: its
    // own), rebuilt after every move
    int nsucc, npred;
    float dout, din;
    auto by_node = [&]() {
        nsucc = __shfl_sync(FULLM, tq, pk + 1 < R ? pk + 1 : 0);
        npred = __shfl_sync(FULLM, tq, pk > 0 ? pk - 1 : R - 1);
        dout = __shfl_sync(FULLM, dq, pk);
        din = __shfl_sync(FULLM, dq, pk > 0 ? pk - 1 : 0);
    };
    by_node();
    uint32_t dlb = first_route ? 0u : 1u; // bit k: don't-look bit of local node k
    int passes = 0;
    bool imp = true;
    // the first half of an examination: node k1 at position q, its tour
    // neighbours, its filtered list entry for this lane and the radii.  It
    // depends only on q and the tour, so the next open position's is loaded
    // while the current examination's ballots resolve (used when no move
    // happens, which is the common case; recomputed after a move).
    struct Head {
        int k1, ks1, kp1, k2;
        bool act;
        float d12, rs, rp;
    };
    auto head = [&](int q) {
        Head h;
        h.k1 = __shfl_sync(FULLM, tq, q);
        h.ks1 = __shfl_sync(FULLM, tq, q + 1 < R ? q + 1 : 0);
        h.kp1 = __shfl_sync(FULLM, tq, q > 0 ? q - 1 : R - 1);
        h.act = lane < (int)lcnt[h.k1];
        h.k2 = h.act ? lnn[h.k1 * kRL + lane] : 0;
        h.d12 = tile[h.k1 * kRL + h.k2];
        h.rs = tile[h.k1 * kRL + h.ks1]; // successor radius
        h.rp = tile[h.kp1 * kRL + h.k1]; // predecessor radius
        return h;
    };
    while (imp) {
        if (pass_limit > 0 && passes >= pass_limit) return ACO_ERR_LS_LIMIT;
        passes++;
        imp = false;
        uint32_t open = __ballot_sync(FULLM, lane < R && !((dlb >> tq) & 1u)) & rmask;
        if (!open) break;
        int q1 = __ffs(open) - 1;
        Head h = head(q1);
        for (;;) {
            const int k1 = h.k1, ks1 = h.ks1, kp1 = h.kp1, k2 = h.k2;
            const bool act = h.act;
            const float d12 = h.d12, rs = h.rs, rp = h.rp;
            // k2's neighbours on the tour and edge lengths, one shuffle level from k2
            const int ks2 = __shfl_sync(FULLM, nsucc, k2);
            const int kpp2 = __shfl_sync(FULLM, npred, k2);
            const float dq2 = __shfl_sync(FULLM, dout, k2);
            const float dqp2 = __shfl_sync(FULLM, din, k2);
            const bool sc = act && __fsub_rn(rs, d12) > kEps;
            const bool pc = act && __fsub_rn(rp, d12) > kEps;
            bool sok = false, pok = false;
            if (sc) {
                const float g = __fsub_rn(__fadd_rn(__fadd_rn(-rs, d12), tile[ks1 * kRL + ks2]), dq2);
                sok = g < -kEps;
            }
            if (pc && !(kpp2 == k1 || kp1 == k2)) {
                const float g = __fsub_rn(__fadd_rn(__fadd_rn(-rp, d12), tile[kp1 * kRL + kpp2]), dqp2);
                pok = g < -kEps;
            }
            // the scan stops at the first lane whose entry ends it: past the radius, or
            // an improving move (kernel.cl:180-198, 202-230); found = that lane moves
            const unsigned sstop = __ballot_sync(FULLM, act && (!sc || sok));
            const unsigned pstop = __ballot_sync(FULLM, act && (!pc || pok));
            const unsigned smove = __ballot_sync(FULLM, sok), pmove = __ballot_sync(FULLM, pok);
            // the next open position if this examination makes no move, and its head
            const uint32_t rest = open & ~((2u << q1) - 1u); // positions > q1 (2u << 31 wraps to 0: none)
            const int qn = __ffs(rest) - 1;                   // -1 when none (the head is then unused)
            const Head hn = head(qn);
            const bool sfound = (sstop & (0u - sstop) & smove) != 0u; // the lowest stop is a move
            const bool pfound = (pstop & (0u - pstop) & pmove) != 0u;
            int h1, h2, h3, h4;
            if (sfound) {
                const int sf = __ffs(sstop) - 1;
                h1 = k1;
                h2 = ks1;
                h3 = __shfl_sync(FULLM, k2, sf);
                h4 = __shfl_sync(FULLM, ks2, sf);
            } else if (pfound) {
                const int pf = __ffs(pstop) - 1;
                h1 = kp1;
                h2 = k1;
                h3 = __shfl_sync(FULLM, kpp2, pf);
                h4 = __shfl_sync(FULLM, k2, pf);
            } else {
                dlb |= 1u << k1; // kernel.cl:232
                open &= ~(1u << q1);
                if (!rest) break;
                q1 = qn;
                h = hn;
                continue;
            }
            // exchange (kernel.cl:235-270)
            imp = true;
            dlb &= ~((1u << h1) | (1u << h2) | (1u << h3) | (1u << h4));
            route_exchange(lane, tile, h1, h2, h3, h4, tq, pk, dq);
            by_node();
            open = __ballot_sync(FULLM, lane < R && !((dlb >> tq) & 1u)) & rmask; // the tour and bits changed
            const uint32_t ahead = open & ~((2u << q1) - 1u); // the scan goes on after q1
            if (!ahead) break;
            q1 = __ffs(ahead) - 1;
            h = head(q1);
        }
    }
    return ACO_OK;
}

// ---------------------------------------------------------------------------
// Best improvement (a non-parity option: the reference improves first in scan
// order): every 2-opt move of the route -- reverse positions i+1..j, 0 <= i <
// j <= R-1, the position after R-1 being the depot at 0 -- is evaluated at once
// from the route's distance tile, lane j taking the pairs (i, j) of one i at a
// time; a warp argmin picks the most negative change of the tour length (ties:
// the lowest (i, j)), which is applied while it is below -EPSILON.  tpos: 32
// bytes of the warp's shared memory for the local node at every position.  At
// most move_limit moves (then ACO_ERR_LS_LIMIT).
// ---------------------------------------------------------------------------
__device__ int two_opt_route_best(int lane, int R, const float *tile, uint8_t *tpos, int &tq, int &pk, float &dq,
                                  int move_limit)
{
    const unsigned FULLM = 0xffffffffu;
    for (int moves = 0;; moves++) {
        if (lane < R) tpos[lane] = (uint8_t)tq;
        __syncwarp();
        unsigned long long best = ~0ull;
        const int j = lane, tj = lane < R ? tpos[lane] : 0, tj1 = lane + 1 < R ? tpos[lane + 1] : tpos[0];
        for (int i = 0; i + 1 < R; i++) {
            if (j > i && j < R) {
                const int ti = tpos[i], ti1 = tpos[i + 1];
                const float add = __fadd_rn(tile[ti * kRL + tj], tile[ti1 * kRL + tj1]);
                const float rem = __fadd_rn(tile[ti * kRL + ti1], tile[tj * kRL + tj1]);
                const uint32_t b = __float_as_uint(__fsub_rn(add, rem));
                const uint32_t ord = (b & 0x80000000u) ? ~b : (b | 0x80000000u); // ascending as the floats
                const unsigned long long key = ((unsigned long long)ord << 32) | (unsigned)(i << 8 | j);
                best = key < best ? key : best;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long w = __shfl_xor_sync(FULLM, best, o);
            best = w < best ? w : best;
        }
        __syncwarp();
        if (best == ~0ull) break;
        const uint32_t ord = (uint32_t)(best >> 32);
        const uint32_t b = (ord & 0x80000000u) ? (ord & 0x7fffffffu) : ~ord;
        if (!(__uint_as_float(b) < -kEps)) break;
        if (move_limit > 0 && moves >= move_limit) return ACO_ERR_LS_LIMIT;
        const int i = (int)((best >> 8) & 0xffu), jj = (int)(best & 0xffu);
        // the exchange of the first-improvement path with h1..h4 = the nodes at i, i+1, jj, jj+1
        const int h1 = tpos[i], h2 = tpos[i + 1], h3 = tpos[jj], h4 = jj + 1 < R ? tpos[jj + 1] : tpos[0];
        const int a = i + 1;
        const float d13 = tile[h1 * kRL + h3], d24 = tile[h2 * kRL + h4];
        const float dsrc = __shfl_sync(FULLM, dq, (lane > i && lane < jj) ? i + jj - lane : lane);
        if (lane == jj) dq = d24;
        else if (lane == i) dq = d13;
        else if (lane > i && lane < jj) dq = dsrc;
        const int tsrc = __shfl_sync(FULLM, tq, (lane >= a && lane <= jj) ? a + jj - lane : lane);
        if (lane >= a && lane <= jj) tq = tsrc;
        if (pk >= a && pk <= jj) pk = a + jj - pk;
    }
    return ACO_OK;
}

} // namespace
} // namespace aco
