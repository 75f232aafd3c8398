// kernels.h -- argument blocks and host launchers of the sm_100a kernels.
//
// Device layout of one instance (all allocations 256-byte aligned):
//   dist, heur, tau, total : n x ld fp32, ld = round_up(n, 32) (128-byte rows);
//                            heur = (1/(d+0.1))^beta, precomputed once
//   demand, tiekey         : n entries, padded to a multiple of 4
//   solutions              : T*(A+1)+1 int32 in the reference layout, T = 2n
//   lens                   : A+1 fp32 (slot A = best so far)
//   seeds                  : A*nloc int32 (one Park-Miller state per work-item lane)
//   nn_ls_list             : n x nn_ls int32 (2-opt); nn16 / cand32 : n x Kp candidate
//                            lists (uint16 node ids / node | demand << 16)
//   chc                    : n x Kp fp32, 1 / total_info of every candidate (throughput
//                            mode: the race's reciprocal weights), written by the pheromone pass
//
// Every kernel except the parity construct reads its instance from an array of
// argument blocks in device memory, so one launch serves one instance or a
// batch of independent instances of different sizes (the batch is a
// concatenation of per-instance buffers; each block holds its own pointers).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/cvrp_aco.h"

namespace aco {

struct ConstructArgs {
    int n, ld, n_ants, T, nloc, log2_nloc, kmax;
    int capacity;
    float max_dist, serv_time;
    const float *total;    // n x ld
    const float *dist;     // n x ld
    const int *demand;     // n (padded)
    const uint32_t *tiekey;// n (padded): ((0xFFFF - prio) << 16) | node
    const uint32_t *jump;  // kmax (padded): 16807^(k+1) mod m
    const uint32_t *adv;   // nloc: 16807^(draws of lane l per step) mod m
    const uint16_t *nn16;  // n x Kp candidate lists (throughput), uint16 node ids
    const uint32_t *cand32;// n x Kp candidate lists, packed node | demand << 16
    const float *chc;      // n x Kp: 1 / total_info of the candidates (+inf for weight 0)
    int K, Kp;             // candidate-list length and padded row length (multiple of 8)
    int smat;              // throughput construct: stage the whole total_info matrix
    int packed;            // throughput construct: use cand32 (else nn16 + demand lookups)
    int gtab;              // throughput construct: read the candidate table from global memory (not staged)
    // fused 2-opt (throughput construct with improving warps): the 2-opt lists, the
    // pass limit, and per global ant whether the 2-opt kernel still has to run
    const int *nn_list;    // n x nn_ls
    int nn_ls, pass_limit, ant_base;
    int ls_best;           // the fused 2-opt improves best-first (aco_params.ls_best)
    uint8_t *ls_needed;    // total ants of the colony
    // route list for the route-level 2-opt (null: not used): every route of at
    // most 255 nodes as {global ant, first position | nodes << 16}; route_ctr[0]
    // counts the entries (capacity route_cap), route_rem[g] the entries of ant g.
    // ls_needed[g]: 2 = none of its routes listed (a longer route, or the list
    // was full) -- the per-ant kernel does those; 1 (fused construct only) = the
    // ant's routes of more than 32 nodes are left to the per-ant kernel.
    int2 *route_desc;
    int *route_ctr, *route_rem;
    int route_cap;
    // the ants whose ls_needed is set, listed for the per-ant 2-opt kernel
    // (route-list mode): ls_list_ctr[0] entries, capacity = the colony's ants
    int *ls_list, *ls_list_ctr;
    int *seeds;
    int *solutions;
    float *lens;
    int *status;
    const int *wait_limit; // polls before a staging wait gives up (device word; <= 0: the default)
};

struct LocalSearchArgs {
    int n, ld, n_ants, T, nn_ls, rmax, pass_limit;
    int best;              // 1: best-improvement 2-opt for routes of at most 32 nodes (aco_params.ls_best)
    const float *dist;     // n x ld
    const int *nn_list;    // n x nn_ls
    int *solutions;
    float *lens;
    int *status;
};

struct StatsArgs {
    int n, n_ants, T, nloc, log2_nloc, ras_ranks, record_cap;
    int do_elites;         // unused on the device (passed per launch)
    int *solutions;
    float *lens;
    int *elites;           // ras_ranks
    int *succ;             // ras_ranks x n: successor of customer i in elite r's tour (-1 if none)
    uint32_t *depmask;     // n: bit r set if elite r's tour goes depot -> i
    float *d_tau;          // ras_ranks: weight / length of elite r
    int *num_bsf;
    aco_record *records;   // record_cap x {iter, length, time}
    int *iteration;        // device iteration counter (incremented here)
    const unsigned long long *t0_ns; // globaltimer at init_aco
    int *status;
};

struct UpdateArgs {
    int n, ld;
    int ras_ranks;
    float evap;              // 1.0f - rho
    float alpha, beta;
    int alpha_int, beta_int; // exponents as integers in [0, 8], or -1
    float rho;
    float *tau;
    float *total;
    float *heur;
    const float *dist;
    const int *succ;
    const uint32_t *depmask;
    const float *d_tau;
    const float *bsf_len;    // lens[A] (trail_0 = 1/(rho * bsf))
    float *chc;              // n x Kp reciprocal candidate weights, or null (no candidate table)
    const uint16_t *nn16;    // n x Kp
    int K, Kp;
};

// Per-row pass modes of the row kernel.
enum RowMode {
    ROW_HEUR = 0,       // heur = eta^beta
    ROW_INIT_TRAIL = 1, // tau = trail, total = trail^alpha * heur
    ROW_INIT_BSF = 2,   // same with trail = 1 / (rho * best-so-far length)
    ROW_UPDATE = 3,     // evaporation + deposit + total_info
    ROW_GATHER = 4,     // candidate table from total_info
    ROW_PRIOR = 5,      // heur = eta^beta * (prior held in heur on entry)
    ROW_TOTAL = 6,      // total = tau^alpha * heur
};

// Launchers (stream-ordered; return cudaGetLastError()).  `d_*args` point to
// arrays of argument blocks in device memory, one per instance.
// Staged host -> device uploads: the pieces of one blob copied to their
// destinations by one kernel.
// The ants' lane seeds on the device (same values as make_seeds on the host).

struct ScatterPiece {
    unsigned long long dst, src_off, bytes;
};
cudaError_t launch_scatter(const ScatterPiece *d_pieces, int count, const unsigned char *d_blob,
                           unsigned long long total_bytes, int sm_count, cudaStream_t st);

cudaError_t launch_construct_parity(const ConstructArgs &a, int warps_per_ant, int ants_per_block, bool stage_total,
                                    cudaStream_t st);
// Throughput construct, persistent: CTAs pull work items {instance, first ant}
// from d_queue[0]; d_queue[1] counts finished CTAs.  Both start at 0 and the
// last CTA to finish sets them back to 0, so consecutive launches need no reset.
// ls_warps > 0: each CTA also runs that many 2-opt warps that improve the
// routes of its ants as soon as they are complete (all instances n <= 1024,
// candidate tables staged); ants with a route of more than 32 nodes are marked
// in ls_needed for the 2-opt kernel.
// lens_later: the route-level 2-opt follows in the same iteration and writes
// the lengths of every ant it gets from the route list; the construct leaves
// them out for instances that have the list.
// wide (no helper draws, no fused 2-opt): the 64-register kernel that runs two
// CTAs per SM; `smem` must then leave room for the second CTA.
cudaError_t launch_construct_nn(const ConstructArgs *d_args, const int2 *d_items, int n_items, int *d_queue,
                                int ants_per_cta, size_t smem, int sm_count, bool finite_maxd, cudaStream_t st,
                                int ls_warps = 0, bool draw = false, bool lens_later = false, bool wide = false);
// 2-opt: one CTA of `warps` warps per ant; d_ant_inst[g] = instance of global ant g,
// d_ant_base[b] = first global ant of instance b.
// Route-level 2-opt over the construct's route list (d_ctr: {entries, next,
// CTAs done}, rewound by the kernel); a persistent grid of `warps`-warp CTAs.
size_t route_opt_smem(int n_max, int warps);
cudaError_t launch_route_opt(const LocalSearchArgs *d_args, const int *d_ant_inst, const int *d_ant_base,
                             const int2 *d_desc, int *d_ctr, int cap, int *d_rem, const uint8_t *d_flagged, int n_max,
                             int warps, int sm_count, cudaStream_t st);
// 2-opt: CTAs of `ants_per_cta` ants (1..8) and `warps` warps pulling routes;
// n_max sizes the per-ant shared buffers.  only (after a fused construct or the
// route-level kernel): skip ants whose flag is 0 and, in the others, routes of
// at most 32 nodes when the flag is 1.  list / list_ctr (with only): the flagged
// ants as the construct listed them (list_ctr[0] entries), taken by a
// persistent grid of at most sm_count x occupancy CTAs, which rewinds the list.
cudaError_t launch_local_search(const LocalSearchArgs *d_args, const int *d_ant_inst, const int *d_ant_base,
                                int total_ants, int ants_per_cta, int n_max, int warps, size_t smem, cudaStream_t st,
                                const uint8_t *only = nullptr, const int *list = nullptr, int *list_ctr = nullptr,
                                int sm_count = 148);
// one: a single instance's arguments passed by value (d_args unused)
cudaError_t launch_stats(const StatsArgs *d_args, int n_inst, int do_elites, size_t smem, cudaStream_t st,
                         const StatsArgs *one = nullptr);
// Row passes (heuristic matrix, pheromone init, fused update, candidate gather):
// one warp per row over all instances; d_row_base[b] = first global row of instance b,
// d_row_inst[g] = the instance of global row g (null: one instance).
cudaError_t launch_rows(const UpdateArgs *d_args, const int *d_row_base, const int *d_row_inst, int total_rows,
                        int mode, float trail, int sm_count, cudaStream_t st);
// lens[A] = +inf, num_bsf = 0, iteration = 0 of every instance (init_aco).
cudaError_t launch_reset_slots(const StatsArgs *d_args, int count, cudaStream_t st);
cudaError_t launch_t0(unsigned long long *t0, cudaStream_t st);

// Shared-memory bytes of the launches (the host picks configurations that fit
// the 227 KB per-CTA limit).
size_t construct_parity_smem(int n, int nloc, int kmax, int warps_per_ant, int ants_per_block, bool stage_total,
                             bool finite_maxd);
// draw: a helper warp per ant makes the race draws ahead (ants_per_cta <= 8;
// ignored with ls_warps > 0)
size_t construct_nn_smem(int n, int K, int Kp, int ants_per_cta, bool stage_total, bool packed,
                         bool global_table = false, int ls_warps = 0, bool draw = false);
size_t local_search_smem(int n_max, int ants_per_cta, int warps);
// resident 2-opt CTAs per SM for this shape (0 = cannot launch)
int local_search_occupancy(int warps, size_t smem);

// Tour validation (validate.cu): flags[slot_base[b] + s] = 1 if slot s of
// instance b (ants, then best-so-far) is a valid tour whose stored length is
// exact; invalid[b] counts the others (zeroed by the caller).
cudaError_t launch_validate(const ConstructArgs *d_args, int n_inst, int max_slots, int max_n, int *flags,
                            const int *slot_base, int *invalid, cudaStream_t st);
// The best-so-far tour, size and length of every instance, packed (validate.cu):
// instance b's 2n ints at tours + tour_base[b], sizes[b], lens[b].
cudaError_t launch_gather_best(const ConstructArgs *d_args, int n_inst, const int *d_tour_base, int *tours,
                               int *sizes, float *lens, cudaStream_t st);

// Inter-route swap stage (swap.cu): one CTA per item {instance, first ant}
// with `apc` ants (one warp each).
size_t swap_smem(int n, int ld, int apc);
cudaError_t launch_swap(const ConstructArgs *d_args, const int2 *d_items, int n_items, int apc, size_t smem,
                        int max_swaps_per_node, cudaStream_t st);

// Random-descent stage (ns.cu): one CTA per item {instance, first ant} with
// `apc` ants, `rounds` neighbourhood-move proposals per ant.
size_t ns_smem(int n, int apc);
cudaError_t launch_ns(const ConstructArgs *d_args, const StatsArgs *d_sargs, const int2 *d_items, int n_items, int apc,
                      size_t smem, int rounds, int rnd_seed, cudaStream_t st);

// Device preprocessing (prep.cu).
bool device_dist_supported(int dist_type);
size_t nn_rows_per_cta(int n);
cudaError_t launch_dist(int n, const float *x, const float *y, int dist_type, float *dist, int ld, int sm_count,
                        cudaStream_t st);
cudaError_t launch_nn(int n, const float *dist, int ld, int depth, int *nn, int *status, cudaStream_t st);

// One instance's inputs and outputs of the batched preprocessing.
struct PrepArgs {
    int n, ld, depth, K, Kp, nn_ls, dist_type;
    int device_prep; // 0: distances and lists came from the host (skipped here, seeds still made)
    int n_ants;
    const float *x, *y;
    float *dist;
    const int *demand;
    uint16_t *nn16;   // n x Kp: first K of the list, padded with node 0
    uint32_t *cand32; // n x Kp: the same with the demand in the high half
    int *nnls;        // n x nn_ls: the 2-opt list
    int *seeds;       // n_ants x nloc
};
// Every instance of a batch in one launch per step (global row g: row g -
// row_base[b] of instance b = row_inst[g]; global ant g: ant g - ant_base[b] of
// b = ant_inst[g]): distances, then the lists (the reference's quicksort per
// row) with the candidate and 2-opt tables, then the lane seeds (rnd_seed + b).
cudaError_t launch_prep_batch(const PrepArgs *d_args, const int *d_row_base, const int *d_row_inst, int total_rows,
                              int n_max, const int *d_ant_base, const int *d_ant_inst, int total_ants, int nloc,
                              int seed_time, int rnd_seed, int *status, int sm_count, cudaStream_t st);

} // namespace aco
