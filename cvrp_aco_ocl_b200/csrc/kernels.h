// kernels.h -- argument blocks and host launchers of the sm_100a kernels.
//
// Device layout of one instance (all allocations 256-byte aligned):
//   dist, heur, tau, total : n x ld fp32, ld = round_up(n, 32) (128-byte rows);
//                            heur = (1/(d+0.1))^beta, precomputed once
//   demand, tiekey         : n entries, padded to a multiple of 4
//   solutions              : T*(A+1)+1 int32 in the reference layout, T = 2n
//   lens                   : A+1 fp32 (slot A = best so far)
//   seeds                  : A*nloc int32 (one Park-Miller state per work-item lane)
//   nn_ls_list             : n x nn_ls int32 (2-opt); nn16 : n x Kp uint16 (candidate lists)
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
    int K, Kp;             // candidate-list length and padded row length (multiple of 8)
    int ants_per_cta;      // throughput construct: ant warps per CTA (the CTA may have helper warps)
    int *seeds;
    int *solutions;
    float *lens;
    int *status;
};

struct LocalSearchArgs {
    int n, ld, n_ants, T, nn_ls, rmax, pass_limit;
    const float *dist;     // n x ld
    const int *nn_list;    // n x nn_ls
    int *solutions;
    float *lens;
    int *status;
};

struct StatsArgs {
    int n, n_ants, T, nloc, log2_nloc, ras_ranks, record_cap;
    int do_elites;         // 0 in the bootstrap of init_aco (g_aco.cpp:87)
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
    int n, ld, q;            // q = float4 chunks per row
    unsigned long long qinv; // ceil(2^40 / q): row = (u * qinv) >> 40
    int ras_ranks;
    float evap;              // 1.0f - rho
    float alpha;
    int alpha_int;           // alpha as an integer exponent in [0, 8], or -1
    float *tau;
    float *total;
    const float *heur;
    const int *succ;
    const uint32_t *depmask;
    const float *d_tau;
};

struct InitArgs {
    int n, ld;
    float trail;             // used when from_bsf == 0
    int from_bsf;            // trail = 1/(rho * lens[A]) (g_aco.cpp:89)
    float rho, alpha;
    int alpha_int;
    const float *bsf_len;
    float *tau;
    float *total;
    const float *heur;
};

// Launchers (stream-ordered; return cudaGetLastError()).
cudaError_t launch_heur(const float *dist, float *heur, int n, int ld, float beta, int beta_int, cudaStream_t st);
cudaError_t launch_pheromone_init(const InitArgs &a, cudaStream_t st);
cudaError_t launch_construct_parity(const ConstructArgs &a, int warps_per_ant, int ants_per_block, bool stage_total,
                                    cudaStream_t st);
cudaError_t launch_construct_nn(const ConstructArgs &a, int ants_per_block, bool stage_total, bool packed,
                                cudaStream_t st);
cudaError_t launch_local_search(const LocalSearchArgs &a, int ants_per_block, bool stage_nn, cudaStream_t st);
cudaError_t launch_stats(const StatsArgs &a, cudaStream_t st);
cudaError_t launch_pheromone_update(const UpdateArgs &a, int sm_count, cudaStream_t st);
cudaError_t launch_t0(unsigned long long *t0, cudaStream_t st);

// Shared-memory bytes the launchers request (the host picks configurations
// that fit the 227 KB per-CTA limit).
size_t construct_parity_smem(int n, int nloc, int kmax, int warps_per_ant, int ants_per_block, bool stage_total,
                             bool finite_maxd);
size_t construct_nn_smem(int n, int K, int Kp, int ants_per_block, bool stage_total, bool packed);
size_t local_search_smem(int n, int nn_ls, int rmax, int ants_per_block, bool stage_nn);

} // namespace aco
