// colony.h -- device state of one or more independent CVRP instances (a
// "colony" each) and the launch sequence of one ACO iteration over all of them.
// A single solver is a colony of one instance; a batch is a colony of many,
// all in one device arena, served by the same launches.
#pragma once

#include <cuda_runtime.h>

#include <chrono>
#include <cstdint>
#include <vector>

#include "../../include/cvrp_aco.h"
#include "kernels.h"

namespace aco {

// The last CUDA error a library call turned into ACO_ERR_CUDA on this thread
// (aco_last_cuda_error reports it).
void note_cuda_error(cudaError_t e);
cudaError_t last_cuda_error();

struct InstanceSpec { // the fields of aco_instance
    int n;
    const float *x, *y;
    const int *demand;
    int capacity;
    float max_dist, serv_time;
    int dist_type;
    const float *dist;
};

struct InstHost {
    int n = 0, ld = 0, n4 = 0, A = 0, T = 0, K = 0, Kp = 8, nn_ls = 0, R = 0, nloc = 0, lg = 0, kmax = 0;
    int capacity = 0;
    float max_dist = 0, serv_time = 0;
    uint64_t data_hash = 0;  // FNV-1a of the instance's data (checkpoint identity)
    uint64_t prior_hash = 0; // of the prior set by set_prior (0: none)
    bool smat = false, packed = false, gtab = false;
    bool device_prep = false;              // distances and lists computed on the device
    const float *x = nullptr, *y = nullptr; // caller's coordinates (valid during create)
    int dist_type = 0;
    std::vector<float> dist; // n*n
    std::vector<int> demand;
    std::vector<int> nn;     // n x depth
    int depth = 0;
    // device pointers inside the arena
    float *dist_d = nullptr, *heur_d = nullptr, *tau_d = nullptr, *total_d = nullptr, *chc_d = nullptr;
    int *dem_d = nullptr, *nnls_d = nullptr, *seeds_d = nullptr, *sol_d = nullptr, *elites_d = nullptr;
    int *succ_d = nullptr, *nbsf_d = nullptr, *iter_d = nullptr;
    uint32_t *key_d = nullptr, *jump_d = nullptr, *adv_d = nullptr, *cand32_d = nullptr, *dep_d = nullptr;
    uint16_t *nn16_d = nullptr;
    float *xy_d = nullptr; // device preprocessing: coordinates (x, then y at n4)
    float *lens_d = nullptr, *dtau_d = nullptr;
    aco_record *rec_d = nullptr;
};

class Colony {
public:
    ~Colony();
    // Host preprocessing (distances, NN lists, seeds, tables), one device arena,
    // uploads.  `parity` allows ACO_MODE_PARITY (single instance only).
    int create(const InstanceSpec *specs, int count, const aco_params &p);

    int init();                  // g_ACO::init_aco for every instance
    int enqueue(int n_iter);     // n_iter iterations (graph replays), no sync
    int sync_status();           // wait for the stream, read the sticky status
    int clear_status();          // sync_status, then reset the sticky status to ACO_OK
    int set_wait_limit(int polls); // poll limit of the device waits (0 = default), from the next launch
    int launches_per_iteration() const; // kernel launches of one iteration (graph nodes)
    // in_iteration: the 2-opt follows (fused 2-opt warps when configured; with the
    // route list the 2-opt writes the tour lengths); false: the phase alone
    int construct(bool in_iteration = false);
    int local_search();
    int neighbourhood(); // the random-descent stage (ns_rounds > 0)
    int stats(bool elites);
    int update();
    int pheromone_init(float trail, bool from_bsf);
    int gather_candidates();     // refresh the compact candidate table from total_info
    // heur = eta^beta * prior for instance b (prior: n x n host array, row stride ld;
    // null restores eta^beta); total_info follows when the colony is initialised
    int set_prior(int b, const float *prior, int ld);
    // Check every tour slot on the device; flags (total slots, or null) and
    // per-instance invalid counts (or null) are copied back.
    int validate(int *flags, int *invalid_per_inst, int *n_invalid);
    // Everything the next iteration reads, to a file / back from it (a colony
    // created with the same instances and parameters; total_info and the
    // candidate table are recomputed from tau).
    int save_checkpoint(const char *path);
    int load_checkpoint(const char *path);
    int time_phases(int n_iter, float *ms4);
    int set_device() const;
    // Every instance's best-so-far tour (2n ints at the prefix sum of 2n),
    // size and length, gathered on the device and copied in one transfer.
    int get_best_all(int *tours, size_t cap_ints, int *sizes, float *lengths);
    // All instances' lengths are one contiguous block: instance b's A+1 floats
    // (ants, then best-so-far) start at lens_base()[b].
    const float *lens_all() const { return lens_all_d_; }
    int lens_total() const { return slot_base_h_.empty() ? 0 : slot_base_h_.back(); }
    int tours_total() const { return tour_base_h_.empty() ? 0 : tour_base_h_.back(); }

    aco_params p{};
    int dev = 0, sm_count = 148;
    cudaStream_t st = nullptr;
    std::vector<InstHost> inst;
    bool initialized = false;
    std::chrono::steady_clock::time_point t_init;
    int *h_pin = nullptr;
    int *status_d = nullptr;
    int *wait_d = nullptr;       // poll limit the construct kernels read at every launch

    // launch configuration
    int cp_wpa = 1, cp_apc = 1;
    bool cp_stage = false;
    int cn_apc = 1, cn_lsw = 0; // throughput construct: ants per CTA, fused 2-opt warps (0 = separate kernel)
    bool cn_draw = false;       // throughput construct: helper warps make the race draws
    bool cn_wide = false;       // throughput construct: two CTAs per SM (64 registers, half the shared memory each)
    StatsArgs stats_one_{};     // a single instance's statistics arguments, passed by value
    size_t cn_smem = 0;
    int ls_warps = 1, ls_apc = 1, ls_nmax = 0; // 2-opt: warps and ants per CTA, largest instance
    int sw_apc = 1, sw_items = 0; // swap stage: ants per CTA, work items
    size_t sw_smem = 0;
    int ns_apc = 1, ns_items = 0; // random-descent stage
    size_t ns_smem_ = 0;
    size_t ls_smem = 0, stats_smem = 0;
    int ld_max = 32, total_ants = 0, total_rows = 0, n_items = 0;
    bool fin_any = false;

private:
    int run_phases();
    int ensure_graph();
    int run_rows(int mode, float trail);
    int run_rows_one(int b, int mode);
    std::vector<void *> allocs_;
    void *arena_ = nullptr;
    bool pooled_ = false; // arena from the device's memory pool (freed stream-ordered)
    unsigned long long *t0_d_ = nullptr;
    int2 *items_d_ = nullptr, *sw_items_d_ = nullptr, *ns_items_d_ = nullptr;
    uint8_t *ls_needed_d_ = nullptr;
    // route-level 2-opt (throughput mode, symmetric distances): the construct's
    // route list, its counters and the listed routes left per ant
    bool use_routes_ = false, routes_pending_ = false;
    int route_cap_ = 0;
    int2 *route_desc_d_ = nullptr;
    int *route_ctr_d_ = nullptr, *route_rem_d_ = nullptr;
    int *ls_list_d_ = nullptr, *ls_list_ctr_d_ = nullptr; // ants left to the per-ant 2-opt
    bool last_fused_ = false;
    int *queue_d_ = nullptr, *ant_inst_d_ = nullptr, *ant_base_d_ = nullptr;
    int *row_base_d_ = nullptr, *zero_base_d_ = nullptr, *row_inst_d_ = nullptr;
    int *slot_base_d_ = nullptr, *valid_d_ = nullptr, *invalid_d_ = nullptr;
    std::vector<int> slot_base_h_, tour_base_h_;
    float *lens_all_d_ = nullptr;
    int *tour_base_d_ = nullptr, *best_tours_d_ = nullptr, *best_sizes_d_ = nullptr;
    float *best_lens_d_ = nullptr;
    ConstructArgs *cargs_d_ = nullptr;
    LocalSearchArgs *largs_d_ = nullptr;
    StatsArgs *sargs_d_ = nullptr;
    UpdateArgs *uargs_d_ = nullptr;
    std::vector<ConstructArgs> cargs_h_;
    cudaGraph_t graph_ = nullptr;
    cudaGraphExec_t exec_ = nullptr;
};

} // namespace aco
