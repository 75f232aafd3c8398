/*
 * cvrp_aco.h -- C ABI of the B200 (sm_100a) CVRP ant-colony solver.
 *
 * Drop-in boundary for the reference's hot path (i-sunny/cvrp_aco_ocl): the
 * C++ class g_ACO (cvrp_ocl/gpu/g_aco.h:16-72) over the Problem struct
 * (cvrp_ocl/problem.h:82-140) and the parameter globals alpha/beta/rho/ras_ranks
 * (cvrp_ocl/problem.h:30-33).  The reference has no FFI of its own; these entry
 * points are what a binding of g_ACO would bind.  Every declaration names the
 * reference routine it replaces.
 *
 * Conventions: plain pointers and sizes, no framework types.  Every call returns
 * an int status: ACO_OK (0) or a negative ACO_ERR_* code; nothing exits or traps.
 * Tours use the reference's layout: a tour is a sequence of node ids that starts
 * and ends at the depot 0 and returns to 0 between routes
 * (cvrp_ocl/problem.h:68-72).  A solver owns its device memory, one CUDA stream
 * and the CUDA graph of one iteration; it is not re-entrant, but separate
 * solvers may be driven from separate host threads.
 */
#ifndef CVRP_ACO_H
#define CVRP_ACO_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (the reference exit(1)s instead: g_aco.cpp:607-614) ---- */
#define ACO_OK 0
#define ACO_ERR_INVALID (-1)        /* bad argument or parameter */
#define ACO_ERR_INFEASIBLE (-2)     /* a customer can never be served (demand > capacity, or out of max distance) */
#define ACO_ERR_CUDA (-3)           /* a CUDA runtime call failed */
#define ACO_ERR_NO_DEVICE (-4)      /* no usable sm_100 device */
#define ACO_ERR_NOMEM (-5)          /* device or host allocation failed */
#define ACO_ERR_STATE (-6)          /* call out of order (e.g. iterate before init) */
#define ACO_ERR_STEP_LIMIT (-7)     /* a construction exceeded 2n-3 steps (would loop forever in the reference) */
#define ACO_ERR_LS_LIMIT (-8)       /* 2-opt exceeded its improvement-pass budget */
#define ACO_ERR_RECORD_OVERFLOW (-9)/* more best-so-far records than record_cap (reference: unchecked, kernel.cl:578-583) */
#define ACO_ERR_CAPACITY (-10)      /* a caller buffer is too small */
#define ACO_ERR_IO (-11)            /* instance file missing or malformed */
#define ACO_ERR_TIMEOUT (-12)       /* a bounded device wait gave up */

/* ---- enums -------------------------------------------------------------- */
enum { ACO_DIST_EUC_2D = 0, ACO_DIST_CEIL_2D = 1, ACO_DIST_GEO = 2, ACO_DIST_ATT = 3 }; /* problem.h:36-38 */
enum {
    ACO_MODE_PARITY = 0,     /* full-row I-Roulette with the reference's RNG stream: bit-exact */
    ACO_MODE_THROUGHPUT = 1  /* nearest-neighbour candidate lists, roulette probabilities drawn as an exponential race */
};

/* Instance: the fields of Problem the path reads (problem.h:82-99).  Either
 * coordinates (x, y + dist_type) or a precomputed row-major n*n distance
 * matrix `dist` must be given; when both are, `dist` wins.  Node 0 is the depot. */
typedef struct aco_instance {
    int n;                /* num_node, depot included */
    const float *x;       /* nodeptr[i].x */
    const float *y;       /* nodeptr[i].y */
    const int *demand;    /* nodeptr[i].demand */
    int capacity;         /* vehicle_capacity */
    float max_distance;   /* max_distance (INFINITY = unlimited, the reader's default io.cpp:348) */
    float service_time;   /* service_time */
    int dist_type;        /* ACO_DIST_* */
    const float *dist;    /* optional precomputed distances */
} aco_instance;

/* Parameters: set_default_parameters (problem.cpp:186-220) plus the values the
 * reference hard-codes or takes from the clock. */
typedef struct aco_params {
    int n_ants;           /* n_ants (default n, problem.cpp:189); at most 57344 */
    float alpha;          /* 1.0 (kernel.cl:10, problem.cpp:207) */
    float beta;           /* 2.0 (kernel.cl:11) */
    float rho;            /* 0.1 (kernel.cl:9) */
    int ras_ranks;        /* 6 (kernel.cl:12): the best-so-far ant + ras_ranks-1 iteration elites */
    int nn_ants;          /* candidate-list length for ACO_MODE_THROUGHPUT (default min(25, n-2)) */
    int nn_ls;            /* 2-opt neighbour-list depth, <= n-2 (default n-2, problem.cpp:191-193) */
    int ls_flag;          /* 1 = 2-opt after every construction (default 1, problem.cpp:203); 3 = 2-opt then
                             the inter-route swap of the CPU local search (localSearch.cpp:51-81,301-410) */
    int mode;             /* ACO_MODE_* (default PARITY) */
    int nloc;             /* work-items per ant of the reference's construct kernel: maxWorkGroupSize/4
                             (g_aco.cpp:41); sets the RNG lane layout; a power of two in [32, 1024], default 256 */
    int seed_time;        /* replaces time(NULL) in the seed formula (g_aco.cpp:718) */
    int rnd_seed;         /* replaces instance->rnd_seed = time(NULL) (problem.cpp:212) */
    int max_iteration;    /* 250 (problem.cpp:196); used by aco_run */
    float max_runtime;    /* 600 s (problem.cpp:213); used by aco_run */
    int ls_pass_limit;    /* 2-opt improvement passes allowed per route before ACO_ERR_LS_LIMIT (default 4096) */
    int record_cap;       /* best-so-far record capacity (default 4096, g_aco.cpp:727-729) */
    int device;           /* CUDA device ordinal (default 0) */
    int use_graph;        /* 1 = replay one CUDA graph per iteration (default 1) */
    int ants_per_block;   /* 0 = autotuned; else ants per CTA of the construct kernel */
    int warps_per_ant;    /* 0 = autotuned; else warps per ant of the parity construct kernel (1,2,4,8) */
    int ls_warps;         /* 0 = autotuned; else warps per 2-opt CTA (1..32, one route per warp at a time) */
    int stage_matrix;     /* throughput construct: 0 = stage the whole total_info matrix in shared memory when
                             it fits (used by the no-candidate fallback); -1 = never, rows are read through L2 */
    int host_prep;        /* 0 = distances and neighbour lists computed on the device when the distance type
                             allows (all but GEO; bit-identical to the host); 1 = on the host */
    int fuse_ls;          /* throughput mode with 2-opt, n <= 1024: 1 = improve each route inside the construct
                             kernel as soon as it is complete (same results); 0 = separate 2-opt kernel (default,
                             faster on the measured workloads) */
    int ns_rounds;        /* random-descent stage after the local search: proposals of the reference's
                             random neighbourhood moves (neighbourSearch.cpp, move.cpp) per ant and iteration,
                             the valid improving ones applied; 0 = off (default) */
    int ls_ants;          /* 0 = autotuned; else ants per 2-opt CTA (1..8), whose routes its warps share */
    int draw_warps;       /* throughput construct: 1 = a helper warp per ant makes the ant's draws ahead of it
                             (at most 8 ants per CTA), -1 = the ant's warp draws, 0 = automatic (helper warps
                             while there are at most 4 ants per SM); same results either way */
    int route_ls;         /* throughput mode with 2-opt, symmetric distances: 1 = the construct lists every route
                             (of at most 255 nodes) and one persistent kernel improves them all, spread over the SMs;
                             -1 = one CTA per group of ants; 0 = automatic (the list above 4 ants per SM); same
                             results either way */
    int wait_limit;       /* polls of an mbarrier before a device wait gives up with ACO_ERR_TIMEOUT (0 = the
                             default, 2^24 polls, about a second); no reference counterpart (kernel.cl has no
                             bounded waits) */
    int ls_best;          /* 2-opt move choice: 0 = first improvement in scan order with don't-look bits, the
                             reference's (kernel.cl:126-277; default); 1 = best improvement, a non-parity option:
                             every move of a route of at most 32 nodes evaluated from its distance tile and the
                             best applied (a warp argmin) until none improves; longer routes keep first
                             improvement.  For symmetric distances. */
    int construct_ctas;   /* throughput construct without helper draws or fused 2-opt: 2 = two 512-thread CTAs per
                             SM at 64 registers a thread, candidate tables that do not fit half of an SM's shared
                             memory read through L2; 1 = one CTA per SM at up to 128 registers, tables staged where
                             they fit; 0 = automatic (two while there are at least 32 ants per SM); same results
                             either way */
} aco_params;

/* One best-so-far record {iteration, length, seconds since init} (problem.h:62-66). */
typedef struct aco_record {
    int iter;
    float length;
    float time;
} aco_record;

typedef struct aco_solver aco_solver;

/* ---- parameters and host-side instance tools ----------------------------- */
/* set_default_parameters (problem.cpp:186-220) for an instance of n nodes. */
int aco_params_default(aco_params *p, int n);

/* read_instance_file (io.cpp:334-517): parses a VRPLIB file.  Call once with
 * x == NULL to get n; then again with arrays of n entries. */
int aco_read_vrplib(const char *path, int *n, float *x, float *y, int *demand, int *capacity,
                    float *max_distance, float *service_time, int *dist_type, float *optimum,
                    char *name, int name_cap);

/* compute_distances (vrpHelper.cpp:160-184): row-major n*n fp32. */
int aco_compute_distances(int n, const float *x, const float *y, int dist_type, float *dist);

/* compute_nn_lists (vrpHelper.cpp:188-236, sort2 tie order utilities.cpp:246-266):
 * depth = min(max(nn_ls, nn_ants), n-1) entries per node, written to nn (n*depth). */
int aco_compute_nn_lists(int n, const float *dist, int nn_ls, int nn_ants, int *nn, int *depth);
/* The same two steps on the device (device pointers; no reference counterpart as an
 * entry point): distances into an n x ld matrix (EUC_2D, CEIL_2D, ATT; GEO is
 * ACO_ERR_INVALID because its cos/acos bits depend on the math library), and
 * the lists (n x depth, depth = min(max(nn_ls, nn_ants), n-1)) from an n x ld
 * matrix, in the reference's quicksort tie order.  Both only enqueue work. */
int aco_compute_distances_device(int n, const float *x, const float *y, int dist_type, float *dist, int ld,
                                 void *stream);
int aco_compute_nn_lists_device(int n, const float *dist, int ld, int nn_ls, int nn_ants, int *nn, int *depth,
                                void *stream);

/* check_solution (problem.cpp:226-319): 1 valid, 0 invalid, <0 error. */
int aco_check_solution(const aco_instance *inst, const int *tour, int tour_size);

/* compute_tour_length (vrpHelper.cpp:244-253) in fp32, and the same sum in fp64. */
int aco_tour_length(int n, const float *dist, const int *tour, int tour_size, float *len32, double *len64);

/* The per-work-item seeds of create_memory_objects (g_aco.cpp:714-722), with
 * time(NULL) = seed_time; *rnd_seed is advanced as the reference advances it. */
int aco_make_seeds(int seed_time, int *rnd_seed, int n_ants, int nloc, int *seeds);

/* ---- solver lifecycle: g_ACO (g_aco.h:16-37) ------------------------------ */
/* g_ACO::g_ACO + create_memory_objects (g_aco.cpp:35-43, 640-761): copies the
 * instance to the device, computes distances / NN lists / seeds. */
int aco_create(const aco_instance *inst, const aco_params *params, aco_solver **out);
/* g_ACO::init_aco (g_aco.cpp:63-93): bootstrap construct, trail_0 = 1/(rho*L). */
int aco_init(aco_solver *s);
/* n_iter x (g_ACO::run_aco_iteration (g_aco.cpp:122-134) + iteration++ (main.cpp:86)). */
int aco_iterate(aco_solver *s, int n_iter);
/* main.cpp:84-88: iterate until max_iteration / max_runtime / optimum (within 10*EPSILON). */
int aco_run(aco_solver *s, float optimum, int *iterations_done);
/* g_ACO::exit_aco + destructor (g_aco.cpp:45-61, 95-117). */
void aco_destroy(aco_solver *s);

/* ---- the individual phases (public methods of g_ACO) -------------------- */
int aco_construct_solutions(aco_solver *s); /* g_aco.cpp:141-177 */
int aco_local_search(aco_solver *s);        /* g_aco.cpp:182-228 */
int aco_update_statistics(aco_solver *s);   /* g_aco.cpp:407-417 (+ iteration++ of the caller) */
int aco_pheromone_update(aco_solver *s);    /* g_aco.cpp:233-243 */
int aco_pheromone_init(aco_solver *s, float trail_0); /* g_aco.cpp:245-263 */

/* ---- results and test taps ----------------------------------------------- */
/* update_best_so_far_from_device (g_aco.cpp:527-552). */
int aco_get_best(aco_solver *s, int *tour, int cap, int *tour_size, float *length);
/* the bsf record stream read by exit_aco (g_aco.cpp:100-113). */
int aco_get_bsf_records(aco_solver *s, aco_record *out, int cap, int *count);
/* solutions_mem / solution_lens_mem in the reference layout (g_aco.cpp:652-665):
 * solutions has 2n*(n_ants+1)+1 ints, lens n_ants+1 floats. */
int aco_get_solutions(aco_solver *s, int *solutions, size_t cap_ints, float *lens, size_t cap_lens);
/* pheromone_mem / total_info_mem as dense row-major n*n. */
int aco_get_pheromone(aco_solver *s, float *tau, float *total_info, size_t cap);
/* seed_mem: n_ants*nloc ints. */
int aco_get_seeds(aco_solver *s, int *seeds, size_t cap);
/* elite_ids_mem: ras_ranks ints. */
int aco_get_elites(aco_solver *s, int *elites, int cap);
/* the current iteration counter (Problem::iteration). */
int aco_get_iteration(aco_solver *s, int *iteration);
/* overwrite state for phase-level tests: pheromone + total_info (dense n*n),
 * solutions + lens (reference layout), seeds.  NULL pointers are skipped. */
int aco_set_state(aco_solver *s, const float *tau, const float *total_info, const int *solutions,
                  const float *lens, const int *seeds);
/* sticky device status of the last launches (ACO_OK or an ACO_ERR_* code). */
int aco_status(aco_solver *s);
/* Waits for the stream, returns the sticky device status and resets it to
 * ACO_OK, so the solver can go on after a reported error (no reference
 * counterpart: the reference exit(1)s, g_aco.cpp:607-614). */
int aco_clear_status(aco_solver *s);
/* Polls of an mbarrier before a device wait gives up (aco_params.wait_limit;
 * 0 = the default); takes effect from the next launch, graph replays included.
 * No reference counterpart. */
int aco_set_wait_limit(aco_solver *s, int polls);
const char *aco_strerror(int code);
/* CUDA's description of the last CUDA error that a call on this thread turned
 * into ACO_ERR_CUDA (diagnostics; no reference counterpart). */
const char *aco_last_cuda_error(void);

/* ---- timing and interop --------------------------------------------------- */
/* the solver's CUDA stream (a cudaStream_t), for event timing by the caller. */
void *aco_get_stream(aco_solver *s);
/* number of kernel launches one iteration makes (graph nodes when graphs are on). */
int aco_launches_per_iteration(aco_solver *s);
/* device-timed run of n_iter iterations on the solver's stream (CUDA events). */
int aco_time_iterations(aco_solver *s, int n_iter, float *ms);
/* enqueue n_iter iterations on the solver's stream and return without waiting
 * (aco_status waits and reports); lets a caller bracket them with its own events. */
int aco_enqueue_iterations(aco_solver *s, int n_iter);
/* Pipelined readback of the A+1 tour lengths (ants, then best-so-far) as the
 * stream stands after the work queued so far: aco_enqueue_lengths queues a copy
 * into one of 4 solver-owned pinned slots and returns a ticket; aco_read_lengths
 * waits for that copy only, writes the lengths to `lens` (cap >= A+1) and
 * returns the device status.  A caller can queue iteration k+1 before reading
 * iteration k, so the GPU does not idle during the host's readback (the
 * reference reads back after every iteration, g_aco.cpp:407-417).  At most 4
 * tickets are outstanding; an older one reads ACO_ERR_STATE.  No reference
 * counterpart. */
int aco_enqueue_lengths(aco_solver *s, long long *ticket);
int aco_read_lengths(aco_solver *s, long long ticket, float *lens, size_t cap);
/* n_iter iterations launched phase by phase with CUDA events between the
 * phases: ms[0] construct, ms[1] 2-opt, ms[2] statistics, ms[3] pheromone pass
 * (device milliseconds summed over the iterations). */
int aco_time_phases(aco_solver *s, int n_iter, float *ms4);
/* the kernel configuration the solver picked: ants per CTA and warps per ant of
 * construct, and whether matrices are staged in shared memory (bit 0: total_info
 * in construct, bit 1: NN lists in 2-opt); bit 2: the throughput construct runs
 * with helper draw warps (construct_nn_draw_kernel); bit 3: it runs two CTAs per
 * SM (construct_nn_wide_kernel). */
int aco_get_config(aco_solver *s, int *ants_per_block, int *warps_per_ant, int *staging_flags);

/* ---- validation and output -------------------------------------------------
 * aco_validate checks every tour slot (ants and best-so-far) on the device with
 * check_solution's rules (problem.cpp:226-319: starts at the depot, every
 * customer exactly once, every route non-empty, within capacity and
 * max_distance) plus node-id range checks and an exact check of the stored
 * length against the fp32 sum of the tour's edges (compute_tour_length,
 * vrpHelper.cpp:244-253).  flags (A+1 ints, or NULL): 1 = valid.  The batch
 * form counts invalid slots per instance (count ints, or NULL).
 * aco_write_solution writes the best-so-far tour as print_solution_to_file
 * does (io.cpp:270-281: "Begin Solution", the tour, "Solution Length %f",
 * "End Solution"); the batch form writes one such block per instance, each
 * after a line "Instance <index>". */
int aco_validate(aco_solver *s, int *flags, int *n_invalid);
int aco_write_solution(aco_solver *s, const char *path);

/* ---- checkpoint and resume (no reference counterpart) ------------------------
 * aco_save_checkpoint writes everything the next iteration reads -- tau, the
 * tours and lengths (best-so-far slot included), the lane seeds, the
 * best-so-far records and the iteration counter -- after aco_init.
 * aco_load_checkpoint restores it into a solver created with the same
 * instance data, seeds and parameters and holding the same prior (the file
 * records a hash of each instance's data and prior; ACO_ERR_INVALID
 * otherwise); total_info and the candidate table are recomputed from tau.  The iterations after a load are bit-identical to the ones the
 * saving solver would have run.  Record times restart from the load. */
int aco_save_checkpoint(aco_solver *s, const char *path);
int aco_load_checkpoint(aco_solver *s, const char *path);

/* ---- autotuner (no reference counterpart) -----------------------------------
 * Times launch configurations on the instance(s) and returns the fastest in
 * *out (a copy of *p with ants_per_block, stage_matrix, draw_warps, route_ls,
 * ls_ants, ls_warps -- and warps_per_ant in ACO_MODE_PARITY -- set where they
 * were 0).  Every configuration computes the same tours, lengths and
 * pheromone bit for bit; only speed differs.  Each candidate runs on a fresh
 * solver from the same seeds: aco_init, 2 warm-up iterations, then `iters`
 * timed iterations (per-kernel CUDA events).  The configuration as given (its
 * 0 fields chosen by the library's create-time model) is the baseline; the
 * construct candidates (ants per CTA x staging x helper draw warps) are timed
 * first, then the route list against the per-ant 2-opt kernel, then (without
 * the list) the 2-opt CTA widths, and a candidate replaces the current choice
 * only when it is more than 2% faster (5% for the 2-opt CTA shape).  ms_out (optional) = the chosen configuration's time per
 * iteration.  The candidate-list length (nn_ants) changes the search itself,
 * not only its speed, so it is not chosen here. */
int aco_autotune(const aco_instance *inst, const aco_params *p, int iters, aco_params *out, float *ms_out);
int aco_batch_autotune(const aco_instance *insts, int count, const aco_params *p, int iters, aco_params *out,
                       float *ms_out);

/* ---- batches: many independent instances in the same launches --------------
 * No reference counterpart (the reference solves one instance per process).
 * ACO_MODE_THROUGHPUT only; every instance has its own device state
 * (pheromone, tours, best-so-far, records); instance b uses the
 * seeds of rnd_seed + b.  Lists deeper than an instance allows are clamped to
 * n-2 for it.  One iteration is four or five launches for the whole batch: a
 * persistent construct kernel over a device work queue of (instance, ant group)
 * items, the route-level 2-opt over the construct's route list (with more than
 * 4 ants per SM) and the per-ant 2-opt for the ants it does not hold,
 * statistics (one CTA per instance) and the row pass over every instance's
 * matrices; replayed as one CUDA graph. */
typedef struct aco_batch aco_batch;
int aco_batch_create(const aco_instance *insts, int count, const aco_params *params, aco_batch **out);
int aco_batch_init(aco_batch *b);
int aco_batch_iterate(aco_batch *b, int n_iter);
int aco_batch_enqueue_iterations(aco_batch *b, int n_iter);
int aco_batch_status(aco_batch *b);
int aco_batch_size(aco_batch *b, int *count, int *total_ants);
int aco_batch_get_best(aco_batch *b, int idx, int *tour, int cap, int *tour_size, float *length);
int aco_batch_get_solutions(aco_batch *b, int idx, int *solutions, size_t cap_ints, float *lens, size_t cap_lens);
int aco_batch_get_pheromone(aco_batch *b, int idx, float *tau, float *total_info, size_t cap);
int aco_batch_time_phases(aco_batch *b, int n_iter, float *ms4);
/* aco_get_config for a batch (its one construct launch over all instances; bit 0
 * describes instance 0). */
int aco_batch_get_config(aco_batch *b, int *ants_per_block, int *warps_per_ant, int *staging_flags);
void *aco_batch_get_stream(aco_batch *b);
/* number of kernel launches one batch iteration makes (graph nodes).  No reference counterpart. */
int aco_batch_launches_per_iteration(aco_batch *b);
/* Pipelined readback of every instance's lengths, as aco_enqueue_lengths /
 * aco_read_lengths for one solver (the reference reads them back after every
 * iteration, g_aco.cpp:407-417): `lens` receives sum over instances of
 * (n_ants + 1) floats, instance b's ants then its best-so-far at offset
 * sum_{c<b} (n_ants + 1).  At most 4 tickets are outstanding.  No reference
 * counterpart. */
int aco_batch_enqueue_lengths(aco_batch *b, long long *ticket);
int aco_batch_read_lengths(aco_batch *b, long long ticket, float *lens, size_t cap);
/* Every instance's best-so-far tour in one transfer (update_best_so_far_from_device,
 * g_aco.cpp:527-552, for the whole batch): tours receives sum of 2n ints,
 * instance b's slot (reference layout, size in its last int) at offset
 * sum_{c<b} 2n_c; tour_sizes and lengths (count entries each) may be NULL. */
int aco_batch_get_best_all(aco_batch *b, int *tours, size_t cap_ints, int *tour_sizes, float *lengths);
void aco_batch_destroy(aco_batch *b);

/* ---- learned prior: edge-scoring network (no reference counterpart) -------
 * A message-passing network on the k-nearest-customer graph of an instance
 * scores every edge (i, j); sigmoid(score) multiplies eta^beta as a sampling
 * prior (aco_set_prior).  Hidden width 64, BF16 tensor-core products with FP32
 * accumulation, FP32 master parameters (aco_mpnn_param_count floats, packed
 * in the order embeddings, layers (W, b, A, a), head (W_h, b_h, w_o, b_o)).
 * Graph arrays hold node i's k out-edges at rows i*k .. i*k+k-1; several
 * graphs are batched by concatenating their nodes (nbr holds global ids).
 * All pointers below are device pointers; stream may be NULL.  The calls only
 * enqueue work; aco_mpnn_status synchronises and returns the sticky status. */
#define ACO_MPNN_HIDDEN 64
#define ACO_MPNN_NODE_FEATURES 5 /* x, y (bounding-box normalised), demand/capacity, is_depot, d(i, depot) */
int aco_mpnn_param_count(int layers);
int aco_mpnn_workspace_bytes(int n_nodes, int k, int layers, size_t *bytes);
/* scores[n_nodes*k]: edge logits. */
int aco_mpnn_forward(int n_nodes, int k, int layers, const float *params, const float *node_feat,
                     const float *edge_feat, const int *nbr, void *workspace, size_t ws_bytes, float *scores,
                     void *stream);
/* Forward + backward of the mean weighted binary cross-entropy against labels
 * (1 = the edge is on the target route): grad (param_count floats) and *loss
 * are overwritten; scores (optional) receives the logits. */
int aco_mpnn_grad(int n_nodes, int k, int layers, const float *params, const float *node_feat, const float *edge_feat,
                  const int *nbr, const float *labels, float pos_weight, void *workspace, size_t ws_bytes, float *grad,
                  float *loss, float *scores, void *stream);
/* One Adam step (bias-corrected, step >= 1) on count parameters. */
int aco_mpnn_adam(int count, float *params, const float *grad, float *m, float *v, float lr, float beta1, float beta2,
                  float eps, int step, void *stream);
int aco_mpnn_status(void *workspace, void *stream);

/* Sampling prior: heur = eta^beta * prior (prior: n x n host array, row stride
 * ld >= n, finite and >= 0), so that total_info = tau^alpha * eta^beta * prior.
 * Tours stay feasible and lengths exact: only the choice weights change.  Call
 * before aco_init (the bootstrap construct uses it) or between iterations
 * (total_info is recomputed from the current tau).  prior = NULL restores plain
 * eta^beta, the fallback.  A non-uniform prior departs from the reference's
 * choice rule: use it with ACO_MODE_THROUGHPUT. */
int aco_set_prior(aco_solver *s, const float *prior, int ld);
int aco_batch_set_prior(aco_batch *b, int idx, const float *prior, int ld);
int aco_batch_validate(aco_batch *b, int *invalid_per_instance, int *n_invalid);
int aco_batch_save_checkpoint(aco_batch *b, const char *path);
int aco_batch_load_checkpoint(aco_batch *b, const char *path);
int aco_batch_write_solutions(aco_batch *b, const char *path);
int aco_batch_get_bsf_records(aco_batch *b, int idx, aco_record *out, int cap, int *count);

/* ---- pheromone update without allocation ---------------------------------
 * No counterpart in the reference.  For callers that cannot let this library
 * allocate device memory: hosts whose memory manager owns all device memory,
 * and loops that cannot take the device-wide synchronisation of cudaMalloc /
 * cudaFree.  Runs the update of aco_update_statistics' elite selection +
 * aco_pheromone_update on the caller's device buffers, enqueued on `stream`
 * (a cudaStream_t, NULL = legacy default stream):
 *   tau, total_info : n rows of ld floats (ld >= n), tau updated in place;
 *   dist            : n rows of ld floats, distances;
 *   solutions, lens : the reference layout (2n*(n_ants+1)+1 ints, n_ants+1
 *                     floats) after the statistics step (best-so-far in slot n_ants);
 *   elites_out      : ras_ranks ints, or NULL.
 * The elite tours are checked before they are used as indices: an elite whose
 * size is outside [2, 2n-1] or that holds a node id outside [0, n) deposits
 * nothing, and its elites_out entry reads ACO_ERR_INVALID instead of its ant id.
 * Scratch is a fixed 148 KB array inside the library (kept by every GPU that
 * loads it until exit): n <= 4096 and ras_ranks <= 8, else ACO_ERR_CAPACITY.
 * The first call on a device (and again after its context is recreated) looks
 * up that array's device address; make it before any stream capture.  Calls
 * share the array, so calls that overlap on the GPU race.  Allocates nothing,
 * frees nothing. */
int aco_pheromone_update_noalloc(int n, int ld, int n_ants, int ras_ranks, float rho, float alpha, float beta,
                                 float *tau, float *total_info, const float *dist, const int *solutions,
                                 const float *lens, int *elites_out, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* CVRP_ACO_H */
