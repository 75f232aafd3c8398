/*
 * aco_oracle.h -- CPU oracle for the CVRP ACO iteration (TEST INFRASTRUCTURE ONLY).
 *
 * This is the checker, never the product: only tests, the smoke check and the
 * benchmark's CPU-baseline leg may load it.  Every function restates one piece of
 * the reference (i-sunny/cvrp_aco_ocl) and names the file:line it follows.
 * Matrices are dense row-major n*n (no pitch); tours use the reference's layout:
 * ant a's tour at solutions[a*T], its size at solutions[a*T + T-1], T = 2n, the
 * best-so-far slot at ant index n_ants and the iteration-best index at
 * solutions[T*(n_ants+1)] (cvrp_ocl/gpu/g_aco.cpp:652-654).
 */
#ifndef ACO_ORACLE_H
#define ACO_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_OK 0
#define ORC_ERR_STEP_LIMIT (-7)
#define ORC_ERR_LS_LIMIT (-8)

typedef struct orc_record {
    int iter;
    float length;
    float time;
} orc_record;

/* All state the reference keeps in device buffers (cvrp_ocl/gpu/g_aco.cpp:640-761). */
typedef struct orc_state {
    int n, n_ants, nloc, nn_ls, ras_ranks;
    int capacity;
    float max_dist, serv_time;
    float alpha, beta, rho;
    int ls_flag;          /* bit 0: 2-opt after every construct (and in the bootstrap);
                             bit 1: then the inter-route swap stage (orc_swap) */
    int step_limit_passes;/* max 2-opt improvement passes per route (0 = unbounded) */
    const float *dist;    /* n*n */
    const int *demand;    /* n */
    const int *nn_list;   /* n*nn_ls */
    float *tau, *total;   /* n*n */
    int *seeds;           /* n_ants*nloc */
    int *solutions;       /* 2n*(n_ants+1)+1 */
    float *lens;          /* n_ants+1 */
    int *elites;          /* ras_ranks */
    orc_record *records;  /* record_cap */
    int record_cap, num_bsf;
    int iteration, update_flag, status;
    int ns_rounds;        /* random-move proposals per ant and iteration after the local search (0 = off) */
    int ns_seed;          /* generator seeds: orc_ns_seed(ns_seed, iteration, ant) */
} orc_state;

/* ---- RNG, seeds -------------------------------------------------------- */
float orc_ran01(int *idum);
int orc_f2i_x86(float v);
/* -ln(u), the throughput sampler's exponential clock (the device's race_exp1) */
float orc_race_exp1(float u);
void orc_make_seeds(int seed_time, int *rnd_seed, int n_ants, int nloc, int *seeds);

/* ---- inputs ------------------------------------------------------------ */
void orc_compute_distances(int n, const float *x, const float *y, int dist_type, float *dist);
int orc_compute_nn_lists(int n, const float *dist, int nn_ls, int nn_ants, int *nn_out);
float orc_tour_length(int n, const float *dist, const int *tour, int tour_size);
double orc_tour_length_f64(int n, const float *dist, const int *tour, int tour_size);
int orc_check_solution(int n, const float *dist, const int *demand, int capacity,
                       float max_dist, float serv_time, const int *tour, int tour_size);
void orc_tournament_priority(int n, int *prio);
float orc_pow_rule(float x, float e);

/* ---- hot path phases --------------------------------------------------- */
int orc_construct(orc_state *s, int n_threads);
int orc_local_search(orc_state *s, int n_threads);
/* LocalSearch::swap (localSearch.cpp:301-410) on one tour; returns the number
 * of swaps, or -1 once more than max_swaps (> 0) were applied. */
#define ORC_SWAP_LIMIT_PER_NODE 64
int orc_swap(int n, const float *dist, const int *demand, int capacity, float max_dist, float serv_time,
             int *tour, int tour_size, int max_swaps);
void orc_find_best(orc_state *s);
void orc_update_best_so_far(orc_state *s, float time);
void orc_get_elites(orc_state *s);
void orc_pheromone_init(orc_state *s, float trail);
void orc_pheromone_evaporation(orc_state *s);
void orc_pheromone_deposit(orc_state *s);
void orc_compute_total_info(orc_state *s);

/* ---- sequencing (g_ACO::init_aco / run_aco_iteration) ------------------ */
int orc_init_aco(orc_state *s, int n_threads);
int orc_run_aco_iteration(orc_state *s, int n_threads);

/* ---- throughput mode (this project's own candidate-list sampler) ------- */
int orc_construct_nn(orc_state *s, const int *nn_ants_list, int nn_ants, int n_threads);
int orc_run_aco_iteration_nn(orc_state *s, const int *nn_ants_list, int nn_ants, int n_threads);
int orc_init_aco_nn(orc_state *s, const int *nn_ants_list, int nn_ants, int n_threads);

#ifdef __cplusplus
}
#endif

/* ---- random neighbourhood moves (ns_oracle.c) ------------------------- */
typedef struct orc_rng { uint32_t r[31]; int f, b; } orc_rng; /* glibc random(), TYPE_3 */
void orc_srandom(orc_rng *g, unsigned seed);
int32_t orc_random(orc_rng *g);
typedef struct orc_move {
    int type; /* 0 exchange, 1 insertion, 2 inversion, -1 none */
    int valid;
    float gain;
    int pos1, pos2;
} orc_move;
void orc_ns_propose(int n, const float *dist, const int *demand, int cap, float max_dist, float serv,
                    const int *tour, int size, orc_rng *g, orc_move *m);
void orc_ns_apply(int *tour, const orc_move *m);
/* seed of ant `ant`'s generator in iteration `iteration` */
unsigned orc_ns_seed(int rnd_seed, int iteration, int ant);
/* `rounds` proposals; the valid ones with gain < -EPSILON are applied */
int orc_ns_descent(int n, const float *dist, const int *demand, int cap, float max_dist, float serv, int *tour,
                   int size, unsigned seed, int rounds);

#endif
